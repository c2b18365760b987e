"""Launch shapes and kernel implementation choices change where the work runs,
not the arithmetic: the k/omega sweeps chained across CTAs through DSMEM,
or pipelined with a cluster barrier per row, give the same bits as the same
sweeps one after another, and a solve on a wide cluster tracks the oracle as
closely as on one CTA."""
import os

import numpy as np
import pytest

import cfd_b200 as cb
from helpers import Case, rel_err
from oracle import port

pytestmark = pytest.mark.gpu

FIELDS = ("U", "V", "P", "MASS_FLUX", "K", "OMEGA", "MUT")


class _env:
    def __init__(self, **values):
        self.values = values

    def __enter__(self):
        self.old = {k: os.environ.get(k) for k in self.values}
        os.environ.update({k: str(v) for k, v in self.values.items()})

    def __exit__(self, *exc):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _medium_sst(iterations, flags, precision=0):
    mesh = cb.cgrid("0012", surface_points=128, wake_points=65, normal_points=97,
                    first_layer_height=1e-5, upstream_chords=10.0, downstream_chords=15.0,
                    vertical_chords=10.0)
    with _env(CFD_KERNEL_FLAGS=flags):
        s = cb.SimpleSolver.create(mesh, cb.freestream_conditions(mesh, 1.0, 4.0),
                                   cb.Settings.defaults(inflow_viscosity_ratio=10.0, precision=precision))
        s.set_turbulence_model(cb.MODEL_SST)
        s.initialise(*cb.uniform_field(mesh, 1.0, 4.0, 1.0, 1e6))
        _, hist = s.iterate(iterations, history=True)
    return {f: s.read(f) for f in FIELDS}, hist


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("flags", [32, 4])
def test_chained_sweeps_are_bit_identical_to_the_other_forms(flags, precision):
    # 384 x 96 cells: a 16-CTA cluster, so the k/omega sweeps run chained
    # over six CTAs by default, pipelined with a cluster barrier per row with
    # flag bit 5 and row after row on two CTAs with flag bit 2 (in the mixed
    # form the same three, on the FP32 corrections).
    a, ha = _medium_sst(6, 0, precision)
    b, hb = _medium_sst(6, flags, precision)
    assert np.array_equal(ha, hb)
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f


def test_a_chain_wait_that_gives_up_is_reported_and_the_device_stays_usable():
    # flag bit 6 makes the second chained k/omega stage also wait for a count
    # that nothing sets: that wait gives up after its poll limit, the launch
    # finishes, and the host reads the fault word as an error.
    with pytest.raises(cb.CfdError) as err:
        _medium_sst(1, 64)
    assert err.value.code == 8  # CFD_INTERNAL
    assert "k/omega sweep stage" in str(err.value)
    a, ha = _medium_sst(2, 0)
    b, hb = _medium_sst(2, 32)
    assert np.all(np.isfinite(ha)) and np.array_equal(ha, hb)


def test_a_halo_wait_that_gives_up_is_reported_and_the_device_stays_usable():
    # flag bit 8 makes the two-pass pressure CG's first iteration also wait
    # for a count that nothing sets: that wait gives up after its poll limit,
    # the halo rows still arrive, the launch finishes, and the host reads the
    # fault word as an error.
    with pytest.raises(cb.CfdError) as err:
        _medium_sst(1, 256)
    assert err.value.code == 8  # CFD_INTERNAL
    assert "halo row" in str(err.value)
    a, ha = _medium_sst(2, 0)
    assert np.all(np.isfinite(ha))


def test_shared_and_global_memory_cg_are_bit_identical():
    # 384 x 96 on 16 CTAs: the pressure CG runs from global memory in two
    # passes by default and keeps its band in shared memory with flag bit 7;
    # one algorithm, the same arithmetic and reduction order
    a, ha = _medium_sst(6, 0)
    b, hb = _medium_sst(6, 128)
    assert np.array_equal(ha, hb)
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f


def test_single_reduction_cg_tracks_the_two_reduction_form():
    # flag bit 3: the reference's two-reduction PCG; the single-reduction
    # rearrangement computes the same iterates, up to rounding
    a, ha = _medium_sst(1, 0)
    b, hb = _medium_sst(1, 8)
    assert np.max(np.abs(ha[:, 5] - hb[:, 5])) <= 1
    for f in FIELDS:
        assert rel_err(a[f], b[f]) < 1e-9, f


@pytest.mark.parametrize("name", ["sst_cgrid", "sst_cambered"])
@pytest.mark.parametrize("ctas", [6, 8])
def test_wide_cluster_tracks_the_oracle(name, ctas):
    c = Case(name)
    o = c.oracle(port.DEVICE_ORDER)
    mo = o.iterate(20)
    with _env(CFD_CLUSTER_SIZE=ctas):
        d = c.device()
    _, hist = d.iterate(20, history=True)
    assert np.max(np.abs(hist[:, 5] - mo[:, 5])) <= 1
    for field, fid in (("U", 0), ("V", 1), ("P", 2), ("K", 22), ("OMEGA", 23), ("MUT", 24)):
        assert rel_err(d.read(field), o.read(fid)) < 1e-7, field


def test_graph_replayed_launches_equal_direct_launches():
    c = Case("sst_cgrid")
    a, b = c.device(), c.device()
    ba, bb = cb.Batch([a]), cb.Batch([b])
    for _ in range(12):
        ba.launch(1)
        bb.graph_launch(1)
    ba.monitors()
    bb.monitors()
    for f in FIELDS:
        assert np.array_equal(a.read(f), b.read(f)), f
    ba.close()
    bb.close()


def _sst_on(ctas, alpha):
    mesh = cb.cgrid("0012", surface_points=64, wake_points=33, normal_points=49,
                    first_layer_height=1e-5, upstream_chords=10.0, downstream_chords=15.0,
                    vertical_chords=10.0)
    with _env(CFD_CLUSTER_SIZE=ctas):
        s = cb.SimpleSolver.create(mesh, cb.freestream_conditions(mesh, 1.0, alpha),
                                   cb.Settings.defaults(inflow_viscosity_ratio=10.0))
    s.set_turbulence_model(cb.MODEL_SST)
    s.initialise(*cb.uniform_field(mesh, 1.0, alpha, 1.0, 1e6))
    return s


@pytest.mark.parametrize("graph", [False, True])
def test_a_batch_of_mixed_cluster_sizes_equals_each_solve_alone(graph):
    # Solves created with different cluster sizes run as one launch per size,
    # side by side on forked streams; each gives the bits it gives alone with
    # its own size, directly or replayed from a captured graph.
    shapes = [(16, 0.0), (8, 2.0), (4, 4.0), (8, 6.0), (16, 8.0)]
    together = [_sst_on(r, a) for r, a in shapes]
    batch = cb.Batch(together)
    assert batch.shape()[0] in (8, 16)
    for _ in range(6):
        if graph:
            batch.graph_launch(1)
        else:
            batch.launch(1)
    batch.monitors()
    batch.close()
    for (r, a), s in zip(shapes, together):
        alone = _sst_on(r, a)
        solo = cb.Batch([alone])
        for _ in range(6):
            solo.launch(1)
        solo.monitors()
        solo.close()
        for f in FIELDS:
            assert np.array_equal(s.read(f), alone.read(f)), (r, a, f)
        alone.close()
        s.close()
