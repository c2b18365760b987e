"""Streamlines on the device (cfd_gpu_streamlines) against the reference's own
tracer, post::traceStreamlines (Streamlines.cpp:80-197), on the reference's
fields (golden vectors from tests/golden/make_streamlines_golden.py): the same
seeds kept and dropped, the same number of points per curve, and the points
to 1e-9 (in chords; the speed's hypot is the only operation that may round
differently on the device)."""
import numpy as np
import pytest

import cfd_b200 as cb
from helpers import golden

pytestmark = pytest.mark.gpu

G = golden("streamlines")
OPTIONS = {"default": dict(), "short": dict(max_steps=150, step_fraction=0.6, trace_backwards=False)}


def _solver(name):
    sp, wp, npn, fl, alpha = G[f"{name}/grid"]
    mesh = cb.cgrid("0012", surface_points=int(sp), wake_points=int(wp), normal_points=int(npn),
                    first_layer_height=float(fl), upstream_chords=10.0, downstream_chords=15.0,
                    vertical_chords=10.0)
    s = cb.SimpleSolver.create(mesh, cb.freestream_conditions(mesh, 1.0, float(alpha)), cb.Settings.defaults())
    s.initialise(*cb.uniform_field(mesh, 1.0, float(alpha), 1.0, 500.0))
    s.load_state(u=G[f"{name}/u"], v=G[f"{name}/v"])
    return s


@pytest.mark.parametrize("option", list(OPTIONS))
@pytest.mark.parametrize("name", ["small", "c1"])
def test_streamlines_match_the_reference(name, option):
    s = _solver(name)
    lengths, pts = s.streamlines(G["seeds"], **OPTIONS[option])
    want = G[f"{name}/{option}/lengths"]
    assert np.array_equal(lengths, want), (lengths.tolist(), want.tolist())
    ref = G[f"{name}/{option}/points"]
    assert pts.shape == ref.shape
    assert np.max(np.abs(pts - ref)) < 1e-9, float(np.max(np.abs(pts - ref)))


def test_streamline_settings_are_validated():
    s = _solver("small")
    with pytest.raises(cb.CfdError):
        s.streamlines(G["seeds"], max_steps=0)
    lengths, pts = s.streamlines(np.zeros((0, 2)))
    assert lengths.size == 0 and pts.size == 0
