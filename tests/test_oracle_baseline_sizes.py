"""The CPU oracle and the library's mesh generator pinned to the reference at
the benchmark grid sizes (192x48 laminar, 384x96 SST, 768x192 SST), against
digests the reference produced (tests/golden/make_baseline_golden.py).

Small cases pin the restatement stage by stage (test_oracle_pinned.py); these
show that nothing size-dependent (the wake-cut map of a long wrap, the CG at
its 200-iteration cap on every iteration, the far-field dead band on a
15-chord domain) breaks the bit-for-bit agreement at the sizes the device is
benchmarked on. In the reference's lexicographic Gauss-Seidel order the
oracle must reproduce every monitor of the first 20 iterations and every bit
of the fields after iterations 1 and 20."""
import numpy as np
import pytest

from helpers import BaselineCase, digest
from oracle import port

CASES = ["c1", "c2", "c3"]
# oracle field ids (CFD_FIELD_*)
FIELDS = {"u": 0, "v": 1, "p": 2, "mu_eff": 4, "mass_flux": 5, "k": 22, "omega": 23, "mut": 24}
SYSTEM = {"p_diag": 17, "p_source": 18, "p_upper": 19}


@pytest.mark.parametrize("name", CASES)
def test_mesh_conditions_and_start_match_the_reference(name):
    c = BaselineCase(name)
    g = c.g
    assert c.mesh.cells == int(g["cells"])
    for key in ("nodes", "centroid", "cell_area", "face_centre", "face_normal", "face_area",
                "owner", "neighbour", "boundary", "partner"):
        assert digest(getattr(c.mesh, key)) == str(g[f"mesh_digest/{key}"]), key
    cond = c.conditions
    for key, a in (("kind", cond.kind), ("bc_velocity", cond.velocity),
                   ("bc_pressure", cond.pressure)):
        assert digest(a) == str(g[f"conditions_digest/{key}"]), key
    for key, a in zip(("u", "v", "p", "rho", "mu"), c.initial):
        assert digest(a) == str(g[f"uniform_digest/{key}"]), key


@pytest.mark.parametrize("name", CASES)
def test_twenty_iterations_match_the_reference_bitwise(name):
    c = BaselineCase(name)
    g = c.g
    s = c.oracle(port.LEXICOGRAPHIC)
    mon = [s.iterate(1)]
    for key, fid in SYSTEM.items():
        assert digest(s.read(fid)) == str(g[f"iter1_digest/{key}"]), key
    keys = [k for k in FIELDS if c.model == 2 or k not in ("k", "omega", "mut")]
    for key in keys:
        assert digest(s.read(FIELDS[key])) == str(g[f"iter1_digest/{key}"]), key
    mon.append(s.iterate(19))
    mon = np.concatenate(mon)
    ref = g["history20"]
    assert np.array_equal(mon[:, :15], ref), float(np.max(np.abs(mon[:, :15] - ref)))
    assert np.all(ref[:, 5] > 0)  # every iteration ran a pressure solve
    for key in keys:
        a = s.read(FIELDS[key])
        if key != "mass_flux":  # per-cell fields also carry sampled values
            assert np.array_equal(a[g["sample_cells"]], g[f"iter20_sample/{key}"]), key
        assert digest(a) == str(g[f"iter20_digest/{key}"]), key
