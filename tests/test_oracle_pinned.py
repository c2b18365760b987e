"""The CPU oracle (oracle/cfd_oracle.c) pinned against the reference's own
outputs: golden vectors produced by the reference solver
(tests/golden/make_golden.py). In lexicographic Gauss-Seidel order the
restatement must reproduce the reference to the last bit."""
import numpy as np
import pytest

from helpers import Case, golden, golden_mesh
from oracle import port

CASES = ["laminar_cgrid", "sst_cgrid", "sst_cambered"]

# oracle field ids (CFD_FIELD_*)
U, V, P, MU_EFF, MF = 0, 1, 2, 4, 5
GRAD_U, GRAD_V, GRAD_P = 8, 9, 10
MOM_DIAG, SRC_U, SRC_V, UPPER, LOWER = 11, 12, 13, 14, 15
P_DIAG, P_SOURCE, P_UPPER, NET = 17, 18, 19, 20
K, OMEGA, MUT, WALL, STRAIN, F1, F2, CD, PROD, GRAD_K, GRAD_OMEGA = range(22, 33)


@pytest.mark.parametrize("name", CASES)
def test_initialise_matches_reference(name):
    c = Case(name)
    s = c.oracle(port.LEXICOGRAPHIC)
    g = c.g
    assert np.array_equal(s.read(MF), g["init/mass_flux"])
    assert np.array_equal(s.read(MU_EFF), g["init/mu_eff"])
    assert s.scalars()[2] == g["init/reference_mass_flow"]
    if c.model == 2:
        assert np.array_equal(s.read(WALL), g["init/wall_distance"])
        assert np.array_equal(s.read(K), g["init/k"])
        assert np.array_equal(s.read(OMEGA), g["init/omega"])
        assert np.array_equal(s.read(MUT), g["init/mut"])
        assert np.array_equal(s.scalars()[:2], g["init/sst_scalars"])


@pytest.mark.parametrize("name", CASES)
def test_first_iteration_stages_match_reference(name):
    c = Case(name)
    g = c.g
    s = c.oracle(port.LEXICOGRAPHIC)
    s.iterate(1, stop_stage=0)
    for fid, key in ((GRAD_U, "grad_u"), (GRAD_V, "grad_v"), (GRAD_P, "grad_p")):
        assert np.array_equal(s.read(fid), g[f"stage1/{key}"]), key
    s = c.oracle(port.LEXICOGRAPHIC)
    s.iterate(1, stop_stage=1)
    for fid, key in ((MOM_DIAG, "mom_diag"), (SRC_U, "mom_source_u"), (SRC_V, "mom_source_v"),
                     (UPPER, "mom_upper"), (LOWER, "mom_lower")):
        assert np.array_equal(s.read(fid), g[f"stage1/{key}"]), key


@pytest.mark.parametrize("name", CASES)
def test_iterations_match_reference_bitwise(name):
    c = Case(name)
    g = c.g
    s = c.oracle(port.LEXICOGRAPHIC)
    mon1 = s.iterate(1)
    for fid, key in ((P_DIAG, "p_diag"), (P_SOURCE, "p_source"), (P_UPPER, "p_upper"),
                     (NET, "net_flux")):
        assert np.array_equal(s.read(fid), g[f"iter1/{key}"]), key
    keys = [(U, "u"), (V, "v"), (P, "p"), (MF, "mass_flux"), (MU_EFF, "mu_eff")]
    if c.model == 2:
        keys += [(K, "k"), (OMEGA, "omega"), (MUT, "mut"), (STRAIN, "strain"), (F1, "f1"),
                 (F2, "f2"), (CD, "cross_diffusion"), (PROD, "production"), (GRAD_K, "grad_k"),
                 (GRAD_OMEGA, "grad_omega")]
    for fid, key in keys:
        assert np.array_equal(s.read(fid), g[f"iter1/{key}"]), key
    mon = np.concatenate([mon1, s.iterate(4)])
    # monitor: the reference's 15 values (no y+); identical bits
    assert np.array_equal(mon[:, :15], g["history5"]), np.max(np.abs(mon[:, :15] - g["history5"]))
    for fid, key in keys[:8 if c.model == 2 else 5]:
        assert np.array_equal(s.read(fid), g[f"iter5/{key}"]), key


def test_converged_laminar_matches_reference():
    """Run the oracle to the same stop rule; the converged fields agree to the
    bit while the iteration paths are the reference's own."""
    c = Case("laminar_cgrid")
    g = c.g
    s = c.oracle(port.LEXICOGRAPHIC)
    n = int(g["converged/iterations"])
    mon = s.iterate(n)
    assert np.array_equal(mon[-1, :15], g["converged/monitor"])
    for fid, key in ((U, "u"), (V, "v"), (P, "p"), (MF, "mass_flux")):
        assert np.array_equal(s.read(fid), g[f"converged/{key}"]), key


def test_red_black_converges_to_the_reference_answer():
    """For the momentum equations Gauss-Seidel order changes the path, not the
    fixed point: the red-black oracle run to convergence lands on the
    reference's converged fields."""
    c = Case("laminar_cgrid")
    g = c.g
    s = c.oracle(port.DEVICE_ORDER)
    mon = s.iterate(int(g["converged/iterations"]))
    worst = np.max(np.abs(mon[:, :3]), axis=1)
    assert worst[-1] < 1e-12
    for fid, key in ((U, "u"), (V, "v"), (P, "p")):
        ref = g[f"converged/{key}"]
        err = np.linalg.norm(s.read(fid) - ref) / np.linalg.norm(ref)
        assert err < 1e-9, (key, err)


def test_linear_algebra_primitives_match_reference():
    g = golden("linalg")
    mesh = golden_mesh("laminar_cgrid")
    assert np.array_equal(port.ldu_multiply(mesh, g["diag"], g["upper"], g["lower"], g["x"]), g["spmv"])
    gs = port.ldu_gauss_seidel(mesh, g["gs_diag"], g["source"], g["gs_upper"], g["gs_lower"], g["x"],
                               3, port.LEXICOGRAPHIC)
    assert np.array_equal(gs, g["gs"])
    x, rep = port.ldu_cg(mesh, g["diag"], g["source"], g["upper"], g["lower"], np.zeros(mesh.cells),
                         0.01, 200)
    assert np.array_equal(x, g["cg"])
    assert np.array_equal(rep, g["cg_report"])
    x, rep = port.ldu_cg(mesh, g["diag"], g["source"], g["upper"], g["lower"], np.zeros(mesh.cells),
                         1e-12, 2000)
    assert np.array_equal(x, g["cg_tight"]) and np.array_equal(rep, g["cg_tight_report"])
    assert np.array_equal(port.green_gauss(mesh, g["face_values"]), g["green_gauss"])


def test_cg_recovers_a_known_solution():
    """LinearSystem CG recovers a known solution to 1e-8 (SolverTests.cpp:365-385)."""
    g = golden("linalg")
    mesh = golden_mesh("laminar_cgrid")
    rng = np.random.default_rng(7)
    truth = rng.standard_normal(mesh.cells)
    # symmetrise the wake pairs' rounding so CG sees an exactly symmetric matrix
    b = port.ldu_multiply(mesh, g["diag"], g["upper"], g["lower"], truth)
    x, rep = port.ldu_cg(mesh, g["diag"], b, g["upper"], g["lower"], np.zeros(mesh.cells), 1e-14, 5000)
    assert np.max(np.abs(x - truth)) < 1e-8 * np.max(np.abs(truth))


@pytest.mark.parametrize("name", ["sst_cgrid", "sst_cambered"])
def test_sst_fixed_point_needs_the_reference_sweep_order(name):
    """The k and omega floors and the wall-cell omega override act after the
    sweeps, so their order moves the converged state. Momentum red-black with
    k and omega in cell order (the device's choice) converges onto the
    reference; red-black everywhere does not."""
    c = Case(name)
    g = c.g
    n = int(g["converged/iterations"])
    s = c.oracle(port.DEVICE_ORDER)
    s.iterate(n)
    for fid, key in ((U, "u"), (V, "v"), (P, "p"), (K, "k"), (OMEGA, "omega"), (MUT, "mut")):
        err = np.linalg.norm(s.read(fid) - g[f"converged/{key}"]) / np.linalg.norm(g[f"converged/{key}"])
        assert err < 1e-9, (key, err)
    s = c.oracle(port.RED_BLACK_ALL)
    s.iterate(n)
    ref = g["converged/k"]
    assert np.linalg.norm(s.read(K) - ref) / np.linalg.norm(ref) > 1e-6
