"""cfd_cg_solve_noalloc: the pressure CG for callers that cannot allocate
device memory (a host application whose memory manager owns the whole GPU,
or a loop that must not block on cudaFree's synchronisation). It uses a fixed
scratch array inside the library instead of cudaMalloc. Checked through the
C ABI against cfd_cg_solve on the same systems, two calls in a row, so that
the second call also shows that what the first left in the shared array does
not leak into its result; against the reference's own CG answer on its first
pressure-correction system; and at the scratch's limit of 65,536 mesh nodes.
Collected last on purpose."""
import numpy as np
import pytest

import cfd_b200 as cb
from helpers import golden, golden_mesh, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-9  # the CG tolerance the other device tests use


def _dev(a, dtype=None):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype or torch.float64, device="cuda")


def _box_system(cells_i, cells_j, across=None, seed=11):
    """A symmetric, diagonally dominant five-point system on a cells_i x cells_j
    block in the reference's LDU layout (j-faces, then i-faces), optionally
    coupled across the j = 0 faces by `across` (a symmetric pairing)."""
    import torch
    rng = np.random.default_rng(seed)
    ni, nj = cells_i, cells_j
    j_faces = ni * (nj + 1)
    faces = j_faces + (ni + 1) * nj
    upper = np.zeros(faces)
    diag = np.full(ni * nj, 0.5)
    # interior j-faces (between rows j-1 and j) and i-faces (between columns)
    for j in range(1, nj):
        c = -1.0 - rng.random(ni)
        upper[j * ni:(j + 1) * ni] = c
        diag[(j - 1) * ni:j * ni] -= c
        diag[j * ni:(j + 1) * ni] -= c
    for i in range(1, ni):
        c = -1.0 - rng.random(nj)
        upper[j_faces + i * nj:j_faces + (i + 1) * nj] = c
        diag[np.arange(nj) * ni + i - 1] -= c
        diag[np.arange(nj) * ni + i] -= c
    if across is not None:
        for i in range(ni):
            a = across[i]
            if a > i:  # one coefficient per pair, on both j = 0 faces
                c = -1.0 - rng.random()
                upper[i] = upper[a] = c
                diag[i] -= c
                diag[a] -= c
    keep = dict(diag=_dev(diag), upper=_dev(upper), source=_dev(rng.standard_normal(ni * nj)))
    if across is not None:
        keep["across"] = _dev(np.asarray(across, np.int32), torch.int32)
    system = cb.CgSystem(ni, nj, keep["diag"].data_ptr(), keep["upper"].data_ptr(),
                         keep["source"].data_ptr(),
                         keep["across"].data_ptr() if across is not None else None)
    return system, ni * nj, keep


def _reference_system():
    """The reference's first pressure-correction system of the laminar C-grid
    case (wake cut), as tests/golden/linalg.npz holds it."""
    import torch
    g = golden("linalg")
    mesh = golden_mesh("laminar_cgrid")
    across = np.full(mesh.cells_i, -1, np.int32)
    for i in range(mesh.cells_i):
        if mesh.boundary[i] == cb.FACE_WAKECUT and mesh.partner[i] >= 0:
            across[i] = mesh.owner[mesh.partner[i]]
    keep = dict(diag=_dev(g["diag"]), upper=_dev(g["upper"]), source=_dev(g["source"]),
                across=_dev(across, torch.int32))
    system = cb.CgSystem(mesh.cells_i, mesh.cells_j, keep["diag"].data_ptr(),
                         keep["upper"].data_ptr(), keep["source"].data_ptr(),
                         keep["across"].data_ptr())
    return system, mesh.cells, keep, g


def _compare(system, cells, tol, cap):
    import torch
    x_ref = torch.zeros(cells, dtype=torch.float64, device="cuda")
    x_new = torch.zeros(cells, dtype=torch.float64, device="cuda")
    rep_ref = cb.cg_solve(system, x_ref.data_ptr(), tol, cap)
    rep_new = cb.cg_solve_noalloc(system, x_new.data_ptr(), tol, cap)
    torch.cuda.synchronize()
    assert rep_new[0] == rep_ref[0] and rep_new[3] == rep_ref[3], (rep_new, rep_ref)
    assert rep_new[1] == pytest.approx(rep_ref[1], rel=TOL)
    assert rep_new[2] == pytest.approx(rep_ref[2], rel=TOL)
    assert rel_err(x_new.cpu().numpy(), x_ref.cpu().numpy()) <= TOL
    return x_new.cpu().numpy(), rep_new


def test_noalloc_matches_the_allocating_solve_twice_in_a_row():
    s1, n1, k1, g = _reference_system()
    box = cb.box(cells_x=40, cells_y=24, grading=2, first_cell_height=0.02)
    s2, n2, k2 = _box_system(box.cells_i, box.cells_j)
    # call 1, then call 2 (other sizes, no wake map) on the shared scratch
    x1, rep1 = _compare(s1, n1, 0.01, 200)
    _compare(s2, n2, 1e-10, 600)
    # and the reference's own answer to system 1 (conjugateGradient at
    # tolerance 0.01, cap 200; dot products summed in another order)
    assert rep1[0] == pytest.approx(g["cg_report"][0], abs=1)
    assert rel_err(x1, g["cg"]) <= TOL
    del k1, k2


@pytest.mark.parametrize("shape", [(255, 255), (32767, 1)])
def test_noalloc_at_the_scratch_limit(shape):
    """Blocks of exactly 65,536 nodes: 255 x 255 runs on a 16-CTA cluster;
    32767 x 1 has the widest wake map the scratch holds, every j = 0 face
    paired across the block (i <-> cells_i - 1 - i, the middle cell alone)."""
    ni, nj = shape
    assert (ni + 1) * (nj + 1) == 65536
    across = None
    if nj == 1:
        across = [ni - 1 - i if ni - 1 - i != i else -1 for i in range(ni)]
    system, cells, keep = _box_system(ni, nj, across, seed=ni)
    _compare(system, cells, 1e-8, 400)
    del keep


def test_noalloc_allocates_nothing_on_a_warm_call():
    import torch
    system, cells, keep = _box_system(120, 80, seed=3)
    x = torch.zeros(cells, dtype=torch.float64, device="cuda")
    cb.cg_solve_noalloc(system, x.data_ptr(), 1e-8, 300)  # resolves the scratch address
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    x.zero_()
    cb.cg_solve_noalloc(system, x.data_ptr(), 1e-8, 300)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    del keep


def test_noalloc_refuses_blocks_beyond_its_scratch():
    s = cb.CgSystem(400, 200, 1, 1, 1, None)  # 401 * 201 nodes > 65,536; never launched
    with pytest.raises(cb.CfdError) as err:
        cb.cg_solve_noalloc(s, 1, 0.01, 10)
    assert err.value.code == 2 and "65536" in str(err.value)


@pytest.mark.parametrize("solve", ["cg_solve", "cg_solve_noalloc"])
def test_a_wake_map_outside_the_block_is_refused(solve):
    """An across_j0 entry that names no cell of the block is an invalid
    argument; the solve does not run and x keeps its values."""
    import torch
    ni, nj = 16, 6
    across = [ni - 1 - i for i in range(ni)]
    system, cells, keep = _box_system(ni, nj, across, seed=5)
    bad = keep["across"].clone()
    bad[3] = cells  # one past the last cell
    system.across_j0 = bad.data_ptr()
    x = torch.full((cells,), 7.0, dtype=torch.float64, device="cuda")
    with pytest.raises(cb.CfdError) as err:
        getattr(cb, solve)(system, x.data_ptr(), 1e-8, 50)
    assert err.value.code == 1 and "across_j0" in str(err.value)
    assert torch.all(x == 7.0)
    del keep, bad
