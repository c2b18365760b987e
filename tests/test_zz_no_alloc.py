"""cfd_cg_solve_noalloc: the pressure CG for callers that cannot allocate
device memory (a host application whose memory manager owns the whole GPU,
or a loop that must not block on cudaFree's synchronisation). It uses a fixed
scratch array inside the library instead of cudaMalloc. Checked through the
C ABI against cfd_cg_solve on the same systems, two calls in a row, so that
the second call also shows that what the first left in the shared array does
not leak into its result. Collected last on purpose."""
import numpy as np
import pytest

import cfd_b200 as cb
from helpers import golden, golden_mesh, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-9  # the CG tolerance the other device tests use


def _systems():
    import torch
    g = golden("linalg")
    mesh = golden_mesh("laminar_cgrid")
    across = np.full(mesh.cells_i, -1, np.int32)
    for i in range(mesh.cells_i):
        if mesh.boundary[i] == cb.FACE_WAKECUT and mesh.partner[i] >= 0:
            across[i] = mesh.owner[mesh.partner[i]]
    dev = lambda a, t=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=t, device="cuda")  # noqa: E731
    keep = []
    # system 1: the reference's first pressure-correction system (wake cut)
    d1 = dict(diag=dev(g["diag"]), upper=dev(g["upper"]), source=dev(g["source"]),
              across=dev(across, torch.int32))
    keep.append(d1)
    s1 = cb.CgSystem(mesh.cells_i, mesh.cells_j, d1["diag"].data_ptr(), d1["upper"].data_ptr(),
                     d1["source"].data_ptr(), d1["across"].data_ptr())
    # system 2: a different block (no wake map) so the second call sees other sizes
    box = cb.box(cells_x=40, cells_y=24, grading=2, first_cell_height=0.02)
    rng = np.random.default_rng(11)
    upper = np.where(box.neighbour >= 0, -1.0 - rng.random(box.faces), 0.0)
    diag = np.zeros(box.cells)
    np.add.at(diag, box.owner, -upper)
    np.add.at(diag, box.neighbour[box.neighbour >= 0], -upper[box.neighbour >= 0])
    diag += 0.5
    d2 = dict(diag=dev(diag), upper=dev(upper), source=dev(rng.standard_normal(box.cells)))
    keep.append(d2)
    s2 = cb.CgSystem(box.cells_i, box.cells_j, d2["diag"].data_ptr(), d2["upper"].data_ptr(),
                     d2["source"].data_ptr(), None)
    return [(s1, mesh.cells, 0.01, 200), (s2, box.cells, 1e-10, 600)], keep


def test_noalloc_matches_the_allocating_solve_twice_in_a_row():
    import torch
    cases, keep = _systems()
    for system, cells, tol, cap in cases:  # call 1 then call 2 on the shared scratch
        x_ref = torch.zeros(cells, dtype=torch.float64, device="cuda")
        x_new = torch.zeros(cells, dtype=torch.float64, device="cuda")
        rep_ref = cb.cg_solve(system, x_ref.data_ptr(), tol, cap)
        rep_new = cb.cg_solve_noalloc(system, x_new.data_ptr(), tol, cap)
        torch.cuda.synchronize()
        assert rep_new[0] == rep_ref[0] and rep_new[3] == rep_ref[3], (rep_new, rep_ref)
        assert rep_new[1] == pytest.approx(rep_ref[1], rel=TOL)
        assert rep_new[2] == pytest.approx(rep_ref[2], rel=TOL)
        assert rel_err(x_new.cpu().numpy(), x_ref.cpu().numpy()) <= TOL
    del keep


def test_noalloc_refuses_blocks_beyond_its_scratch():
    s = cb.CgSystem(400, 200, 1, 1, 1, None)  # 401 * 201 nodes > 65,536; never launched
    with pytest.raises(cb.CfdError) as err:
        cb.cg_solve_noalloc(s, 1, 0.01, 10)
    assert err.value.code == 2 and "65536" in str(err.value)
