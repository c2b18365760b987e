"""The device CG primitive (cfd_cg_solve) against the CPU oracle's
conjugateGradient on the reference's own pressure-correction system (golden
vectors), through the C ABI with device buffers."""
import numpy as np
import pytest

import cfd_b200 as cb
from helpers import golden, golden_mesh, rel_err
from oracle import port

pytestmark = pytest.mark.gpu


def _device(a, dtype):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _system(g, mesh):
    import torch
    across = np.full(mesh.cells_i, -1, np.int32)
    for i in range(mesh.cells_i):
        if mesh.boundary[i] == cb.FACE_WAKECUT and mesh.partner[i] >= 0:
            across[i] = mesh.owner[mesh.partner[i]]
    bufs = dict(diag=_device(g["diag"], torch.float64), upper=_device(g["upper"], torch.float64),
                source=_device(g["source"], torch.float64), across=_device(across, torch.int32))
    sys_ = cb.CgSystem(mesh.cells_i, mesh.cells_j, bufs["diag"].data_ptr(), bufs["upper"].data_ptr(),
                       bufs["source"].data_ptr(), bufs["across"].data_ptr())
    return sys_, bufs


@pytest.mark.parametrize("tol,cap", [(0.01, 200), (1e-12, 2000)])
def test_device_cg_matches_the_reference_solve(tol, cap):
    import torch
    g = golden("linalg")
    mesh = golden_mesh("laminar_cgrid")
    sys_, bufs = _system(g, mesh)
    x = torch.zeros(mesh.cells, dtype=torch.float64, device="cuda")
    report = cb.cg_solve(sys_, x.data_ptr(), tol, cap)
    torch.cuda.synchronize()
    ref_x = g["cg"] if tol == 0.01 else g["cg_tight"]
    ref_rep = g["cg_report"] if tol == 0.01 else g["cg_tight_report"]
    assert abs(report[0] - ref_rep[0]) <= 1, (report, ref_rep)
    assert report[3] == ref_rep[3]
    assert report[1] == pytest.approx(ref_rep[1], rel=1e-13)
    assert rel_err(x.cpu().numpy(), ref_x) < 1e-9


def test_device_cg_with_a_start_vector_and_no_wake_map():
    """x0 != 0 and across_j0 = NULL on a box system built from the oracle."""
    import torch
    mesh = cb.box(cells_x=30, cells_y=20, grading=2, first_cell_height=0.02)
    rng = np.random.default_rng(3)
    # an SPD five-point system: -1 couplings per interior face, diag = 4.5
    upper = np.where(mesh.neighbour >= 0, -1.0, 0.0)
    diag = np.full(mesh.cells, 4.5)
    src = rng.standard_normal(mesh.cells)
    x0 = rng.standard_normal(mesh.cells)
    ref_x, ref_rep = port.ldu_cg(mesh, diag, src, upper, upper, x0, 1e-10, 500)
    d = {k: _device(v, torch.float64) for k, v in dict(diag=diag, upper=upper, source=src).items()}
    sys_ = cb.CgSystem(mesh.cells_i, mesh.cells_j, d["diag"].data_ptr(), d["upper"].data_ptr(),
                       d["source"].data_ptr(), None)
    x = _device(x0, torch.float64)
    rep = cb.cg_solve(sys_, x.data_ptr(), 1e-10, 500)
    assert abs(rep[0] - ref_rep[0]) <= 1
    assert rel_err(x.cpu().numpy(), ref_x) < 1e-9


def test_invalid_systems_are_rejected():
    s = cb.CgSystem(0, 4, None, None, None, None)
    with pytest.raises(cb.CfdError):
        cb.cg_solve(s, 0, 0.01, 10)
