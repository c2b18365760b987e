"""Algorithmic HBM bytes of one SIMPLE outer iteration, per cell.

    B = s * (A_outer + 12 * n_cg)

A_outer counts the array accesses (reads + writes) per cell of everything
outside the pressure CG, n_cg the CG iterations actually executed, 12 the
accesses per cell of one CG iteration (3 matrix + d + 2 Ad + 2 x + 2 r + 2 d),
s the stored width in bytes (8 in the plain FP64 form).

A_outer, laminar = 108:
    gradients 9 (read u, v, p; write 3 Vec2), momentum assembly shared by u
    and v 18, residual + 3 Gauss-Seidel sweeps for u and v 42, Rhie-Chow 8,
    pressure-correction assembly 7, correction 12, divergence 2, and geometry
    read by five stages, 2 accesses each, 10.
A_outer, SST = 218 = 108 + 110:
    strain 5, grad k and grad omega 6, blending / cross-diffusion / production
    12, k and omega assembly 2 x 9, residual + 3 sweeps per equation 2 x 30,
    wall omega and mu_t 7, effective viscosity 2.

Counting by what an ideal kernel must move, not what the implementation
moves: the measured DRAM traffic (ncu) sits beside this in the profiles.
"""

A_OUTER_LAMINAR = 108
A_OUTER_SST = 218
CG_ACCESSES = 12


def bytes_per_cell_iteration(sst: bool, mean_cg_iterations: float, width: int = 8) -> float:
    a_outer = A_OUTER_SST if sst else A_OUTER_LAMINAR
    return float(width) * (a_outer + CG_ACCESSES * mean_cg_iterations)


# The mixed FP32/FP64 form: the outer stages as above (assembly and state in
# FP64, 8 B), plus per inner (multigrid-CG) iteration, in FP32 (4 B):
#   flexible CG 20 accesses per cell: A d' (z and d, five coefficients,
#   write d and q: 9), the update (e, d, r, q, 1/D; write e, r, z: 8), the
#   dot products (r, z, z_old: 3);
#   one V-cycle 40 per fine cell: on the fine level a black half sweep
#   before (5.5: six row values and four neighbours per black cell, write),
#   the residual restriction (11.5), the black half sweep after with the
#   coarse correction (7.5) and the last red one (5.5), 30 together, and a
#   third of that again for all coarser levels;
# and per outer iteration 12 FP64 accesses for the refinement (x += e;
# r = b - A x) and 9 for the FP32 copy of the pressure-correction rows.
MG_CG_ACCESSES = 20
MG_VCYCLE_ACCESSES = 40
MG_OUTER_FP64 = 12 + 9


def bytes_per_cell_iteration_mixed(sst: bool, mean_inner_iterations: float) -> float:
    a_outer = A_OUTER_SST if sst else A_OUTER_LAMINAR
    return 8.0 * (a_outer + MG_OUTER_FP64) + 4.0 * (MG_CG_ACCESSES + MG_VCYCLE_ACCESSES) * mean_inner_iterations
