"""voxphoton_b200: B200-native piecewise-constant JVIE-II frequency solve.

Hot path (hand-written sm_100a CUDA in libvox.so, C-ABI in include/vox.h):
FFT-circulant matvec, level-1 circulant preconditioner and device GMRES with
an FP32 + FP64-refinement solver.  See voxphoton_b200.vie for the
MATLAB-facing calls (mv_AN_const, chan_mvp_idx, pgmres), voxphoton_b200.solvers
for pgmresDR / bicgstab and voxphoton_b200.mor for the reduced-order sweep.
"""
from .vie import (E_field_Nop_const, JVIE_Solver_const, Lane, Operator, Preconditioner, assemble_toeplitz, chan_mvp_idx,
                  face3_from_Mr, jvie_rhs, mv_AN_const, mv_L_const, pgmres, singular_integrals,
                  solve_refined, solve_refined_batch, transmitted_power)
from .solvers import bicgstab, pgmresDR
from .mor import ReducedModel

__all__ = ["E_field_Nop_const", "JVIE_Solver_const", "Lane", "transmitted_power", "Operator", "Preconditioner", "assemble_toeplitz", "chan_mvp_idx", "face3_from_Mr",
           "jvie_rhs", "mv_AN_const", "mv_L_const", "pgmres", "singular_integrals",
           "solve_refined", "solve_refined_batch", "pgmresDR", "bicgstab", "ReducedModel"]
