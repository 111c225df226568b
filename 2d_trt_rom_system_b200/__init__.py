"""B200-native SCB transport sweep and QD-factor moments for the 2D TRT solver of
jmc9/2D_TRT_ROM_System (drop-in for MODULE TRANSPORT_SOLVES and the QD-factor routines).

The compute path is libtrt_sweep.so (CUDA, sm_100a) behind the C ABI of include/trt_sweep.h; this
package is its Python mirror plus the problem and quadrature generators used by tests and the bench.
"""
from . import problems, quadrature, ranks, serving, sharded  # noqa: F401
from .api import (COLLAPSE_INTENSITIES, COLLAPSE_MG_EF, DMD_Calc, DMD_RECONSTRUCT, EGP_FV_NEWT, FMAP,  # noqa: F401
                  GENERATE_GRIDS_T, GENERATE_GRIDS_XY, GRIDMAP_GEN, GRIDMAP_GEN_BND, MAP_GRIDS, GQD_In_Calc, GREY_COEFS,
                  DMD_RECONSTRUCT_BCg, DMD_RECONSTRUCT_fg, POD_RECONSTRUCT_BCg, POD_RECONSTRUCT_fg, POD_TRUNCATE, RRANK_CALC,
                  MGQD_In_Calc, MLOQD_FV, OLD_GREY_COEFS, OLD_MGQD_COEFS, POD_RECONSTRUCT, POD_Calc, RT_BC_UPDATE,
                  LINEAR_INTERPOLATION, TRANSPORT_SCB, Batch,
                  Bg_planck_calc, Cbar_Calc, Cg_Calc, TransportSweep, fg_Calc, kernel_launches, mgqd_last_stats,
                  mgqd_set_fused_levels, mgqd_set_graphs, mgqd_set_smem_vcycle, mgqd_set_tolerance,
                  required_bytes)
from ._lib import LIB_PATH, TrtError, check, lib  # noqa: F401
