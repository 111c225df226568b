"""Python mirror of the reference interface for the sweep path, over the C ABI (include/trt_sweep.h).

Reference-signature functions take numpy arrays in the reference's Fortran layouts (shape (nx, ny, ...)
with order='F'), in the argument order of the Fortran subroutine they replace; INTENT(OUT) arrays are
passed in and filled, as in Fortran.  ``TransportSweep`` wraps the resident-state handle.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, dptr, iptr


def _f64(a, shape=None):
    a = np.asarray(a, dtype=np.float64)
    if shape is not None and a.shape != tuple(shape):
        raise ValueError(f"expected shape {tuple(shape)}, got {a.shape}")
    return np.asfortranarray(a)


def _out(a, shape):
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.f_contiguous and a.shape == tuple(shape)):
        raise ValueError(f"output must be a Fortran-ordered float64 array of shape {tuple(shape)}")
    return a


# --------------------------------------------------------------------------------------------
# Reference-signature entry points
# --------------------------------------------------------------------------------------------
def TRANSPORT_SCB(I_avg, I_edgV, I_edgH, I_crn, Ic_edgV, Ic_edgH, Omega_x, Omega_y, Delx, Dely, A, KapE_in, Src_in,
                  I_crn_old, c, Delt, Open_Threads, RT_Residual, RT_ResLoc_x, RT_ResLoc_y, Res_Calc):
    """SUBROUTINE TRANSPORT_SCB, MainSrc/TRANSPORT_SOLVES.f08:14-327."""
    nx, ny = len(Delx), len(Dely)
    nm, ng = I_avg.shape[2], I_avg.shape[3]
    _out(I_avg, (nx, ny, nm, ng)); _out(I_edgV, (nx + 1, ny, nm, ng)); _out(I_edgH, (nx, ny + 1, nm, ng))
    _out(I_crn, (2 * nx, 2 * ny, nm, ng)); _out(Ic_edgV, (nx + 1, 2 * ny, nm, ng)); _out(Ic_edgH, (2 * nx, ny + 1, nm, ng))
    ox, oy, dx, dy = _f64(Omega_x, (nm,)), _f64(Omega_y, (nm,)), _f64(Delx), _f64(Dely)
    A_, K, S, Io = _f64(A, (nx, ny)), _f64(KapE_in, (nx, ny, ng)), _f64(Src_in, (2 * nx, 2 * ny, nm, ng)), \
        _f64(I_crn_old, (2 * nx, 2 * ny, nm, ng))
    if Res_Calc:
        _out(RT_Residual, (4, ng, 5))
        assert RT_ResLoc_x.dtype == np.int32 and RT_ResLoc_y.dtype == np.int32
    rc = _lib.lib().trt_transport_scb(nx, ny, nm, ng, dptr(I_avg), dptr(I_edgV), dptr(I_edgH), dptr(I_crn),
                                      dptr(Ic_edgV), dptr(Ic_edgH), dptr(ox), dptr(oy), dptr(dx), dptr(dy), dptr(A_),
                                      dptr(K), dptr(S), dptr(Io), float(c), float(Delt), int(Open_Threads),
                                      dptr(RT_Residual) if Res_Calc else None,
                                      iptr(RT_ResLoc_x) if Res_Calc else None,
                                      iptr(RT_ResLoc_y) if Res_Calc else None, 1 if Res_Calc else 0)
    check(rc, "TRANSPORT_SCB")


def COLLAPSE_INTENSITIES(Open_Threads, I_avg, I_edgV, I_edgH, Omega_x, Omega_y, quad_weight, Comp_Unit, Hg_avg_xx,
                         Hg_avg_yy, Hg_avg_xy, Hg_edgV_xx, Hg_edgV_xy, Hg_edgH_yy, Hg_edgH_xy, Eg_edgV, Eg_edgH,
                         Eg_avg, Fxg_edgV, Fyg_edgH, E_edgV, E_edgH, E_avg, Fx_edgV, Fy_edgH):
    """SUBROUTINE COLLAPSE_INTENSITIES, MainSrc/TRANSPORT_SOLVES.f08:381-511."""
    nx, ny, nm, ng = I_avg.shape
    Ia, Iv, Ih = _f64(I_avg), _f64(I_edgV, (nx + 1, ny, nm, ng)), _f64(I_edgH, (nx, ny + 1, nm, ng))
    outs = [Hg_avg_xx, Hg_avg_yy, Hg_avg_xy, Hg_edgV_xx, Hg_edgV_xy, Hg_edgH_yy, Hg_edgH_xy, Eg_edgV, Eg_edgH, Eg_avg,
            Fxg_edgV, Fyg_edgH, E_edgV, E_edgH, E_avg, Fx_edgV, Fy_edgH]
    A, V, H = (nx, ny), (nx + 1, ny), (nx, ny + 1)
    shapes = [A + (ng,)] * 3 + [V + (ng,)] * 2 + [H + (ng,)] * 2 + [V + (ng,), H + (ng,), A + (ng,), V + (ng,),
                                                                   H + (ng,), V, H, A, V, H]
    for o, s in zip(outs, shapes):
        _out(o, s)
    rc = _lib.lib().trt_collapse_intensities(nx, ny, nm, ng, int(Open_Threads), dptr(Ia), dptr(Iv), dptr(Ih),
                                             dptr(_f64(Omega_x)), dptr(_f64(Omega_y)), dptr(_f64(quad_weight)),
                                             float(Comp_Unit), *[dptr(o) for o in outs])
    check(rc, "COLLAPSE_INTENSITIES")


def fg_Calc(fg_avg_xx, fg_avg_yy, fg_avg_xy, fg_edgV_xx, fg_edgV_xy, fg_edgH_yy, fg_edgH_xy, Hg_avg_xx, Hg_avg_yy,
            Hg_avg_xy, Hg_edgV_xx, Hg_edgV_xy, Hg_edgH_yy, Hg_edgH_xy, HO_Eg_avg, HO_Eg_edgV, HO_Eg_edgH, c,
            Open_Threads):
    """SUBROUTINE fg_Calc, MainSrc/MLOQD_SOLVES.f08:619-678."""
    nx, ny, ng = fg_avg_xx.shape
    outs = [fg_avg_xx, fg_avg_yy, fg_avg_xy, fg_edgV_xx, fg_edgV_xy, fg_edgH_yy, fg_edgH_xy]
    for o, s in zip(outs, [(nx, ny, ng)] * 3 + [(nx + 1, ny, ng)] * 2 + [(nx, ny + 1, ng)] * 2):
        _out(o, s)
    ins = [_f64(a) for a in (Hg_avg_xx, Hg_avg_yy, Hg_avg_xy, Hg_edgV_xx, Hg_edgV_xy, Hg_edgH_yy, Hg_edgH_xy,
                             HO_Eg_avg, HO_Eg_edgV, HO_Eg_edgH)]
    rc = _lib.lib().trt_fg_calc(nx, ny, ng, *[dptr(o) for o in outs], *[dptr(a) for a in ins], float(c),
                                int(Open_Threads))
    check(rc, "fg_Calc")


def Cg_Calc(Cg_L, Cg_B, Cg_R, Cg_T, I_edgV, I_edgH, Omega_x, Omega_y, quad_weight, Comp_Unit, BC_Type, Open_Threads):
    """SUBROUTINE Cg_Calc, MainSrc/MLOQD_SOLVES.f08:367-488."""
    ny, ng = Cg_L.shape
    nx = Cg_B.shape[0]
    nm = len(quad_weight)
    for o, s in zip((Cg_L, Cg_B, Cg_R, Cg_T), ((ny, ng), (nx, ng), (ny, ng), (nx, ng))):
        _out(o, s)
    bc = np.ascontiguousarray(BC_Type, dtype=np.int32)
    rc = _lib.lib().trt_cg_calc(nx, ny, nm, ng, dptr(Cg_L), dptr(Cg_B), dptr(Cg_R), dptr(Cg_T),
                                dptr(_f64(I_edgV, (nx + 1, ny, nm, ng))), dptr(_f64(I_edgH, (nx, ny + 1, nm, ng))),
                                dptr(_f64(Omega_x)), dptr(_f64(Omega_y)), dptr(_f64(quad_weight)), float(Comp_Unit),
                                iptr(bc), int(Open_Threads))
    check(rc, "Cg_Calc")


def MGQD_In_Calc(Eg_in_L, Eg_in_B, Eg_in_R, Eg_in_T, Fg_in_L, Fg_in_B, Fg_in_R, Fg_in_T, I_edgV, I_edgH, Omega_x,
                 Omega_y, quad_weight, c, Comp_Unit, BC_Type, Open_Threads):
    """SUBROUTINE MGQD_In_Calc, MainSrc/MLOQD_SOLVES.f08:493-614."""
    ny, ng = Eg_in_L.shape
    nx = Eg_in_B.shape[0]
    nm = len(quad_weight)
    outs = (Eg_in_L, Eg_in_B, Eg_in_R, Eg_in_T, Fg_in_L, Fg_in_B, Fg_in_R, Fg_in_T)
    for o, s in zip(outs, ((ny, ng), (nx, ng)) * 4):
        _out(o, s)
    bc = np.ascontiguousarray(BC_Type, dtype=np.int32)
    rc = _lib.lib().trt_mgqd_in_calc(nx, ny, nm, ng, *[dptr(o) for o in outs],
                                     dptr(_f64(I_edgV, (nx + 1, ny, nm, ng))), dptr(_f64(I_edgH, (nx, ny + 1, nm, ng))),
                                     dptr(_f64(Omega_x)), dptr(_f64(Omega_y)), dptr(_f64(quad_weight)), float(c),
                                     float(Comp_Unit), iptr(bc), int(Open_Threads))
    check(rc, "MGQD_In_Calc")


def GQD_In_Calc(E_in_L, E_in_B, E_in_R, E_in_T, F_in_L, F_in_B, F_in_R, F_in_T, Eg_in_L, Eg_in_B, Eg_in_R, Eg_in_T,
                Fg_in_L, Fg_in_B, Fg_in_R, Fg_in_T):
    """SUBROUTINE GQD_In_Calc, MainSrc/GLOQD_SOLVES.f08:263-290."""
    ny, ng = Eg_in_L.shape
    nx = Eg_in_B.shape[0]
    outs = (E_in_L, E_in_B, E_in_R, E_in_T, F_in_L, F_in_B, F_in_R, F_in_T)
    for o, s in zip(outs, ((ny,), (nx,)) * 4):
        _out(o, s)
    ins = [_f64(a) for a in (Eg_in_L, Eg_in_B, Eg_in_R, Eg_in_T, Fg_in_L, Fg_in_B, Fg_in_R, Fg_in_T)]
    rc = _lib.lib().trt_gqd_in_calc(nx, ny, ng, *[dptr(o) for o in outs], *[dptr(a) for a in ins])
    check(rc, "GQD_In_Calc")


def RT_BC_UPDATE(BC_Type, bcT_left, bcT_lower, bcT_right, bcT_upper, Comp_Unit, Nu_g, I_edgV, I_edgH, Ic_edgV,
                 Ic_edgH):
    """SUBROUTINE RT_BC_UPDATE, MainSrc/UPDATES.f08:12-105."""
    nx = I_edgH.shape[0]
    ny = I_edgV.shape[1]
    nm, ng = I_edgV.shape[2], I_edgV.shape[3]
    _out(I_edgV, (nx + 1, ny, nm, ng)); _out(I_edgH, (nx, ny + 1, nm, ng))
    _out(Ic_edgV, (nx + 1, 2 * ny, nm, ng)); _out(Ic_edgH, (2 * nx, ny + 1, nm, ng))
    bc = np.ascontiguousarray(BC_Type, dtype=np.int32)
    rc = _lib.lib().trt_rt_bc_update(nx, ny, nm, ng, iptr(bc), float(bcT_left), float(bcT_lower), float(bcT_right),
                                     float(bcT_upper), float(Comp_Unit), dptr(_f64(Nu_g, (ng + 1,))), dptr(I_edgV),
                                     dptr(I_edgH), dptr(Ic_edgV), dptr(Ic_edgH))
    check(rc, "RT_BC_UPDATE")


def OLD_MGQD_COEFS(Eg_avg_old, Eg_edgV_old, Eg_edgH_old, Fxg_edgV_old, Fyg_edgH_old, fg_avg_xx_old, fg_avg_yy_old,
                   fg_edgV_xx_old, fg_edgV_xy_old, fg_edgH_yy_old, fg_edgH_xy_old, KapE_old, KapR_old, Src_old, Delx,
                   Dely, A, c, Delt, Theta, G_old, Pold_L, Pold_B, Pold_R, Pold_T, Open_Threads):
    """SUBROUTINE OLD_MGQD_COEFS, MainSrc/MLOQD_SOLVES.f08:12-73."""
    nx, ny, ng = Eg_avg_old.shape
    C, V, H = (nx, ny, ng), (nx + 1, ny, ng), (nx, ny + 1, ng)
    shapes = (C, V, H, V, H, C, C, V, V, H, H, C, C, C, (nx,), (ny,), (nx, ny))
    ins = [_f64(a, s) for a, s in zip((Eg_avg_old, Eg_edgV_old, Eg_edgH_old, Fxg_edgV_old, Fyg_edgH_old,
                                       fg_avg_xx_old, fg_avg_yy_old, fg_edgV_xx_old, fg_edgV_xy_old, fg_edgH_yy_old,
                                       fg_edgH_xy_old, KapE_old, KapR_old, Src_old, Delx, Dely, A), shapes)]
    outs = [_out(o, C) for o in (G_old, Pold_L, Pold_B, Pold_R, Pold_T)]
    rc = _lib.lib().trt_old_mgqd_coefs(nx, ny, ng, *[dptr(a) for a in ins], float(c), float(Delt), float(Theta),
                                       *[dptr(o) for o in outs], int(Open_Threads))
    check(rc, "OLD_MGQD_COEFS")


def MLOQD_FV(Eg_avg, Eg_edgV, Eg_edgH, Fxg_edgV, Fyg_edgH, fg_avg_xx, fg_avg_yy, fg_edgV_xx, fg_edgV_xy, fg_edgH_yy,
             fg_edgH_xy, Cg_L, Cg_B, Cg_R, Cg_T, Eg_in_L, Eg_in_B, Eg_in_R, Eg_in_T, Fg_in_L, Fg_in_B, Fg_in_R, Fg_in_T,
             Src, KapE, KapR, Delx, Dely, A, c, Delt, Theta, Open_Threads, Res_Calc, MGQD_Residual, MGQD_BC_Residual,
             G_old, Pold_L, Pold_B, Pold_R, Pold_T, Eg_avg_old, Fxg_edgV_old, Fyg_edgH_old, MGQD_Kits, Fdt_Weight,
             Fin_Weight, Ein_Weight):
    """SUBROUTINE MLOQD_FV, MainSrc/MLOQD_SOLVES.f08:78-362, with QD_FV (QD_SOLVERS.f08:40-538) on the
    device.  Eg_avg/Eg_edgV/Eg_edgH are the initial guess and are overwritten with the solution;
    MGQD_Kits must be an int32 array of n_g entries.  Raises TrtError (TRT_ERR_NOCONV) when a group does
    not converge, after filling the outputs with the last iterate."""
    nx, ny, ng = Eg_avg.shape
    C, V, H = (nx, ny, ng), (nx + 1, ny, ng), (nx, ny + 1, ng)
    for o, s in ((Eg_avg, C), (Eg_edgV, V), (Eg_edgH, H), (Fxg_edgV, V), (Fyg_edgH, H), (MGQD_Residual, (ng, 5, 5)),
                 (MGQD_BC_Residual, (ng, 4))):
        _out(o, s)
    if not (isinstance(MGQD_Kits, np.ndarray) and MGQD_Kits.dtype == np.int32 and MGQD_Kits.shape == (ng,)):
        raise ValueError("MGQD_Kits must be an int32 array of n_g entries")
    by, bx = (ny, ng), (nx, ng)
    ins = [_f64(a, s) for a, s in zip(
        (fg_avg_xx, fg_avg_yy, fg_edgV_xx, fg_edgV_xy, fg_edgH_yy, fg_edgH_xy, Cg_L, Cg_B, Cg_R, Cg_T, Eg_in_L, Eg_in_B,
         Eg_in_R, Eg_in_T, Fg_in_L, Fg_in_B, Fg_in_R, Fg_in_T, Src, KapE, KapR, Delx, Dely, A),
        (C, C, V, V, H, H, by, bx, by, bx, by, bx, by, bx, by, bx, by, bx, C, C, C, (nx,), (ny,), (nx, ny)))]
    old = [_f64(a, s) for a, s in zip((G_old, Pold_L, Pold_B, Pold_R, Pold_T, Eg_avg_old, Fxg_edgV_old, Fyg_edgH_old),
                                      (C, C, C, C, C, C, V, H))]
    rc = _lib.lib().trt_mloqd_fv(nx, ny, ng, dptr(Eg_avg), dptr(Eg_edgV), dptr(Eg_edgH), dptr(Fxg_edgV), dptr(Fyg_edgH),
                                 *[dptr(a) for a in ins], float(c), float(Delt), float(Theta), int(Open_Threads),
                                 int(bool(Res_Calc)), dptr(MGQD_Residual), dptr(MGQD_BC_Residual),
                                 *[dptr(a) for a in old], iptr(MGQD_Kits), float(Fdt_Weight), float(Fin_Weight),
                                 float(Ein_Weight))
    check(rc, "MLOQD_FV")


def COLLAPSE_MG_EF(Eg_avg, Eg_edgV, Eg_edgH, Fxg_edgV, Fyg_edgH, Open_Threads, E_avg, E_edgV, E_edgH, Fx_edgV, Fy_edgH):
    """SUBROUTINE COLLAPSE_MG_EF, MainSrc/MLOQD_SOLVES.f08:687-730."""
    nx, ny, ng = Eg_avg.shape
    ins = [_f64(a, s) for a, s in zip((Eg_avg, Eg_edgV, Eg_edgH, Fxg_edgV, Fyg_edgH),
                                      ((nx, ny, ng), (nx + 1, ny, ng), (nx, ny + 1, ng), (nx + 1, ny, ng),
                                       (nx, ny + 1, ng)))]
    outs = [_out(o, s) for o, s in zip((E_avg, E_edgV, E_edgH, Fx_edgV, Fy_edgH),
                                       ((nx, ny), (nx + 1, ny), (nx, ny + 1), (nx + 1, ny), (nx, ny + 1)))]
    check(_lib.lib().trt_collapse_mg_ef(nx, ny, ng, *[dptr(a) for a in ins], int(Open_Threads),
                                        *[dptr(o) for o in outs]), "COLLAPSE_MG_EF")


def Cbar_Calc(Cb_L, Cb_B, Cb_R, Cb_T, Cg_L, Cg_B, Cg_R, Cg_T, Eg_avg, Eg_edgV, Eg_edgH, Eg_in_L, Eg_in_B, Eg_in_R,
              Eg_in_T):
    """SUBROUTINE Cbar_Calc, MainSrc/GLOQD_SOLVES.f08:177-231."""
    nx, ny, ng = Eg_avg.shape
    outs = [_out(o, s) for o, s in zip((Cb_L, Cb_B, Cb_R, Cb_T), ((ny,), (nx,), (ny,), (nx,)))]
    by, bx = (ny, ng), (nx, ng)
    ins = [_f64(a, s) for a, s in zip((Cg_L, Cg_B, Cg_R, Cg_T, Eg_avg, Eg_edgV, Eg_edgH, Eg_in_L, Eg_in_B, Eg_in_R,
                                       Eg_in_T),
                                      (by, bx, by, bx, (nx, ny, ng), (nx + 1, ny, ng), (nx, ny + 1, ng), by, bx, by, bx))]
    check(_lib.lib().trt_cbar_calc(nx, ny, ng, *[dptr(o) for o in outs], *[dptr(a) for a in ins]), "Cbar_Calc")


def OLD_GREY_COEFS(c, Delt, Theta, cv, A, Gold, Temp_old, KapE_bar_old, E_avg_old, GQD_Src_old, Gold_Hat, Rhat_old):
    """SUBROUTINE OLD_GREY_COEFS, MainSrc/GLOQD_SOLVES.f08:12-42."""
    nx, ny, ng = Gold.shape
    ins = [_f64(A, (nx, ny)), _f64(Gold, (nx, ny, ng))] + [_f64(a, (nx, ny)) for a in (Temp_old, KapE_bar_old,
                                                                                       E_avg_old, GQD_Src_old)]
    outs = [_out(Gold_Hat, (nx, ny)), _out(Rhat_old, (nx, ny))]
    check(_lib.lib().trt_old_grey_coefs(nx, ny, ng, float(c), float(Delt), float(Theta), float(cv),
                                        *[dptr(a) for a in ins], *[dptr(o) for o in outs]), "OLD_GREY_COEFS")


def GREY_COEFS(Eg_avg, Eg_edgV, Eg_edgH, Fxg_edgV_old, Fyg_edgH_old, fg_avg_xx, fg_avg_yy, fg_edgV_xx, fg_edgV_xy,
               fg_edgH_yy, fg_edgH_xy, KapE, KapR, A, c, Delt, Theta, Pold_L, Pold_R, Pold_B, Pold_T, KapE_Bar, DC_xx,
               DL_xx, DR_xx, DC_yy, DB_yy, DT_yy, DL_xy, DR_xy, DB_xy, DT_xy, PL, PR, PB, PT, Fdt_Weight):
    """SUBROUTINE GREY_COEFS, MainSrc/GLOQD_SOLVES.f08:47-146."""
    nx, ny, ng = Eg_avg.shape
    C, V, H = (nx, ny, ng), (nx + 1, ny, ng), (nx, ny + 1, ng)
    ins = [_f64(a, s) for a, s in zip((Eg_avg, Eg_edgV, Eg_edgH, Fxg_edgV_old, Fyg_edgH_old, fg_avg_xx, fg_avg_yy,
                                       fg_edgV_xx, fg_edgV_xy, fg_edgH_yy, fg_edgH_xy, KapE, KapR, A),
                                      (C, V, H, V, H, C, C, V, V, H, H, C, C, (nx, ny)))]
    olds = [_f64(a, C) for a in (Pold_L, Pold_R, Pold_B, Pold_T)]
    outs = [_out(o, (nx, ny)) for o in (KapE_Bar, DC_xx, DL_xx, DR_xx, DC_yy, DB_yy, DT_yy, DL_xy, DR_xy, DB_xy, DT_xy,
                                        PL, PR, PB, PT)]
    check(_lib.lib().trt_grey_coefs(nx, ny, ng, *[dptr(a) for a in ins], float(c), float(Delt), float(Theta),
                                    *[dptr(a) for a in olds], *[dptr(o) for o in outs], float(Fdt_Weight)), "GREY_COEFS")


def EGP_FV_NEWT(E_avg, E_edgV, E_edgH, Temp, KapE_Bar, Fx_edgV, Fy_edgH, Q_bar, KapE_Bar_dT, Temp_Mold, KapE_bar_Mold,
                Theta, Delt, Delx, Dely, A, Cb_L, Cb_B, Cb_R, Cb_T, E_in_L, E_in_B, E_in_R, E_in_T, F_in_L, F_in_B,
                F_in_R, F_in_T, DC_xx, DL_xx, DR_xx, DC_yy, DB_yy, DT_yy, DL_xy, DR_xy, DB_xy, DT_xy, PL, PR, PB, PT,
                Gold_Hat, Rhat_old, Kap0, cv, Comp_Unit, Chi, line_src, E_Bound_Low, T_Bound_Low, Eps1, Eps2, Maxits,
                MGQD_It, Use_Line_Search, Use_Safety_Search, Res_Calc, kapE_dT_flag, Fin_Weight, Ein_Weight):
    """SUBROUTINE EGP_FV_NEWT, MainSrc/GLOQD_SOLVES.f08:305-860, with every linear solve on the device.
    The INTENT(INOUT)/(OUT) arrays are updated in place; returns (Its, GQD_Kits, Deltas (Its, 6),
    dresiduals (Its, 6))."""
    nx, ny = Temp.shape
    for o, s in ((E_avg, (nx, ny)), (E_edgV, (nx + 1, ny)), (E_edgH, (nx, ny + 1)), (Temp, (nx, ny)),
                 (KapE_Bar, (nx, ny)), (Fx_edgV, (nx + 1, ny)), (Fy_edgH, (nx, ny + 1)), (Q_bar, (nx, ny)),
                 (KapE_Bar_dT, (nx, ny))):
        _out(o, s)
    its = ctypes.c_int(0)
    Dl = np.zeros((Maxits, 6), order="F")
    dr = np.zeros((Maxits, 6), order="F")
    kits = np.zeros(Maxits, dtype=np.int32)
    cells = [_f64(a, (nx, ny)) for a in (DC_xx, DL_xx, DR_xx, DC_yy, DB_yy, DT_yy, DL_xy, DR_xy, DB_xy, DT_xy, PL, PR,
                                         PB, PT, Gold_Hat, Rhat_old)]
    bnd = [_f64(a, ((ny,) if k % 2 == 0 else (nx,))) for k, a in
           enumerate((Cb_L, Cb_B, Cb_R, Cb_T, E_in_L, E_in_B, E_in_R, E_in_T, F_in_L, F_in_B, F_in_R, F_in_T))]
    rc = _lib.lib().trt_egp_fv_newt(
        nx, ny, *[dptr(o) for o in (E_avg, E_edgV, E_edgH, Temp, KapE_Bar, Fx_edgV, Fy_edgH, Q_bar, KapE_Bar_dT)],
        ctypes.byref(its), dptr(Dl), dptr(dr), dptr(_f64(Temp_Mold, (nx, ny))), dptr(_f64(KapE_bar_Mold, (nx, ny))),
        float(Theta), float(Delt), dptr(_f64(Delx, (nx,))), dptr(_f64(Dely, (ny,))), dptr(_f64(A, (nx, ny))),
        *[dptr(a) for a in bnd], *[dptr(a) for a in cells], float(Kap0), float(cv), float(Comp_Unit), float(Chi),
        float(line_src), float(E_Bound_Low), float(T_Bound_Low), float(Eps1), float(Eps2), int(Maxits), int(MGQD_It),
        int(bool(Use_Line_Search)), int(bool(Use_Safety_Search)), int(bool(Res_Calc)), int(bool(kapE_dT_flag)),
        iptr(kits), float(Fin_Weight), float(Ein_Weight))
    check(rc, "EGP_FV_NEWT")
    n = its.value
    return n, kits[:n], Dl[:n], dr[:n]


def mgqd_set_tolerance(tol=1e-13, maxit=1000):
    """Convergence settings of MLOQD_FV's device solve (process-wide)."""
    check(_lib.lib().trt_mgqd_set_tolerance(float(tol), int(maxit)), "mgqd_set_tolerance")


def mgqd_set_graphs(on=True):
    """Replay the low-order solves' iteration blocks as CUDA graphs (default) or launch kernel by kernel."""
    check(_lib.lib().trt_mgqd_set_graphs(int(bool(on))), "mgqd_set_graphs")


def mgqd_set_fused_levels(on=True):
    """Run the multigrid preconditioner's fine-level passes as one tiled kernel per level and direction (default)
    or one kernel per half-sweep; the results are identical."""
    check(_lib.lib().trt_mgqd_set_fused_levels(int(bool(on))), "mgqd_set_fused_levels")


def mgqd_set_smem_vcycle(on=True):
    """Run the multigrid levels of at most 64 x 64 cells in the shared-memory kernel (default) or in the tiled
    level passes and the global-memory one-CTA kernel; the results are identical."""
    check(_lib.lib().trt_mgqd_set_smem_vcycle(int(bool(on))), "mgqd_set_smem_vcycle")


def mgqd_last_stats():
    """(device ms of the last MLOQD_FV solve without its copies, largest iteration count, device ms of
    its first matrix-vector product)."""
    ms, its, mv = ctypes.c_double(0), ctypes.c_int(0), ctypes.c_double(0)
    check(_lib.lib().trt_mgqd_last_stats(ctypes.byref(ms), ctypes.byref(its), ctypes.byref(mv)), "mgqd_last_stats")
    return ms.value, its.value, mv.value


def POD_Calc(data, N_t, N_g, clen, g):
    """POD of block g of data(clen, N_g, N_t) (trt_pod_calc): (center, umat, sig, vtmat), k = min(clen, N_t)."""
    k = min(clen, N_t)
    d = np.asarray(data, dtype=np.float64).reshape(-1, order="F")
    if d.size != clen * max(N_g, 1) * N_t:
        raise ValueError(f"data holds {d.size} values, expected clen * max(N_g, 1) * N_t")
    d = np.ascontiguousarray(d)
    c, u, s, vt = np.empty(clen), np.empty((clen, k), order="F"), np.empty(k), np.empty((k, N_t), order="F")
    check(_lib.lib().trt_pod_calc(dptr(d), int(N_t), int(N_g), int(clen), int(g), dptr(c), dptr(u), dptr(s),
                                  dptr(vt)), "trt_pod_calc")
    return c, u, s, vt


def POD_RECONSTRUCT(dat, C, S, U, V, rank, len_, N_g, N_t, t, PODgsum):
    """trt_pod_reconstruct into dat (float64, len_ values)."""
    r = np.ascontiguousarray(rank, dtype=np.int32)
    arrs = [np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, order="F")) for a in (C, S, U, V)]
    check(_lib.lib().trt_pod_reconstruct(dptr(dat), *[dptr(a) for a in arrs], iptr(r), int(len_), int(N_g), int(N_t),
                                         int(t), int(PODgsum)), "trt_pod_reconstruct")


def DMD_Calc(data, N_t, N_g, clen, g, base_subtract=0, svd_eps=-1.0, delt=1.0):
    """DMD of block g of data(clen, N_g, N_t) (trt_dmd_calc).  Returns a dict with lambda, omega, b (xr),
    wmat, wmat_proj (clen, xr) complex, umat (clen, xr), wmat_tild (xr, xr) complex, cvec (clen)."""
    shift = 2 if base_subtract else 1
    k = min(clen, N_t - shift)
    d = np.ascontiguousarray(np.asarray(data, dtype=np.float64).reshape(-1, order="F"))
    if d.size != clen * max(N_g, 1) * N_t:
        raise ValueError("data holds the wrong number of values")
    lam, om, b = (np.zeros(k, dtype=np.complex128) for _ in range(3))
    wm, wp = np.zeros(clen * k, dtype=np.complex128), np.zeros(clen * k, dtype=np.complex128)
    um, wt, cv = np.zeros(clen * k), np.zeros(k * k, dtype=np.complex128), np.zeros(clen)
    nm = ctypes.c_longlong(0)
    f = lambda a: a.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    check(_lib.lib().trt_dmd_calc(dptr(d), int(N_t), int(N_g), int(clen), int(g), int(bool(base_subtract)),
                                  float(svd_eps), float(delt), ctypes.byref(nm), f(lam), f(om), f(b), f(wm), f(wp),
                                  dptr(um), f(wt), dptr(cv)), "trt_dmd_calc")
    xr = nm.value
    return dict(lambda_=lam[:xr], omega=om[:xr], b=b[:xr], wmat=wm[:clen * xr].reshape(clen, xr, order="F"),
                wmat_proj=wp[:clen * xr].reshape(clen, xr, order="F"), umat=um[:clen * xr].reshape(clen, xr, order="F"),
                wmat_tild=wt[:xr * xr].reshape(xr, xr, order="F"), cvec=cv)


def DMD_RECONSTRUCT(dat, L, B, W, C, rank, len_, N_g, DMDgsum, Time):
    """trt_dmd_reconstruct into dat (float64, len_ values); L, B, W complex."""
    r = np.ascontiguousarray(rank, dtype=np.int32)
    cplx = [np.ascontiguousarray(np.asarray(a, dtype=np.complex128).reshape(-1, order="F")).view(np.float64)
            for a in (L, B, W)]
    c = np.ascontiguousarray(np.asarray(C, dtype=np.float64).reshape(-1, order="F"))
    check(_lib.lib().trt_dmd_reconstruct(dptr(dat), *[dptr(a) for a in cplx], dptr(c), iptr(r), int(len_), int(N_g),
                                         int(DMDgsum), float(Time)), "trt_dmd_reconstruct")


def FMAP(f1, Grid1, Grid2, GMap, VMap, Glen1, Glen2, flen2):
    """trt_fmap: returns f2 (flen2 values) mapped from f1 on grid 1 to grid 2."""
    a = np.ascontiguousarray(np.asarray(f1, dtype=np.float64).reshape(-1, order="F"))
    g1 = np.ascontiguousarray(Grid1, dtype=np.float64)
    g2 = np.ascontiguousarray(Grid2, dtype=np.float64)
    gm = np.ascontiguousarray(np.asarray(GMap).reshape(-1, order="F"), dtype=np.int32)
    vm = np.ascontiguousarray(np.asarray(VMap).reshape(-1, order="F"), dtype=np.int32)
    f2 = np.zeros(flen2)
    check(_lib.lib().trt_fmap(dptr(a), dptr(f2), dptr(g1), dptr(g2), iptr(gm), iptr(vm), int(Glen1), int(Glen2),
                              int(a.size), int(flen2)), "trt_fmap")
    return f2


def GRIDMAP_GEN(kind, Delx, Dely, N_x, N_y):
    """trt_gridmap_gen: (x, y) pairs of cell centres (kind 0), vertical edges (1) or horizontal edges (2)."""
    out = np.zeros(2 * N_x * N_y)
    check(_lib.lib().trt_gridmap_gen(int(kind), dptr(_f64(Delx)), dptr(_f64(Dely)), int(N_x), int(N_y), dptr(out)),
          "trt_gridmap_gen")
    return out


def MAP_GRIDS(Grid1, Grid2, xlen1):
    """trt_map_grids: (GMap, VMap) of every Grid2 point's four bracketing Grid1 points (1-based)."""
    g1 = np.ascontiguousarray(Grid1, dtype=np.float64)
    g2 = np.ascontiguousarray(Grid2, dtype=np.float64)
    gm = np.zeros(2 * g2.size, dtype=np.int32)
    vm = np.zeros(2 * g2.size, dtype=np.int32)
    check(_lib.lib().trt_map_grids(iptr(gm), dptr(g1), dptr(g2), int(g1.size), int(g2.size), int(xlen1), iptr(vm)),
          "trt_map_grids")
    return gm, vm


def GRIDMAP_GEN_BND(side, Del, pos, N):
    """trt_gridmap_gen_bnd: the N points of the left/right (side 0, x = pos) or bottom/top (side 1, y = pos) side."""
    out = np.zeros(2 * N)
    check(_lib.lib().trt_gridmap_gen_bnd(int(side), dptr(_f64(Del)), float(pos), int(N), dptr(out)),
          "trt_gridmap_gen_bnd")
    return out


def GENERATE_GRIDS_XY(Delx_d, Dely_d, Delx, Dely, xlen_d, ylen_d, xlen, ylen):
    """trt_generate_grids_xy: dict of the simulation (Sim_Grid_*) and padded data (Dat_Grid_*) point sets and the
    maps between them (GMap_xy*, VMap_xy*), keyed by the reference's names."""
    Delx_d, Dely_d, Delx, Dely = _f64(Delx_d), _f64(Dely_d), _f64(Delx), _f64(Dely)
    dN_x, dN_y, N_x, N_y = Delx_d.size, Dely_d.size, Delx.size, Dely.size
    sets = {"Avg": (N_x * N_y, (dN_x + 2) * (dN_y + 2)), "EdgV": ((N_x + 1) * N_y, (dN_x + 1) * (dN_y + 2)),
            "EdgH": (N_x * (N_y + 1), (dN_x + 2) * (dN_y + 1)), "Bnds": (2 * (N_x + N_y), 2 * (dN_x + dN_y) + 8)}
    out = {}
    for k, (ns, nd) in sets.items():
        out["Sim_Grid_" + k], out["Dat_Grid_" + k] = np.zeros(2 * ns), np.zeros(2 * nd)
        out["GMap_xy" + k], out["VMap_xy" + k] = np.zeros(4 * ns, dtype=np.int32), np.zeros(4 * ns, dtype=np.int32)
    args = [dptr(out[p + k]) for p in ("Sim_Grid_", "Dat_Grid_") for k in sets] + \
        [iptr(out[p + k]) for p in ("GMap_xy", "VMap_xy") for k in sets]
    check(_lib.lib().trt_generate_grids_xy(dptr(Delx_d), dptr(Dely_d), dptr(Delx), dptr(Dely), float(xlen_d),
                                           float(ylen_d), float(xlen), float(ylen), dN_x, dN_y, N_x, N_y, *args),
          "trt_generate_grids_xy")
    return out


def RRANK_CALC(sig, eps):
    """trt_rrank_calc: the reduced rank of the singular values sig for the error level eps."""
    s = _f64(sig)
    r = ctypes.c_int(0)
    check(_lib.lib().trt_rrank_calc(dptr(s), float(eps), int(s.size), ctypes.byref(r)), "trt_rrank_calc")
    return r.value


def POD_TRUNCATE(parts, eps):
    """Packs per-group decompositions [(center, U (clen x k), sig (k), Vt (k x N_t)), ...] (POD_Calc's outputs)
    into the drivers' (C, S, U, V, rank) arrays, each group truncated to RRANK_CALC(sig, eps) modes and appended
    after the earlier groups' as READ_POD_GPART (MainSrc/POD_ROUTINES.f08:700-774) assembles them: U the first
    columns, V the first rows of Vt."""
    C, S, U, V, rank = [], [], [], [], []
    for c, u, sig, vt in parts:
        r = RRANK_CALC(sig, eps)
        C.append(np.asarray(c, dtype=np.float64).reshape(-1))
        S.append(np.asarray(sig[:r], dtype=np.float64))
        U.append(np.asarray(u)[:, :r].reshape(-1, order="F"))
        V.append(np.asarray(vt)[:r, :].reshape(-1, order="F"))
        rank.append(r)
    return (np.concatenate(C), np.concatenate(S), np.concatenate(U), np.concatenate(V),
            np.array(rank, dtype=np.int32))


def GENERATE_GRIDS_T(Delt_d, Delt, Start_Time_d, Start_Time, dN_t, N_t):
    """trt_generate_grids_t: (Sim_TGrid, Dat_TGrid, TMap) with TMap's data levels 1-based."""
    sim, dat, tmap = np.zeros(N_t), np.zeros(dN_t), np.zeros(2 * N_t, dtype=np.int32)
    check(_lib.lib().trt_generate_grids_t(float(Delt_d), float(Delt), float(Start_Time_d), float(Start_Time),
                                          int(dN_t), int(N_t), dptr(sim), dptr(dat), iptr(tmap)),
          "trt_generate_grids_t")
    return sim, dat, tmap


_FG_FIELDS = ("avg_xx", "edgV_xx", "avg_yy", "edgH_yy", "edgV_xy", "edgH_xy")   # the decompositions' order
_FG_OUT = ("fg_avg_xx", "fg_avg_yy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy")


def _fg_out(dN_x, dN_y, N_x, N_y, N_g):
    na, nv, nh = N_x * N_y * N_g, (N_x + 1) * N_y * N_g, N_x * (N_y + 1) * N_g
    return {k: np.zeros(n) for k, n in zip(_FG_OUT, (na, na, nv, nv, nh, nh))}


def _grid_args(grids, sets):
    return [dptr(np.ascontiguousarray(grids[p + k], dtype=np.float64)) for p in ("Sim_Grid_", "Dat_Grid_")
            for k in sets], [iptr(np.ascontiguousarray(grids[p + k], dtype=np.int32)) for p in ("GMap_xy", "VMap_xy")
                             for k in sets]


def _dec_args(parts, n_real):
    """Pointers of one decomposition: the first n_real arrays float64, the rest complex128 (as interleaved
    doubles), then the rank array."""
    keep, ptrs = [], []
    for i, a in enumerate(parts[:-1]):
        if i < n_real:
            v = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, order="F"))
        else:
            v = np.ascontiguousarray(np.asarray(a, dtype=np.complex128).reshape(-1, order="F")).view(np.float64)
        keep.append(v)
        ptrs.append(dptr(v))
    r = np.ascontiguousarray(parts[-1], dtype=np.int32)
    keep.append(r)
    return keep, ptrs, iptr(r)


def POD_RECONSTRUCT_fg(dec, dN, N, t, PODgsum, grids, tgrids):
    """trt_pod_reconstruct_fg: dict of the six QD factors on the simulation grid at simulation level t.
    dec[name] = (C, S, U, V, rank) for name in avg_xx, edgV_xx, avg_yy, edgH_yy, edgV_xy, edgH_xy;
    dN = (dN_x, dN_y, dN_g, dN_t), N = (N_x, N_y, N_g, N_t); grids from GENERATE_GRIDS_XY; tgrids =
    (Sim_TGrid, Dat_TGrid, TMap)."""
    dN_x, dN_y, dN_g, dN_t = dN
    N_x, N_y, N_g, N_t = N
    out = _fg_out(dN_x, dN_y, N_x, N_y, N_g)
    keep, dec_ptrs, ranks = [], [], []
    for name in _FG_FIELDS:
        k, p, r = _dec_args(dec[name], 4)
        keep += k
        dec_ptrs += p
        ranks.append(r)
    g, m = _grid_args(grids, ("Avg", "EdgV", "EdgH"))
    tg = [np.ascontiguousarray(a, dtype=np.float64) for a in tgrids[:2]]
    tm = np.ascontiguousarray(tgrids[2], dtype=np.int32)
    check(_lib.lib().trt_pod_reconstruct_fg(*[dptr(out[k]) for k in _FG_OUT], *dec_ptrs, *ranks, dN_x, dN_y, dN_g,
                                            dN_t, N_x, N_y, N_g, N_t, int(t), int(PODgsum), *g, *[dptr(a) for a in tg],
                                            *m, iptr(tm)), "trt_pod_reconstruct_fg")
    return out


def POD_RECONSTRUCT_BCg(dec, dN, N, t, PODgsum, grids, tgrids):
    """trt_pod_reconstruct_bcg: (Cg_L, Cg_B, Cg_R, Cg_T) at simulation level t; dec = (C, S, U, V, rank)."""
    dN_x, dN_y, dN_g, dN_t = dN
    N_x, N_y, N_g, N_t = N
    out = [np.zeros(N_g * n) for n in (N_y, N_x, N_y, N_x)]
    keep, p, r = _dec_args(dec, 4)
    tg = [np.ascontiguousarray(a, dtype=np.float64) for a in tgrids[:2]]
    tm = np.ascontiguousarray(tgrids[2], dtype=np.int32)
    gb = [np.ascontiguousarray(grids[k], dtype=np.float64) for k in ("Sim_Grid_Bnds", "Dat_Grid_Bnds")]
    mb = [np.ascontiguousarray(grids[k], dtype=np.int32) for k in ("GMap_xyBnds", "VMap_xyBnds")]
    check(_lib.lib().trt_pod_reconstruct_bcg(*[dptr(o) for o in out], *p, r, dN_x, dN_y, dN_g, dN_t, N_x, N_y, N_g,
                                             N_t, int(t), int(PODgsum), *[dptr(a) for a in gb + tg],
                                             *[iptr(a) for a in mb], iptr(tm)), "trt_pod_reconstruct_bcg")
    return tuple(out)


def DMD_RECONSTRUCT_fg(dec, dN, N, Time, DMDgsum, grids):
    """trt_dmd_reconstruct_fg: dict of the six QD factors on the simulation grid at Time.
    dec[name] = (L, B, W, C, rank) (L, B, W complex); dN = (dN_x, dN_y, dN_g), N = (N_x, N_y, N_g)."""
    dN_x, dN_y, dN_g = dN
    N_x, N_y, N_g = N
    out = _fg_out(dN_x, dN_y, N_x, N_y, N_g)
    keep, dec_ptrs, ranks = [], [], []
    for name in _FG_FIELDS:
        L_, B_, W_, C_, r_ = dec[name]
        k, p, r = _dec_args((C_, L_, B_, W_, r_), 1)
        keep += k
        dec_ptrs += [p[1], p[2], p[3], p[0]]
        ranks.append(r)
    g, m = _grid_args(grids, ("Avg", "EdgV", "EdgH"))
    check(_lib.lib().trt_dmd_reconstruct_fg(*[dptr(out[k]) for k in _FG_OUT], *dec_ptrs, *ranks, dN_x, dN_y, dN_g,
                                            N_x, N_y, N_g, float(Time), int(DMDgsum), *g, *m),
          "trt_dmd_reconstruct_fg")
    return out


def DMD_RECONSTRUCT_BCg(dec, dN, N, Time, DMDgsum, grids):
    """trt_dmd_reconstruct_bcg: (Cg_L, Cg_B, Cg_R, Cg_T) at Time; dec = (L, B, W, C, rank)."""
    dN_x, dN_y, dN_g = dN
    N_x, N_y, N_g = N
    out = [np.zeros(N_g * n) for n in (N_y, N_x, N_y, N_x)]
    L_, B_, W_, C_, r_ = dec
    keep, p, r = _dec_args((C_, L_, B_, W_, r_), 1)
    gb = [np.ascontiguousarray(grids[k], dtype=np.float64) for k in ("Sim_Grid_Bnds", "Dat_Grid_Bnds")]
    mb = [np.ascontiguousarray(grids[k], dtype=np.int32) for k in ("GMap_xyBnds", "VMap_xyBnds")]
    check(_lib.lib().trt_dmd_reconstruct_bcg(*[dptr(o) for o in out], p[1], p[2], p[3], p[0], r, dN_x, dN_y, dN_g,
                                             N_x, N_y, N_g, float(Time), int(DMDgsum), *[dptr(a) for a in gb],
                                             *[iptr(a) for a in mb]), "trt_dmd_reconstruct_bcg")
    return tuple(out)


def LINEAR_INTERPOLATION(v1, v2, xm, x1, x2, len_):
    """trt_linear_interpolation, in place on v1 (float64)."""
    b = np.ascontiguousarray(np.asarray(v2, dtype=np.float64).reshape(-1))
    check(_lib.lib().trt_linear_interpolation(dptr(v1), dptr(b), float(xm), float(x1), float(x2), int(len_)),
          "trt_linear_interpolation")


def Bg_planck_calc(T, nu_low, nu_high, comp_unit):
    """FUNCTION Bg_planck_calc, MainSrc/TEMP_FUNCTIONS.f08:90-108 (host evaluation in the library)."""
    return _lib.lib().trt_bg_planck(float(T), float(nu_low), float(nu_high), float(comp_unit))


# --------------------------------------------------------------------------------------------
# Resident-state handle
# --------------------------------------------------------------------------------------------
class TransportSweep:
    """A device-resident sweep instance (trt_create ... trt_destroy).

    Typical time step (Tgen_QDf, ALGORITHMS.f08:1035-1101):
        s.set_material(KapE, src_iso, c, dt, comp_unit)
        s.sweep(roll=True, moments=True)
        out = s.moments(["fg_avg_xx", ...])
    """

    def __init__(self, nx, ny, Omega_x, Omega_y, quad_weight, Delx, Dely, ng, precision="fp64", hbm_budget=0,
                 inplace=False):
        L = _lib.lib()
        self.nx, self.ny, self.ng = int(nx), int(ny), int(ng)
        self.Omega_x, self.Omega_y, self.w = _f64(Omega_x), _f64(Omega_y), _f64(quad_weight)
        self.nm = len(self.Omega_x)
        self.Delx, self.Dely = _f64(Delx, (nx,)), _f64(Dely, (ny,))
        self.precision = {"fp64": _lib.TRT_PREC_FP64, "fp32": _lib.TRT_PREC_FP32, "mixed": _lib.TRT_PREC_FP32}[precision]
        st = ctypes.c_int(0)
        flags = _lib.TRT_CREATE_INPLACE if inplace else 0
        self._h = L.trt_create(self.nx, self.ny, self.nm, self.ng, dptr(self.Omega_x), dptr(self.Omega_y),
                               dptr(self.w), dptr(self.Delx), dptr(self.Dely), self.precision | flags,
                               int(hbm_budget), ctypes.byref(st))
        if not self._h:
            raise _lib.TrtError(st.value, "trt_create")

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().trt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_tiling(self, warps=0, slices=0, stages=0, splits=0):
        """Kernel tiling (0 = default for each); re-lays out the state, which must be put again."""
        check(_lib.lib().trt_set_tiling(self._h, int(warps), int(slices), int(stages), int(splits)),
              "trt_set_tiling")

    def autotune(self):
        """Pick the fastest tiling by timing one sweep per candidate (re-lays out and zeroes the state:
        call before init_state / put_state).  Returns the tiling and its sweep time in ms."""
        w, sl, sp, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0), ctypes.c_float(0)
        check(_lib.lib().trt_autotune(self._h, ctypes.byref(w), ctypes.byref(sl), ctypes.byref(sp), ctypes.byref(ms)),
              "trt_autotune")
        return dict(self.tiling(), sweep_ms=ms.value)

    def set_bands(self, bands):
        """Band CTAs per (group, quadrant, split) sweep (spatial row tiles on a tile-diagonal wavefront,
        one thread-block cluster each); 0/1 = one CTA per sweep.  Re-lays out (zeroes) the state."""
        check(_lib.lib().trt_set_bands(self._h, int(bands)), "trt_set_bands")

    def set_inplace(self, on=True):
        """One corner-state buffer swept in place (each sweep consumes I_crn_old: the next sweep must roll).
        Re-lays out (zeroes) the state."""
        check(_lib.lib().trt_set_inplace(self._h, 1 if on else 0), "trt_set_inplace")

    def state_bytes(self):
        return int(_lib.lib().trt_state_bytes(self._h))

    def bind_state(self, device_ptr, nbytes):
        """In-place handles: sweep a caller-owned device buffer (raw state bytes of this layout)."""
        check(_lib.lib().trt_bind_state(self._h, ctypes.c_void_p(int(device_ptr)), ctypes.c_size_t(int(nbytes))),
              "trt_bind_state")

    def state_written(self):
        """The bound state now holds I_crn_old (raw bytes copied in by the caller)."""
        check(_lib.lib().trt_state_written(self._h), "trt_state_written")

    def snapshot_angular(self, device_ptr):
        """FP32 I_avg of every group into device memory (n_x, n_y, n_m, n_g), on the handle's stream."""
        check(_lib.lib().trt_snapshot_angular(self._h, ctypes.c_void_p(int(device_ptr))), "trt_snapshot_angular")

    def snapshot_angular_groups(self, g0, n_groups, device_ptr):
        """FP32 I_avg of groups g0..g0+n_groups-1 into device memory (n_x, n_y, n_m, n_groups), on the stream."""
        check(_lib.lib().trt_snapshot_angular_groups(self._h, int(g0), int(n_groups), ctypes.c_void_p(int(device_ptr))),
              "trt_snapshot_angular_groups")

    def set_register_mode(self, mode):
        """Cap the sweep kernel's register level (0: <= 128, 1: <= 170, 2: <= 255 registers per thread);
        -1 = the highest level that keeps the whole grid resident.  Re-lays out (zeroes) the state."""
        check(_lib.lib().trt_set_register_mode(self._h, int(mode)), "trt_set_register_mode")

    def tiling(self):
        v = [ctypes.c_int(0) for _ in range(5)]
        check(_lib.lib().trt_get_tiling(self._h, *[ctypes.byref(x) for x in v]), "trt_get_tiling")
        out = dict(zip(("warps", "slices", "dirs_per_lane", "stages", "splits"), [x.value for x in v]))
        out["wide_registers"] = int(_lib.lib().trt_get_register_mode(self._h))
        out["bands"] = int(_lib.lib().trt_get_bands(self._h))
        return out

    def set_material(self, KapE_in, src_iso, c, Delt, Comp_Unit):
        K = _f64(KapE_in, (self.nx, self.ny, self.ng))
        S = _f64(src_iso, (self.nx, self.ny, self.ng))
        check(_lib.lib().trt_set_material(self._h, dptr(K), dptr(S), float(c), float(Delt), float(Comp_Unit)),
              "trt_set_material")

    def set_material_async(self, KapE_in, src_iso, c, Delt, Comp_Unit):
        """Enqueue the material upload on the handle's input copy stream (trt_set_material_async).  The
        arrays must be contiguous float64 (pinned for overlap) and stay unchanged until sync()."""
        check(_lib.lib().trt_set_material_async(self._h, dptr(KapE_in), dptr(src_iso), float(c), float(Delt),
                                                float(Comp_Unit)), "trt_set_material_async")

    def set_material_device(self, d_kap, d_src, c, Delt, Comp_Unit):
        """Device pointers (ints) to FP64 (nx, ny, ng) Fortran arrays."""
        check(_lib.lib().trt_set_material_device(self._h, ctypes.c_void_p(d_kap), ctypes.c_void_p(d_src), float(c),
                                                 float(Delt), float(Comp_Unit)), "trt_set_material_device")

    def set_source_full(self, Src_in):
        S = None if Src_in is None else _f64(Src_in, (2 * self.nx, 2 * self.ny, self.nm, self.ng))
        check(_lib.lib().trt_set_source_full(self._h, dptr(S)), "trt_set_source_full")

    def set_boundary(self, Ic_edgV, Ic_edgH, BC_Type=(0, 0, 0, 0)):
        V = _f64(Ic_edgV, (self.nx + 1, 2 * self.ny, self.nm, self.ng))
        H = _f64(Ic_edgH, (2 * self.nx, self.ny + 1, self.nm, self.ng))
        bc = np.ascontiguousarray(BC_Type, dtype=np.int32)
        check(_lib.lib().trt_set_boundary(self._h, dptr(V), dptr(H), iptr(bc)), "trt_set_boundary")

    def bc_update(self, BC_Type, bcT, Comp_Unit, Nu_g):
        bc = np.ascontiguousarray(BC_Type, dtype=np.int32)
        check(_lib.lib().trt_bc_update(self._h, iptr(bc), *[float(t) for t in bcT], float(Comp_Unit),
                                       dptr(_f64(Nu_g, (self.ng + 1,)))), "trt_bc_update")

    def init_state(self, Tini, bcT, Comp_Unit, Nu_g):
        check(_lib.lib().trt_init_state(self._h, float(Tini), *[float(t) for t in bcT], float(Comp_Unit),
                                        dptr(_f64(Nu_g, (self.ng + 1,)))), "trt_init_state")

    def tstep_setup(self, Nu_g, kappa_mult, cV, Temp, Kap0, Comp_Unit, c, Delt, BC_Type=(0, 0, 0, 0),
                    bcT=(0.0, 0.0, 0.0, 0.0), conv_type=2, conv_ho=1e-12, maxit_rte=150, law=0):
        """Device time stepping with the reference's run_type 'tr_no_qd' (temperatures in eV);
        kappa_mult(i,j) = Kappa_Mult(Mat(i,j)); cV per cell or a scalar.  law 0: the reference's
        Fleck-Cummings material and MEB_SOLVE; law 1 (TRT_LAW_CONFIG): the configurations' opacity law
        with kappa_mult = kappa0(i,j) and the T^4-linearised energy balance (Kap0 unused)."""
        shp = (self.nx, self.ny)
        check(_lib.lib().trt_tstep_set_law(self._h, int(law)), "trt_tstep_set_law")
        cv = _f64(np.broadcast_to(np.asarray(cV, dtype=np.float64), shp), shp)
        bc = np.ascontiguousarray(BC_Type, dtype=np.int32)
        bt = np.ascontiguousarray(bcT, dtype=np.float64)
        check(_lib.lib().trt_tstep_setup(self._h, dptr(_f64(Nu_g, (self.ng + 1,))), dptr(_f64(kappa_mult, shp)),
                                         dptr(cv), dptr(_f64(Temp, shp)), float(Kap0), float(Comp_Unit), float(c),
                                         float(Delt), iptr(bc), dptr(bt), int(conv_type), float(conv_ho),
                                         int(maxit_rte)), "trt_tstep_setup")

    # group-split time step (sharded.ShardedTimeLoop): the phases of trt_tstep for a handle that holds a
    # range of the instance's groups
    def tstep_begin(self):
        check(_lib.lib().trt_tstep_begin(self._h), "trt_tstep_begin")

    def tstep_sweep(self, its):
        check(_lib.lib().trt_tstep_sweep(self._h, int(its)), "trt_tstep_sweep")

    def tstep_partials(self, buf):
        """Group sums of the energy balance (3 n_x n_y doubles) into the device tensor `buf`."""
        check(_lib.lib().trt_tstep_partials(self._h, ctypes.c_void_p(buf.data_ptr())), "trt_tstep_partials")

    def tstep_finish(self, total, its):
        """Temperature, material and convergence from the summed partials (device tensor `total`)."""
        conv, tn, en = ctypes.c_int(0), ctypes.c_double(0), ctypes.c_double(0)
        check(_lib.lib().trt_tstep_finish(self._h, ctypes.c_void_p(total.data_ptr()), int(its), ctypes.byref(conv),
                                          ctypes.byref(tn), ctypes.byref(en)), "trt_tstep_finish")
        return bool(conv.value), tn.value, en.value

    def tstep(self):
        """One backward-Euler time step; returns (outer iterations, T norm, E norm)."""
        its, tn, en = ctypes.c_int(0), ctypes.c_double(0), ctypes.c_double(0)
        check(_lib.lib().trt_tstep(self._h, ctypes.byref(its), ctypes.byref(tn), ctypes.byref(en)), "trt_tstep")
        return its.value, tn.value, en.value

    def mlqd_setup(self, Tini, conv_lo=1e-10, conv_gr1=1e-14, conv_gr2=1e-15, maxit_mloqd=50, maxit_gloqd=20,
                   chi=0.7, line_src=2.0, E_Bound_Low=0.0, T_Bound_Low=0.0, use_line_search=True,
                   use_safety_search=False, kapE_dT_flag=True, Theta=1.0, ho_form=0, group_range=None):
        """Device time stepping with the reference's run_type 'mlqd' (after init_state and tstep_setup):
        the initial low-order state of MGQD_INIT / GQD_INIT at Tini.  group_range = (g_first, Nu_g of the
        whole instance): the handle holds groups g_first .. g_first + ng - 1 of it (trt_mlqd_setup_range; the
        steps then run through the exchange phases, sharded.ShardedMlqd)."""
        p = _lib.MlqdParams(float(conv_lo), float(conv_gr1), float(conv_gr2), int(maxit_mloqd), int(maxit_gloqd),
                            float(chi), float(line_src), float(E_Bound_Low), float(T_Bound_Low),
                            int(bool(use_line_search)), int(bool(use_safety_search)), int(bool(kapE_dT_flag)),
                            float(Theta), int(ho_form))
        self.mlqd_maxit_mloqd = int(maxit_mloqd)
        if group_range is None:
            check(_lib.lib().trt_mlqd_setup(self._h, float(Tini), ctypes.byref(p)), "trt_mlqd_setup")
            return
        g_first, nu_all = group_range
        nu_all = np.ascontiguousarray(np.asarray(nu_all, dtype=np.float64))
        check(_lib.lib().trt_mlqd_setup_range(self._h, float(Tini), ctypes.byref(p), len(nu_all) - 1, int(g_first),
                                              dptr(nu_all)), "trt_mlqd_setup_range")

    # The phases of an mlqd step for groups split over handles (include/trt_sweep.h); buffers are device
    # tensors (torch) of mlqd_exchange_size() doubles.
    def mlqd_exchange_size(self):
        n = _lib.lib().trt_mlqd_exchange_size(self._h)
        if n < 0:
            check(int(n), "trt_mlqd_exchange_size")
        return int(n)

    def mlqd_step_begin(self, part):
        check(_lib.lib().trt_mlqd_step_begin(self._h, ctypes.c_void_p(part.data_ptr())), "trt_mlqd_step_begin")

    def mlqd_step_begin_finish(self, tot):
        check(_lib.lib().trt_mlqd_step_begin_finish(self._h, ctypes.c_void_p(tot.data_ptr())),
              "trt_mlqd_step_begin_finish")

    def mlqd_outer_begin(self, rt, part):
        check(_lib.lib().trt_mlqd_outer_begin(self._h, int(rt), ctypes.c_void_p(part.data_ptr())),
              "trt_mlqd_outer_begin")

    def mlqd_outer_begin_finish(self, tot):
        check(_lib.lib().trt_mlqd_outer_begin_finish(self._h, ctypes.c_void_p(tot.data_ptr())),
              "trt_mlqd_outer_begin_finish")

    def mlqd_mgqd_local(self, part):
        check(_lib.lib().trt_mlqd_mgqd_local(self._h, ctypes.c_void_p(part.data_ptr())), "trt_mlqd_mgqd_local")

    def mlqd_mgqd_finish(self, mg, tot):
        c = ctypes.c_int(0)
        check(_lib.lib().trt_mlqd_mgqd_finish(self._h, int(mg), ctypes.c_void_p(tot.data_ptr()), ctypes.byref(c)),
              "trt_mlqd_mgqd_finish")
        return bool(c.value)

    def mlqd_outer_end(self, rt):
        c = ctypes.c_int(0)
        check(_lib.lib().trt_mlqd_outer_end(self._h, int(rt), ctypes.byref(c)), "trt_mlqd_outer_end")
        return bool(c.value)

    def mlqd_step_end(self):
        st = _lib.MlqdStats()
        check(_lib.lib().trt_mlqd_step_end(self._h, ctypes.byref(st)), "trt_mlqd_step_end")
        return self._mlqd_stats(st)

    def mlqd_step(self):
        """One mlqd time step; returns its statistics (dict) with the MGQD iterations of each outer iteration
        and the EGP iterations of each MGQD iteration."""
        st = _lib.MlqdStats()
        check(_lib.lib().trt_mlqd_step(self._h, ctypes.byref(st)), "trt_mlqd_step")
        return self._mlqd_stats(st)

    def _mlqd_stats(self, st):
        out = {k: getattr(st, k) for k, _ in _lib.MlqdStats._fields_}
        a, b = np.zeros(4096, dtype=np.int32), np.zeros(65536, dtype=np.int32)
        n1, n2 = ctypes.c_int(0), ctypes.c_int(0)
        check(_lib.lib().trt_mlqd_counts(self._h, iptr(a), len(a), iptr(b), len(b), ctypes.byref(n1),
                                         ctypes.byref(n2)), "trt_mlqd_counts")
        out["mgqd_per_outer"] = a[:n1.value].tolist()
        out["egp_per_mgqd"] = b[:n2.value].tolist()
        return out

    def mlqd_put(self, name, values):
        """Overwrite a QD or boundary factor field (fg_*, Cg_*) from a host array (trt_mlqd_put)."""
        a = np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(-1, order="F"))
        check(_lib.lib().trt_mlqd_put(self._h, name.encode(), a.ctypes.data_as(ctypes.c_void_p), a.size, 0),
              "trt_mlqd_put")

    def mlqd_field(self, name):
        """A field of the device mlqd state (trt_mlqd_get), Fortran layout."""
        nx, ny, ng = self.nx, self.ny, self.ng
        grey = {"avg": (nx, ny), "edgV": (nx + 1, ny), "edgH": (nx, ny + 1)}
        keys = [k for k in grey if k in name]
        if name.startswith("Cb_"):
            shp = (ny if name[-1] in "LR" else nx,)
        elif name in ("Temp", "KapE_Bar", "KapE_Bar_dT", "GQD_Src", "MGQD_E_avg", "HO_E_avg", "HO_E_avg_own"):
            shp = (nx, ny)
        elif name == "MGQD_Src":
            shp = (nx, ny, ng)
        elif keys:
            shp = grey[keys[0]] + ((ng,) if name.startswith(("Eg_", "Fxg", "Fyg")) else ())
        else:
            shp = (1,)   # unknown name: the library rejects it
        out = np.empty(shp, order="F")
        check(_lib.lib().trt_mlqd_get(self._h, name.encode(), dptr(out), out.size), "trt_mlqd_get")
        return out

    def temperature(self):
        T = np.empty((self.nx, self.ny), order="F")
        check(_lib.lib().trt_get_temperature(self._h, dptr(T)), "trt_get_temperature")
        return T

    def put_temperature(self, Temp):
        check(_lib.lib().trt_put_temperature(self._h, dptr(_f64(Temp, (self.nx, self.ny)))), "trt_put_temperature")

    def put_state(self, I_crn):
        I = _f64(I_crn, (2 * self.nx, 2 * self.ny, self.nm, self.ng))
        check(_lib.lib().trt_put_state(self._h, dptr(I)), "trt_put_state")

    def get_state(self):
        I = np.empty((2 * self.nx, 2 * self.ny, self.nm, self.ng), order="F")
        check(_lib.lib().trt_get_state(self._h, dptr(I)), "trt_get_state")
        return I

    def sweep(self, roll=False, moments=True, res_calc=False, sync=True):
        flags = (_lib.TRT_ROLL_STATE if roll else 0) | (_lib.TRT_MOMENTS if moments else 0) | \
            (_lib.TRT_RES_CALC if res_calc else 0)
        check(_lib.lib().trt_sweep(self._h, flags), "trt_sweep")
        if sync:
            self.sync()

    def sync(self):
        check(_lib.lib().trt_sync(self._h), "trt_sync")

    def moments(self, names=None):
        names = list(_lib.MOMENT_FIELDS) if names is None else list(names)
        out = {n: np.zeros(_lib.moment_shape(n, self.nx, self.ny, self.ng), order="F") for n in names}
        mh = _lib.MomentsHost()
        for n, a in out.items():
            setattr(mh, n, dptr(a))
        check(_lib.lib().trt_moments(self._h, ctypes.byref(mh)), "trt_moments")
        return out

    def moments_into(self, mh):
        """Fill a prepared MomentsHost (pinned buffers) without allocating."""
        check(_lib.lib().trt_moments(self._h, ctypes.byref(mh)), "trt_moments")

    def moments_async(self, mh):
        """Enqueue the output download into a prepared MomentsHost (trt_moments_async); read after sync()."""
        check(_lib.lib().trt_moments_async(self._h, ctypes.byref(mh)), "trt_moments_async")

    def angular(self, which=("I_avg", "I_edgV", "I_edgH", "Ic_edgV", "Ic_edgH")):
        nx, ny, nm, ng = self.nx, self.ny, self.nm, self.ng
        shapes = {"I_avg": (nx, ny, nm, ng), "I_edgV": (nx + 1, ny, nm, ng), "I_edgH": (nx, ny + 1, nm, ng),
                  "Ic_edgV": (nx + 1, 2 * ny, nm, ng), "Ic_edgH": (2 * nx, ny + 1, nm, ng)}
        out = {k: np.zeros(shapes[k], order="F") for k in which}
        args = [dptr(out.get(k)) for k in ("I_avg", "I_edgV", "I_edgH", "Ic_edgV", "Ic_edgH")]
        check(_lib.lib().trt_get_angular(self._h, *args), "trt_get_angular")
        return out

    def residual(self):
        R = np.zeros((4, self.ng, 5), order="F")
        lx = np.zeros((4, self.ng, 5), dtype=np.int32, order="F")
        ly = np.zeros((4, self.ng, 5), dtype=np.int32, order="F")
        check(_lib.lib().trt_get_residual(self._h, dptr(R), iptr(lx), iptr(ly)), "trt_get_residual")
        return R, lx, ly

    def stream(self):
        return _lib.lib().trt_stream(self._h)

    def device_output(self, name):
        return _lib.lib().trt_device_output(self._h, name.encode())


def required_bytes(nx, ny, nm, ng, precision="fp64"):
    p = {"fp64": _lib.TRT_PREC_FP64, "fp32": _lib.TRT_PREC_FP32, "mixed": _lib.TRT_PREC_FP32}[precision]
    return int(_lib.lib().trt_required_bytes(nx, ny, nm, ng, p))


def kernel_launches():
    return int(_lib.lib().trt_kernel_launches())


class Batch:
    """Many TransportSweep handles stepped together: the sweeps of handles that share a tiling class
    run as one kernel launch over all their (handle, group, quadrant, split) CTAs.  Results are
    bit-identical to stepping each handle alone.  The handles stay owned by the caller and must
    outlive the batch."""

    def __init__(self, sweeps):
        self.sweeps = list(sweeps)
        arr = (ctypes.c_void_p * len(self.sweeps))(*[s.handle for s in self.sweeps])
        st = ctypes.c_int(0)
        self._b = _lib.lib().trt_batch_create(arr, len(self.sweeps), ctypes.byref(st))
        if not self._b:
            raise _lib.TrtError(st.value, "trt_batch_create")

    def close(self):
        if getattr(self, "_b", None):
            _lib.lib().trt_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_persistent(self, on=True):
        """Persistent work-queue launches (default) or one CTA per sweep; results are identical."""
        check(_lib.lib().trt_batch_set_persistent(self._b, 1 if on else 0), "trt_batch_set_persistent")

    def sweep(self, roll=False, moments=True, sync=True):
        flags = (_lib.TRT_ROLL_STATE if roll else 0) | (_lib.TRT_MOMENTS if moments else 0)
        check(_lib.lib().trt_batch_sweep(self._b, flags), "trt_batch_sweep")
        if sync:
            check(_lib.lib().trt_batch_sync(self._b), "trt_batch_sync")

    def tstep(self):
        """One time step of every handle's transport-only loop; returns (iterations, T norms, E norms)."""
        n = len(self.sweeps)
        its = np.zeros(n, dtype=np.int32)
        tn = np.zeros(n)
        en = np.zeros(n)
        check(_lib.lib().trt_batch_tstep(self._b, iptr(its), dptr(tn), dptr(en)), "trt_batch_tstep")
        return its, tn, en
