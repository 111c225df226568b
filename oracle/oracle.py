"""ctypes wrapper of the CPU oracle (liboracle.so, trt_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU-baseline leg of bench.py,
as the checker.  Parity status of the oracle: UNPINNED (see trt_oracle.cpp).

Functions mirror the reference subroutines (Fortran argument order, Fortran-ordered numpy arrays).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_i, _d = ctypes.c_int, ctypes.c_double

_SIG = {
    "oracle_sigint": (_d, [_d]),
    "oracle_bg_planck": (_d, [_d, _d, _d, _d]),
    "oracle_kapb": (_d, [_d, _d, _d]),
    "oracle_scb_cell_ge": (None, [_d, _d, _d, _d, _d, _D]),
    "oracle_transport_scb": (_i, [_i, _i, _i, _i] + [_D] * 6 + [_D] * 8 + [_d, _d, _i, _D, _I, _I, _i, _i]),
    "oracle_collapse_intensities": (_i, [_i, _i, _i, _i, _i, _D, _D, _D, _D, _D, _D, _d] + [_D] * 17),
    "oracle_fg_calc": (_i, [_i, _i, _i] + [_D] * 17 + [_d, _i]),
    "oracle_cg_calc": (_i, [_i, _i, _i, _i] + [_D] * 9 + [_d, _I, _i]),
    "oracle_mgqd_in_calc": (_i, [_i, _i, _i, _i] + [_D] * 13 + [_d, _d, _I, _i]),
    "oracle_gqd_in_calc": (_i, [_i, _i, _i] + [_D] * 16),
    "oracle_rt_bc_update": (_i, [_i, _i, _i, _i, _I, _d, _d, _d, _d, _d, _D, _D, _D, _D, _D]),
    "oracle_openmp_max_threads": (_i, []),
    "oracle_material_update": (_i, [_i, _i, _i, _D, _D, _D, _d, _D, _D, _D]),
    "oracle_meb_solve": (_i, [_i, _i, _i, _D, _D, _D, _D, _d, _D, _d, _d]),
    "oracle_material_update_law": (_i, [_i, _i, _i, _D, _D, _D, _d, _D, _D, _D]),
    "oracle_meb_solve_law": (_i, [_i, _i, _i, _D, _D, _D, _D, _d, _D, _D, _d, _d]),
    "oracle_meb_partial": (_i, [_i, _i, _i, _i, _i, _i, _D, _D, _D, _D, _d, _d, _D]),
    "oracle_meb_finish": (_i, [_i, _i, _i, _D, _D, _D, _d, _d, _d, _D, _D]),
    "oracle_convergence": (_i, [_i, _d, _D, _D, _D, _i, _i, _D, _D]),
    "oracle_old_mgqd_coefs": (_i, [_i, _i, _i] + [_D] * 17 + [_d, _d, _d] + [_D] * 5),
    "oracle_mloqd_fv": (_i, [_i, _i, _i] + [_D] * 29 + [_d, _d, _d, _i, _i] + [_D] * 10 + [_I, _d, _d, _d]),
    "oracle_mloqd_fv_solver": (_i, [_i, _i, _i, _i] + [_D] * 29 + [_d, _d, _d, _i, _i] + [_D] * 10 + [_I, _d, _d, _d]),
    "oracle_collapse_mg_ef": (_i, [_i, _i, _i] + [_D] * 5 + [_i] + [_D] * 5),
    "oracle_cbar_calc": (_i, [_i, _i, _i] + [_D] * 15),
    "oracle_old_grey_coefs": (_i, [_i, _i, _i, _d, _d, _d, _d] + [_D] * 8),
    "oracle_old_grey_coefs_cells": (_i, [_i, _i, _i, _d, _d, _d, _d] + [_D] * 9),
    "oracle_grey_coefs": (_i, [_i, _i, _i] + [_D] * 14 + [_d, _d, _d] + [_D] * 4 + [_D] * 15 + [_d]),
    "oracle_egp_fv_newt": (_i, [_i, _i] + [_D] * 9 + [_I, _D, _D, _D, _D, _d, _d] + [_D] * 3 + [_D] * 12 + [_D] * 14
                           + [_D] * 2 + [_d] * 9 + [_i] * 6 + [_I, _d, _d]),
    "oracle_egp_fv_newt_cells": (_i, [_i, _i] + [_D] * 9 + [_I, _D, _D, _D, _D, _d, _d] + [_D] * 3 + [_D] * 12
                                 + [_D] * 14 + [_D] * 2 + [_d] * 9 + [_i] * 6 + [_I, _d, _d, _D]),
}

_lib = None


def build():
    """Compile liboracle.so with the Makefile beside this file (g++, -O2 -fopenmp)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        for n, (r, a) in _SIG.items():
            f = getattr(L, n)
            f.restype, f.argtypes = r, a
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    if a.dtype == np.int32:
        return a.ctypes.data_as(_I)
    assert a.dtype == np.float64 and a.flags.f_contiguous
    return a.ctypes.data_as(_D)


def F(a, dtype=np.float64):
    return np.asfortranarray(np.asarray(a, dtype=dtype))


def zeros(*shape):
    return np.zeros(shape, order="F")


def transport_scb(I_edgV, I_edgH, Ic_edgV, Ic_edgH, Omega_x, Omega_y, Delx, Dely, A, KapE_in, Src_in, I_crn_old, c,
                  Delt, threads=1, res_calc=False, solver=0, RT_ResLoc_init=0):
    """TRANSPORT_SCB.  I_edgV/I_edgH/Ic_edgV/Ic_edgH are copied (in/out in the reference); returns a dict."""
    nx, ny = len(Delx), len(Dely)
    nm = len(Omega_x)
    ng = KapE_in.shape[2]
    out = dict(I_avg=zeros(nx, ny, nm, ng), I_edgV=F(I_edgV).copy(order="F"), I_edgH=F(I_edgH).copy(order="F"),
               I_crn=zeros(2 * nx, 2 * ny, nm, ng), Ic_edgV=F(Ic_edgV).copy(order="F"),
               Ic_edgH=F(Ic_edgH).copy(order="F"), RT_Residual=zeros(4, ng, 5),
               RT_ResLoc_x=np.full((4, ng, 5), RT_ResLoc_init, dtype=np.int32, order="F"),
               RT_ResLoc_y=np.full((4, ng, 5), RT_ResLoc_init, dtype=np.int32, order="F"))
    args = [F(Omega_x), F(Omega_y), F(Delx), F(Dely), F(A), F(KapE_in), F(Src_in), F(I_crn_old)]
    rc = lib().oracle_transport_scb(nx, ny, nm, ng, _p(out["I_avg"]), _p(out["I_edgV"]), _p(out["I_edgH"]),
                                    _p(out["I_crn"]), _p(out["Ic_edgV"]), _p(out["Ic_edgH"]), *[_p(a) for a in args],
                                    float(c), float(Delt), int(threads), _p(out["RT_Residual"]),
                                    _p(out["RT_ResLoc_x"]), _p(out["RT_ResLoc_y"]), 1 if res_calc else 0, int(solver))
    assert rc == 0
    return out


COLLAPSE_OUT = ["Hg_avg_xx", "Hg_avg_yy", "Hg_avg_xy", "Hg_edgV_xx", "Hg_edgV_xy", "Hg_edgH_yy", "Hg_edgH_xy",
                "Eg_edgV", "Eg_edgH", "Eg_avg", "Fxg_edgV", "Fyg_edgH", "E_edgV", "E_edgH", "E_avg", "Fx_edgV",
                "Fy_edgH"]


def collapse_intensities(I_avg, I_edgV, I_edgH, Omega_x, Omega_y, quad_weight, comp_unit, threads=1):
    nx, ny, nm, ng = I_avg.shape
    A, V, H = (nx, ny), (nx + 1, ny), (nx, ny + 1)
    shapes = [A + (ng,)] * 3 + [V + (ng,)] * 2 + [H + (ng,)] * 2 + [V + (ng,), H + (ng,), A + (ng,), V + (ng,),
                                                                   H + (ng,), V, H, A, V, H]
    out = {k: zeros(*s) for k, s in zip(COLLAPSE_OUT, shapes)}
    rc = lib().oracle_collapse_intensities(nx, ny, nm, ng, int(threads), _p(F(I_avg)), _p(F(I_edgV)), _p(F(I_edgH)),
                                           _p(F(Omega_x)), _p(F(Omega_y)), _p(F(quad_weight)), float(comp_unit),
                                           *[_p(out[k]) for k in COLLAPSE_OUT])
    assert rc == 0
    return out


FG_OUT = ["fg_avg_xx", "fg_avg_yy", "fg_avg_xy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy"]


def fg_calc(m, c, threads=1):
    """m: dict with Hg_* and Eg_avg/Eg_edgV/Eg_edgH (HO_Eg_*)."""
    nx, ny, ng = m["Hg_avg_xx"].shape
    shapes = [(nx, ny, ng)] * 3 + [(nx + 1, ny, ng)] * 2 + [(nx, ny + 1, ng)] * 2
    out = {k: zeros(*s) for k, s in zip(FG_OUT, shapes)}
    ins = [F(m[k]) for k in ("Hg_avg_xx", "Hg_avg_yy", "Hg_avg_xy", "Hg_edgV_xx", "Hg_edgV_xy", "Hg_edgH_yy",
                             "Hg_edgH_xy", "Eg_avg", "Eg_edgV", "Eg_edgH")]
    rc = lib().oracle_fg_calc(nx, ny, ng, *[_p(out[k]) for k in FG_OUT], *[_p(a) for a in ins], float(c), int(threads))
    assert rc == 0
    return out


def cg_calc(I_edgV, I_edgH, Omega_x, Omega_y, quad_weight, comp_unit, bc_type, threads=1):
    nxp, ny, nm, ng = I_edgV.shape
    nx = nxp - 1
    out = dict(Cg_L=zeros(ny, ng), Cg_B=zeros(nx, ng), Cg_R=zeros(ny, ng), Cg_T=zeros(nx, ng))
    rc = lib().oracle_cg_calc(nx, ny, nm, ng, _p(out["Cg_L"]), _p(out["Cg_B"]), _p(out["Cg_R"]), _p(out["Cg_T"]),
                              _p(F(I_edgV)), _p(F(I_edgH)), _p(F(Omega_x)), _p(F(Omega_y)), _p(F(quad_weight)),
                              float(comp_unit), _p(np.ascontiguousarray(bc_type, dtype=np.int32)), int(threads))
    assert rc == 0
    return out


IN_OUT = ["Eg_in_L", "Eg_in_B", "Eg_in_R", "Eg_in_T", "Fg_in_L", "Fg_in_B", "Fg_in_R", "Fg_in_T"]


def mgqd_in_calc(I_edgV, I_edgH, Omega_x, Omega_y, quad_weight, c, comp_unit, bc_type, threads=1):
    nxp, ny, nm, ng = I_edgV.shape
    nx = nxp - 1
    out = {k: zeros(ny if k[-1] in "LR" else nx, ng) for k in IN_OUT}
    rc = lib().oracle_mgqd_in_calc(nx, ny, nm, ng, *[_p(out[k]) for k in IN_OUT], _p(F(I_edgV)), _p(F(I_edgH)),
                                   _p(F(Omega_x)), _p(F(Omega_y)), _p(F(quad_weight)), float(c), float(comp_unit),
                                   _p(np.ascontiguousarray(bc_type, dtype=np.int32)), int(threads))
    assert rc == 0
    return out


def gqd_in_calc(m):
    nx = m["Eg_in_B"].shape[0]
    ny, ng = m["Eg_in_L"].shape
    keys = ["E_in_L", "E_in_B", "E_in_R", "E_in_T", "F_in_L", "F_in_B", "F_in_R", "F_in_T"]
    out = {k: zeros(ny if k[-1] in "LR" else nx) for k in keys}
    rc = lib().oracle_gqd_in_calc(nx, ny, ng, *[_p(out[k]) for k in keys], *[_p(F(m[k])) for k in IN_OUT])
    assert rc == 0
    return out


def rt_bc_update(bc_type, bcT_left, bcT_lower, bcT_right, bcT_upper, comp_unit, nu_g, I_edgV, I_edgH, Ic_edgV,
                 Ic_edgH):
    """In-place on Fortran-ordered copies; returns them."""
    arrs = [F(a).copy(order="F") for a in (I_edgV, I_edgH, Ic_edgV, Ic_edgH)]
    nx = arrs[1].shape[0]
    ny, nm, ng = arrs[0].shape[1], arrs[0].shape[2], arrs[0].shape[3]
    rc = lib().oracle_rt_bc_update(nx, ny, nm, ng, _p(np.ascontiguousarray(bc_type, dtype=np.int32)),
                                   float(bcT_left), float(bcT_lower), float(bcT_right), float(bcT_upper),
                                   float(comp_unit), _p(F(nu_g)), *[_p(a) for a in arrs])
    assert rc == 0
    return arrs


def bg_planck(T, nu_lo, nu_hi, comp_unit):
    return lib().oracle_bg_planck(float(T), float(nu_lo), float(nu_hi), float(comp_unit))


def sigint(z):
    return lib().oracle_sigint(float(z))


def scb_cell_ge(omx, omy, dx, dy, kapE, Q):
    q = np.ascontiguousarray(Q, dtype=np.float64).copy()
    lib().oracle_scb_cell_ge(float(omx), float(omy), float(dx), float(dy), float(kapE), q.ctypes.data_as(_D))
    return q


def max_threads():
    return lib().oracle_openmp_max_threads()


def material_update(Temp, Nu_g, kappa_mult, comp_unit):
    """MATERIAL_UPDATE (UPDATES.f08:110-152): KapE = kapB_calc * Kappa_Mult, src = KapB * Bg, Bg; (nx,ny,ng)."""
    nx, ny = Temp.shape
    ng = len(Nu_g) - 1
    K, S, B = zeros(nx, ny, ng), zeros(nx, ny, ng), zeros(nx, ny, ng)
    rc = lib().oracle_material_update(nx, ny, ng, _p(F(Temp)), _p(F(Nu_g)), _p(F(kappa_mult)), float(comp_unit),
                                      _p(K), _p(S), _p(B))
    assert rc == 0
    return K, S, B


def meb_solve(Temp_old, Eg_HO, KapE, Delt, cV, Kap0, comp_unit):
    """MEB_SOLVE (UPDATES.f08:185-230) with cV per cell; returns the new Temp."""
    nx, ny, ng = Eg_HO.shape
    T = zeros(nx, ny)
    rc = lib().oracle_meb_solve(nx, ny, ng, _p(T), _p(F(Eg_HO)), _p(F(KapE)), _p(F(Temp_old)), float(Delt),
                                _p(F(np.broadcast_to(cV, (nx, ny)))), float(Kap0), float(comp_unit))
    assert rc == 0
    return T


def material_update_law(Temp, Nu_g, kappa0, comp_unit):
    """The configurations' opacity law in place of kapB_calc (MATERIAL_UPDATE's template,
    UPDATES.f08:130-150): KapE = kappa0 (1 - exp(-nu/T)) / (nu^3 sqrt(T)) (keV), src = KapE * Bg, Bg."""
    nx, ny = Temp.shape
    ng = len(Nu_g) - 1
    K, S, B = zeros(nx, ny, ng), zeros(nx, ny, ng), zeros(nx, ny, ng)
    rc = lib().oracle_material_update_law(nx, ny, ng, _p(F(Temp)), _p(F(Nu_g)), _p(F(kappa0)), float(comp_unit),
                                          _p(K), _p(S), _p(B))
    assert rc == 0
    return K, S, B


def meb_solve_law(Temp, Temp_old, Eg_HO, KapE, Delt, cV, Nu_g, comp_unit, c):
    """Backward-Euler energy balance of the configurations with the emission linearised about Temp (one
    Newton step); returns the new Temp."""
    nx, ny, ng = Eg_HO.shape
    T = F(Temp).copy(order="F")
    rc = lib().oracle_meb_solve_law(nx, ny, ng, _p(T), _p(F(Eg_HO)), _p(F(KapE)), _p(F(Temp_old)), float(Delt),
                                    _p(F(np.broadcast_to(cV, (nx, ny)))), _p(F(Nu_g)), float(comp_unit), float(c))
    assert rc == 0
    return T


def meb_partial(Eg_HO, KapE, Temp, Nu_g, comp_unit, c, g0, g1, law=0):
    """Group sums over groups [g0, g1) of the energy balance, (nx, ny, 3) Fortran-ordered: the split form of
    MEB_SOLVE (law 0) or of the configurations' balance (law 1)."""
    nx, ny, ng = Eg_HO.shape
    part = zeros(nx, ny, 3)
    rc = lib().oracle_meb_partial(nx, ny, ng, int(g0), int(g1), int(law), _p(F(Eg_HO)), _p(F(KapE)), _p(F(Temp)),
                                  _p(F(Nu_g)), float(comp_unit), float(c), _p(part))
    assert rc == 0
    return part


def meb_finish(sums, Temp_old, cV, Delt, Kap0, comp_unit, law=0):
    """Temperature and transport E from the group sums over all ranges (sums: (nx, ny, 3) Fortran-ordered)."""
    nx, ny = Temp_old.shape
    sums = F(sums)
    T, E = zeros(nx, ny), zeros(nx, ny)
    rc = lib().oracle_meb_finish(nx, ny, int(law), _p(sums), _p(F(Temp_old)), _p(F(np.broadcast_to(cV, (nx, ny)))),
                                 float(Delt), float(Kap0), float(comp_unit), _p(T), _p(E))
    assert rc == 0
    return T, E


def convergence(conv_type, eps, x, x_old, x_old2, its):
    """CONVERGENCE (CONVERGENCE_CHECKS.f08:7-44): (converged, norm, rho)."""
    n = int(np.asarray(x).size)
    nrm, rho = ctypes.c_double(0), ctypes.c_double(0)
    ok = lib().oracle_convergence(int(conv_type), float(eps), _p(F(x)), _p(F(x_old)), _p(F(x_old2)), n, int(its),
                                  ctypes.byref(nrm), ctypes.byref(rho))
    return bool(ok), nrm.value, rho.value


def tr_no_qd_steps(st, Omega_x, Omega_y, quad_weight, Delx, Dely, Nu_g, kappa_mult, cV, Kap0, comp_unit, c, Delt,
                   steps, conv_type=2, conv_ho=1e-12, maxit=150, bc_type=(0, 0, 0, 0), bcT=(0.0, 0.0, 0.0, 0.0),
                   threads=4, solver=1, law=0, record=None):
    """Time steps of TRT_MLQD_ALGORITHM with run_type 'tr_no_qd' (ALGORITHMS.f08:389-421, 518-572,
    662-668, 816-836).  st: dict with I_crn, Ic_edgV, Ic_edgH, I_edgV, I_edgH, Temp (updated in place).
    solver: the sweep's cell solve (0 = SCB_BGEN + Gaussian elimination, the reference's form; 1 = the
    closed form).  law 0: the reference's material (kapB_calc * kappa_mult, MEB_SOLVE); law 1: the
    configurations' opacity law with kappa_mult = kappa0 and the T^4-linearised energy balance.
    record: optional list; after every step a dict of the step's fg factors and corner state is appended.
    Returns one (Temp, HO_E_avg, outer iterations, T norm, E norm) tuple per step."""
    A = F(np.outer(Delx, Dely))
    nm = len(Omega_x)
    mat = material_update_law if law == 1 else material_update
    KapE, src, _ = mat(st["Temp"], Nu_g, kappa_mult, comp_unit)   # INITIALIZERS.f08:137
    hist = []
    for _ in range(steps):
        Temp_old = st["Temp"].copy(order="F")
        I_crn_old = st["I_crn"].copy(order="F")
        shp = Temp_old.shape
        T_rt1, T_rt2 = zeros(*shp), zeros(*shp)
        E_rt1, E_rt2 = zeros(*shp), zeros(*shp)
        its, conv = 0, False
        while not conv and its < maxit:
            its += 1
            Src_in = F(np.repeat(np.repeat(src, 2, axis=0), 2, axis=1)[:, :, None, :].repeat(nm, axis=2))
            s = transport_scb(st["I_edgV"], st["I_edgH"], st["Ic_edgV"], st["Ic_edgH"], Omega_x, Omega_y, Delx, Dely,
                              A, KapE, Src_in, I_crn_old, c, Delt, threads=threads, solver=solver)
            for k in ("I_crn", "I_edgV", "I_edgH", "Ic_edgV", "Ic_edgH"):
                st[k] = s[k]
            m = collapse_intensities(s["I_avg"], s["I_edgV"], s["I_edgH"], Omega_x, Omega_y, quad_weight, comp_unit,
                                     threads=threads)
            if max(bc_type) > 0:
                st["I_edgV"], st["I_edgH"], st["Ic_edgV"], st["Ic_edgH"] = rt_bc_update(
                    bc_type, bcT[0], bcT[1], bcT[2], bcT[3], comp_unit, Nu_g, st["I_edgV"], st["I_edgH"],
                    st["Ic_edgV"], st["Ic_edgH"])
            if law == 1:
                st["Temp"] = meb_solve_law(st["Temp"], Temp_old, m["Eg_avg"], KapE, Delt, cV, Nu_g, comp_unit, c)
            else:
                st["Temp"] = meb_solve(Temp_old, m["Eg_avg"], KapE, Delt, cV, Kap0, comp_unit)
            KapE, src, _ = mat(st["Temp"], Nu_g, kappa_mult, comp_unit)
            tc, tn, _ = convergence(conv_type, conv_ho, st["Temp"], T_rt1, T_rt2, its)
            ec, en, _ = convergence(conv_type, conv_ho, m["E_avg"], E_rt1, E_rt2, its)
            conv = tc and ec
            E_rt2, E_rt1 = E_rt1, m["E_avg"].copy(order="F")
            T_rt2, T_rt1 = T_rt1, st["Temp"].copy(order="F")
        hist.append((st["Temp"].copy(order="F"), m["E_avg"].copy(order="F"), its, tn, en))
        if record is not None:
            f = fg_calc(m, c, threads=threads)
            record.append(dict(f, I_crn=st["I_crn"].copy(order="F"), Eg_avg=m["Eg_avg"].copy(order="F")))
    return hist


# Low-order (MGQD) solve: argument names of MLOQD_FV / OLD_MGQD_COEFS (MLOQD_SOLVES.f08:12-362).
MLOQD_FACTORS = ("fg_avg_xx", "fg_avg_yy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy")
MLOQD_BOUNDARY = ("Cg_L", "Cg_B", "Cg_R", "Cg_T", "Eg_in_L", "Eg_in_B", "Eg_in_R", "Eg_in_T",
                  "Fg_in_L", "Fg_in_B", "Fg_in_R", "Fg_in_T")
MLOQD_MATERIAL = ("Src", "KapE", "KapR", "Delx", "Dely", "A")
MLOQD_OLD = ("G_old", "Pold_L", "Pold_B", "Pold_R", "Pold_T", "Eg_avg_old", "Fxg_edgV_old", "Fyg_edgH_old")
OLD_MGQD_IN = ("Eg_avg_old", "Eg_edgV_old", "Eg_edgH_old", "Fxg_edgV_old", "Fyg_edgH_old", "fg_avg_xx_old",
               "fg_avg_yy_old", "fg_edgV_xx_old", "fg_edgV_xy_old", "fg_edgH_yy_old", "fg_edgH_xy_old", "KapE_old",
               "KapR_old", "Src_old", "Delx", "Dely", "A")


def old_mgqd_coefs(d, c, Delt, Theta):
    """OLD_MGQD_COEFS (MLOQD_SOLVES.f08:12-73): returns G_old, Pold_L, Pold_B, Pold_R, Pold_T (nx,ny,ng)."""
    nx, ny, ng = d["Eg_avg_old"].shape
    out = {k: zeros(nx, ny, ng) for k in ("G_old", "Pold_L", "Pold_B", "Pold_R", "Pold_T")}
    rc = lib().oracle_old_mgqd_coefs(nx, ny, ng, *[_p(F(d[k])) for k in OLD_MGQD_IN], float(c), float(Delt),
                                     float(Theta), *[_p(v) for v in out.values()])
    assert rc == 0
    return out


def mloqd_fv(d, c, Delt, Theta=1.0, res_calc=True, threads=1, Fdt_Weight=1.0, Fin_Weight=1.0, Ein_Weight=1.0,
             solver=0):
    """MLOQD_FV (MLOQD_SOLVES.f08:78-362).  solver 0: the reduced system solved directly (the checker);
    solver 1: the reference's ILUT + BiCGSTAB procedure in its unknown numbering (the CPU baseline);
    see mgqd_oracle.cpp.  d holds the subroutine's inputs by name plus Eg_avg/Eg_edgV/Eg_edgH (initial
    guess).  Returns Eg_avg, Eg_edgV, Eg_edgH, Fxg_edgV, Fyg_edgH, MGQD_Residual (ng,5,5),
    MGQD_BC_Residual (ng,4), MGQD_Kits (ng)."""
    nx, ny, ng = d["Eg_avg"].shape
    o = {k: F(d[k]).copy(order="F") for k in ("Eg_avg", "Eg_edgV", "Eg_edgH")}
    o["Fxg_edgV"], o["Fyg_edgH"] = zeros(nx + 1, ny, ng), zeros(nx, ny + 1, ng)
    o["MGQD_Residual"], o["MGQD_BC_Residual"] = zeros(ng, 5, 5), zeros(ng, 4)
    o["MGQD_Kits"] = np.zeros(ng, dtype=np.int32)
    rc = lib().oracle_mloqd_fv_solver(
        int(solver), nx, ny, ng, *[_p(o[k]) for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH")],
        *[_p(F(d[k])) for k in MLOQD_FACTORS + MLOQD_BOUNDARY + MLOQD_MATERIAL], float(c), float(Delt),
        float(Theta), int(threads), int(bool(res_calc)), _p(o["MGQD_Residual"]), _p(o["MGQD_BC_Residual"]),
        *[_p(F(d[k])) for k in MLOQD_OLD], _p(o["MGQD_Kits"]), float(Fdt_Weight), float(Fin_Weight),
        float(Ein_Weight))
    assert rc == 0, rc
    return o


# Grey low-order side (GLOQD_SOLVES.f08, MLOQD_SOLVES.f08:687-730).
GREY_D = ("DC_xx", "DL_xx", "DR_xx", "DC_yy", "DB_yy", "DT_yy", "DL_xy", "DR_xy", "DB_xy", "DT_xy")
GREY_P = ("PL", "PR", "PB", "PT")
SIDES = ("L", "B", "R", "T")


def collapse_mg_ef(d):
    """COLLAPSE_MG_EF: group sums of Eg_avg/Eg_edgV/Eg_edgH/Fxg_edgV/Fyg_edgH."""
    nx, ny, ng = d["Eg_avg"].shape
    o = {"E_avg": zeros(nx, ny), "E_edgV": zeros(nx + 1, ny), "E_edgH": zeros(nx, ny + 1),
         "Fx_edgV": zeros(nx + 1, ny), "Fy_edgH": zeros(nx, ny + 1)}
    rc = lib().oracle_collapse_mg_ef(nx, ny, ng, *[_p(F(d[k])) for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV",
                                                                       "Fyg_edgH")], 1, *[_p(v) for v in o.values()])
    assert rc == 0
    return o


def cbar_calc(d):
    """Cbar_Calc: Cb_L, Cb_B, Cb_R, Cb_T."""
    nx, ny, ng = d["Eg_avg"].shape
    o = {"Cb_" + s: zeros(ny if s in "LR" else nx) for s in SIDES}
    rc = lib().oracle_cbar_calc(nx, ny, ng, *[_p(v) for v in o.values()], *[_p(F(d["Cg_" + s])) for s in SIDES],
                                *[_p(F(d[k])) for k in ("Eg_avg", "Eg_edgV", "Eg_edgH")],
                                *[_p(F(d["Eg_in_" + s])) for s in SIDES])
    assert rc == 0
    return o


def old_grey_coefs(c, Delt, Theta, cv, A, Gold, Temp_old, KapE_bar_old, E_avg_old, GQD_Src_old):
    """OLD_GREY_COEFS: (Gold_Hat, Rhat_old).  cv: the reference's scalar, or an (nx, ny) array per cell."""
    nx, ny, ng = Gold.shape
    gh, rh = zeros(nx, ny), zeros(nx, ny)
    args = [nx, ny, ng, float(c), float(Delt), float(Theta), 0.0 if np.ndim(cv) else float(cv), _p(F(A)), _p(F(Gold)),
            _p(F(Temp_old)), _p(F(KapE_bar_old)), _p(F(E_avg_old)), _p(F(GQD_Src_old)), _p(gh), _p(rh)]
    if np.ndim(cv):
        cvc = F(np.broadcast_to(cv, (nx, ny)))
        rc = lib().oracle_old_grey_coefs_cells(*args, _p(cvc))
    else:
        rc = lib().oracle_old_grey_coefs(*args)
    assert rc == 0
    return gh, rh


def grey_coefs(d, c, Delt, Theta, Fdt_Weight=1.0):
    """GREY_COEFS: KapE_Bar, the ten D's and the four P's (nx, ny)."""
    nx, ny, ng = d["Eg_avg"].shape
    o = {k: zeros(nx, ny) for k in ("KapE_Bar",) + GREY_D + GREY_P}
    ins = ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV_old", "Fyg_edgH_old", "fg_avg_xx", "fg_avg_yy", "fg_edgV_xx",
           "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy", "KapE", "KapR", "A")
    rc = lib().oracle_grey_coefs(nx, ny, ng, *[_p(F(d[k])) for k in ins], float(c), float(Delt), float(Theta),
                                 *[_p(F(d[k])) for k in ("Pold_L", "Pold_R", "Pold_B", "Pold_T")],
                                 *[_p(v) for v in o.values()], float(Fdt_Weight))
    assert rc == 0
    return o


def grey_sums(d, c, Delt, Theta, Fdt_Weight=1.0):
    """The group sums behind COLLAPSE_MG_EF (MLOQD_SOLVES.f08:687-730), Cbar_Calc (GLOQD_SOLVES.f08:191-229) and
    GREY_COEFS (:89-143) over the groups d holds (one range of a split instance), groups added in order, in the
    exchange layout of the library (trt_mlqd_exchange_size): E (nx,ny), EV (nx+1,ny), EH (nx,ny+1), FV, FH;
    per left/right point (l, s1, r, s2) and per bottom/top point (b, s1, t, s2) of Cbar_Calc; the 15 numerators
    of GREY_COEFS (KapE_Bar's, the ten D's, the four P's), each field in Fortran order, concatenated."""
    Eg, EgV, EgH = F(d["Eg_avg"]), F(d["Eg_edgV"]), F(d["Eg_edgH"])
    Fx, Fy = F(d["Fxg_edgV"]), F(d["Fyg_edgH"])
    nx, ny, ng = Eg.shape
    E, EV, EH, FV, FH = zeros(nx, ny), zeros(nx + 1, ny), zeros(nx, ny + 1), zeros(nx + 1, ny), zeros(nx, ny + 1)
    for g in range(ng):
        E = E + Eg[:, :, g]
        EV = EV + EgV[:, :, g]
        EH = EH + EgH[:, :, g]
        FV = FV + Fx[:, :, g]
        FH = FH + Fy[:, :, g]
    lr, bt = zeros(4, ny), zeros(4, nx)
    for g in range(ng):
        q = EgV[0, :, g] - F(d["Eg_in_L"])[:, g]
        lr[0] = lr[0] + F(d["Cg_L"])[:, g] * q
        lr[1] = lr[1] + q
        q = EgV[nx, :, g] - F(d["Eg_in_R"])[:, g]
        lr[2] = lr[2] + F(d["Cg_R"])[:, g] * q
        lr[3] = lr[3] + q
        q = EgH[:, 0, g] - F(d["Eg_in_B"])[:, g]
        bt[0] = bt[0] + F(d["Cg_B"])[:, g] * q
        bt[1] = bt[1] + q
        q = EgH[:, ny, g] - F(d["Eg_in_T"])[:, g]
        bt[2] = bt[2] + F(d["Cg_T"])[:, g] * q
        bt[3] = bt[3] + q
    num = zeros(nx, ny, 15)
    A = F(d["A"])
    fxx, fyy = F(d["fg_avg_xx"]), F(d["fg_avg_yy"])
    fVxx, fVxy, fHyy, fHxy = F(d["fg_edgV_xx"]), F(d["fg_edgV_xy"]), F(d["fg_edgH_yy"]), F(d["fg_edgH_xy"])
    FxO, FyO = F(d["Fxg_edgV_old"]), F(d["Fyg_edgH_old"])
    Pold = [F(d[k]) for k in ("Pold_L", "Pold_R", "Pold_B", "Pold_T")]
    w = Fdt_Weight * A / (2.0 * Theta * c * Delt)
    for g in range(ng):
        tk = F(d["KapR"])[:, :, g] + Fdt_Weight / (Theta * c * Delt)
        L, R, B, T = (slice(0, nx), slice(None)), (slice(1, nx + 1), slice(None)), (slice(None), slice(0, ny)), \
            (slice(None), slice(1, ny + 1))
        terms = [F(d["KapE"])[:, :, g] * Eg[:, :, g],
                 fxx[:, :, g] * Eg[:, :, g] / tk,
                 fVxx[L + (g,)] * EgV[L + (g,)] / tk,
                 fVxx[R + (g,)] * EgV[R + (g,)] / tk,
                 fyy[:, :, g] * Eg[:, :, g] / tk,
                 fHyy[B + (g,)] * EgH[B + (g,)] / tk,
                 fHyy[T + (g,)] * EgH[T + (g,)] / tk,
                 fVxy[L + (g,)] * EgV[L + (g,)] / tk,
                 fVxy[R + (g,)] * EgV[R + (g,)] / tk,
                 fHxy[B + (g,)] * EgH[B + (g,)] / tk,
                 fHxy[T + (g,)] * EgH[T + (g,)] / tk,
                 (w * FxO[L + (g,)] + Pold[0][:, :, g]) / tk,
                 (w * FxO[R + (g,)] + Pold[1][:, :, g]) / tk,
                 (w * FyO[B + (g,)] + Pold[2][:, :, g]) / tk,
                 (w * FyO[T + (g,)] + Pold[3][:, :, g]) / tk]
        for q_, t_ in enumerate(terms):
            num[:, :, q_] = num[:, :, q_] + t_
    return np.concatenate([a.reshape(-1, order="F") for a in (E, EV, EH, FV, FH, lr, bt, num)])


def grey_from_sums(tot, nx, ny):
    """The grey fields, Cbar_Calc's boundary factors and GREY_COEFS's coefficients from the group sums of
    grey_sums added over every range."""
    sizes = [("E_avg", (nx, ny)), ("E_edgV", (nx + 1, ny)), ("E_edgH", (nx, ny + 1)), ("Fx_edgV", (nx + 1, ny)),
             ("Fy_edgH", (nx, ny + 1)), ("lr", (4, ny)), ("bt", (4, nx)), ("num", (nx, ny, 15))]
    out, k = {}, 0
    for name, shp in sizes:
        n = int(np.prod(shp))
        out[name] = F(np.array(tot[k:k + n], dtype=np.float64).reshape(shp, order="F"))
        k += n
    lr, bt, num = out.pop("lr"), out.pop("bt"), out.pop("num")
    out.update(Cb_L=F(lr[0] / lr[1]), Cb_R=F(lr[2] / lr[3]), Cb_B=F(bt[0] / bt[1]), Cb_T=F(bt[2] / bt[3]))
    E, EV, EH = out["E_avg"], out["E_edgV"], out["E_edgH"]
    div = [E, E, EV[:nx], EV[1:], E, EH[:, :ny], EH[:, 1:], EV[:nx], EV[1:], EH[:, :ny], EH[:, 1:]]
    out["KapE_Bar"] = F(num[:, :, 0] / div[0])
    for q_, name in enumerate(GREY_D):
        out[name] = F(num[:, :, q_ + 1] / div[q_ + 1])
    for q_, name in enumerate(GREY_P):
        out[name] = F(num[:, :, 11 + q_])
    return out


EGP_STATE = ("E_avg", "E_edgV", "E_edgH", "Temp", "KapE_Bar", "Fx_edgV", "Fy_edgH")


def egp_fv_newt(g, Theta, Delt, Kap0, cv, Comp_Unit, Chi=0.7, line_src=2.0, E_Bound_Low=0.0, T_Bound_Low=0.0,
                Eps1=1e-14, Eps2=1e-15, Maxits=10, MGQD_It=1, Use_Line_Search=True, Use_Safety_Search=False,
                Res_Calc=True, kapE_dT_flag=True, Fin_Weight=1.0, Ein_Weight=1.0):
    """EGP_FV_NEWT (GLOQD_SOLVES.f08:305-860) on copies of g's state (E_avg, E_edgV, E_edgH, Temp, KapE_Bar,
    Fx_edgV, Fy_edgH); g also holds Temp_Mold, KapE_bar_Mold, Delx, Dely, A, Cb_*, E_in_*, F_in_*, the D's,
    the P's, Gold_Hat and Rhat_old.  Returns the new state plus Q_bar, KapE_Bar_dT, Its, GQD_Kits,
    Deltas (Its, 6), dresiduals (Its, 6).  cv: the reference's scalar, or an (nx, ny) array per cell."""
    nx, ny = g["Temp"].shape
    o = {k: F(g[k]).copy(order="F") for k in EGP_STATE}
    o["Q_bar"], o["KapE_Bar_dT"] = zeros(nx, ny), zeros(nx, ny)
    its = ctypes.c_int(0)
    Dl, dr = zeros(Maxits, 6), zeros(Maxits, 6)
    kits = np.zeros(Maxits, dtype=np.int32)
    cvc = F(np.broadcast_to(cv, (nx, ny))) if np.ndim(cv) else None
    fn = lib().oracle_egp_fv_newt_cells if cvc is not None else lib().oracle_egp_fv_newt
    extra = (_p(cvc),) if cvc is not None else ()
    rc = fn(
        nx, ny, *[_p(o[k]) for k in EGP_STATE], _p(o["Q_bar"]), _p(o["KapE_Bar_dT"]), ctypes.byref(its), _p(Dl),
        _p(dr), _p(F(g["Temp_Mold"])), _p(F(g["KapE_bar_Mold"])), float(Theta), float(Delt), _p(F(g["Delx"])),
        _p(F(g["Dely"])), _p(F(g["A"])), *[_p(F(g["Cb_" + s])) for s in SIDES], *[_p(F(g["E_in_" + s])) for s in SIDES],
        *[_p(F(g["F_in_" + s])) for s in SIDES], *[_p(F(g[k])) for k in GREY_D + GREY_P],
        _p(F(g["Gold_Hat"])), _p(F(g["Rhat_old"])), float(Kap0), 0.0 if cvc is not None else float(cv),
        float(Comp_Unit), float(Chi), float(line_src), float(E_Bound_Low), float(T_Bound_Low), float(Eps1), float(Eps2),
        int(Maxits), int(MGQD_It), int(bool(Use_Line_Search)), int(bool(Use_Safety_Search)), int(bool(Res_Calc)),
        int(bool(kapE_dT_flag)), _p(kits), float(Fin_Weight), float(Ein_Weight), *extra)
    assert rc == 0, rc
    n = its.value
    o["Its"], o["GQD_Kits"], o["Deltas"], o["dresiduals"] = n, kits[:n], Dl[:n], dr[:n]
    return o



# ------------------------------------------------------------------------------------------------
# The mlqd time loop: TRT_MLQD_ALGORITHM with run_type 'mlqd' and use_grey = 1 (HO_Form 0, RT_start_Its 2,
# Fdt/Fin/Ein weights 1; ALGORITHMS.f08:294-302, 389-416, 518-572, 670-836).
# ------------------------------------------------------------------------------------------------

def mlqd_init(nx, ny, Omega_x, Omega_y, quad_weight, Nu_g, Tini, comp_unit, c, bc_type=(0, 0, 0, 0),
              bcT=(0.0, 0.0, 0.0, 0.0)):
    """The initial state of the mlqd algorithm: RT_INIT (INITIALIZERS.f08:15-109), Temp = Tini (TEMP_INIT,
    :114-139; the material follows from Temp), MGQD_INIT (:159-321) and GQD_INIT (:326-427).  KapE_Bar and
    GQD_Src are left unset by the reference (allocated, never written before the first step); they are
    zero here, and with Theta = 1 they do not enter the first step."""
    nm, ng = len(Omega_x), len(Nu_g) - 1
    pi = np.pi
    bg = np.array([bg_planck(Tini, Nu_g[g], Nu_g[g + 1], comp_unit) for g in range(ng)])
    st = {}
    st["I_crn"] = F(np.broadcast_to(bg, (2 * nx, 2 * ny, nm, ng)))
    I_edgV = F(np.broadcast_to(bg, (nx + 1, ny, nm, ng)))
    I_edgH = F(np.broadcast_to(bg, (nx, ny + 1, nm, ng)))
    Ic_edgV = F(np.broadcast_to(bg, (nx + 1, 2 * ny, nm, ng)))
    Ic_edgH = F(np.broadcast_to(bg, (2 * nx, ny + 1, nm, ng)))
    st["I_edgV"], st["I_edgH"], st["Ic_edgV"], st["Ic_edgH"] = rt_bc_update(
        (0, 0, 0, 0), bcT[0], bcT[1], bcT[2], bcT[3], comp_unit, Nu_g, I_edgV, I_edgH, Ic_edgV, Ic_edgH)
    eg = 4.0 * pi * bg / c
    E0 = zeros(nx, ny)
    for g in range(ng):
        E0 = E0 + eg[g]
    st["HO_E_avg"] = E0.copy(order="F")
    st["Temp"] = F(np.full((nx, ny), float(Tini)))
    st["Eg_avg"] = F(np.broadcast_to(eg, (nx, ny, ng)))
    st["Eg_edgV"] = F(np.broadcast_to(eg, (nx + 1, ny, ng)))
    st["Eg_edgH"] = F(np.broadcast_to(eg, (nx, ny + 1, ng)))
    st["Fxg_edgV"], st["Fyg_edgH"] = zeros(nx + 1, ny, ng), zeros(nx, ny + 1, ng)
    third = 1.0 / 3.0
    st["fg_avg_xx"], st["fg_avg_yy"] = F(np.full((nx, ny, ng), third)), F(np.full((nx, ny, ng), third))
    st["fg_edgV_xx"], st["fg_edgV_xy"] = F(np.full((nx + 1, ny, ng), third)), zeros(nx + 1, ny, ng)
    st["fg_edgH_yy"], st["fg_edgH_xy"] = F(np.full((nx, ny + 1, ng), third)), zeros(nx, ny + 1, ng)
    for s, v in zip(SIDES, (-0.5, -0.5, 0.5, 0.5)):
        n = ny if s in "LR" else nx
        k = SIDES.index(s)
        st["Cg_" + s] = F(np.full((n, ng), v if bc_type[k] == 0 else 0.0))
        st["Cb_" + s] = F(np.full(n, v if bc_type[k] == 0 else 0.0))
    st.update(mgqd_in_calc(st["I_edgV"], st["I_edgH"], Omega_x, Omega_y, quad_weight, c, comp_unit, bc_type))
    st.update(gqd_in_calc(st))
    st["E_avg"] = E0.copy(order="F")
    st["E_edgV"] = F(np.broadcast_to(E0[:1, :1], (nx + 1, ny)))
    st["E_edgH"] = F(np.broadcast_to(E0[:1, :1], (nx, ny + 1)))
    st["Fx_edgV"], st["Fy_edgH"] = zeros(nx + 1, ny), zeros(nx, ny + 1)
    st["KapE_Bar"], st["GQD_Src"], st["KapE_Bar_dT"] = zeros(nx, ny), zeros(nx, ny), zeros(nx, ny)
    return st


def mlqd_steps(st, Omega_x, Omega_y, quad_weight, Delx, Dely, Nu_g, kappa_mult, cV, Kap0, comp_unit, c, Delt, steps,
               Theta=1.0, conv_type=2, conv_ho=1e-10, conv_lo=1e-10, conv_gr1=1e-14, conv_gr2=1e-15, maxit_rte=50,
               maxit_mloqd=50, maxit_gloqd=20, chi=0.7, line_src=2.0, E_Bound_Low=0.0, T_Bound_Low=0.0,
               use_line_search=True, use_safety_search=False, kapE_dT_flag=True, bc_type=(0, 0, 0, 0),
               bcT=(0.0, 0.0, 0.0, 0.0), threads=4, solver=1):
    """Time steps of TRT_MLQD_ALGORITHM with run_type 'mlqd' (ALGORITHMS.f08:389-416, 518-572, 670-836), on
    the state dict of mlqd_init (updated in place).  Per step: the _old copies (:395-416), OLD_MGQD_COEFS and
    OLD_GREY_COEFS; then outer iterations, each (from the second on) TRANSPORT_SCB + COLLAPSE_INTENSITIES
    (+ RT_BC_UPDATE, MGQD_In_Calc, GQD_In_Calc when a side is reflective) + fg_Calc + Cg_Calc, then MGQD
    iterations of MLOQD_FV (solved directly), COLLAPSE_MG_EF, Cbar_Calc, GREY_COEFS, EGP_FV_NEWT and
    MATERIAL_UPDATE with CONVERGENCE(conv_lo) on T and the MGQD E, then CONVERGENCE(conv_ho) on T and the
    transport E.  cV is a scalar or an (nx, ny) array.  Returns one dict per step (Temp, E_avg, HO_E_avg,
    RT_Its, MGQD_Its per outer iteration, EGP_Its per MGQD iteration, the last MGQD T/E norms of each outer
    iteration, the outer T/E norms).  solver: the sweep's cell solve (0 = Gaussian elimination, 1 = closed
    form)."""
    nx, ny = st["Temp"].shape
    nm, ng = len(Omega_x), len(Nu_g) - 1
    A = F(np.outer(Delx, Dely))
    cv = F(np.broadcast_to(cV, (nx, ny))) if np.ndim(cV) else float(cV)
    KapE, rt_src, Bg = material_update(st["Temp"], Nu_g, kappa_mult, comp_unit)   # TEMP_INIT
    MGQD_Src = F(4.0 * np.pi * KapE * Bg)
    rt_start = 2
    hist = []
    for _ in range(steps):
        Temp_old = st["Temp"].copy(order="F")
        I_crn_old = st["I_crn"].copy(order="F")
        od = {k + "_old": F(st[k]).copy(order="F") for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV",
                                                              "Fyg_edgH") + MLOQD_FACTORS}
        od.update(KapE_old=KapE.copy(order="F"), KapR_old=KapE.copy(order="F"), Src_old=MGQD_Src.copy(order="F"),
                  Delx=Delx, Dely=Dely, A=A)
        E_avg_old, GQD_Src_old, KapE_Bar_old = st["E_avg"].copy(order="F"), st["GQD_Src"].copy(order="F"), \
            st["KapE_Bar"].copy(order="F")
        old = old_mgqd_coefs(od, c, Delt, Theta)
        Gold_Hat, Rhat_old = old_grey_coefs(c, Delt, Theta, cv, A, old["G_old"], Temp_old, KapE_Bar_old, E_avg_old,
                                            GQD_Src_old)
        T_rt1, T_rt2, E_rt1, E_rt2 = zeros(nx, ny), zeros(nx, ny), zeros(nx, ny), zeros(nx, ny)
        rt_its, rt_conv = 0, False
        mg_hist, egp_hist, lo_norms = [], [], []
        while not rt_conv and rt_its < maxit_rte:
            rt_its += 1
            if rt_its >= rt_start:
                Src_in = F(np.repeat(np.repeat(rt_src, 2, axis=0), 2, axis=1)[:, :, None, :].repeat(nm, axis=2))
                s = transport_scb(st["I_edgV"], st["I_edgH"], st["Ic_edgV"], st["Ic_edgH"], Omega_x, Omega_y, Delx,
                                  Dely, A, KapE, Src_in, I_crn_old, c, Delt, threads=threads, solver=solver)
                for k in ("I_crn", "I_edgV", "I_edgH", "Ic_edgV", "Ic_edgH"):
                    st[k] = s[k]
                m = collapse_intensities(s["I_avg"], s["I_edgV"], s["I_edgH"], Omega_x, Omega_y, quad_weight,
                                         comp_unit, threads=threads)
                st["HO_E_avg"] = m["E_avg"]
                if max(bc_type) > 0:
                    st["I_edgV"], st["I_edgH"], st["Ic_edgV"], st["Ic_edgH"] = rt_bc_update(
                        bc_type, bcT[0], bcT[1], bcT[2], bcT[3], comp_unit, Nu_g, st["I_edgV"], st["I_edgH"],
                        st["Ic_edgV"], st["Ic_edgH"])
                    st.update(mgqd_in_calc(st["I_edgV"], st["I_edgH"], Omega_x, Omega_y, quad_weight, c, comp_unit,
                                           bc_type))
                    st.update(gqd_in_calc(st))
                st.update({k: v for k, v in fg_calc(m, c).items() if k != "fg_avg_xy"})
                st.update(cg_calc(st["I_edgV"], st["I_edgH"], Omega_x, Omega_y, quad_weight, comp_unit, bc_type))
            E_mg1, E_mg2 = st["HO_E_avg"].copy(order="F"), zeros(nx, ny)
            T_mg1, T_mg2 = st["Temp"].copy(order="F"), zeros(nx, ny)
            mg_its, mg_conv = 0, False
            while not mg_conv and mg_its < maxit_mloqd:
                mg_its += 1
                d = {k: st[k] for k in MLOQD_FACTORS + MLOQD_BOUNDARY + ("Eg_avg", "Eg_edgV", "Eg_edgH")}
                d.update(Src=MGQD_Src, KapE=KapE, KapR=KapE, Delx=Delx, Dely=Dely, A=A, G_old=old["G_old"],
                         Pold_L=old["Pold_L"], Pold_B=old["Pold_B"], Pold_R=old["Pold_R"], Pold_T=old["Pold_T"],
                         Eg_avg_old=od["Eg_avg_old"], Fxg_edgV_old=od["Fxg_edgV_old"], Fyg_edgH_old=od["Fyg_edgH_old"])
                sol = mloqd_fv(d, c, Delt, Theta, res_calc=False, solver=0)
                for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH"):
                    st[k] = sol[k]
                mg = collapse_mg_ef(st)
                cb = cbar_calc(st)
                KapE_bar_MGQDold = st["KapE_Bar"].copy(order="F")
                gd = dict(st, Fxg_edgV_old=od["Fxg_edgV_old"], Fyg_edgH_old=od["Fyg_edgH_old"], KapE=KapE, KapR=KapE,
                          A=A, Pold_L=old["Pold_L"], Pold_R=old["Pold_R"], Pold_B=old["Pold_B"], Pold_T=old["Pold_T"])
                gc = grey_coefs(gd, c, Delt, Theta)
                g = dict(gc, **cb)
                for k in ("E_avg", "E_edgV", "E_edgH", "Fx_edgV", "Fy_edgH"):
                    g[k] = mg[k]
                for k in ("E_in_", "F_in_"):
                    for s_ in SIDES:
                        g[k + s_] = st[k + s_]
                g.update(Temp=st["Temp"], Temp_Mold=T_mg2, KapE_bar_Mold=KapE_bar_MGQDold, Delx=Delx, Dely=Dely, A=A,
                         Gold_Hat=Gold_Hat, Rhat_old=Rhat_old)
                o = egp_fv_newt(g, Theta, Delt, Kap0, cv, comp_unit, Chi=chi, line_src=line_src,
                                E_Bound_Low=E_Bound_Low, T_Bound_Low=T_Bound_Low, Eps1=conv_gr1, Eps2=conv_gr2,
                                Maxits=maxit_gloqd, MGQD_It=mg_its, Use_Line_Search=use_line_search,
                                Use_Safety_Search=use_safety_search, Res_Calc=False, kapE_dT_flag=kapE_dT_flag)
                for k in EGP_STATE:
                    st[k] = o[k]
                st["GQD_Src"], st["KapE_Bar_dT"] = o["Q_bar"], o["KapE_Bar_dT"]
                st.update({k: gc[k] for k in GREY_D + GREY_P})
                st.update(cb)
                st["MGQD_E_avg"] = mg["E_avg"]
                egp_hist.append(o["Its"])
                KapE, rt_src, Bg = material_update(st["Temp"], Nu_g, kappa_mult, comp_unit)
                MGQD_Src = F(4.0 * np.pi * KapE * Bg)
                tc, tn_lo, _ = convergence(conv_type, conv_lo, st["Temp"], T_mg1, T_mg2, mg_its)
                ec, en_lo, _ = convergence(conv_type, conv_lo, mg["E_avg"], E_mg1, E_mg2, mg_its)
                mg_conv = tc and ec
                E_mg2, E_mg1 = E_mg1, mg["E_avg"].copy(order="F")
                T_mg2, T_mg1 = T_mg1, st["Temp"].copy(order="F")
            mg_hist.append(mg_its)
            lo_norms.append((tn_lo, en_lo))
            tc, tn, _ = convergence(conv_type, conv_ho, st["Temp"], T_rt1, T_rt2, rt_its)
            ec, en, _ = convergence(conv_type, conv_ho, st["HO_E_avg"], E_rt1, E_rt2, rt_its)
            rt_conv = tc and ec
            E_rt2, E_rt1 = E_rt1, st["HO_E_avg"].copy(order="F")
            T_rt2, T_rt1 = T_rt1, st["Temp"].copy(order="F")
        hist.append(dict(Temp=st["Temp"].copy(order="F"), E_avg=st["E_avg"].copy(order="F"),
                         HO_E_avg=st["HO_E_avg"].copy(order="F"), Eg_avg=st["Eg_avg"].copy(order="F"),
                         RT_Its=rt_its, MGQD_Its=mg_hist, EGP_Its=egp_hist, T_norm=tn, E_norm=en,
                         MGQD_norms=lo_norms))
    st["KapE"], st["MGQD_Src"] = KapE, MGQD_Src
    return hist


# ------------------------------------------------------------------------------------------------
# Reduced-order model: POD of snapshots and its reconstruction.
# ------------------------------------------------------------------------------------------------

def pod_calc(data, n_t, n_g, clen, g):
    """POD_Calc with SVD_Calc_Cntr (Decomposer/DecompSrc/POD_ROUTINES.c:75-120, LA_ROUTINES.c:50-170): the
    columns of block g (gdat_reform, LA_ROUTINES.c:279-294) of data(clen, n_g, n_t) (n_g = 0: one block),
    centred by their mean over t (summed in t order), then the thin SVD (LAPACK, as dgesvd).  Returns
    (center(clen), umat(clen, k), sig(k), vtmat(k, n_t)), k = min(clen, n_t)."""
    ng = max(n_g, 1)
    d = np.asarray(data, dtype=np.float64).reshape(-1, order="F")
    X = np.empty((clen, n_t), order="F")
    for t in range(n_t):
        p = g * clen + t * ng * clen
        X[:, t] = d[p:p + clen]
    center = np.zeros(clen)
    for t in range(n_t):
        center = center + X[:, t]
    center = center / float(n_t)
    Xc = X - center[:, None]
    U, S, VT = np.linalg.svd(Xc, full_matrices=False)
    return center, F(U), S.copy(), F(VT)


def pod_reconstruct(C, S, U, V, rank, length, N_g, N_t, t, PODgsum):
    """POD_RECONSTRUCT (MainSrc/POD_ROUTINES.f08:372-432), with its loop order: modes in order, each term
    (S U) V added to a zeroed vector, then the centring vector; t is 1-based."""
    C, S, U, V = (np.asarray(a, dtype=np.float64).reshape(-1, order="F") for a in (C, S, U, V))
    dat = np.zeros(length)
    if PODgsum == 0:
        glen = length // N_g
        p2 = p3 = 0
        for g in range(N_g):
            rg = int(rank[g])
            p4 = N_t * p3 + (t - 1) * rg
            for r in range(rg):
                seg = slice(g * glen, (g + 1) * glen)
                dat[seg] = dat[seg] + (S[p3 + r] * U[p2:p2 + glen]) * V[p4 + r]
                p2 += glen
            p3 += rg
    else:
        r1 = int(rank[0])
        for r in range(r1):
            dat = dat + (S[r] * U[r * length:(r + 1) * length]) * V[r + (t - 1) * r1]
    return dat + C


def dmd_reconstruct(L, B, W, C, rank, length, N_g, DMDgsum, Time):
    """DMD_RECONSTRUCT (MainSrc/DMD_ROUTINES.f08:28-109): dat = Re(sum_r B(r) W(., r) exp(L(r) Time)) + C, modes
    in order, each term (B W) e with the complex products written out (re = ac - bd, im = ad + bc) and
    e = exp(L Time) evaluated once per mode (with the host's libm, as the library does)."""
    import math
    L, B, W = (np.asarray(a, dtype=np.complex128).reshape(-1, order="F") for a in (L, B, W))
    C = np.asarray(C, dtype=np.float64).reshape(-1, order="F")
    nb = N_g if DMDgsum == 0 else 1
    glen = length // nb
    re, im = np.zeros(length), np.zeros(length)
    p3 = 0
    for g in range(nb):
        for r in range(int(rank[g])):
            b, lam = B[p3 + r], L[p3 + r]
            zr, zi = lam.real * Time, lam.imag * Time
            m = math.exp(zr)
            er, ei = m * math.cos(zi), m * math.sin(zi)
            w = W[glen * (p3 + r):glen * (p3 + r + 1)]
            pr = b.real * w.real - b.imag * w.imag
            pi = b.real * w.imag + b.imag * w.real
            seg = slice(g * glen, (g + 1) * glen)
            re[seg] = re[seg] + (pr * er - pi * ei)
            im[seg] = im[seg] + (pr * ei + pi * er)
        p3 += int(rank[g])
    return re + C


def _omega(lam, delt):
    """Omega_Calc (DMD_ROUTINES.c:100-152): log(lambda)/delt with the reference's argument branches."""
    import math
    pi = 4.0 * math.atan(1.0)
    c, r = lam.imag, lam.real
    if c == 0.0:
        if r > 0.0:
            return complex(math.log(abs(r)) / delt, 0.0)
        if r < 0.0:
            return complex(math.log(abs(r)), pi) / delt
        return 0j
    if r == 0.0:
        return complex(math.log(abs(c)), pi / 2.0 if c > 0.0 else 3.0 * pi / 2.0) / delt
    theta = math.atan(abs(c) / abs(r))
    radius = math.sqrt(r ** 2 + c ** 2)
    if r < 0.0 < c:
        theta = pi - theta
    elif r < 0.0 and c < 0.0:
        theta += pi
    elif r > 0.0 > c:
        theta = 2.0 * pi - theta
    return complex(math.log(radius), theta) / delt


def dmd_calc(data, N_t, N_g, clen, g, base_subtract=0, svd_eps=-1.0, delt=1.0):
    """DMD_Calc, Coef_Calc and Omega_Calc (Decomposer/DecompSrc/DMD_ROUTINES.c:100-470) restated with numpy/LAPACK:
    X, Y (snapshots 0..n-1 and 1..n less the base vector), thin SVD of X truncated by SVD_Rank_Calc's rule,
    A~ = U^T Y V S^-1, eig(A~), modes Y V S^-1 W~ / lambda and U W~, amplitudes W~ b = U^T a0, omega."""
    ng = max(N_g, 1)
    d = np.asarray(data, dtype=np.float64).reshape(-1, order="F")
    col = lambda t: d[g * clen + t * ng * clen:g * clen + t * ng * clen + clen]
    shift = 2 if base_subtract else 1
    n = N_t - shift
    cvec = col(N_t - 1).copy() if base_subtract else np.zeros(clen)
    X = np.stack([col(t) - cvec for t in range(n)], axis=1)
    Y = np.stack([col(t + 1) - cvec for t in range(n)], axis=1)
    U, S, VT = np.linalg.svd(X, full_matrices=False)
    k = len(S)
    xr = k
    if svd_eps >= 0.0:
        fsum = np.sqrt(np.sum(S ** 2))
        for i in range(k):
            if np.sqrt(np.sum(S[i:] ** 2)) / fsum <= svd_eps:
                xr = i
                break
    Ur = U[:, :xr]
    XV = VT[:xr].T / S[:xr]
    Xm = Y @ XV
    At = Ur.T @ Xm
    lam, Wt = np.linalg.eig(At)
    wmat = (Xm @ Wt) / lam
    wmat_proj = Ur @ Wt
    a0 = col(0) if N_g > 0 else col(0) - cvec
    b = np.linalg.solve(Wt, Ur.T @ a0)
    omega = np.array([_omega(x, delt) for x in lam])
    return dict(lambda_=lam, omega=omega, b=b, wmat=wmat, wmat_proj=wmat_proj, umat=Ur, wmat_tild=Wt, cvec=cvec)


def _bilinear(f11, f12, f21, f22, x, x1, x2, y, y1, y2):
    """BILINEAR_INTERPOLATE (MainSrc/GRID_FUNCTIONS.f08:366-401), its branches and operation order."""
    if (x2 - x1) == 0.0:
        if (y2 - y1) == 0.0:
            return f11
        yy1, yy2 = y - y1, y2 - y
        return (f11 * yy2 + f12 * yy1) / (y2 - y1)
    if (y2 - y1) == 0.0:
        xx1, xx2 = x - x1, x2 - x
        return (f11 * xx2 + f21 * xx1) / (x2 - x1)
    xx1, xx2, yy1, yy2 = x - x1, x2 - x, y - y1, y2 - y
    return (f11 * xx2 * yy2 + f21 * xx1 * yy2 + f12 * xx2 * yy1 + f22 * xx1 * yy1) / ((x2 - x1) * (y2 - y1))


def fmap(f1, Grid1, Grid2, GMap, VMap, Glen1, Glen2, flen2):
    """FMAP (MainSrc/GRID_FUNCTIONS.f08:14-44), the Fortran loop with 1-based maps."""
    f1 = np.asarray(f1, dtype=np.float64).reshape(-1, order="F")
    G1, G2 = np.asarray(Grid1, dtype=np.float64), np.asarray(Grid2, dtype=np.float64)
    GM, VM = np.asarray(GMap).reshape(-1, order="F"), np.asarray(VMap).reshape(-1, order="F")
    f2 = np.zeros(flen2)
    for i in range(flen2 // Glen2):
        p1 = i * Glen1
        for j in range(1, Glen2 + 1):
            f2[i * Glen2 + j - 1] = _bilinear(
                f1[p1 + VM[4 * j - 4] - 1], f1[p1 + VM[4 * j - 2] - 1], f1[p1 + VM[4 * j - 3] - 1],
                f1[p1 + VM[4 * j - 1] - 1], G2[2 * j - 2], G1[GM[4 * j - 4] - 1], G1[GM[4 * j - 1] - 1], G2[2 * j - 1],
                G1[GM[4 * j - 4]], G1[GM[4 * j - 1]])
    return f2


def linear_interpolation(v1, v2, xm, x1, x2):
    """LINEAR_INTERPOLATION (MainSrc/GRID_FUNCTIONS.f08:819-836): v1 + (xm - x1) (v2 - v1) / (x2 - x1)."""
    v1, v2 = np.asarray(v1, dtype=np.float64), np.asarray(v2, dtype=np.float64)
    return v1 + (xm - x1) * (v2 - v1) / (x2 - x1)


def gridmap_gen(kind, Delx, Dely, N_x, N_y):
    """GRIDMAP_GEN_AVG (kind 0) / _EDGV (1) / _EDGH (2), MainSrc/GRID_FUNCTIONS.f08:49-133: (x, y) pairs."""
    xloc = [0.0] * N_x
    if kind == 1:
        for i in range(1, N_x):
            xloc[i] = xloc[i - 1] + Delx[i - 1]
    else:
        xloc[0] = Delx[0] / 2.0
        for i in range(1, N_x):
            xloc[i] = xloc[i - 1] + (Delx[i - 1] + Delx[i]) / 2.0
    out, yloc = [], 0.0
    for j in range(N_y):
        if kind != 2:
            yloc = yloc + Dely[j] / 2.0
        for i in range(N_x):
            out += [xloc[i], yloc]
        if kind != 2:
            yloc = yloc + Dely[j] / 2.0
        elif j + 1 < N_y:
            yloc = yloc + Dely[j]
    return np.array(out)


def map_grids(Grid1, Grid2, xlen1, len1=None, len2=None):
    """MAP_GRIDS (MainSrc/GRID_FUNCTIONS.f08:222-327): GMap (1-based x indices of the four bracketing points of
    grid 1 for every grid-2 point) and VMap = (GMap + 1) / 2.  len1 / len2 (default: the arrays' lengths) are the
    reference's counts of values searched and mapped, which its boundary maps set below the arrays' lengths."""
    import math
    len1 = len(Grid1) if len1 is None else len1
    len2 = len(Grid2) if len2 is None else len2
    G1 = lambda i: Grid1[i - 1]
    G2 = lambda j: Grid2[j - 1]
    Map = []
    for j in range(1, len2 + 1, 2):
        d, l1 = np.finfo(np.float64).max, 0
        for i in range(1, len1 + 1, 2):
            ddx, ddy = G1(i) - G2(j), G1(i + 1) - G2(j + 1)   # DIST's integer powers are products
            r = abs(math.sqrt(ddx * ddx + ddy * ddy))
            if r < d:
                d, l1 = r, i
        dx, dy = G1(l1) - G2(j), G1(l1 + 1) - G2(j + 1)
        if dx < -1e-10:
            if dy < -1e-10:
                l = [l1, l1 + 2, l1 + xlen1, l1 + xlen1 + 2]
            elif dy > 1e-10:
                l = [l1 - xlen1, l1 - xlen1 + 2, l1, l1 + 2]
            else:
                l = [l1, l1 + 2, l1, l1 + 2]
        elif dx > 1e-10:
            if dy < -1e-10:
                l = [l1 - 2, l1, l1 - 2 + xlen1, l1 + xlen1]
            elif dy > 1e-10:
                l = [l1 - xlen1 - 2, l1 - xlen1, l1 - 2, l1]
            else:
                l = [l1 - 2, l1, l1 - 2, l1]
        else:
            if dy < -1e-10:
                l = [l1, l1, l1 + xlen1, l1 + xlen1]
            elif dy > 1e-10:
                l = [l1 - xlen1, l1 - xlen1, l1, l1]
            else:
                l = [l1, l1, l1, l1]
        Map += l
    Map = np.array(Map, dtype=np.int32)
    return Map, (Map + 1) // 2


def gridmap_gen_bnd(side, Del, pos, N):
    """GRIDMAP_GEN_LR_BND (side 0, x = pos) / GRIDMAP_GEN_BT_BND (side 1, y = pos),
    MainSrc/GRID_FUNCTIONS.f08:158-200: the side's N points at the midpoints of Del."""
    out, loc = [], 0.0
    for i in range(N):
        loc = loc + Del[i] / 2.0
        out += [pos, loc] if side == 0 else [loc, pos]
        loc = loc + Del[i] / 2.0
    return np.array(out)


def generate_grids_xy(Delx_d, Dely_d, Delx, Dely, xlen_d, ylen_d, xlen, ylen):
    """GENERATE_GRIDS_XY (MainSrc/GRID_FUNCTIONS.f08:689-749), its calls in order, on square grids (N_x = N_y,
    dN_x = dN_y): the reference's boundary maps pass the left side's counts for all four sides and read past the
    point sets elsewhere.  Returns the dict of point sets and maps keyed by the reference's names."""
    dN_x, dN_y, N_x, N_y = len(Delx_d), len(Dely_d), len(Delx), len(Dely)
    assert N_x == N_y and dN_x == dN_y, "the reference's boundary maps are defined on square grids"
    Dx2, Dy2 = [0.0] + list(Delx_d) + [0.0], [0.0] + list(Dely_d) + [0.0]
    o = {"Sim_Grid_Avg": gridmap_gen(0, Delx, Dely, N_x, N_y), "Sim_Grid_EdgV": gridmap_gen(1, Delx, Dely, N_x + 1, N_y),
         "Sim_Grid_EdgH": gridmap_gen(2, Delx, Dely, N_x, N_y + 1),
         "Sim_Grid_Bnds": np.concatenate([gridmap_gen_bnd(0, Dely, 0.0, N_y), gridmap_gen_bnd(1, Delx, 0.0, N_x),
                                          gridmap_gen_bnd(0, Dely, ylen, N_y), gridmap_gen_bnd(1, Delx, xlen, N_x)]),
         "Dat_Grid_Avg": gridmap_gen(0, Dx2, Dy2, dN_x + 2, dN_y + 2),
         "Dat_Grid_EdgV": gridmap_gen(1, Delx_d, Dy2, dN_x + 1, dN_y + 2),
         "Dat_Grid_EdgH": gridmap_gen(2, Dx2, Dely_d, dN_x + 2, dN_y + 1),
         "Dat_Grid_Bnds": np.concatenate([gridmap_gen_bnd(0, Dy2, 0.0, dN_y + 2), gridmap_gen_bnd(1, Dx2, 0.0, dN_x + 2),
                                          gridmap_gen_bnd(0, Dy2, ylen_d, dN_y + 2),
                                          gridmap_gen_bnd(1, Dx2, xlen_d, dN_x + 2)])}
    for k, xl in (("Avg", 2 * (dN_x + 2)), ("EdgV", 2 * (dN_x + 1)), ("EdgH", 2 * (dN_x + 2))):
        o["GMap_xy" + k], o["VMap_xy" + k] = map_grids(o["Dat_Grid_" + k], o["Sim_Grid_" + k], xl)
    gm, vm = np.zeros(8 * (N_x + N_y), dtype=np.int32), np.zeros(8 * (N_x + N_y), dtype=np.int32)
    for go, do, so, xl in ((0, 0, 0, 2), (4 * N_y, 2 * dN_y + 4, 2 * N_y, 0),
                           (4 * (N_y + N_x), 2 * (dN_y + dN_x) + 8, 2 * (N_y + N_x), 2),
                           (8 * N_y + 4 * N_x, 4 * dN_y + 2 * dN_x + 12, 4 * N_y + 2 * N_x, 0)):
        g, v = map_grids(o["Dat_Grid_Bnds"][do:], o["Sim_Grid_Bnds"][so:], xl, 2 * dN_y + 2, 2 * N_y)
        gm[go:go + g.size], vm[go:go + v.size] = g, v
    o["GMap_xyBnds"], o["VMap_xyBnds"] = gm, vm
    return o


def generate_grids_t(Delt_d, Delt, Start_Time_d, Start_Time, dN_t, N_t):
    """GENERATE_GRIDS_T (MainSrc/GRID_FUNCTIONS.f08:754-814): (Sim_TGrid, Dat_TGrid, TMap(2 N_t), 1-based)."""
    dat = [Start_Time_d + Delt_d]
    for _ in range(1, dN_t):
        dat.append(dat[-1] + Delt_d)
    sim = [Start_Time + Delt]
    for _ in range(1, N_t):
        sim.append(sim[-1] + Delt)
    tmap = []
    for ts in sim:
        if dat[0] >= ts:
            tmap += [1, 1]
        elif dat[-1] <= ts:
            tmap += [dN_t, dN_t]
        else:
            for j in range(1, dN_t):
                if abs(dat[j] - ts) / dat[j] <= 1e-14:
                    tmap += [j + 1, j + 1]
                    break
                if dat[j] > ts:
                    tmap += [j + 1, j]
                    break
    return np.array(sim), np.array(dat), np.array(tmap, dtype=np.int32)


def _blocks(f, N_g, N_y, N_x):
    return np.asarray(f, dtype=np.float64).reshape(N_g, N_y, N_x)


def collect_lr_bnd(f, N_g, N_y, N_x):
    """COLLECT_LR_BND: first and last value of every row, row by row."""
    b = _blocks(f, N_g, N_y, N_x)
    return np.stack([b[:, :, 0], b[:, :, -1]], axis=2).reshape(-1)


def collect_bt_bnd(f, N_g, N_y, N_x):
    """COLLECT_BT_BND: the first and the last row of every block."""
    b = _blocks(f, N_g, N_y, N_x)
    return np.concatenate([b[:, 0, :], b[:, -1, :]], axis=1).reshape(-1)


def collect_crn_bnd(f, N_g, N_y, N_x):
    """COLLECT_CRN_BND: the four corners of every block (bottom left, bottom right, top left, top right)."""
    b = _blocks(f, N_g, N_y, N_x)
    return np.stack([b[:, 0, 0], b[:, 0, -1], b[:, -1, 0], b[:, -1, -1]], axis=1).reshape(-1)


def extnd_bt_bnd(f, N_g, N_y, N_x):
    """EXTND_BT_BND: the first and last rows repeated below and above."""
    b = _blocks(f, N_g, N_y, N_x)
    return np.concatenate([b[:, :1, :], b, b[:, -1:, :]], axis=1).reshape(-1)


def extnd_lr_bnd(f, N_g, N_y, N_x):
    """EXTND_LR_BND: the first and last values of every row repeated left and right."""
    b = _blocks(f, N_g, N_y, N_x)
    return np.concatenate([b[:, :, :1], b, b[:, :, -1:]], axis=2).reshape(-1)


def avg_apnd_bnd(f, LR, BT, Crn, N_g, N_y, N_x):
    """AVG_APND_BND: the field framed by its left/right values (2 per row), bottom/top rows and 4 corners."""
    b = _blocks(f, N_g, N_y, N_x)
    lr = np.asarray(LR).reshape(N_g, N_y, 2)
    bt = np.asarray(BT).reshape(N_g, 2, N_x)
    c = np.asarray(Crn).reshape(N_g, 4)
    out = np.empty((N_g, N_y + 2, N_x + 2))
    out[:, 0, 0], out[:, 0, -1], out[:, -1, 0], out[:, -1, -1] = c[:, 0], c[:, 1], c[:, 2], c[:, 3]
    out[:, 0, 1:-1], out[:, -1, 1:-1] = bt[:, 0], bt[:, 1]
    out[:, 1:-1, 0], out[:, 1:-1, -1] = lr[:, :, 0], lr[:, :, 1]
    out[:, 1:-1, 1:-1] = b
    return out.reshape(-1)


# ------------------------------------------------------------------------------------------------------------
# Online reconstruction drivers: POD_RECONSTRUCT_fg / _BCg (MainSrc/POD_ROUTINES.f08:28-353) and
# DMD_RECONSTRUCT_fg / _BCg (MainSrc/DMD_ROUTINES.f08:131-424), their calls in order.  dec maps a field name
# (avg_xx, edgV_xx, avg_yy, edgH_yy, edgV_xy, edgH_xy, BCg) to its decomposition; grids is the dict of
# generate_grids_xy; tgrids = (Sim_TGrid, Dat_TGrid, TMap) of generate_grids_t.
# ------------------------------------------------------------------------------------------------------------
FG_FIELDS = ("avg_xx", "edgV_xx", "avg_yy", "edgH_yy", "edgV_xy", "edgH_xy")


def _pod_at_step(d, length, dN_g, dN_t, t, PODgsum, tgrids):
    """POD_RECONSTRUCT at data level TMap(2t) when TMap(2t-1) equals it, else at both levels with
    LINEAR_INTERPOLATION between them (the drivers' time handling)."""
    C, S, U, V, rank = d
    sim_t, dat_t, tmap = tgrids
    a, b = int(tmap[2 * t - 2]), int(tmap[2 * t - 1])
    if a == b:
        return pod_reconstruct(C, S, U, V, rank, length, dN_g, dN_t, b, PODgsum)
    f = pod_reconstruct(C, S, U, V, rank, length, dN_g, dN_t, a, PODgsum)
    f3 = pod_reconstruct(C, S, U, V, rank, length, dN_g, dN_t, b, PODgsum)
    return linear_interpolation(f, f3, sim_t[t - 1], dat_t[a - 1], dat_t[b - 1])


def _fg_map(rec, dN_x, dN_y, dN_g, N_x, N_y, N_g, grids):
    out = {}
    G = grids
    nv1, nv2 = (dN_x + 1) * (dN_y + 2), (N_x + 1) * N_y
    f = rec("edgV_xx", (dN_x + 1) * dN_y * dN_g)
    xxbnd = collect_lr_bnd(f, dN_g, dN_y, dN_x + 1)
    f2 = extnd_bt_bnd(f, dN_g, dN_y, dN_x + 1)
    out["fg_edgV_xx"] = fmap(f2, G["Dat_Grid_EdgV"], G["Sim_Grid_EdgV"], G["GMap_xyEdgV"], G["VMap_xyEdgV"], nv1, nv2,
                             nv2 * N_g)
    f = rec("edgV_xy", (dN_x + 1) * dN_y * dN_g)
    f2 = extnd_bt_bnd(f, dN_g, dN_y, dN_x + 1)
    out["fg_edgV_xy"] = fmap(f2, G["Dat_Grid_EdgV"], G["Sim_Grid_EdgV"], G["GMap_xyEdgV"], G["VMap_xyEdgV"], nv1, nv2,
                             nv2 * N_g)
    nh1, nh2 = (dN_x + 2) * (dN_y + 1), N_x * (N_y + 1)
    f = rec("edgH_yy", dN_x * (dN_y + 1) * dN_g)
    yybnd = collect_bt_bnd(f, dN_g, dN_y + 1, dN_x)
    f2 = extnd_lr_bnd(f, dN_g, dN_y + 1, dN_x)
    out["fg_edgH_yy"] = fmap(f2, G["Dat_Grid_EdgH"], G["Sim_Grid_EdgH"], G["GMap_xyEdgH"], G["VMap_xyEdgH"], nh1, nh2,
                             nh2 * N_g)
    f = rec("edgH_xy", dN_x * (dN_y + 1) * dN_g)
    f2 = extnd_lr_bnd(f, dN_g, dN_y + 1, dN_x)
    out["fg_edgH_xy"] = fmap(f2, G["Dat_Grid_EdgH"], G["Sim_Grid_EdgH"], G["GMap_xyEdgH"], G["VMap_xyEdgH"], nh1, nh2,
                             nh2 * N_g)
    na1, na2 = (dN_x + 2) * (dN_y + 2), N_x * N_y
    f = rec("avg_xx", dN_x * dN_y * dN_g)
    f2 = avg_apnd_bnd(f, xxbnd, collect_bt_bnd(f, dN_g, dN_y, dN_x), collect_crn_bnd(f, dN_g, dN_y, dN_x), dN_g, dN_y,
                      dN_x)
    out["fg_avg_xx"] = fmap(f2, G["Dat_Grid_Avg"], G["Sim_Grid_Avg"], G["GMap_xyAvg"], G["VMap_xyAvg"], na1, na2,
                            na2 * N_g)
    f = rec("avg_yy", dN_x * dN_y * dN_g)
    f2 = avg_apnd_bnd(f, collect_lr_bnd(f, dN_g, dN_y, dN_x), yybnd, collect_crn_bnd(f, dN_g, dN_y, dN_x), dN_g, dN_y,
                      dN_x)
    out["fg_avg_yy"] = fmap(f2, G["Dat_Grid_Avg"], G["Sim_Grid_Avg"], G["GMap_xyAvg"], G["VMap_xyAvg"], na1, na2,
                            na2 * N_g)
    return out


def _bcg_map(BC, dN_x, dN_y, dN_g, N_x, N_y, N_g, grids):
    """The BCg drivers' side vectors CL2, CB2, CR2, CT2 (each side with its end values repeated) and their FMAPs."""
    sides = ([], [], [], [])
    p = 0
    for _ in range(dN_g):
        for s, n in enumerate((dN_y, dN_x, dN_y, dN_x)):
            sides[s].append(BC[p])
            for _i in range(n):
                p += 1
                sides[s].append(BC[p - 1])
            sides[s].append(BC[p - 1])
    G = grids
    out = []
    for s, (do, so, mo, n1, n2) in enumerate(((0, 0, 0, dN_y + 2, N_y),
                                              (2 * dN_y + 4, 2 * N_y, 4 * N_y, dN_x + 2, N_x),
                                              (2 * (dN_y + dN_x) + 8, 2 * (N_y + N_x), 4 * (N_y + N_x), dN_y + 2, N_y),
                                              (4 * dN_y + 2 * dN_x + 12, 4 * N_y + 2 * N_x, 8 * N_y + 4 * N_x, dN_x + 2,
                                               N_x))):
        out.append(fmap(np.array(sides[s]), G["Dat_Grid_Bnds"][do:], G["Sim_Grid_Bnds"][so:], G["GMap_xyBnds"][mo:],
                        G["VMap_xyBnds"][mo:], n1, n2, N_g * n2))
    return tuple(out)


def rrank_calc(sig, eps):
    """RRANK_CALC (MainSrc/POD_ROUTINES.f08:791-819): sums of squares in index order, the first i whose tail
    norm is at most eps times the total norm."""
    import math
    n = len(sig)
    sum1 = 0.0
    for v in sig:
        sum1 = sum1 + v * v
    eps2 = eps * math.sqrt(sum1)
    for i in range(1, n + 1):
        sum2 = 0.0
        for j in range(i + 1, n + 1):
            sum2 = sum2 + sig[j - 1] * sig[j - 1]
        if math.sqrt(sum2) <= eps2:
            return i
    return n


def pod_reconstruct_fg(dec, dN, N, t, PODgsum, grids, tgrids):
    """POD_RECONSTRUCT_fg: dN = (dN_x, dN_y, dN_g, dN_t), N = (N_x, N_y, N_g); dec[name] = (C, S, U, V, rank)."""
    dN_x, dN_y, dN_g, dN_t = dN
    rec = lambda name, length: _pod_at_step(dec[name], length, dN_g, dN_t, t, PODgsum, tgrids)
    return _fg_map(rec, dN_x, dN_y, dN_g, *N, grids)


def pod_reconstruct_bcg(dec, dN, N, t, PODgsum, grids, tgrids):
    """POD_RECONSTRUCT_BCg: (Cg_L, Cg_B, Cg_R, Cg_T); dec = (C, S, U, V, rank) of the boundary factors."""
    dN_x, dN_y, dN_g, dN_t = dN
    BC = _pod_at_step(dec, dN_g * 2 * (dN_x + dN_y), dN_g, dN_t, t, PODgsum, tgrids)
    return _bcg_map(BC, dN_x, dN_y, dN_g, *N, grids)


def dmd_reconstruct_fg(dec, dN, N, Time, DMDgsum, grids):
    """DMD_RECONSTRUCT_fg: dN = (dN_x, dN_y, dN_g), N = (N_x, N_y, N_g); dec[name] = (L, B, W, C, rank)."""
    dN_x, dN_y, dN_g = dN
    rec = lambda name, length: dmd_reconstruct(*dec[name], length, N[2], DMDgsum, Time)
    return _fg_map(rec, dN_x, dN_y, dN_g, *N, grids)


def dmd_reconstruct_bcg(dec, dN, N, Time, DMDgsum, grids):
    """DMD_RECONSTRUCT_BCg: (Cg_L, Cg_B, Cg_R, Cg_T); dec = (L, B, W, C, rank) of the boundary factors."""
    dN_x, dN_y, dN_g = dN
    BC = dmd_reconstruct(*dec, dN_g * 2 * (dN_x + dN_y), N[2], DMDgsum, Time)
    return _bcg_map(BC, dN_x, dN_y, dN_g, *N, grids)
