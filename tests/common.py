"""Shared helpers of the tests: inputs for a problem in the reference layouts, comparison norms."""
import importlib
import json
import os

import numpy as np

pkg = importlib.import_module("2d_trt_rom_system_b200")
HERE = os.path.dirname(os.path.abspath(__file__))

C = pkg.problems.C_LIGHT
CU = pkg.problems.COMP_UNIT


def rel_err(a, b, scale=None):
    """max |a - b| / max |b| (or / scale)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.max(np.abs(b)) if scale is None else scale
    if s == 0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / s)


def rel_err_per_group(a, b, gaxis=-1):
    """Worst over groups of max|a-b| / max|b| within each group slice (intensity arrays span many
    orders of magnitude across groups)."""
    a = np.moveaxis(np.asarray(a), gaxis, 0)
    b = np.moveaxis(np.asarray(b), gaxis, 0)
    worst = 0.0
    for ag, bg in zip(a, b):
        s = np.max(np.abs(bg))
        d = np.max(np.abs(ag - bg))
        worst = max(worst, d / s if s > 0 else d)
    return worst


def sweep_inputs(prob, T=None, seed=0, random_old=True):
    """Reference-layout inputs of one sweep for a Problem: dict with Omega_x, Omega_y, w, Delx, Dely, A,
    KapE_in, src_iso, Src_in (per corner), I_crn_old, Ic_edgV, Ic_edgH, I_edgV, I_edgH, c, dt."""
    ox, oy, w = prob.directions()
    nx, ny, nm, ng = prob.nx, prob.ny, len(ox), prob.ng
    rng = np.random.default_rng(seed)
    if T is None:
        T = np.full((nx, ny), prob.T0)
    kap, src = prob.material(T)
    Src_in = np.asfortranarray(np.repeat(np.repeat(src, 2, axis=0), 2, axis=1)[:, :, None, :].repeat(nm, axis=2))
    nu = prob.nu_eV
    Bg0 = np.array([pkg.problems.bg_planck(prob.T0 * 1e3, nu[g], nu[g + 1]) for g in range(ng)])
    if random_old:
        I_old = np.asfortranarray(Bg0[None, None, None, :] * rng.uniform(0.5, 1.5, (2 * nx, 2 * ny, nm, ng)))
    else:
        I_old = np.asfortranarray(np.broadcast_to(Bg0, (2 * nx, 2 * ny, nm, ng)).copy())
    # RT_INIT: everything Bg(Tini), then Planck inflow faces (RT_BC_UPDATE with all-zero types)
    Ic_edgV = np.asfortranarray(np.broadcast_to(Bg0, (nx + 1, 2 * ny, nm, ng)).copy())
    Ic_edgH = np.asfortranarray(np.broadcast_to(Bg0, (2 * nx, ny + 1, nm, ng)).copy())
    I_edgV = np.asfortranarray(np.broadcast_to(Bg0, (nx + 1, ny, nm, ng)).copy())
    I_edgH = np.asfortranarray(np.broadcast_to(Bg0, (nx, ny + 1, nm, ng)).copy())
    bT = [t * 1e3 for t in prob.bcT]
    from oracle import oracle as O
    I_edgV, I_edgH, Ic_edgV, Ic_edgH = O.rt_bc_update((0, 0, 0, 0), bT[0], bT[1], bT[2], bT[3], CU, nu, I_edgV, I_edgH,
                                                      Ic_edgV, Ic_edgH)
    delx, dely = prob.delx, prob.dely
    return dict(Omega_x=ox, Omega_y=oy, w=w, Delx=delx, Dely=dely, A=np.asfortranarray(np.outer(delx, dely)),
                KapE_in=kap, src_iso=src, Src_in=Src_in, I_crn_old=I_old, Ic_edgV=Ic_edgV, Ic_edgH=Ic_edgH,
                I_edgV=I_edgV, I_edgH=I_edgH, c=C, dt=prob.dt, nu=nu, bcT_eV=bT)


def oracle_full(inp, solver=0, res_calc=False, bc_type=(0, 0, 0, 0), threads=4):
    """Oracle sweep + COLLAPSE_INTENSITIES + fg_Calc + Cg_Calc + MGQD_In_Calc + GQD_In_Calc."""
    from oracle import oracle as O
    s = O.transport_scb(inp["I_edgV"], inp["I_edgH"], inp["Ic_edgV"], inp["Ic_edgH"], inp["Omega_x"], inp["Omega_y"],
                        inp["Delx"], inp["Dely"], inp["A"], inp["KapE_in"], inp["Src_in"], inp["I_crn_old"], inp["c"],
                        inp["dt"], threads=threads, res_calc=res_calc, solver=solver)
    m = O.collapse_intensities(s["I_avg"], s["I_edgV"], s["I_edgH"], inp["Omega_x"], inp["Omega_y"], inp["w"], CU,
                               threads=threads)
    s.update(m)
    s.update(O.fg_calc(m, inp["c"], threads=threads))
    s.update(O.cg_calc(s["I_edgV"], s["I_edgH"], inp["Omega_x"], inp["Omega_y"], inp["w"], CU, bc_type,
                       threads=threads))
    s.update(O.mgqd_in_calc(s["I_edgV"], s["I_edgH"], inp["Omega_x"], inp["Omega_y"], inp["w"], inp["c"], CU, bc_type,
                            threads=threads))
    s.update(O.gqd_in_calc(s))
    return s


def load_golden():
    with open(os.path.join(HERE, "golden", "scb_exact.json")) as f:
        return json.load(f)["cases"]


def golden_arrays(case):
    nx, ny, nm, ng = case["nx"], case["ny"], case["nm"], case["ng"]

    def arr(name, shape):
        return np.asfortranarray(np.array(case[name], dtype=np.float64).reshape(shape, order="F"))

    d = dict(nx=nx, ny=ny, nm=nm, ng=ng, c=case["c"], dt=case["dt"], comp_unit=case["comp_unit"])
    d["Omega_x"] = arr("Omega_x", (nm,))
    d["Omega_y"] = arr("Omega_y", (nm,))
    d["w"] = arr("w", (nm,))
    d["Delx"] = arr("dx", (nx,))
    d["Dely"] = arr("dy", (ny,))
    d["A"] = arr("A", (nx, ny))
    d["KapE_in"] = arr("kap", (nx, ny, ng))
    src = arr("src", (nx, ny, ng))
    d["src_iso"] = src
    d["Src_in"] = np.asfortranarray(np.repeat(np.repeat(src, 2, axis=0), 2, axis=1)[:, :, None, :].repeat(nm, axis=2))
    d["I_crn_old"] = arr("I_crn_old", (2 * nx, 2 * ny, nm, ng))
    bV = arr("bV", (2, 2 * ny, nm, ng))
    bH = arr("bH", (2, 2 * nx, nm, ng))
    IcV = np.zeros((nx + 1, 2 * ny, nm, ng), order="F")
    IcV[0] = bV[0]
    IcV[nx] = bV[1]
    IcH = np.zeros((2 * nx, ny + 1, nm, ng), order="F")
    IcH[:, 0] = bH[0]
    IcH[:, ny] = bH[1]
    d["Ic_edgV"], d["Ic_edgH"] = IcV, IcH
    d["I_edgV"] = np.asfortranarray(0.5 * (IcV[:, 0::2] + IcV[:, 1::2]))
    d["I_edgH"] = np.asfortranarray(0.5 * (IcH[0::2] + IcH[1::2]))
    exp = {}
    for k, shp in (("I_crn", (2 * nx, 2 * ny, nm, ng)), ("I_avg", (nx, ny, nm, ng)),
                   ("Ic_edgV", (nx + 1, 2 * ny, nm, ng)), ("Ic_edgH", (2 * nx, ny + 1, nm, ng)),
                   ("Eg_avg", (nx, ny, ng)), ("fg_avg_xx", (nx, ny, ng)), ("fg_avg_yy", (nx, ny, ng)),
                   ("fg_avg_xy", (nx, ny, ng)), ("Eg_edgV", (nx + 1, ny, ng)), ("Fxg_edgV", (nx + 1, ny, ng)),
                   ("Eg_edgH", (nx, ny + 1, ng))):
        exp[k] = arr(k, shp)
    return d, exp
