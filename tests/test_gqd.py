"""Grey low-order side: COLLAPSE_MG_EF (MainSrc/MLOQD_SOLVES.f08:687-730), Cbar_Calc, OLD_GREY_COEFS,
GREY_COEFS and the Newton iteration EGP_FV_NEWT of the effective grey problem (MainSrc/GLOQD_SOLVES.f08).

The grey problems are built the way TRT_MLQD_ALGORITHM builds them (ALGORITHMS.f08:686-728): a multigroup
low-order solution, its group sums, boundary factors and grey coefficients, with temperatures, old-state
terms and material constants chosen so that the Newton iteration converges.
"""
import numpy as np
import pytest

from common import pkg

P = pkg.problems
CU = 1e13


def multigroup_state(nx, ny, ng, seed, oracle, theta=1.0):
    d, c, dt, th = P.mgqd_inputs(nx, ny, ng, seed=seed, theta=theta)
    d.update(oracle.old_mgqd_coefs(d, c, dt, th))
    m = oracle.mloqd_fv(d, c, dt, th)
    dd = dict(d)
    dd.update({k: m[k] for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH")})
    return dd, c, dt, th


def grey_problem(nx, ny, ng, seed, oracle, mgqd_it=2, theta=1.0):
    dd, c, dt, th = multigroup_state(nx, ny, ng, seed, oracle, theta)
    g = dict(oracle.grey_coefs(dd, c, dt, th))
    g.update(oracle.cbar_calc(dd))
    g.update(oracle.collapse_mg_ef(dd))
    for s in oracle.SIDES:
        g["E_in_" + s] = np.asfortranarray(dd["Eg_in_" + s].sum(axis=1))
        g["F_in_" + s] = np.asfortranarray(dd["Fg_in_" + s].sum(axis=1))
    rng = np.random.default_rng(seed)
    g["Temp"] = np.asfortranarray(rng.uniform(0.9, 1.1, (nx, ny)))
    g["Temp_Mold"] = np.asfortranarray(g["Temp"] * rng.uniform(0.9, 0.99, (nx, ny)))
    g["KapE_bar_Mold"] = np.asfortranarray(g["KapE_Bar"] * rng.uniform(0.9, 1.1, (nx, ny)))
    g["Delx"], g["Dely"], g["A"] = dd["Delx"], dd["Dely"], dd["A"]
    h, cc, pi, erg = 6.62613e-19, 2.99792458e2, np.pi, 6.24150934e11
    aR = 4 * (2 * pi ** 5 / (15 * cc ** 2 * h ** 3 * erg ** 4 * CU)) / cc
    # emission comparable to absorption, heat capacity comparable to the absorbed energy of a step
    kap0 = float(np.mean(cc * g["KapE_Bar"] * g["E_avg"]) / np.mean(15 * cc * aR * g["Temp"] / pi ** 4))
    cv = float(np.mean(cc * g["KapE_Bar"] * g["E_avg"]) * dt)
    Qold = 15 * kap0 * cc * aR * g["Temp"] / pi ** 4
    g["Gold_Hat"], g["Rhat_old"] = oracle.old_grey_coefs(c, dt, th, cv, dd["A"], dd["G_old"], g["Temp"], g["KapE_Bar"],
                                                         g["E_avg"] * 0.9, Qold)
    return g, dict(Theta=th, Delt=dt, Kap0=kap0, cv=cv, Comp_Unit=CU, MGQD_It=mgqd_it)


# ------------------------------------------------------------------------------------------------ CPU

def test_grey_coefficients_oracle_definitions(oracle):
    dd, c, dt, th = multigroup_state(7, 5, 4, 3, oracle, theta=0.5)
    col = oracle.collapse_mg_ef(dd)
    assert np.allclose(col["E_avg"], dd["Eg_avg"].sum(axis=2), rtol=1e-14, atol=0)
    assert np.allclose(col["Fy_edgH"], dd["Fyg_edgH"].sum(axis=2), rtol=1e-13, atol=1e-13 * np.abs(col["Fy_edgH"]).max())
    cb = oracle.cbar_calc(dd)
    q = dd["Eg_edgV"][0] - dd["Eg_in_L"]
    assert np.allclose(cb["Cb_L"], (dd["Cg_L"] * q).sum(axis=1) / q.sum(axis=1), rtol=1e-12)
    gc = oracle.grey_coefs(dd, c, dt, th)
    tk = dd["KapR"] + 1.0 / (th * c * dt)
    assert np.allclose(gc["KapE_Bar"], (dd["KapE"] * dd["Eg_avg"]).sum(axis=2) / dd["Eg_avg"].sum(axis=2), rtol=1e-13)
    assert np.allclose(gc["DR_xx"], (dd["fg_edgV_xx"][1:] * dd["Eg_edgV"][1:] / tk).sum(axis=2)
                       / dd["Eg_edgV"][1:].sum(axis=2), rtol=1e-12)
    w = dd["A"][:, :, None] / (2 * th * c * dt)
    PT = ((w * dd["Fyg_edgH_old"][:, 1:] + dd["Pold_T"]) / tk).sum(axis=2)
    assert np.allclose(gc["PT"], PT, rtol=1e-12, atol=1e-12 * np.abs(PT).max())


@pytest.mark.parametrize("mgqd_it", [1, 2])
def test_oracle_newton_converges_and_zeroes_its_residuals(mgqd_it, oracle):
    g, kw = grey_problem(6, 5, 4, 1, oracle, mgqd_it)
    o = oracle.egp_fv_newt(g, **kw)
    assert o["Its"] < 10
    D, R = o["Deltas"], o["dresiduals"]
    assert D[-1, 0] <= 1e-14 * np.abs(o["Temp"]).max() + 1e-15
    # the residuals of the last iterate's equations are at round-off relative to the first
    assert (R[-1] <= 1e-9 * R[0] + 1e-12).all()
    if mgqd_it == 1:   # KapE_Bar_dT = 0: the problem is linear, one step solves it
        assert o["Its"] <= 3 and np.abs(o["KapE_Bar_dT"]).max() == 0.0
    else:
        assert o["Its"] >= 3 and np.abs(o["KapE_Bar_dT"]).max() > 0.0


# ------------------------------------------------------------------------------------------------ GPU

def device_egp(g, kw, **opts):
    o = {k: np.asfortranarray(np.array(g[k], dtype=np.float64)) for k in
         ("E_avg", "E_edgV", "E_edgH", "Temp", "KapE_Bar", "Fx_edgV", "Fy_edgH")}
    nx, ny = g["Temp"].shape
    o["Q_bar"], o["KapE_Bar_dT"] = np.zeros((nx, ny), order="F"), np.zeros((nx, ny), order="F")
    a = dict(Chi=0.7, line_src=2.0, E_Bound_Low=0.0, T_Bound_Low=0.0, Eps1=1e-14, Eps2=1e-15, Maxits=10,
             Use_Line_Search=True, Use_Safety_Search=False, Res_Calc=True, kapE_dT_flag=True, Fin_Weight=1.0,
             Ein_Weight=1.0)
    a.update(opts)
    its, kits, D, R = pkg.EGP_FV_NEWT(
        o["E_avg"], o["E_edgV"], o["E_edgH"], o["Temp"], o["KapE_Bar"], o["Fx_edgV"], o["Fy_edgH"], o["Q_bar"],
        o["KapE_Bar_dT"], g["Temp_Mold"], g["KapE_bar_Mold"], kw["Theta"], kw["Delt"], g["Delx"], g["Dely"], g["A"],
        *[g["Cb_" + s] for s in "LBRT"], *[g["E_in_" + s] for s in "LBRT"], *[g["F_in_" + s] for s in "LBRT"],
        *[g[k] for k in ("DC_xx", "DL_xx", "DR_xx", "DC_yy", "DB_yy", "DT_yy", "DL_xy", "DR_xy", "DB_xy", "DT_xy",
                         "PL", "PR", "PB", "PT", "Gold_Hat", "Rhat_old")],
        kw["Kap0"], kw["cv"], kw["Comp_Unit"], a["Chi"], a["line_src"], a["E_Bound_Low"], a["T_Bound_Low"], a["Eps1"],
        a["Eps2"], a["Maxits"], kw["MGQD_It"], a["Use_Line_Search"], a["Use_Safety_Search"], a["Res_Calc"],
        a["kapE_dT_flag"], a["Fin_Weight"], a["Ein_Weight"])
    o.update(Its=its, GQD_Kits=kits, Deltas=D, dresiduals=R)
    return o


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.gpu
def test_device_grey_coefficient_routines_match_oracle(oracle):
    dd, c, dt, th = multigroup_state(9, 7, 5, 4, oracle, theta=0.5)
    nx, ny, ng = dd["Eg_avg"].shape
    ref = oracle.collapse_mg_ef(dd)
    out = {k: np.zeros(v.shape, order="F") for k, v in ref.items()}
    pkg.COLLAPSE_MG_EF(dd["Eg_avg"], dd["Eg_edgV"], dd["Eg_edgH"], dd["Fxg_edgV"], dd["Fyg_edgH"], 1, *out.values())
    for k in ref:
        assert np.array_equal(out[k], ref[k]), k
    ref = oracle.cbar_calc(dd)
    out = {k: np.zeros(v.shape, order="F") for k, v in ref.items()}
    pkg.Cbar_Calc(*out.values(), *[dd["Cg_" + s] for s in "LBRT"], dd["Eg_avg"], dd["Eg_edgV"], dd["Eg_edgH"],
                  *[dd["Eg_in_" + s] for s in "LBRT"])
    for k in ref:
        assert np.array_equal(out[k], ref[k]), k
    ref = oracle.grey_coefs(dd, c, dt, th)
    out = {k: np.zeros(v.shape, order="F") for k, v in ref.items()}
    pkg.GREY_COEFS(*[dd[k] for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV_old", "Fyg_edgH_old", "fg_avg_xx",
                                     "fg_avg_yy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy", "KapE", "KapR",
                                     "A")],
                   c, dt, th, dd["Pold_L"], dd["Pold_R"], dd["Pold_B"], dd["Pold_T"], *out.values(), 1.0)
    for k in ref:
        assert rel(out[k], ref[k]) <= 1e-14, k
    rng = np.random.default_rng(5)
    T0, Kb, E0, Q0 = (np.asfortranarray(rng.uniform(0.5, 1.5, (nx, ny))) for _ in range(4))
    gh, rh = oracle.old_grey_coefs(c, dt, th, 3.0, dd["A"], dd["G_old"], T0, Kb, E0, Q0)
    ogh, orh = np.zeros((nx, ny), order="F"), np.zeros((nx, ny), order="F")
    pkg.OLD_GREY_COEFS(c, dt, th, 3.0, dd["A"], dd["G_old"], T0, Kb, E0, Q0, ogh, orh)
    assert rel(ogh, gh) <= 1e-14 and rel(orh, rh) <= 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("case", [(6, 5, 4, 1, 1), (6, 5, 4, 1, 2), (16, 12, 8, 2, 2), (11, 3, 5, 5, 3)])
def test_device_egp_newton_matches_oracle(case, oracle):
    nx, ny, ng, seed, mgqd_it = case
    g, kw = grey_problem(nx, ny, ng, seed, oracle, mgqd_it)
    ref = oracle.egp_fv_newt(g, **kw)
    out = device_egp(g, kw)
    assert ref["Its"] < 10 and out["Its"] == ref["Its"]
    for k in ("Temp", "E_avg", "E_edgV", "E_edgH", "Fx_edgV", "Fy_edgH", "KapE_Bar", "Q_bar", "KapE_Bar_dT"):
        assert rel(out[k], ref[k]) < 1e-9, k
    assert (out["GQD_Kits"] > 0).all()
    np.testing.assert_allclose(out["Deltas"][0], ref["Deltas"][0], rtol=1e-8)


@pytest.mark.gpu
def test_device_egp_without_line_search_and_with_safety_pass(oracle):
    g, kw = grey_problem(8, 6, 4, 6, oracle, 2)
    for opts in (dict(Use_Line_Search=False), dict(Use_Safety_Search=True, T_Bound_Low=0.5, E_Bound_Low=0.0)):
        ref = oracle.egp_fv_newt(g, **kw, **opts)
        out = device_egp(g, kw, **opts)
        assert out["Its"] == ref["Its"]
        for k in ("Temp", "E_avg", "Fx_edgV"):
            assert rel(out[k], ref[k]) < 1e-9, (opts, k)
        assert out["Temp"].min() >= 0.5 - 1e-12 or not opts.get("Use_Safety_Search")
