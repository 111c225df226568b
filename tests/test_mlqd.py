"""The mlqd time step (TRT_MLQD_ALGORITHM with run_type 'mlqd', MainSrc/ALGORITHMS.f08:389-416, 518-572,
670-836): one sweep per outer iteration after the first, MGQD iterations of MLOQD_FV, COLLAPSE_MG_EF,
Cbar_Calc, GREY_COEFS, EGP_FV_NEWT and MATERIAL_UPDATE, with the reference's convergence tests.

The device step (trt_mlqd_step, FP64 sweep) is checked against the oracle's restatement of the same loop
(oracle.mlqd_steps: the sweep restated, the multigroup system solved directly).  Both iterative solves on
the device stop at relative tolerances near 1e-13, so fields agree to 1e-9 relative, not bit for bit.

Problems: the reference's Fleck-Cummings material with Kappa_Mult = 1 (the grey emission Q_bar uses Kap0
without Kappa_Mult, so only a uniform material gives the grey problem the multigroup emission) on small
seeded grids, a hot left boundary and a warm initial temperature, where the MGQD iteration converges.
"""
import numpy as np
import pytest

from common import C, CU, pkg

P = pkg.problems


def setup_problem(nx, ny, G, quad, seed, Tini=100.0, bcT=(1000.0, 0.0, 0.0, 0.0)):
    prob = P.random_small(seed, nx, ny, G, quad)
    ts = P.fc_timestep_setup(prob, Tini_eV=Tini)
    km = np.ones((nx, ny), order="F")
    return prob, ts, km, tuple(bcT), P.fc_cv(1000.0)


def oracle_run(oracle, prob, ts, km, bcT, cv, steps, bc_type=(0, 0, 0, 0), **kw):
    ox, oy, w = prob.directions()
    st = oracle.mlqd_init(prob.nx, prob.ny, ox, oy, w, ts.nu_eV, ts.Tini_eV, CU, C, bc_type=bc_type, bcT=bcT)
    hist = oracle.mlqd_steps(st, ox, oy, w, prob.delx, prob.dely, ts.nu_eV, km, cv, ts.Kap0, CU, C, ts.dt, steps,
                             bc_type=bc_type, bcT=bcT, **kw)
    return st, hist


def device(prob, ts, km, bcT, cv, precision="fp64", bc_type=(0, 0, 0, 0), conv_type=2, conv_ho=0.0, maxit_rte=3,
           law=0, **kw):
    ox, oy, w = prob.directions()
    s = pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng, precision=precision)
    s.init_state(ts.Tini_eV, list(bcT), CU, ts.nu_eV)
    s.tstep_setup(ts.nu_eV, km, cv, np.full((prob.nx, prob.ny), ts.Tini_eV), ts.Kap0, CU, C, ts.dt,
                  BC_Type=bc_type, bcT=bcT, conv_type=conv_type, conv_ho=conv_ho, maxit_rte=maxit_rte, law=law)
    s.mlqd_setup(ts.Tini_eV, **kw)
    return s


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


# ------------------------------------------------------------------------------------------------ CPU

def test_oracle_mlqd_converges_and_heats_from_the_left(oracle):
    prob, ts, km, bcT, cv = setup_problem(8, 6, 10, "S8", 31)
    st, hist = oracle_run(oracle, prob, ts, km, bcT, cv, 2, conv_ho=1e-7, conv_lo=1e-8, maxit_rte=30,
                          maxit_mloqd=60)
    for h in hist:
        assert 2 <= h["RT_Its"] < 30 and max(h["MGQD_Its"]) < 60
        T = h["Temp"]
        assert np.isfinite(T).all() and T.min() > 0.5 * ts.Tini_eV and T.max() < 1000.0
        # the hot side is the left one
        assert T[0].mean() > T[-1].mean()
    # the first outer iteration of a step has no sweep; later ones do, so the transport E is no longer
    # the uniform field of RT_INIT
    assert np.ptp(hist[0]["HO_E_avg"]) > 0.1 * hist[0]["HO_E_avg"].max()


def test_oracle_mlqd_cell_heat_capacity_matches_scalar(oracle):
    prob, ts, km, bcT, cv = setup_problem(5, 4, 2, "S8", 32)
    _, h1 = oracle_run(oracle, prob, ts, km, bcT, cv, 1, conv_ho=0.0, conv_lo=0.0, maxit_rte=2, maxit_mloqd=2)
    _, h2 = oracle_run(oracle, prob, ts, km, bcT, np.full((5, 4), cv), 1, conv_ho=0.0, conv_lo=0.0, maxit_rte=2,
                       maxit_mloqd=2)
    assert np.array_equal(h1[0]["Temp"], h2[0]["Temp"])


# ------------------------------------------------------------------------------------------------ GPU

@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(7, 6, 3, "S8", 33), (6, 7, 4, "S12", 34)])
def test_mlqd_step_fp64_matches_oracle_fixed_iterations(oracle, shape):
    nx, ny, G, quad, seed = shape
    prob, ts, km, bcT, cv = setup_problem(nx, ny, G, quad, seed)
    st, ref = oracle_run(oracle, prob, ts, km, bcT, cv, 2, conv_ho=0.0, conv_lo=0.0, maxit_rte=3, maxit_mloqd=3)
    with device(prob, ts, km, bcT, cv, conv_ho=0.0, maxit_rte=3, conv_lo=0.0, maxit_mloqd=3) as s:
        for r in ref:
            out = s.mlqd_step()
            assert out["rt_its"] == r["RT_Its"] == 3 and out["sweeps"] == 2
            assert out["mgqd_per_outer"] == r["MGQD_Its"] == [3, 3, 3]
            # Newton iterations stop on a relative change of 1e-14; the iterative device solves and the
            # oracle's direct ones may cross that threshold one iteration apart
            assert len(out["egp_per_mgqd"]) == len(r["EGP_Its"])
            assert np.abs(np.subtract(out["egp_per_mgqd"], r["EGP_Its"])).max() <= 1
            assert out["mgqd_nonconv"] == 0
            assert rel(s.mlqd_field("Temp"), r["Temp"]) < 1e-9
            assert rel(s.mlqd_field("E_avg"), r["E_avg"]) < 1e-9
            assert rel(s.mlqd_field("HO_E_avg"), r["HO_E_avg"]) < 1e-9
            assert rel(s.mlqd_field("Eg_avg"), r["Eg_avg"]) < 1e-9
        for k in ("Fx_edgV", "Fy_edgH", "KapE_Bar", "GQD_Src", "Cb_L", "Cb_T", "Eg_edgV", "Fxg_edgV", "MGQD_Src"):
            assert rel(s.mlqd_field(k), st[k]) < 1e-8, k
        assert rel(s.get_state(), st["I_crn"]) < 1e-9


@pytest.mark.gpu
def test_mlqd_step_theta_half_matches_oracle(oracle):
    """Theta = 0.5 brings in every old-time term of OLD_MGQD_COEFS and OLD_GREY_COEFS (with Theta = 1 they
    vanish), including the KapE_Bar and GQD_Src that the reference leaves unset before the first step."""
    prob, ts, km, bcT, cv = setup_problem(7, 6, 4, "S8", 39)
    kw = dict(conv_lo=0.0, maxit_mloqd=3, Theta=0.5)
    st, ref = oracle_run(oracle, prob, ts, km, bcT, cv, 2, conv_ho=0.0, maxit_rte=3, **kw)
    with device(prob, ts, km, bcT, cv, conv_ho=0.0, maxit_rte=3, **kw) as s:
        for r in ref:
            s.mlqd_step()
            assert rel(s.mlqd_field("Temp"), r["Temp"]) < 1e-9
            assert rel(s.mlqd_field("E_avg"), r["E_avg"]) < 1e-9


@pytest.mark.gpu
def test_mlqd_convergence_path_matches_oracle(oracle):
    prob, ts, km, bcT, cv = setup_problem(8, 6, 10, "S8", 31)
    kw = dict(conv_lo=1e-8, maxit_mloqd=60)
    _, ref = oracle_run(oracle, prob, ts, km, bcT, cv, 2, conv_ho=1e-7, maxit_rte=30, **kw)
    with device(prob, ts, km, bcT, cv, conv_ho=1e-7, maxit_rte=30, **kw) as s:
        for r in ref:
            out = s.mlqd_step()
            assert out["rt_its"] == r["RT_Its"] < 30
            assert out["mgqd_per_outer"] == r["MGQD_Its"]
            # the multigroup solves converge; a Newton linear solve whose right-hand side has fallen to round-off
            # may end in a BiCGSTAB breakdown (counted in egp_nonconv), which leaves the iteration unharmed
            assert out["mgqd_nonconv"] == 0 and out["egp_nonconv"] == 0
            assert out["T_norm"] == pytest.approx(r["T_norm"], rel=1e-4, abs=1e-12)
            assert rel(s.mlqd_field("Temp"), r["Temp"]) < 1e-9


@pytest.mark.gpu
def test_mlqd_reflective_sides_and_no_kapE_dT(oracle):
    prob, ts, km, bcT, cv = setup_problem(6, 5, 2, "S8", 35)
    bc = (0, 1, 0, 1)
    kw = dict(conv_lo=0.0, maxit_mloqd=2, kapE_dT_flag=False)
    st, ref = oracle_run(oracle, prob, ts, km, bcT, cv, 2, bc_type=bc, conv_ho=0.0, maxit_rte=3, **kw)
    with device(prob, ts, km, bcT, cv, bc_type=bc, conv_ho=0.0, maxit_rte=3, **kw) as s:
        for r in ref:
            s.mlqd_step()
            assert rel(s.mlqd_field("Temp"), r["Temp"]) < 1e-9
        assert np.array_equal(s.mlqd_field("Cb_B"), st["Cb_B"]) and (st["Cb_B"] == 0).all()


@pytest.mark.gpu
def test_mlqd_mixed_precision_temperature_error():
    """FP32 sweep with the FP64 low-order solves against the FP64 step, converged."""
    prob, ts, km, bcT, cv = setup_problem(16, 16, 10, "S8", 36)
    kw = dict(conv_ho=1e-8, maxit_rte=40, conv_lo=1e-9, maxit_mloqd=80)
    T = {}
    for prec in ("fp64", "fp32"):
        with device(prob, ts, km, bcT, cv, precision=prec, **kw) as s:
            T[prec] = []
            for _ in range(3):
                s.mlqd_step()
                T[prec].append(s.mlqd_field("Temp"))
    for a, b in zip(T["fp32"], T["fp64"]):
        assert rel(a, b) < 1e-5


@pytest.mark.gpu
def test_mlqd_call_order_and_arguments():
    prob, ts, km, bcT, cv = setup_problem(4, 4, 2, "S8", 37)
    ox, oy, w = prob.directions()
    with pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng) as s:
        with pytest.raises(pkg.TrtError):
            s.mlqd_step()                    # no mlqd state yet
        with pytest.raises(pkg.TrtError):
            s.mlqd_setup(ts.Tini_eV)         # trt_tstep_setup has not run
        s.init_state(ts.Tini_eV, list(bcT), CU, ts.nu_eV)
        s.tstep_setup(ts.nu_eV, km, cv, np.full((4, 4), ts.Tini_eV), ts.Kap0, CU, C, ts.dt, bcT=bcT)
        with pytest.raises(pkg.TrtError):
            s.mlqd_setup(ts.Tini_eV, line_src=1.0)
        s.mlqd_setup(ts.Tini_eV, maxit_mloqd=2)
        with pytest.raises(pkg.TrtError):
            s.mlqd_field("no_such_field")
        s.mlqd_setup(ts.Tini_eV, maxit_mloqd=2)   # a second setup replaces the first
        assert s.mlqd_step()["rt_its"] >= 1
        with pytest.raises(pkg.TrtError):
            s.mlqd_put("fg_avg_xx", np.ones(3))                # wrong size
        with pytest.raises(pkg.TrtError):
            s.mlqd_put("no_such_factor", np.ones(16 * prob.ng))
        s.mlqd_put("fg_avg_xx", np.full(16 * prob.ng, 0.3))
        assert np.array_equal(s.moments(["fg_avg_xx"])["fg_avg_xx"], np.full((4, 4, prob.ng), 0.3))

