"""Device time stepping with the reference's transport-only outer iteration (run_type 'tr_no_qd'):
the FP64 library against the oracle's restatement of the same loop (ALGORITHMS.f08, UPDATES.f08
MEB_SOLVE / MATERIAL_UPDATE, CONVERGENCE_CHECKS.f08), and the FP32 sweep's temperature error against
FP64.  Bars: FP64 temperatures and energies <= 1e-12 relative to the oracle (the device and host
exponentials differ by an ulp); iteration counts equal; mixed precision <= 1e-5 relative in T."""
import numpy as np
import pytest

from common import CU, C, pkg, sweep_inputs

pytestmark = pytest.mark.gpu


def _oracle_state(prob, ts):
    d = sweep_inputs(prob, random_old=False)     # RT_INIT at prob.T0 (= ts.Tini_eV): Bg(Tini) + Planck faces
    return d, dict(I_crn=d["I_crn_old"].copy(order="F"), Ic_edgV=d["Ic_edgV"], Ic_edgH=d["Ic_edgH"],
                   I_edgV=d["I_edgV"], I_edgH=d["I_edgH"],
                   Temp=np.full((prob.nx, prob.ny), ts.Tini_eV, order="F"))


def _device(prob, ts, precision, conv_type, conv_ho, maxit, bc_type=(0, 0, 0, 0), law=0):
    ox, oy, w = prob.directions()
    s = pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng, precision=precision)
    s.init_state(ts.Tini_eV, list(ts.bcT_eV), CU, ts.nu_eV)
    s.tstep_setup(ts.nu_eV, ts.kappa_mult, ts.cv, np.full((prob.nx, prob.ny), ts.Tini_eV), ts.Kap0, CU, C, ts.dt,
                  BC_Type=bc_type, bcT=ts.bcT_eV, conv_type=conv_type, conv_ho=conv_ho, maxit_rte=maxit, law=law)
    return s


FG_KEYS = ("fg_avg_xx", "fg_avg_yy", "fg_avg_xy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy")


def _rel_per_group(a, b):
    """Worst over the groups that carry intensity of max|a - b| / max|b| within the group."""
    worst = 0.0
    for g in range(b.shape[-1]):
        s = np.max(np.abs(b[..., g]))
        if s > 0:
            worst = max(worst, float(np.max(np.abs(a[..., g] - b[..., g])) / s))
        else:
            assert np.max(np.abs(a[..., g])) == 0
    return worst


def test_config0_time_loop_matches_gaussian_elimination_oracle_every_step(oracle):
    """Config 0 as specified: 20x20 cells on [0,6]^2, 17 log-spaced groups, S8, the opacity law
    kappa0 (1 - exp(-nu/T)) / (nu^3 sqrt(T)) with kappa0 = 10 / 1000 (central block), c_v = 0.5, Planck
    T = 1 keV on the left, T0 = 0.01 keV, backward Euler dt = 2e-3, 10 steps.  The oracle sweeps with
    SCB_BGEN + Gaussian elimination (the reference's form, no code shared with the library).  Every
    step: temperature, transport E, every QD factor and the corner state within 1e-12.  The
    transport-only iteration is not accelerated, so each step runs a fixed 20 outer iterations on both
    sides (in this optically thick problem it converges one cell per few dozen iterations)."""
    prob = pkg.problems.config0()
    ts = pkg.problems.config_timestep_setup(prob)
    d, st = _oracle_state(prob, ts)
    rec = []
    ref = oracle.tr_no_qd_steps(st, d["Omega_x"], d["Omega_y"], d["w"], d["Delx"], d["Dely"], ts.nu_eV, ts.kappa_mult,
                                ts.cv, ts.Kap0, CU, C, ts.dt, 10, conv_type=2, conv_ho=0.0, maxit=20, threads=8,
                                solver=0, law=1, record=rec)
    with _device(prob, ts, "fp64", 2, 0.0, 20, law=1) as s:
        for (T_ref, E_ref, its_ref, _, _), r in zip(ref, rec):
            its, _, _ = s.tstep()
            assert its == its_ref == 20
            assert _rel(s.temperature(), T_ref) < 1e-12
            m = s.moments(("E_avg", "Eg_avg") + FG_KEYS)
            assert _rel(m["E_avg"], E_ref) < 1e-12
            assert _rel_per_group(m["Eg_avg"], r["Eg_avg"]) < 1e-12
            for k in FG_KEYS:
                assert np.max(np.abs(m[k] - r[k])) < 1e-12, k
            assert _rel_per_group(s.get_state(), r["I_crn"]) < 1e-12
    T_final = ref[-1][0]
    assert T_final.max() > 10 * ts.Tini_eV      # the hot boundary has heated the left of the domain


def test_config0_time_loop_mixed_precision_temperature_error():
    """The same 10 steps with the FP32 sweep (FP64 moment sums, energy balance and material): temperature
    within 1e-5 of the FP64 run at every step."""
    prob = pkg.problems.config0()
    ts = pkg.problems.config_timestep_setup(prob)
    out = {}
    for prec in ("fp64", "fp32"):
        with _device(prob, ts, prec, 2, 0.0, 20, law=1) as s:
            out[prec] = [(s.tstep(), s.temperature()) for _ in range(10)]
    for (_, T64), (_, T32) in zip(out["fp64"], out["fp32"]):
        assert _rel(T32, T64) < 1e-5


def _rel(a, b):
    return float(np.max(np.abs(a - b) / np.abs(b)))


@pytest.mark.parametrize("shape", [(7, 6, 3, "S8"), (5, 9, 2, "S12")])
def test_tstep_fp64_matches_oracle_fixed_iterations(oracle, shape):
    nx, ny, G, quad = shape
    prob = pkg.problems.random_small(22, nx, ny, G, quad)
    ts = pkg.problems.fc_timestep_setup(prob)
    d, st = _oracle_state(prob, ts)
    ref = oracle.tr_no_qd_steps(st, d["Omega_x"], d["Omega_y"], d["w"], d["Delx"], d["Dely"], ts.nu_eV, ts.kappa_mult,
                                ts.cv, ts.Kap0, CU, C, ts.dt, 3, conv_type=2, conv_ho=0.0, maxit=5)
    with _device(prob, ts, "fp64", 2, 0.0, 5) as s:
        for T_ref, E_ref, its_ref, _, _ in ref:
            its, _, _ = s.tstep()
            assert its == its_ref == 5
            assert _rel(s.temperature(), T_ref) < 1e-12
            assert _rel(s.moments(["E_avg"])["E_avg"], E_ref) < 1e-12
        I = s.get_state()
    assert _rel(I, st["I_crn"]) < 1e-11


def test_tstep_convergence_path_matches_oracle(oracle):
    prob = pkg.problems.random_small(23, 6, 6, 3, "S8")
    ts = pkg.problems.fc_timestep_setup(prob)
    d, st = _oracle_state(prob, ts)
    for conv_type in (1, 2, 3):
        d, st = _oracle_state(prob, ts)
        ref = oracle.tr_no_qd_steps(st, d["Omega_x"], d["Omega_y"], d["w"], d["Delx"], d["Dely"], ts.nu_eV,
                                    ts.kappa_mult, ts.cv, ts.Kap0, CU, C, ts.dt, 2, conv_type=conv_type,
                                    conv_ho=1e-7, maxit=60)
        with _device(prob, ts, "fp64", conv_type, 1e-7, 60) as s:
            for T_ref, _, its_ref, tn_ref, en_ref in ref:
                its, tn, en = s.tstep()
                assert its == its_ref < 60, conv_type
                assert tn == pytest.approx(tn_ref, rel=1e-6) and en == pytest.approx(en_ref, rel=1e-6)
                assert _rel(s.temperature(), T_ref) < 1e-12


def test_tstep_reflective_sides_match_oracle(oracle):
    prob = pkg.problems.random_small(24, 6, 5, 2, "S8")
    ts = pkg.problems.fc_timestep_setup(prob)
    bc = (0, 1, 0, 1)
    d, st = _oracle_state(prob, ts)
    ref = oracle.tr_no_qd_steps(st, d["Omega_x"], d["Omega_y"], d["w"], d["Delx"], d["Dely"], ts.nu_eV, ts.kappa_mult,
                                ts.cv, ts.Kap0, CU, C, ts.dt, 2, conv_type=2, conv_ho=0.0, maxit=4, bc_type=bc,
                                bcT=ts.bcT_eV)
    with _device(prob, ts, "fp64", 2, 0.0, 4, bc_type=bc) as s:
        for T_ref, _, _, _, _ in ref:
            s.tstep()
            assert _rel(s.temperature(), T_ref) < 1e-12


def test_tstep_mixed_precision_temperature_error():
    """C0 grid and groups with the reference physics, 3 time steps: the FP32 sweep with FP64 moment sums,
    MEB and material update stays within 1e-5 of the FP64 temperatures."""
    prob = pkg.problems.config0()
    ts = pkg.problems.fc_timestep_setup(prob)
    out = {}
    for prec in ("fp64", "fp32"):
        with _device(prob, ts, prec, 2, 0.0, 8) as s:
            out[prec] = [(s.tstep(), s.temperature()) for _ in range(3)]
    for (_, T64), (_, T32) in zip(out["fp64"], out["fp32"]):
        assert _rel(T32, T64) < 1e-5


def test_tstep_argument_and_state_errors():
    prob = pkg.problems.random_small(25, 3, 3, 1, "S8")
    ox, oy, w = prob.directions()
    with pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng) as s:
        with pytest.raises(pkg.TrtError):
            s.tstep()                               # no setup
        with pytest.raises(pkg.TrtError):
            s.temperature()
        ts = pkg.problems.fc_timestep_setup(prob)
        with pytest.raises(pkg.TrtError):
            s.tstep_setup(ts.nu_eV, ts.kappa_mult, ts.cv, np.ones((3, 3)), ts.Kap0, CU, C, ts.dt, conv_type=4)
