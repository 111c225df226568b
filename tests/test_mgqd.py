"""Low-order multigroup QD solve: MLOQD_FV / OLD_MGQD_COEFS (MainSrc/MLOQD_SOLVES.f08:12-362) with its
linear solver QD_FV (MainSrc/QD_SOLVERS.f08:40-538).

CPU tests pin the oracle through the reference's own residual formulas (written on the un-reduced
equations, MLOQD_SOLVES.f08:277-345); GPU tests compare the device solve with the oracle's direct solve.
"""
import numpy as np
import pytest

from common import pkg

P = pkg.problems

CASES = [  # nx, ny, ng, theta, seed, uniform grid
    (5, 4, 3, 1.0, 1, True),
    (12, 9, 6, 0.5, 2, False),
    (20, 20, 17, 1.0, 3, True),
    (1, 6, 2, 1.0, 4, False),
    (7, 1, 2, 0.5, 5, False),
]


def make(nx, ny, ng, theta, seed, uniform, oracle):
    d, c, dt, th = P.mgqd_inputs(nx, ny, ng, seed=seed, theta=theta, uniform=uniform)
    d.update(oracle.old_mgqd_coefs(d, c, dt, th))
    return d, c, dt, th


def eq_scale(d, o, c, dt, theta):
    """Per-group magnitude of the energy-balance terms (for relative residuals)."""
    return np.abs(d["A"][:, :, None] * (1 / (theta * dt) + c * d["KapE"]) * o["Eg_avg"]).max(axis=(0, 1))


def mom_scale(d, o, c, dt=2e-3, theta=1.0):
    """Magnitude of the terms of the momentum balances and boundary conditions (for relative residuals):
    the absorption term A (1/(theta c dt) + KapR) F / 2 and the pressure term c dy f E."""
    kr = np.abs(d["A"][:, :, None] * (1 / (theta * c * dt) + d["KapR"])).max()
    f = max(np.abs(o["Fxg_edgV"]).max(), np.abs(o["Fyg_edgH"]).max())
    e = max(np.abs(o["Eg_avg"]).max(), np.abs(o["Eg_edgV"]).max(), np.abs(o["Eg_edgH"]).max())
    fold = max(np.abs(d["Fxg_edgV_old"]).max(), np.abs(d["Fyg_edgH_old"]).max()) * d["A"].max() / (2 * theta * c * dt)
    pold = max(np.abs(d[k]).max() for k in ("Pold_L", "Pold_B", "Pold_R", "Pold_T"))
    return max(kr * f / 2, c * max(d["Delx"].max(), d["Dely"].max()) * e, fold, pold)


@pytest.mark.parametrize("case", CASES)
def test_oracle_solution_satisfies_the_reference_residual_equations(case, oracle):
    d, c, dt, th = make(*case, oracle)
    o = oracle.mloqd_fv(d, c, dt, th, res_calc=True, threads=2)
    R, RB = o["MGQD_Residual"], o["MGQD_BC_Residual"]
    # round-off level: the equations mix terms up to G_old ~ 1e6 times the result's magnitude
    assert (R[:, 0, 0] <= 1e-11 * eq_scale(d, o, c, dt, th)).all()
    assert R[:, 1:, 0].max() <= 1e-11 * mom_scale(d, o, c, dt, th)
    assert RB.max() <= 1e-11 * mom_scale(d, o, c, dt, th)
    assert (o["MGQD_Kits"] == -1).all()
    # the norms follow their definitions: max <= L2 <= L1 (per equation and group)
    assert (R[:, :, 0] <= R[:, :, 2] * (1 + 1e-12)).all() and (R[:, :, 2] <= R[:, :, 1] * (1 + 1e-12) + 1e-300).all()


def test_old_mgqd_coefs_oracle_matches_its_definition(oracle):
    nx, ny, ng = 6, 5, 3
    d, c, dt, _ = P.mgqd_inputs(nx, ny, ng, seed=9)
    o1 = oracle.old_mgqd_coefs(d, c, dt, 1.0)
    assert all(np.abs(v).max() == 0.0 for v in o1.values())      # (Theta-1)/Theta = 0: backward Euler
    th = 0.5
    o = oracle.old_mgqd_coefs(d, c, dt, th)
    w = (th - 1) / th
    dx, dy, A = d["Delx"][:, None, None], d["Dely"][None, :, None], d["A"][:, :, None]
    G = w * (dy * (d["Fxg_edgV_old"][1:] - d["Fxg_edgV_old"][:-1]) + dx * (d["Fyg_edgH_old"][:, 1:] - d["Fyg_edgH_old"][:, :-1])
             + A * (c * d["KapE_old"] * d["Eg_avg_old"] - d["Src_old"]))
    np.testing.assert_allclose(o["G_old"], G, rtol=1e-13, atol=1e-13 * np.abs(G).max())
    PL = w * (c * dy * (d["fg_avg_xx_old"] * d["Eg_avg_old"] - d["fg_edgV_xx_old"][:-1] * d["Eg_edgV_old"][:-1])
              + c * dx * (d["fg_edgH_xy_old"][:, 1:] * d["Eg_edgH_old"][:, 1:]
                          - d["fg_edgH_xy_old"][:, :-1] * d["Eg_edgH_old"][:, :-1]) / 2
              + A * (d["KapR_old"] * d["Fxg_edgV_old"][:-1]) / 2)
    np.testing.assert_allclose(o["Pold_L"], PL, rtol=1e-12, atol=1e-13 * np.abs(PL).max())


def test_oracle_direct_solve_is_independent_of_the_initial_guess(oracle):
    d, c, dt, th = make(8, 7, 4, 1.0, 11, False, oracle)
    a = oracle.mloqd_fv(d, c, dt, th)
    d2 = dict(d)
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH"):
        d2[k] = np.asfortranarray(np.zeros_like(d[k]))
    b = oracle.mloqd_fv(d2, c, dt, th)
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH"):
        assert np.array_equal(a[k], b[k])


# ------------------------------------------------------------------------------------------------ GPU

def call_device(d, c, dt, th, res_calc=True, fdt=1.0, fin=1.0, ein=1.0):
    nx, ny, ng = d["Eg_avg"].shape
    o = {k: np.asfortranarray(d[k].copy()) for k in ("Eg_avg", "Eg_edgV", "Eg_edgH")}
    o["Fxg_edgV"] = np.zeros((nx + 1, ny, ng), order="F")
    o["Fyg_edgH"] = np.zeros((nx, ny + 1, ng), order="F")
    o["MGQD_Residual"] = np.zeros((ng, 5, 5), order="F")
    o["MGQD_BC_Residual"] = np.zeros((ng, 4), order="F")
    o["MGQD_Kits"] = np.zeros(ng, dtype=np.int32)
    pkg.MLOQD_FV(o["Eg_avg"], o["Eg_edgV"], o["Eg_edgH"], o["Fxg_edgV"], o["Fyg_edgH"],
                 *[d[k] for k in ("fg_avg_xx", "fg_avg_yy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy",
                                  "Cg_L", "Cg_B", "Cg_R", "Cg_T", "Eg_in_L", "Eg_in_B", "Eg_in_R", "Eg_in_T",
                                  "Fg_in_L", "Fg_in_B", "Fg_in_R", "Fg_in_T", "Src", "KapE", "KapR", "Delx", "Dely",
                                  "A")],
                 c, dt, th, 1, res_calc, o["MGQD_Residual"], o["MGQD_BC_Residual"],
                 *[d[k] for k in ("G_old", "Pold_L", "Pold_B", "Pold_R", "Pold_T", "Eg_avg_old", "Fxg_edgV_old",
                                  "Fyg_edgH_old")],
                 o["MGQD_Kits"], fdt, fin, ein)
    return o


def rel_err(a, b):
    """max |a - b| over a group / max |b| over the group, maximised over groups."""
    ng = a.shape[-1]
    a2, b2 = a.reshape(-1, ng), b.reshape(-1, ng)
    return float((np.abs(a2 - b2).max(axis=0) / np.abs(b2).max(axis=0)).max())


@pytest.mark.gpu
# (100, 72): a fine level above the shared-memory V-cycle, in ragged tiles of the fused level passes
@pytest.mark.parametrize("case", CASES + [(48, 40, 12, 1.0, 6, False), (33, 64, 5, 0.5, 7, True),
                                          (100, 72, 3, 1.0, 8, False)])
def test_device_mloqd_fv_matches_oracle(case, oracle):
    d, c, dt, th = make(*case, oracle)
    ref = oracle.mloqd_fv(d, c, dt, th, res_calc=True, threads=4)
    out = call_device(d, c, dt, th)
    # the device iteration stops at a Jacobi-scaled residual of 1e-13 max|E|; the direct solution is
    # within the system's condition number times that
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH"):
        assert rel_err(out[k], ref[k]) < 1e-9, k
    assert (out["MGQD_Kits"] >= 1).all()
    R, RB = out["MGQD_Residual"], out["MGQD_BC_Residual"]
    assert (R[:, 0, 0] <= 1e-9 * eq_scale(d, ref, c, dt, th)).all()
    assert R[:, 1:, 0].max() <= 1e-9 * mom_scale(d, ref, c, dt, th)
    assert RB.max() <= 1e-9 * mom_scale(d, ref, c, dt, th)


@pytest.mark.gpu
def test_device_mloqd_fv_weights_and_thin_groups(oracle):
    # opacities down to 1e-6: diffusion-dominated groups (c dt / dx = 13), non-unit weights
    d, c, dt, th = P.mgqd_inputs(32, 32, 6, seed=21, kap_range=(1e-6, 1e2), uniform=True)
    d.update(oracle.old_mgqd_coefs(d, c, dt, th))
    ref = oracle.mloqd_fv(d, c, dt, th, Fdt_Weight=0.5, Fin_Weight=0.0, Ein_Weight=2.0, threads=4)
    out = call_device(d, c, dt, th, fdt=0.5, fin=0.0, ein=2.0)
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH"):
        assert rel_err(out[k], ref[k]) < 1e-9, k
    # the edge-elimination + multigrid preconditioner keeps thin and thick groups at a few iterations
    assert (out["MGQD_Kits"] <= 41).all()


@pytest.mark.gpu
def test_device_mloqd_fv_is_reproducible_and_guess_independent(oracle):
    d, c, dt, th = make(24, 17, 5, 1.0, 12, False, oracle)
    a = call_device(d, c, dt, th)
    b = call_device(d, c, dt, th)
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH", "MGQD_Residual", "MGQD_BC_Residual"):
        assert np.array_equal(a[k], b[k]), k
    d0 = dict(d)
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH"):
        d0[k] = np.zeros_like(d[k], order="F")
    z = call_device(d0, c, dt, th)
    assert rel_err(z["Eg_avg"], a["Eg_avg"]) < 1e-10
    # a converged guess needs no iterations
    d1 = dict(d)
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH"):
        d1[k] = a[k]
    again = call_device(d1, c, dt, th)
    assert (again["MGQD_Kits"] <= 3).all()


@pytest.mark.gpu
def test_graph_replayed_iterations_are_bit_identical(oracle):
    """The iteration blocks replayed as CUDA graphs run the same kernels in the same order as direct launches."""
    d, c, dt, th = make(48, 40, 6, 1.0, 14, False, oracle)
    try:
        pkg.mgqd_set_graphs(False)
        a = call_device(d, c, dt, th)
        pkg.mgqd_set_graphs(True)
        b = call_device(d, c, dt, th)
        c2 = call_device(d, c, dt, th)   # the recorded graph replayed again
    finally:
        pkg.mgqd_set_graphs(True)
    assert (a["MGQD_Kits"] > 9).any()    # more than one block of iterations
    for k in ("Eg_avg", "Eg_edgV", "Fxg_edgV", "MGQD_Residual", "MGQD_Kits"):
        assert np.array_equal(a[k], b[k]) and np.array_equal(b[k], c2[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(300, 140, 3), (512, 384, 4)])
def test_fused_level_passes_are_bit_identical(shape, oracle):
    """The V-cycle's fine levels run as one tiled kernel per level and direction (pre-smoothing + restriction,
    prolongation + post-smoothing) or as one kernel per half-sweep: the same iterates, bit for bit, and the same
    again on a repeat (a tile's halo is its neighbours' interior, written by other CTAs of the same launch: no pass
    may read what it writes).  300 x 140 has two levels above the shared-memory V-cycle in ragged tiles; 512 x 384
    x 4 groups runs 1536 tiles per launch on its finest level, several waves of CTAs."""
    d, c, dt, th = make(*shape, 1.0, 21, False, oracle)
    try:
        pkg.mgqd_set_fused_levels(False)
        a = call_device(d, c, dt, th)
        pkg.mgqd_set_fused_levels(True)
        b = call_device(d, c, dt, th)
        b2 = call_device(d, c, dt, th)
    finally:
        pkg.mgqd_set_fused_levels(True)
    assert (a["MGQD_Kits"] > 4).all()
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH", "MGQD_Residual", "MGQD_Kits"):
        assert np.array_equal(a[k], b[k]) and np.array_equal(b[k], b2[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(96, 80, 4), (300, 140, 3)])
def test_smem_vcycle_is_bit_identical(shape, oracle):
    """The multigrid levels of at most 64 x 64 cells in the shared-memory kernel (its coarsest level solved in
    registers by one warp) or in the tiled level passes and the global-memory one-CTA kernel: the same cell
    arithmetic in the same order, so the same iterates bit for bit.  96 x 80 starts the shared-memory levels at
    48 x 40 (a 2 x 2 coarsest level), 300 x 140 at 75 x 35 (ragged levels, a 2 x 1 coarsest level)."""
    d, c, dt, th = make(*shape, 1.0, 23, False, oracle)
    try:
        pkg.mgqd_set_smem_vcycle(False)
        a = call_device(d, c, dt, th)
        pkg.mgqd_set_smem_vcycle(True)
        b = call_device(d, c, dt, th)
        b2 = call_device(d, c, dt, th)
    finally:
        pkg.mgqd_set_smem_vcycle(True)
    assert (a["MGQD_Kits"] > 4).all()
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH", "MGQD_Residual", "MGQD_Kits"):
        assert np.array_equal(a[k], b[k]) and np.array_equal(b[k], b2[k]), k


@pytest.mark.gpu
def test_res_calc_off_skips_only_the_residuals(oracle):
    """Res_Calc = .FALSE.: the same solution and fluxes bit for bit, and MGQD_Residual / MGQD_BC_Residual left as
    the caller passed them (the reference forms them under Res_Calc only)."""
    d, c, dt, th = make(20, 16, 3, 1.0, 29, False, oracle)
    a = call_device(d, c, dt, th, res_calc=True)
    b = call_device(d, c, dt, th, res_calc=False)
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH", "MGQD_Kits"):
        assert np.array_equal(a[k], b[k]), k
    assert np.any(a["MGQD_Residual"] != 0.0)
    assert not np.any(b["MGQD_Residual"]) and not np.any(b["MGQD_BC_Residual"])


@pytest.mark.gpu
def test_device_mloqd_fv_reports_non_convergence(oracle):
    d, c, dt, th = make(16, 16, 3, 1.0, 13, True, oracle)
    try:
        pkg.mgqd_set_tolerance(1e-30, 2)
        with pytest.raises(pkg.TrtError) as e:
            call_device(d, c, dt, th)
        assert e.value.code == -10
    finally:
        pkg.mgqd_set_tolerance(1e-13, 1000)
    out = call_device(d, c, dt, th)
    assert (out["MGQD_Kits"] > 0).all()


@pytest.mark.gpu
def test_device_old_mgqd_coefs_matches_oracle(oracle):
    d, c, dt, _ = P.mgqd_inputs(11, 8, 4, seed=14)
    for th in (1.0, 0.5):
        ref = oracle.old_mgqd_coefs(d, c, dt, th)
        nx, ny, ng = d["Eg_avg_old"].shape
        out = {k: np.zeros((nx, ny, ng), order="F") for k in ref}
        pkg.OLD_MGQD_COEFS(*[d[k] for k in oracle.OLD_MGQD_IN], c, dt, th, out["G_old"], out["Pold_L"],
                           out["Pold_B"], out["Pold_R"], out["Pold_T"], 1)
        for k in ref:
            scale = max(np.abs(ref[k]).max(), 1e-300)
            assert np.abs(out[k] - ref[k]).max() <= 1e-14 * scale, k


@pytest.mark.gpu
def test_device_mloqd_fv_on_factors_from_the_sweep(oracle):
    """QD factors, boundary factors and incoming E/F produced by the device sweep of a small problem feed
    the low-order solve, as ALGORITHMS.f08:686 does inside an outer iteration."""
    from common import CU, sweep_inputs
    prob = P.random_small(31, 10, 9, 4, "S8")
    sd = sweep_inputs(prob, seed=31)
    nx, ny, ng = len(sd["Delx"]), len(sd["Dely"]), sd["KapE_in"].shape[2]
    with pkg.TransportSweep(nx, ny, sd["Omega_x"], sd["Omega_y"], sd["w"], sd["Delx"], sd["Dely"], ng) as s:
        s.put_state(sd["I_crn_old"])
        s.set_boundary(sd["Ic_edgV"], sd["Ic_edgH"], (0, 0, 0, 0))
        s.set_material(sd["KapE_in"], sd["src_iso"], sd["c"], sd["dt"], CU)
        s.sweep(moments=True)
        m = s.moments(["fg_avg_xx", "fg_avg_yy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy", "Cg_L",
                       "Cg_B", "Cg_R", "Cg_T", "Eg_in_L", "Eg_in_B", "Eg_in_R", "Eg_in_T", "Fg_in_L", "Fg_in_B",
                       "Fg_in_R", "Fg_in_T", "Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH"])
    d, c, dt, th = P.mgqd_inputs(nx, ny, ng, seed=31)
    for k, v in m.items():
        if k.startswith(("fg_", "Cg_", "Eg_in", "Fg_in")):
            d[k] = np.asfortranarray(v)
    d["Eg_avg_old"], d["Eg_avg"] = np.asfortranarray(m["Eg_avg"]), np.asfortranarray(m["Eg_avg"])
    d["Eg_edgV"], d["Eg_edgH"] = np.asfortranarray(m["Eg_edgV"]), np.asfortranarray(m["Eg_edgH"])
    d["Fxg_edgV_old"], d["Fyg_edgH_old"] = np.asfortranarray(m["Fxg_edgV"]), np.asfortranarray(m["Fyg_edgH"])
    d["Delx"], d["Dely"] = np.asarray(sd["Delx"]), np.asarray(sd["Dely"])
    d["A"] = np.asfortranarray(np.outer(d["Delx"], d["Dely"]))
    d["KapE"] = d["KapR"] = np.asfortranarray(sd["KapE_in"])
    d.update(oracle.old_mgqd_coefs(d, c, dt, th))
    ref = oracle.mloqd_fv(d, c, dt, th, threads=4)
    out = call_device(d, c, dt, th)
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH"):
        assert rel_err(out[k], ref[k]) < 1e-9, k


@pytest.mark.parametrize("case", [(5, 4, 3, 1.0, 1, True), (12, 9, 6, 0.5, 2, False), (1, 6, 2, 1.0, 4, False),
                                  (7, 1, 2, 0.5, 5, False), (30, 26, 8, 1.0, 15, False)])
def test_oracle_reference_procedure_matches_the_direct_solve(case, oracle):
    """The reference's own procedure (its unknown numbering, ILUT(3, 1e-6), BiCGSTAB to 1e-13) lands on
    the direct solution of the reduced system."""
    d, c, dt, th = make(*case, oracle)
    a = oracle.mloqd_fv(d, c, dt, th, threads=2)
    b = oracle.mloqd_fv(d, c, dt, th, threads=2, solver=1)
    assert (b["MGQD_Kits"] > 0).all()
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH"):
        assert rel_err(b[k], a[k]) < 1e-9, k
