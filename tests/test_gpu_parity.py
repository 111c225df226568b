"""GPU parity: the CUDA library, called through its C ABI, against the CPU oracle.

Bars:
  * FP64 sweep vs the oracle's device-arithmetic mode (closed-form cell solve, solver 1): bit-identical;
  * FP64 sweep vs the reference restatement (Gaussian elimination with complete pivoting, solver 0):
    <= 1e-12 relative per group;
  * moments / QD factors / boundary factors (fused epilogue, different summation order): <= 1e-13;
  * reference-signature moment routines (same summation order): bit-identical;
  * FP32 ("mixed") sweep: <= 1e-5 relative per group.
"""
import ctypes

import numpy as np
import pytest

from common import CU, C, golden_arrays, load_golden, oracle_full, pkg, rel_err, rel_err_per_group, sweep_inputs

pytestmark = pytest.mark.gpu

MOM_KEYS = ("Hg_avg_xx", "Hg_avg_yy", "Hg_avg_xy", "Hg_edgV_xx", "Hg_edgV_xy", "Hg_edgH_yy", "Hg_edgH_xy",
            "Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH", "E_avg", "E_edgV", "E_edgH", "Fx_edgV",
            "Fy_edgH")
FG_KEYS = ("fg_avg_xx", "fg_avg_yy", "fg_avg_xy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy")
BND_KEYS = ("Cg_L", "Cg_B", "Cg_R", "Cg_T", "Eg_in_L", "Eg_in_B", "Eg_in_R", "Eg_in_T", "Fg_in_L", "Fg_in_B",
            "Fg_in_R", "Fg_in_T", "E_in_L", "E_in_B", "E_in_R", "E_in_T", "F_in_L", "F_in_B", "F_in_R", "F_in_T")


def moment_err(m, ref, k):
    """max |a - b| over the scale of the matching energy sum: moments with cancelling terms (H_xy, F)
    are compared against sum w I of the same group and location, not against their own size."""
    loc = "avg" if "avg" in k else ("edgV" if "edgV" in k else "edgH")
    E = ref[{"avg": "Eg_avg", "edgV": "Eg_edgV", "edgH": "Eg_edgH"}[loc]] if ref[k].ndim == 3 else \
        ref[{"avg": "E_avg", "edgV": "E_edgV", "edgH": "E_edgH"}[loc]]
    diff = np.abs(np.asarray(m[k]) - ref[k])
    if ref[k].ndim == 3:
        scale = C * np.max(np.abs(E), axis=(0, 1))
        return float(np.max(np.max(diff, axis=(0, 1)) / scale))
    return float(np.max(diff) / (C * np.max(np.abs(E))))


def dropin_sweep(d, res_calc=False):
    nx, ny, nm, ng = len(d["Delx"]), len(d["Dely"]), len(d["Omega_x"]), d["KapE_in"].shape[2]
    out = dict(I_avg=np.zeros((nx, ny, nm, ng), order="F"), I_edgV=d["I_edgV"].copy(order="F"),
               I_edgH=d["I_edgH"].copy(order="F"), I_crn=np.zeros((2 * nx, 2 * ny, nm, ng), order="F"),
               Ic_edgV=d["Ic_edgV"].copy(order="F"), Ic_edgH=d["Ic_edgH"].copy(order="F"),
               RT_Residual=np.zeros((4, ng, 5), order="F"),
               RT_ResLoc_x=np.zeros((4, ng, 5), dtype=np.int32, order="F"),
               RT_ResLoc_y=np.zeros((4, ng, 5), dtype=np.int32, order="F"))
    pkg.TRANSPORT_SCB(out["I_avg"], out["I_edgV"], out["I_edgH"], out["I_crn"], out["Ic_edgV"], out["Ic_edgH"],
                      d["Omega_x"], d["Omega_y"], d["Delx"], d["Dely"], d["A"], d["KapE_in"], d["Src_in"],
                      d["I_crn_old"], d["c"], d["dt"], 1, out["RT_Residual"], out["RT_ResLoc_x"], out["RT_ResLoc_y"],
                      res_calc)
    return out


def resident(d, precision="fp64", tiling=None, bc_type=(0, 0, 0, 0), bands=0):
    nx, ny, ng = len(d["Delx"]), len(d["Dely"]), d["KapE_in"].shape[2]
    s = pkg.TransportSweep(nx, ny, d["Omega_x"], d["Omega_y"], d["w"], d["Delx"], d["Dely"], ng, precision=precision)
    if tiling:
        s.set_tiling(**tiling)
    if bands:
        s.set_bands(bands)
    s.put_state(d["I_crn_old"])
    s.set_boundary(d["Ic_edgV"], d["Ic_edgH"], bc_type)
    s.set_material(d["KapE_in"], d["src_iso"], d["c"], d["dt"], CU)
    return s


SHAPES = [("C0", lambda: pkg.problems.config0()),
          ("3x4_S8", lambda: pkg.problems.random_small(1, 3, 4, 3, "S8")),
          ("1x1_S8", lambda: pkg.problems.random_small(2, 1, 1, 2, "S8")),
          ("5x7_S12", lambda: pkg.problems.random_small(3, 5, 7, 2, "S12")),
          ("37x21_S16", lambda: pkg.problems.random_small(4, 37, 21, 2, "S16")),
          ("2x3_1dtest", lambda: pkg.problems.random_small(5, 2, 3, 2, "1d_test")),
          ("9x40_abu20", lambda: pkg.problems.random_small(6, 9, 40, 1, "abu20"))]


@pytest.mark.parametrize("name,make", SHAPES, ids=[s[0] for s in SHAPES])
def test_dropin_transport_scb_bit_identical_to_oracle(oracle, name, make):
    d = sweep_inputs(make(), seed=7)
    g = dropin_sweep(d, res_calc=True)
    r1 = oracle_full(d, solver=1, res_calc=True)
    for k in ("I_crn", "I_avg", "I_edgV", "I_edgH", "Ic_edgV", "Ic_edgH"):
        assert np.array_equal(g[k], r1[k]), k
    assert np.array_equal(g["RT_Residual"], r1["RT_Residual"])
    assert np.array_equal(g["RT_ResLoc_x"], r1["RT_ResLoc_x"]) and np.array_equal(g["RT_ResLoc_y"], r1["RT_ResLoc_y"])
    r0 = oracle_full(d, solver=0)
    for k in ("I_crn", "I_avg", "I_edgV", "I_edgH"):
        assert rel_err_per_group(g[k], r0[k]) <= 1e-12, k


@pytest.mark.parametrize("case", load_golden(), ids=lambda c: c["name"])
def test_dropin_matches_exact_rational_sweep(case):
    d, exp = golden_arrays(case)
    g = dropin_sweep(d)
    for k in ("I_crn", "I_avg", "Ic_edgV", "Ic_edgH"):
        assert rel_err_per_group(g[k], exp[k]) < 2e-14, k


@pytest.mark.parametrize("name,make", SHAPES[:5], ids=[s[0] for s in SHAPES[:5]])
def test_resident_sweep_and_fused_moments(oracle, name, make):
    prob = make()
    d = sweep_inputs(prob, seed=11)
    ref = oracle_full(d, solver=1)
    with resident(d) as s:
        s.sweep(moments=True)
        I = s.get_state()
        m = s.moments()
    assert np.array_equal(I, ref["I_crn"])
    for k in MOM_KEYS:
        assert moment_err(m, ref, k) < 1e-13, k
    for k in FG_KEYS:
        assert np.max(np.abs(m[k] - ref[k])) < 1e-13, k
    for k in BND_KEYS:
        assert rel_err(m[k], ref[k]) < 1e-13 or np.max(np.abs(m[k] - ref[k])) < 1e-300, k
    # Omega_y-weighted horizontal flux (the reference's Fyg_edgH is Omega_x-weighted, :469): the
    # oracle's collapse with Omega_y passed as the x cosine yields it
    rc = oracle.collapse_intensities(ref["I_avg"], ref["I_edgV"], ref["I_edgH"], d["Omega_y"], d["Omega_y"], d["w"],
                                     CU)
    m2 = dict(m, Fyg_edgH=m["Fyg_edgH_true"])
    assert moment_err(m2, dict(ref, Fyg_edgH=rc["Fyg_edgH"]), "Fyg_edgH") < 1e-13


@pytest.mark.parametrize("tiling", [dict(warps=1), dict(warps=2, stages=1), dict(warps=8, stages=2),
                                    dict(warps=3, stages=4), dict(warps=16)])
def test_tiling_does_not_change_results(tiling):
    prob = pkg.problems.random_small(8, 33, 29, 2, "S16")
    d = sweep_inputs(prob, seed=5)
    with resident(d) as s:
        s.sweep()
        I0, m0 = s.get_state(), s.moments(["Eg_avg", "fg_edgV_xy", "Cg_T"])
    with resident(d, tiling=tiling) as s:
        s.sweep()
        I1, m1 = s.get_state(), s.moments(["Eg_avg", "fg_edgV_xy", "Cg_T"])
    assert np.array_equal(I0, I1)
    for k in m0:
        assert np.array_equal(m0[k], m1[k]), k


@pytest.mark.parametrize("slices", [1, 2, 4, 8, 16, 32])
def test_direction_slicing_variants(oracle, slices):
    prob = pkg.problems.random_small(9, 12, 10, 2, "S8")
    d = sweep_inputs(prob, seed=9)
    ref = oracle_full(d, solver=1)
    try:
        s = resident(d, tiling=dict(slices=slices))
    except pkg.TrtError:
        pytest.skip(f"no compiled kernel with {slices} slices for 10 directions per quadrant")
    with s:
        s.sweep()
        I = s.get_state()
        m = s.moments(["Eg_avg", "fg_avg_xy"])
    assert np.array_equal(I, ref["I_crn"])
    assert rel_err_per_group(m["Eg_avg"], ref["Eg_avg"]) < 1e-13


@pytest.mark.parametrize("splits,slices", [(2, 0), (3, 0), (3, 2), (4, 0), (5, 0), (10, 0)])
def test_direction_splits(oracle, splits, slices):
    """Each quadrant's 10 directions split over several CTAs (ragged splits included): the state is
    unchanged bit for bit, the moments only change in the order the split partials are added."""
    prob = pkg.problems.random_small(12, 13, 11, 2, "S8")
    d = sweep_inputs(prob, seed=12)
    ref = oracle_full(d, solver=1)
    with resident(d, tiling=dict(splits=splits, slices=slices)) as s:
        assert s.tiling()["splits"] == splits
        s.sweep(moments=True)
        I = s.get_state()
        m = s.moments()
        ang = s.angular()
    assert np.array_equal(I, ref["I_crn"])
    for k in ("I_avg", "I_edgV", "I_edgH"):
        assert np.array_equal(ang[k], ref[k]), k
    for k in MOM_KEYS:
        assert moment_err(m, ref, k) < 1e-13, k
    for k in BND_KEYS:
        assert rel_err(m[k], ref[k]) < 1e-13 or np.max(np.abs(m[k] - ref[k])) < 1e-300, k


def test_direction_splits_fp32_state_unchanged():
    prob = pkg.problems.random_small(13, 17, 19, 2, "S12")
    d = sweep_inputs(prob, seed=13)
    out = []
    for splits in (1, 2, 7):
        with resident(d, precision="fp32", tiling=dict(splits=splits)) as s:
            s.sweep(moments=True)
            out.append((s.get_state(), s.moments(["Eg_avg", "Fxg_edgV"])))
    # FP32 partial records are rounded once per (cell, quadrant, split): splitting changes that
    # rounding, at the FP32 unit roundoff
    for I, m in out[1:]:
        assert np.array_equal(I, out[0][0])
        for k in m:
            assert rel_err_per_group(m[k], out[0][1][k]) < 1e-6, k


def test_split_count_limits():
    prob = pkg.problems.random_small(14, 4, 4, 1, "S8")
    d = sweep_inputs(prob, seed=14)
    with resident(d) as s:
        with pytest.raises(pkg.TrtError):
            s.set_tiling(splits=11)          # more splits than directions per quadrant
        s.set_tiling(splits=10)
        assert s.tiling()["splits"] == 10


def test_multi_step_state_roll(oracle):
    """Three time steps: I_crn_old <- I_crn between steps (ALGORITHMS.f08:397), with a new material each step."""
    prob = pkg.problems.random_small(10, 11, 9, 3, "S8")
    d = sweep_inputs(prob, seed=1)
    rng = np.random.default_rng(3)
    with resident(d) as s:
        I_old = d["I_crn_old"]
        for step in range(3):
            T = prob.T0 * rng.uniform(0.5, 3.0, (prob.nx, prob.ny))
            kap, src = prob.material(T)
            dd = dict(d, KapE_in=kap, src_iso=src,
                      Src_in=np.asfortranarray(np.repeat(np.repeat(src, 2, 0), 2, 1)[:, :, None, :].repeat(prob.nm, 2)),
                      I_crn_old=I_old)
            ref = oracle_full(dd, solver=1)
            s.set_material(kap, src, d["c"], d["dt"], CU)
            s.sweep(roll=(step > 0), moments=True)
            I = s.get_state()
            assert np.array_equal(I, ref["I_crn"]), step
            m = s.moments(["fg_avg_xx", "Cg_L"])
            assert np.max(np.abs(m["fg_avg_xx"] - ref["fg_avg_xx"])) < 1e-13
            I_old = ref["I_crn"]


def test_reflective_boundaries(oracle):
    """Reflective left and top sides: sweep, combine, RT_BC_UPDATE (mirror copies), sweep again."""
    prob = pkg.problems.random_small(12, 6, 5, 2, "S8")
    d = sweep_inputs(prob, seed=4)
    bc = (1, 0, 0, 1)
    bT = d["bcT_eV"]
    with resident(d, bc_type=bc) as s:
        ref = oracle_full(d, solver=1, bc_type=bc)
        s.sweep(moments=True)
        assert np.array_equal(s.get_state(), ref["I_crn"])
        m = s.moments(["Cg_L", "Cg_T", "Cg_R", "Eg_in_L", "Eg_in_R", "E_in_L", "F_in_R"])
        for k in m:
            assert rel_err(m[k], ref[k]) < 1e-13 or np.max(np.abs(m[k] - ref[k])) == 0, k
        s.bc_update(bc, bT, CU, d["nu"])
        IV, IH, IcV, IcH = oracle.rt_bc_update(bc, *bT, CU, d["nu"], ref["I_edgV"], ref["I_edgH"], ref["Ic_edgV"],
                                               ref["Ic_edgH"])
        d2 = dict(d, I_edgV=IV, I_edgH=IH, Ic_edgV=IcV, Ic_edgH=IcH)
        ref2 = oracle_full(d2, solver=1, bc_type=bc)
        s.sweep(moments=True)
        assert np.array_equal(s.get_state(), ref2["I_crn"])
        ang = s.angular(("Ic_edgV", "Ic_edgH"))
        assert np.array_equal(ang["Ic_edgV"], ref2["Ic_edgV"]) and np.array_equal(ang["Ic_edgH"], ref2["Ic_edgH"])


def test_init_state_matches_rt_init(oracle):
    """RT_INIT: corners and boundaries at Bg(Tini), then the Planck inflow faces."""
    prob = pkg.problems.random_small(13, 4, 6, 3, "S12")
    ox, oy, w = prob.directions()
    with pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng) as s:
        s.init_state(prob.T0 * 1e3, [t * 1e3 for t in prob.bcT], CU, prob.nu_eV)
        I = s.get_state()
        ang = s.angular(("Ic_edgV", "Ic_edgH"))
    d = sweep_inputs(prob, random_old=False)
    # the host Planck evaluations differ only in the exp of the C library vs numpy (<= 1 ulp)
    assert rel_err_per_group(I, d["I_crn_old"]) < 1e-15
    assert rel_err_per_group(ang["Ic_edgV"], d["Ic_edgV"]) < 1e-15
    assert rel_err_per_group(ang["Ic_edgH"], d["Ic_edgH"]) < 1e-15


def test_fp32_mixed_sweep_against_fp64_oracle(oracle):
    prob = pkg.problems.config0()
    d = sweep_inputs(prob, seed=2)
    ref = oracle_full(d, solver=0)
    with resident(d, precision="fp32") as s:
        s.sweep(moments=True)
        I = s.get_state()
        m = s.moments(["Eg_avg", "E_avg", "fg_avg_xx", "fg_edgV_xx", "Cg_L", "Fx_edgV"])
    # groups carrying energy (the others sit at FP32 underflow / the eps floor) to 1e-5 per group
    gmax = np.max(np.abs(ref["I_crn"]), axis=(0, 1, 2))
    live = gmax > 1e-20 * gmax.max()
    assert rel_err_per_group(I[..., live], ref["I_crn"][..., live]) < 1e-5
    assert rel_err(m["E_avg"], ref["E_avg"]) < 1e-5
    assert rel_err(m["Fx_edgV"], ref["Fx_edgV"], scale=C * np.max(ref["E_edgV"])) < 1e-5
    assert np.max(np.abs(m["fg_avg_xx"] - ref["fg_avg_xx"])[..., live]) < 1e-5
    assert np.all(np.isfinite(m["fg_edgV_xx"])) and np.all(np.isfinite(m["Cg_L"]))


def test_reference_signature_moment_routines_bit_identical(oracle):
    prob = pkg.problems.random_small(14, 7, 6, 3, "S12")
    d = sweep_inputs(prob, seed=8)
    r = oracle_full(d, solver=0)
    nx, ny, ng = prob.nx, prob.ny, prob.ng
    A, V, H = (nx, ny), (nx + 1, ny), (nx, ny + 1)
    shapes = [A + (ng,)] * 3 + [V + (ng,)] * 2 + [H + (ng,)] * 2 + [V + (ng,), H + (ng,), A + (ng,), V + (ng,),
                                                                   H + (ng,), V, H, A, V, H]
    names = oracle.COLLAPSE_OUT
    out = {k: np.zeros(s, order="F") for k, s in zip(names, shapes)}
    pkg.COLLAPSE_INTENSITIES(4, r["I_avg"], r["I_edgV"], r["I_edgH"], d["Omega_x"], d["Omega_y"], d["w"], CU,
                             *[out[k] for k in names])
    for k in names:
        assert np.array_equal(out[k], r[k]), k
    fg = {k: np.zeros_like(r[k], order="F") for k in oracle.FG_OUT}
    pkg.fg_Calc(*[fg[k] for k in oracle.FG_OUT], *[r[k] for k in ("Hg_avg_xx", "Hg_avg_yy", "Hg_avg_xy",
                                                                   "Hg_edgV_xx", "Hg_edgV_xy", "Hg_edgH_yy",
                                                                   "Hg_edgH_xy", "Eg_avg", "Eg_edgV", "Eg_edgH")],
                C, 4)
    for k in oracle.FG_OUT:
        assert np.array_equal(fg[k], r[k]), k
    for bc in ((0, 0, 0, 0), (1, 0, 1, 0), (0, 1, 0, 1)):
        rr = oracle.cg_calc(r["I_edgV"], r["I_edgH"], d["Omega_x"], d["Omega_y"], d["w"], CU, bc)
        cg = {k: np.zeros_like(rr[k], order="F") for k in ("Cg_L", "Cg_B", "Cg_R", "Cg_T")}
        pkg.Cg_Calc(cg["Cg_L"], cg["Cg_B"], cg["Cg_R"], cg["Cg_T"], r["I_edgV"], r["I_edgH"], d["Omega_x"],
                    d["Omega_y"], d["w"], CU, bc, 4)
        for k in cg:
            assert np.array_equal(cg[k], rr[k]), (bc, k)
        ri = oracle.mgqd_in_calc(r["I_edgV"], r["I_edgH"], d["Omega_x"], d["Omega_y"], d["w"], C, CU, bc)
        gi = {k: np.zeros_like(ri[k], order="F") for k in oracle.IN_OUT}
        pkg.MGQD_In_Calc(*[gi[k] for k in oracle.IN_OUT], r["I_edgV"], r["I_edgH"], d["Omega_x"], d["Omega_y"],
                         d["w"], C, CU, bc, 4)
        for k in gi:
            assert np.array_equal(gi[k], ri[k]), (bc, k)
        rg = oracle.gqd_in_calc(ri)
        gg = {k: np.zeros_like(rg[k]) for k in rg}
        pkg.GQD_In_Calc(*[gg[k] for k in ("E_in_L", "E_in_B", "E_in_R", "E_in_T", "F_in_L", "F_in_B", "F_in_R",
                                          "F_in_T")], *[ri[k] for k in oracle.IN_OUT])
        for k in gg:
            assert np.array_equal(gg[k], rg[k]), k


def test_rt_bc_update_signature_bit_identical(oracle):
    prob = pkg.problems.random_small(15, 5, 4, 2, "S8")
    d = sweep_inputs(prob, seed=3)
    r = oracle_full(d, solver=1)
    for bc in ((0, 0, 0, 0), (1, 1, 1, 1), (1, 0, 0, 1)):
        exp = oracle.rt_bc_update(bc, 800.0, 0.0, 300.0, 50.0, CU, d["nu"], r["I_edgV"], r["I_edgH"], r["Ic_edgV"],
                                  r["Ic_edgH"])
        got = [r[k].copy(order="F") for k in ("I_edgV", "I_edgH", "Ic_edgV", "Ic_edgH")]
        pkg.RT_BC_UPDATE(bc, 800.0, 0.0, 300.0, 50.0, CU, d["nu"], *got)
        for a, b in zip(got, exp):
            assert np.array_equal(a, b), bc


def _c1_moments(s, prob, kap, src, Tini, bcT, names=("E_avg", "Fx_edgV", "Eg_avg", "fg_avg_xx")):
    s.init_state(Tini, bcT, CU, prob.nu_eV)
    s.set_material(kap, src, C, prob.dt, CU)
    s.sweep(moments=True)
    return s.moments(names)


def test_superposition_and_scaling_at_full_c1_size():
    """Size-independent properties at the C1 size (256^2 cells, 50 groups, S16): the sweep is linear in
    (source, inflow) from a zero state -- inflow+source = inflow alone + source alone -- and doubling
    the source doubles every intensity moment."""
    prob = pkg.problems.config1()
    ox, oy, w = prob.directions()
    kap, src = prob.material(np.full((prob.nx, prob.ny), 0.3))
    zero = np.zeros_like(src, order="F")
    with pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng) as s:
        both = _c1_moments(s, prob, kap, src, 0.0, [1000.0, 0.0, 0.0, 0.0])
        only_src = _c1_moments(s, prob, kap, src, 0.0, [0.0, 0.0, 0.0, 0.0])
        only_bc = _c1_moments(s, prob, kap, zero, 0.0, [1000.0, 0.0, 0.0, 0.0])
        twice = _c1_moments(s, prob, kap, np.asfortranarray(2.0 * src), 0.0, [0.0, 0.0, 0.0, 0.0])
    assert np.all(np.isfinite(both["E_avg"])) and np.all(both["E_avg"] > 0)
    assert rel_err(both["E_avg"], only_src["E_avg"] + only_bc["E_avg"]) < 1e-12
    assert rel_err(both["Fx_edgV"], only_src["Fx_edgV"] + only_bc["Fx_edgV"]) < 1e-12
    # E_g = (sum w I + eps sum w) / c: remove the eps floor before comparing the doubled source
    floor = 1e-25 / CU * np.sum(w) / C
    big = np.max(only_src["Eg_avg"], axis=(0, 1)) > 1e6 * floor
    assert rel_err_per_group((twice["Eg_avg"] - floor)[..., big], 2.0 * (only_src["Eg_avg"] - floor)[..., big]) < 1e-12


def test_equilibrium_at_full_c1_size():
    """Infinite-medium equilibrium at the C1 size: state, inflow and source at one temperature keep
    every intensity at B_g, so E_g = 4 pi B_g / c and the QD and boundary factors are the quadrature's
    moments."""
    prob = pkg.problems.config1()
    ox, oy, w = prob.directions()
    T = 0.05
    kap, src = prob.material(np.full((prob.nx, prob.ny), T))
    with pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng) as s:
        m = _c1_moments(s, prob, kap, src, T * 1e3, [T * 1e3] * 4,
                        names=("Eg_avg", "fg_avg_xx", "fg_avg_xy", "fg_edgH_yy", "Cg_B"))
    nu = prob.nu_eV
    B = np.array([pkg.problems.bg_planck(T * 1e3, nu[g], nu[g + 1]) for g in range(prob.ng)])
    live = B > 1e-200
    expE = 4 * np.pi * B / C
    got = m["Eg_avg"][:, :, live] - 1e-38 * np.sum(w) / C
    assert np.max(np.abs(got / expE[live] - 1.0)) < 1e-11
    assert np.max(np.abs(m["fg_avg_xx"][:, :, live] - np.sum(w * ox * ox) / np.sum(w))) < 1e-12
    assert np.max(np.abs(m["fg_avg_xy"][:, :, live])) < 1e-12
    q = len(w) // 4
    out_B = slice(2 * q, 4 * q)
    assert np.max(np.abs(m["Cg_B"][:, live] - np.sum(oy[out_B] * w[out_B]) / np.sum(w[out_B]))) < 1e-12


def test_api_errors_and_timeout_path():
    prob = pkg.problems.random_small(16, 8, 8, 2, "S8")
    d = sweep_inputs(prob, seed=1)
    ox, oy, w = d["Omega_x"], d["Omega_y"], d["w"]
    with pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, d["Delx"], d["Dely"], prob.ng) as s:
        with pytest.raises(pkg.TrtError) as e:
            s.sweep()
        assert e.value.code == pkg._lib.TRT_ERR_STATE
    with pytest.raises(pkg.TrtError) as e:
        pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, d["Delx"], d["Dely"], prob.ng, hbm_budget=1024)
    assert e.value.code == pkg._lib.TRT_ERR_BUDGET
    # a wait that never completes: every poll budget zero -> error status, then the handle recovers
    ref = oracle_full(d, solver=1)
    with resident(d) as s:
        L = pkg.lib()
        assert L.trt_set_wait_limit_zero(s.handle) == 0
        assert L.trt_sweep(s.handle, 2) == 0
        assert L.trt_sync(s.handle) == pkg._lib.TRT_ERR_TIMEOUT
        assert L.trt_set_wait_limit(s.handle, 0) == 0
        s.sweep(moments=True)
        assert np.array_equal(s.get_state(), ref["I_crn"])


def test_launch_counter_counts_library_kernels():
    before = pkg.kernel_launches()
    prob = pkg.problems.random_small(17, 4, 4, 1, "S8")
    d = sweep_inputs(prob)
    with resident(d) as s:
        s.sweep(moments=True)
    assert pkg.kernel_launches() - before >= 3


def test_autotune_picks_a_resident_tiling_and_keeps_results(oracle):
    prob = pkg.problems.random_small(30, 33, 29, 3, "S16")
    d = sweep_inputs(prob, seed=30)
    ref = oracle_full(d, solver=1)
    nx, ny, ng = len(d["Delx"]), len(d["Dely"]), d["KapE_in"].shape[2]
    with pkg.TransportSweep(nx, ny, d["Omega_x"], d["Omega_y"], d["w"], d["Delx"], d["Dely"], ng) as s:
        t = s.autotune()
        assert t["splits"] in (1, 2, 3, 4) and t["warps"] in (2, 3, 4, 5, 6, 8) and t["sweep_ms"] > 0
        s.put_state(d["I_crn_old"])
        s.set_boundary(d["Ic_edgV"], d["Ic_edgH"], (0, 0, 0, 0))
        s.set_material(d["KapE_in"], d["src_iso"], d["c"], d["dt"], CU)
        s.sweep(moments=True)
        assert np.array_equal(s.get_state(), ref["I_crn"])
        m = s.moments(["Eg_avg", "E_avg"])
    assert moment_err(m, ref, "Eg_avg") < 1e-13


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_register_variant_does_not_change_results(precision):
    """The up-to-170-register kernel variant computes the same operations: bit-identical outputs."""
    prob = pkg.problems.random_small(31, 40, 36, 4, "S16")
    d = sweep_inputs(prob, seed=31)
    out = []
    for mode in (0, -1):
        with resident(d, precision=precision, tiling=dict(warps=4)) as s:
            s.set_register_mode(mode)
            s.put_state(d["I_crn_old"])
            s.sweep(moments=True)
            out.append((s.tiling()["wide_registers"], s.get_state(), s.moments(["Eg_avg", "Fxg_edgV", "Cg_B"])))
    assert out[0][0] == 0 and out[1][0] >= 1
    assert np.array_equal(out[0][1], out[1][1])
    for k in out[0][2]:
        assert np.array_equal(out[0][2][k], out[1][2][k]), k


@pytest.mark.parametrize("name,make", SHAPES[:5], ids=[s[0] for s in SHAPES[:5]])
def test_resident_sweep_matches_gaussian_elimination_oracle(oracle, name, make):
    """The resident sweep with the isotropic per-cell source (the kernel the benchmark times) against the
    oracle's SCB_BGEN + Gaussian-elimination form (solver 0), which shares no code with the library:
    corner state, group energies and QD/boundary factors within 1e-12."""
    d = sweep_inputs(make(), seed=13)
    r0 = oracle_full(d, solver=0)
    with resident(d) as s:
        s.sweep(moments=True)
        I = s.get_state()
        m = s.moments()
    assert rel_err_per_group(I, r0["I_crn"]) <= 1e-12
    for k in ("Eg_avg", "Eg_edgV", "Eg_edgH"):
        assert rel_err_per_group(m[k], r0[k]) <= 1e-12, k
    for k in FG_KEYS + ("Cg_L", "Cg_B", "Cg_R", "Cg_T"):
        assert np.max(np.abs(m[k] - r0[k])) <= 1e-12, k


def fg_weighted_err(m, ref, k, groups=None):
    """max over cells of |fg - fg_ref| E / max E of the group (E at the factor's location): the error of the
    factor as it weights the low-order equations.  Where the group's energy is negligible (E/max E below
    1e-15 or so, a cold far corner, or the slightly negative intensities SCB produces in thick cells) the
    ratio H/(cE) is round-off noise, in the oracle's two cell solves as well."""
    loc = "avg" if "avg" in k else ("edgV" if "edgV" in k else "edgH")
    E = ref["Eg_" + loc]
    a = np.asarray(m[k]) if groups is None else np.asarray(m[k])[..., groups]
    w = np.abs(E) / np.max(np.abs(E), axis=(0, 1))
    return float(np.max(np.abs(a - ref[k]) * w))


def _c1_group_inputs(prob, sel, T):
    """Reference-layout sweep inputs of config C1 restricted to the groups `sel`, in the state the
    benchmark's handle starts from (trt_init_state: every corner at Bg(T0), Planck inflow on the left)
    and with the material at temperature field T."""
    from oracle import oracle as O
    ox, oy, w = prob.directions()
    nx, ny, nm = prob.nx, prob.ny, len(ox)
    kap, src = prob.material(T)
    nu = prob.nu_eV
    ns = len(sel)
    Bg0 = np.array([pkg.problems.bg_planck(prob.T0 * 1e3, nu[g], nu[g + 1]) for g in sel])
    I_old = np.asfortranarray(np.broadcast_to(Bg0, (2 * nx, 2 * ny, nm, ns)).copy())
    src_s = np.asfortranarray(src[:, :, sel])
    Src_in = np.asfortranarray(np.repeat(np.repeat(src_s, 2, axis=0), 2, axis=1)[:, :, None, :].repeat(nm, axis=2))
    faces = [np.zeros((nx + 1, 2 * ny, nm, ns), order="F"), np.zeros((2 * nx, ny + 1, nm, ns), order="F"),
             np.zeros((nx + 1, ny, nm, ns), order="F"), np.zeros((nx, ny + 1, nm, ns), order="F")]
    bT = [t * 1e3 for t in prob.bcT]
    for k, g in enumerate(sel):   # RT_INIT's boundary update, one group at a time (edges g, g+1)
        b = Bg0[k]
        IcV = np.full((nx + 1, 2 * ny, nm, 1), b, order="F")
        IcH = np.full((2 * nx, ny + 1, nm, 1), b, order="F")
        IV = np.full((nx + 1, ny, nm, 1), b, order="F")
        IH = np.full((nx, ny + 1, nm, 1), b, order="F")
        IV, IH, IcV, IcH = O.rt_bc_update((0, 0, 0, 0), bT[0], bT[1], bT[2], bT[3], CU, nu[g:g + 2], IV, IH, IcV, IcH)
        for f, v in zip(faces, (IcV, IcH, IV, IH)):
            f[..., k] = v[..., 0]
    return dict(Omega_x=ox, Omega_y=oy, w=w, Delx=prob.delx, Dely=prob.dely, A=np.asfortranarray(np.outer(prob.delx,
                prob.dely)), KapE_in=np.asfortranarray(kap[:, :, sel]), src_iso=src_s, Src_in=Src_in, I_crn_old=I_old,
                Ic_edgV=faces[0], Ic_edgH=faces[1], I_edgV=faces[2], I_edgH=faces[3], c=C, dt=prob.dt)


def test_c1_full_size_sweep_matches_gaussian_elimination_oracle(oracle):
    """Config C1 at full size (256x256 cells, 50 groups, S16) through the resident handle with the
    benchmark's set-up (initial state, material at the benchmark's temperature field): the group
    energies, QD factors and boundary factors of 8 groups spread over the group range (opacities from
    optically thin to thick) against the oracle's Gaussian-elimination sweep of those groups, within
    1e-12 (QD factors weighted by the cell's share of the group energy: in cells whose energy is 1e-17 of
    the group's and below, the two oracle cell solves differ by 1e-10 as well)."""
    prob = pkg.problems.config1()
    ox, oy, w = prob.directions()
    x = (np.arange(prob.nx) + 0.5) / prob.nx
    T = np.asfortranarray(np.broadcast_to((prob.T0 + 0.5 * np.exp(-8 * x))[:, None], (prob.nx, prob.ny)))
    kap, src = prob.material(T)
    s = pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng, precision="fp64")
    try:
        s.init_state(prob.T0 * 1e3, [t * 1e3 for t in prob.bcT], CU, prob.nu_eV)
        s.set_material(kap, src, C, prob.dt, CU)
        s.sweep(roll=True, moments=True)
        m = s.moments(("Eg_avg", "Eg_edgV", "Eg_edgH") + FG_KEYS + ("Cg_L", "Cg_B", "Cg_R", "Cg_T"))
    finally:
        s.close()
    sel = [int(g) for g in np.linspace(0, prob.ng - 1, 8).round()]
    for chunk in (sel[0:2], sel[2:4], sel[4:6], sel[6:8]):
        d = _c1_group_inputs(prob, chunk, T)
        r0 = oracle_full(d, solver=0, threads=2)
        for k in ("Eg_avg", "Eg_edgV", "Eg_edgH"):
            assert rel_err_per_group(m[k][..., chunk], r0[k]) <= 1e-12, (k, chunk)
        for k in FG_KEYS:
            assert fg_weighted_err(m, r0, k, chunk) <= 1e-12, (k, chunk)
        for k in ("Cg_L", "Cg_B", "Cg_R", "Cg_T"):
            assert np.max(np.abs(m[k][..., chunk] - r0[k])) <= 1e-12, (k, chunk)
        del d, r0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("bands,tiling", [(2, dict(warps=1, slices=4)), (3, dict(warps=2, slices=8)),
                                          (4, dict(warps=1, slices=8)), (8, dict(warps=1, slices=8, splits=2))],
                         ids=["b2", "b3", "b4", "b8"])
def test_band_ctas_bit_identical(precision, bands, tiling):
    """Spatial row tiles: the rounds of each sweep dealt to `bands` CTAs of one cluster, handed over
    through the L2 wrap buffer, give the same corner state and moments as one CTA per sweep, bit for bit,
    over two rolled steps."""
    prob = pkg.problems.random_small(8, 33, 29, 2, "S16")
    d = sweep_inputs(prob, seed=5)
    out = []
    for nb in (0, bands):
        with resident(d, precision=precision, tiling=tiling, bands=nb) as s:
            t = s.tiling()
            s.sweep(moments=True)
            s.sweep(roll=True, moments=True)
            out.append((t, s.get_state(), s.moments(["Eg_avg", "fg_avg_xy", "fg_edgV_xx", "Cg_T", "Eg_in_L"])))
    (t0, I0, m0), (t1, I1, m1) = out
    assert t0["bands"] == 1 and t1["bands"] > 1
    assert np.array_equal(I0, I1)
    for k in m0:
        assert np.array_equal(m0[k], m1[k]), k


def test_band_ctas_time_loop_matches_single_cta():
    """The config-0 time loop (three steps of the transport-only iteration) with band CTAs equals the
    default tiling bit for bit."""
    from test_gpu_tstep import _device
    prob = pkg.problems.config0()
    ts = pkg.problems.config_timestep_setup(prob)
    res = []
    for nb in (1, 3):
        s = _device(prob, ts, "fp64", 2, 0.0, 5, law=1)
        try:
            if nb > 1:
                s.set_tiling(warps=1, slices=8)
                s.set_bands(nb)
                s.init_state(ts.Tini_eV, list(ts.bcT_eV), CU, ts.nu_eV)
            else:
                s.set_tiling(warps=1, slices=8)
                s.init_state(ts.Tini_eV, list(ts.bcT_eV), CU, ts.nu_eV)
            Ts = [(s.tstep(), s.temperature()) for _ in range(3)]
            res.append((s.tiling()["bands"], Ts, s.get_state()))
        finally:
            s.close()
    assert res[0][0] == 1 and res[1][0] == 3
    for (_, Ta), (_, Tb) in zip(res[0][1], res[1][1]):
        assert np.array_equal(Ta, Tb)
    assert np.array_equal(res[0][2], res[1][2])
