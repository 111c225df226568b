"""The mlqd time step with the groups split over several handles (sharded.ShardedMlqd): the group ranges of a
multi-GPU run.  The groups meet only in group sums (OLD_GREY_COEFS's sum of G_old, the transport E of the outer
convergence test, and per MGQD iteration the sums behind COLLAPSE_MG_EF, Cbar_Calc and GREY_COEFS), which
the driver adds across the ranges; the grey Newton solve runs on every range with the same totals.

CPU: the split grey sums against the oracle's unsplit routines; the driver over oracle-backed members (each
range sweeps and solves its groups with the oracle's restatements, the real driver in between) against the
oracle's unsplit loop, in one process and as two gloo ranks.  GPU: the driver over library handles, one handle
through the phases against trt_mlqd_step bit for bit, two group-range handles on one device against one
handle."""
import os
import tempfile

import numpy as np
import pytest

from common import C, CU, pkg

P = pkg.problems
S = pkg.sharded

PER_GROUP = ("I_crn", "I_edgV", "I_edgH", "Ic_edgV", "Ic_edgH", "Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV",
             "Fyg_edgH", "fg_avg_xx", "fg_avg_yy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy",
             "Cg_L", "Cg_B", "Cg_R", "Cg_T", "Eg_in_L", "Eg_in_B", "Eg_in_R", "Eg_in_T", "Fg_in_L", "Fg_in_B",
             "Fg_in_R", "Fg_in_T")


def setup_problem(nx=7, ny=6, G=5, quad="S8", seed=61, Tini=100.0, bcT=(1000.0, 0.0, 0.0, 0.0)):
    prob = P.random_small(seed, nx, ny, G, quad)
    ts = P.fc_timestep_setup(prob, Tini_eV=Tini)
    km = np.ones((nx, ny), order="F")
    return prob, ts, km, tuple(bcT), P.fc_cv(1000.0)


class OracleMlqdMember:
    """A group range [g0, g1) of the mlqd time step on the CPU oracle (test infrastructure): the phases of
    include/trt_sweep.h restated over the oracle's routines, in the order of oracle.mlqd_steps."""

    def __init__(self, prob, ts, km, bcT, cv, g0, g1, conv_ho, conv_lo, maxit_gloqd=20, Theta=1.0):
        from oracle import oracle as O
        self.O, self.prob, self.ts, self.km, self.cv = O, prob, ts, km, cv
        self.g0, self.g1 = g0, g1
        self.conv_ho, self.conv_lo, self.maxit_gloqd, self.Theta = conv_ho, conv_lo, maxit_gloqd, Theta
        self.ox, self.oy, self.w = prob.directions()
        full = O.mlqd_init(prob.nx, prob.ny, self.ox, self.oy, self.w, ts.nu_eV, ts.Tini_eV, CU, C, bcT=bcT)
        sl = slice(g0, g1)
        self.st = {k: (np.asfortranarray(v[..., sl]) if k in PER_GROUP else v) for k, v in full.items()}
        self.nu = ts.nu_eV[g0:g1 + 1]
        self.A = O.F(np.outer(prob.delx, prob.dely))
        self.HO_own = O.zeros(prob.nx, prob.ny)
        for g in range(g1 - g0):
            self.HO_own = self.HO_own + self.st["Eg_avg"][:, :, g]
        self.KapE, self.rt_src, Bg = O.material_update(self.st["Temp"], self.nu, km, CU)
        self.MGQD_Src = O.F(4.0 * np.pi * self.KapE * Bg)

    def mlqd_exchange_size(self):
        nx, ny = self.prob.nx, self.prob.ny
        return 16 * nx * ny + 2 * (nx + 1) * ny + 2 * nx * (ny + 1) + 4 * (nx + ny)

    def _put(self, buf, v):
        buf.zero_()
        buf[:v.size] = __import__("torch").from_numpy(np.ascontiguousarray(v.reshape(-1, order="F")))

    def _get(self, tot, n, shape):
        return self.O.F(tot[:n].numpy().reshape(shape, order="F").copy(order="F"))   # tot is reused

    def mlqd_step_begin(self, buf):
        O, st = self.O, self.st
        nx, ny = self.prob.nx, self.prob.ny
        self.Temp_old = st["Temp"].copy(order="F")
        self.I_crn_old = st["I_crn"].copy(order="F")
        od = {k + "_old": O.F(st[k]).copy(order="F") for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV",
                                                                "Fyg_edgH") + O.MLOQD_FACTORS}
        od.update(KapE_old=self.KapE.copy(order="F"), KapR_old=self.KapE.copy(order="F"),
                  Src_old=self.MGQD_Src.copy(order="F"), Delx=self.prob.delx, Dely=self.prob.dely, A=self.A)
        self.od = od
        self.old_grey = (st["E_avg"].copy(order="F"), st["GQD_Src"].copy(order="F"), st["KapE_Bar"].copy(order="F"))
        self.old = O.old_mgqd_coefs(od, C, self.ts.dt, self.Theta)
        gs = O.zeros(nx, ny)
        for g in range(self.g1 - self.g0):
            gs = gs + self.old["G_old"][:, :, g]
        self._put(buf, gs)
        self.mg_hist, self.egp_hist = [], []

    def mlqd_step_begin_finish(self, tot):
        O = self.O
        nx, ny = self.prob.nx, self.prob.ny
        gsum = self._get(tot, nx * ny, (nx, ny, 1))
        E_old, Q_old, Kb_old = self.old_grey
        self.Gold_Hat, self.Rhat_old = O.old_grey_coefs(C, self.ts.dt, self.Theta, self.cv, self.A, gsum,
                                                        self.Temp_old, Kb_old, E_old, Q_old)
        self.rt_hist = [O.zeros(nx, ny) for _ in range(4)]   # T_rt1, T_rt2, E_rt1, E_rt2

    def mlqd_outer_begin(self, rt, buf):
        O, st, prob = self.O, self.st, self.prob
        if rt >= 2:
            nm = len(self.ox)
            Src_in = O.F(np.repeat(np.repeat(self.rt_src, 2, axis=0), 2, axis=1)[:, :, None, :].repeat(nm, axis=2))
            s = O.transport_scb(st["I_edgV"], st["I_edgH"], st["Ic_edgV"], st["Ic_edgH"], self.ox, self.oy, prob.delx,
                                prob.dely, self.A, self.KapE, Src_in, self.I_crn_old, C, self.ts.dt, solver=0)
            for k in ("I_crn", "I_edgV", "I_edgH", "Ic_edgV", "Ic_edgH"):
                st[k] = s[k]
            m = O.collapse_intensities(s["I_avg"], s["I_edgV"], s["I_edgH"], self.ox, self.oy, self.w, CU)
            self.HO_own = m["E_avg"]
            st.update({k: v for k, v in O.fg_calc(m, C).items() if k != "fg_avg_xy"})
            st.update(O.cg_calc(st["I_edgV"], st["I_edgH"], self.ox, self.oy, self.w, CU, (0, 0, 0, 0)))
        self._put(buf, self.HO_own)

    def mlqd_outer_begin_finish(self, tot):
        nx, ny = self.prob.nx, self.prob.ny
        self.HO_tot = self._get(tot, nx * ny, (nx, ny))
        self.mg = [self.HO_tot.copy(order="F"), self.O.zeros(nx, ny), self.st["Temp"].copy(order="F"),
                   self.O.zeros(nx, ny)]   # E_mg1, E_mg2, T_mg1, T_mg2
        self.mg_its = 0

    def mlqd_mgqd_local(self, buf):
        O, st, old, od = self.O, self.st, self.old, self.od
        d = {k: st[k] for k in O.MLOQD_FACTORS + O.MLOQD_BOUNDARY + ("Eg_avg", "Eg_edgV", "Eg_edgH")}
        d.update(Src=self.MGQD_Src, KapE=self.KapE, KapR=self.KapE, Delx=self.prob.delx, Dely=self.prob.dely, A=self.A,
                 G_old=old["G_old"], Pold_L=old["Pold_L"], Pold_B=old["Pold_B"], Pold_R=old["Pold_R"],
                 Pold_T=old["Pold_T"], Eg_avg_old=od["Eg_avg_old"], Fxg_edgV_old=od["Fxg_edgV_old"],
                 Fyg_edgH_old=od["Fyg_edgH_old"])
        sol = O.mloqd_fv(d, C, self.ts.dt, self.Theta, res_calc=False, solver=0)
        for k in ("Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH"):
            st[k] = sol[k]
        gd = dict(st, Fxg_edgV_old=od["Fxg_edgV_old"], Fyg_edgH_old=od["Fyg_edgH_old"], KapE=self.KapE,
                  KapR=self.KapE, A=self.A, Pold_L=old["Pold_L"], Pold_R=old["Pold_R"], Pold_B=old["Pold_B"],
                  Pold_T=old["Pold_T"])
        self._put(buf, O.grey_sums(gd, C, self.ts.dt, self.Theta))

    def mlqd_mgqd_finish(self, mg, tot):
        O, st = self.O, self.st
        nx, ny = self.prob.nx, self.prob.ny
        gf = O.grey_from_sums(tot.numpy(), nx, ny)
        g = {k: gf[k] for k in ("KapE_Bar",) + O.GREY_D + O.GREY_P + tuple("Cb_" + s for s in O.SIDES)}
        for k in ("E_avg", "E_edgV", "E_edgH", "Fx_edgV", "Fy_edgH"):
            g[k] = gf[k]
        for k in ("E_in_", "F_in_"):
            for s_ in O.SIDES:
                g[k + s_] = st[k + s_]
        E_mg1, E_mg2, T_mg1, T_mg2 = self.mg
        g.update(Temp=st["Temp"], Temp_Mold=T_mg2, KapE_bar_Mold=st["KapE_Bar"].copy(order="F"), Delx=self.prob.delx,
                 Dely=self.prob.dely, A=self.A, Gold_Hat=self.Gold_Hat, Rhat_old=self.Rhat_old)
        o = O.egp_fv_newt(g, self.Theta, self.ts.dt, self.ts.Kap0, self.cv, CU, Maxits=self.maxit_gloqd, MGQD_It=mg,
                          Res_Calc=False)
        for k in O.EGP_STATE:
            st[k] = o[k]
        st["GQD_Src"], st["KapE_Bar_dT"] = o["Q_bar"], o["KapE_Bar_dT"]
        self.egp_hist.append(o["Its"])
        self.KapE, self.rt_src, Bg = O.material_update(st["Temp"], self.nu, self.km, CU)
        self.MGQD_Src = O.F(4.0 * np.pi * self.KapE * Bg)
        tc, _, _ = O.convergence(2, self.conv_lo, st["Temp"], T_mg1, T_mg2, mg)
        ec, _, _ = O.convergence(2, self.conv_lo, gf["E_avg"], E_mg1, E_mg2, mg)
        self.mg = [gf["E_avg"].copy(order="F"), E_mg1, st["Temp"].copy(order="F"), T_mg1]
        self.mg_its = mg
        return bool(tc and ec)

    def mlqd_outer_end(self, rt):
        O, st = self.O, self.st
        T_rt1, T_rt2, E_rt1, E_rt2 = self.rt_hist
        tc, _, _ = O.convergence(2, self.conv_ho, st["Temp"], T_rt1, T_rt2, rt)
        ec, _, _ = O.convergence(2, self.conv_ho, self.HO_tot, E_rt1, E_rt2, rt)
        self.rt_hist = [st["Temp"].copy(order="F"), T_rt1, self.HO_tot.copy(order="F"), E_rt1]
        self.mg_hist.append(self.mg_its)
        return bool(tc and ec)

    def mlqd_step_end(self):
        return {"mgqd_per_outer": list(self.mg_hist), "egp_per_mgqd": list(self.egp_hist)}


def _oracle_reference(prob, ts, km, bcT, cv, steps, **kw):
    from oracle import oracle as O
    ox, oy, w = prob.directions()
    st = O.mlqd_init(prob.nx, prob.ny, ox, oy, w, ts.nu_eV, ts.Tini_eV, CU, C, bcT=bcT)
    hist = O.mlqd_steps(st, ox, oy, w, prob.delx, prob.dely, ts.nu_eV, km, cv, ts.Kap0, CU, C, ts.dt, steps, bcT=bcT,
                        solver=0, **kw)
    return st, hist


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


# ------------------------------------------------------------------------------------------------ CPU

def test_split_grey_sums_reproduce_the_unsplit_routines(oracle):
    """grey_from_sums(sum over ranges of grey_sums) = COLLAPSE_MG_EF, Cbar_Calc and GREY_COEFS."""
    rng = np.random.default_rng(5)
    nx, ny, ng = 5, 4, 6
    F = oracle.F
    d = {"Eg_avg": F(rng.uniform(1, 2, (nx, ny, ng))), "Eg_edgV": F(rng.uniform(1, 2, (nx + 1, ny, ng))),
         "Eg_edgH": F(rng.uniform(1, 2, (nx, ny + 1, ng))), "Fxg_edgV": F(rng.normal(size=(nx + 1, ny, ng))),
         "Fyg_edgH": F(rng.normal(size=(nx, ny + 1, ng))), "Fxg_edgV_old": F(rng.normal(size=(nx + 1, ny, ng))),
         "Fyg_edgH_old": F(rng.normal(size=(nx, ny + 1, ng))), "KapE": F(rng.uniform(0.1, 5, (nx, ny, ng))),
         "A": F(rng.uniform(0.5, 1, (nx, ny)))}
    d["KapR"] = d["KapE"]
    for k, shp in (("fg_avg_xx", (nx, ny)), ("fg_avg_yy", (nx, ny)), ("fg_edgV_xx", (nx + 1, ny)),
                   ("fg_edgV_xy", (nx + 1, ny)), ("fg_edgH_yy", (nx, ny + 1)), ("fg_edgH_xy", (nx, ny + 1))):
        d[k] = F(rng.uniform(0.2, 0.5, shp + (ng,)))
    for s, n in zip("LBRT", (ny, nx, ny, nx)):
        d["Cg_" + s] = F(rng.uniform(-0.6, 0.6, (n, ng)))
        d["Eg_in_" + s] = F(rng.uniform(0.0, 0.5, (n, ng)))
    for k in ("Pold_L", "Pold_R", "Pold_B", "Pold_T"):
        d[k] = F(rng.normal(size=(nx, ny, ng)))
    c, dt, th = 3.0, 0.01, 1.0
    tot = oracle.grey_sums({k: (v[..., :2] if v.ndim == 3 or k[:2] in ("Cg", "Eg") and v.ndim == 2 else v)
                            for k, v in d.items()}, c, dt, th)
    tot = tot + oracle.grey_sums({k: (v[..., 2:] if v.ndim == 3 or k[:2] in ("Cg", "Eg") and v.ndim == 2 else v)
                                  for k, v in d.items()}, c, dt, th)
    out = oracle.grey_from_sums(tot, nx, ny)
    ref = oracle.collapse_mg_ef(d)
    ref.update(oracle.cbar_calc(d))
    ref.update(oracle.grey_coefs(d, c, dt, th))
    for k, v in ref.items():
        assert rel(out[k], v) < 1e-14, k


def _run_members(members, steps, maxit_rte, maxit_mloqd, allreduce=None):
    import torch
    drv = S.ShardedMlqd(members, maxit_rte, maxit_mloqd, allreduce=allreduce, device=torch.device("cpu"))
    return [drv.step() for _ in range(steps)], drv


def test_two_group_ranges_match_the_unsplit_oracle_loop(oracle):
    prob, ts, km, bcT, cv = setup_problem()
    kw = dict(conv_ho=0.0, conv_lo=0.0, maxit_rte=3, maxit_mloqd=3)
    st, ref = _oracle_reference(prob, ts, km, bcT, cv, 2, **kw)
    members = [OracleMlqdMember(prob, ts, km, bcT, cv, g0, g1, 0.0, 0.0) for g0, g1 in S.group_ranges(prob.ng, 2)]
    hist, drv = _run_members(members, 2, 3, 3)
    # per step: one exchange for G_old, then per outer iteration one for the transport E and one per MGQD iteration
    assert drv.exchanges == 2 * (1 + 3 * (1 + 3))
    for step in hist:
        for h in step:
            assert h["mgqd_per_outer"] == [3, 3, 3]
    for m in members:
        assert rel(m.st["Temp"], st["Temp"]) < 1e-12
        assert rel(m.st["E_avg"], st["E_avg"]) < 1e-12
        assert rel(m.HO_tot, st["HO_E_avg"]) < 1e-12
        assert rel(m.st["KapE_Bar"], st["KapE_Bar"]) < 1e-12
    sl = [slice(g0, g1) for g0, g1 in S.group_ranges(prob.ng, 2)]
    for m, s_ in zip(members, sl):
        assert rel(m.st["Eg_avg"], st["Eg_avg"][..., s_]) < 1e-12
        assert rel(m.st["I_crn"], st["I_crn"][..., s_]) < 1e-12


def test_two_group_ranges_converge_like_the_unsplit_loop(oracle):
    prob, ts, km, bcT, cv = setup_problem(6, 5, 4, "S8", 62)
    kw = dict(conv_ho=1e-6, conv_lo=1e-7, maxit_rte=20, maxit_mloqd=40)
    st, ref = _oracle_reference(prob, ts, km, bcT, cv, 1, **kw)
    members = [OracleMlqdMember(prob, ts, km, bcT, cv, g0, g1, 1e-6, 1e-7) for g0, g1 in S.group_ranges(prob.ng, 2)]
    hist, _ = _run_members(members, 1, 20, 40)
    assert hist[0][0]["mgqd_per_outer"] == ref[0]["MGQD_Its"]
    assert rel(members[0].st["Temp"], st["Temp"]) < 1e-10


def _gloo_worker(rank, world, path, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"file://{path}", rank=rank, world_size=world)
    try:
        prob, ts, km, bcT, cv = setup_problem()
        g0, g1 = S.group_ranges(prob.ng, world)[rank]
        m = OracleMlqdMember(prob, ts, km, bcT, cv, g0, g1, 0.0, 0.0)
        hist, drv = _run_members([m], 2, 3, 3, allreduce=S.torch_allreduce())
        np.savez(f"{out}_{rank}.npz", Temp=m.st["Temp"], E_avg=m.st["E_avg"], Eg_avg=m.st["Eg_avg"],
                 exchanges=drv.exchanges)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_the_unsplit_oracle_loop(oracle):
    import torch.multiprocessing as mp
    prob, ts, km, bcT, cv = setup_problem()
    st, _ = _oracle_reference(prob, ts, km, bcT, cv, 2, conv_ho=0.0, conv_lo=0.0, maxit_rte=3, maxit_mloqd=3)
    with tempfile.TemporaryDirectory() as tmp:
        path, out = os.path.join(tmp, "rdv"), os.path.join(tmp, "r")
        mp.start_processes(_gloo_worker, args=(2, path, out), nprocs=2, join=True, start_method="spawn")
        r = [np.load(f"{out}_{k}.npz") for k in range(2)]
    for k, (g0, g1) in enumerate(S.group_ranges(prob.ng, 2)):
        assert int(r[k]["exchanges"]) == 2 * (1 + 3 * (1 + 3))
        assert rel(r[k]["Temp"], st["Temp"]) < 1e-12
        assert rel(r[k]["E_avg"], st["E_avg"]) < 1e-12
        assert rel(r[k]["Eg_avg"], st["Eg_avg"][..., g0:g1]) < 1e-12


# ------------------------------------------------------------------------------------------------ GPU

def _handle(prob, ts, km, bcT, cv, g0=0, g1=None, split=False, **kw):
    g1 = prob.ng if g1 is None else g1
    ox, oy, w = prob.directions()
    nu = ts.nu_eV[g0:g1 + 1]
    s = pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, g1 - g0, precision="fp64")
    s.init_state(ts.Tini_eV, list(bcT), CU, nu)
    s.tstep_setup(nu, km, cv, np.full((prob.nx, prob.ny), ts.Tini_eV), ts.Kap0, CU, C, ts.dt, bcT=bcT,
                  conv_type=2, conv_ho=kw.pop("conv_ho", 0.0), maxit_rte=kw.pop("maxit_rte", 3))
    s.mlqd_setup(ts.Tini_eV, group_range=(g0, ts.nu_eV) if split else None, **kw)
    return s


@pytest.mark.gpu
def test_one_handle_through_the_phases_equals_trt_mlqd_step():
    prob, ts, km, bcT, cv = setup_problem(9, 7, 5, "S8", 63)
    kw = dict(conv_ho=1e-7, conv_lo=1e-8, maxit_rte=10, maxit_mloqd=30)
    with _handle(prob, ts, km, bcT, cv, **dict(kw)) as a, _handle(prob, ts, km, bcT, cv, **dict(kw)) as b:
        drv = S.ShardedMlqd([b], 10, 30)
        for _ in range(2):
            ra = a.mlqd_step()
            rb = drv.step()[0]
            assert ra["mgqd_per_outer"] == rb["mgqd_per_outer"] and ra["egp_per_mgqd"] == rb["egp_per_mgqd"]
            for k in ("Temp", "E_avg", "HO_E_avg", "Eg_avg", "KapE_Bar", "Cb_L", "Fx_edgV", "MGQD_Src"):
                assert np.array_equal(a.mlqd_field(k), b.mlqd_field(k)), k
        assert np.array_equal(a.get_state(), b.get_state())


@pytest.mark.gpu
def test_two_group_range_handles_match_one_handle():
    prob, ts, km, bcT, cv = setup_problem(9, 7, 6, "S8", 64)
    kw = dict(conv_ho=0.0, conv_lo=0.0, maxit_rte=3, maxit_mloqd=3)
    ranges = S.group_ranges(prob.ng, 2)
    with _handle(prob, ts, km, bcT, cv, **dict(kw)) as a:
        parts = [_handle(prob, ts, km, bcT, cv, g0, g1, split=True, **dict(kw)) for g0, g1 in ranges]
        try:
            drv = S.ShardedMlqd(parts, 3, 3)
            for _ in range(2):
                ra = a.mlqd_step()
                rb = drv.step()
                for r in rb:
                    assert r["mgqd_per_outer"] == ra["mgqd_per_outer"] == [3, 3, 3]
                for p in parts:
                    assert rel(p.mlqd_field("Temp"), a.mlqd_field("Temp")) < 1e-12
                    assert rel(p.mlqd_field("E_avg"), a.mlqd_field("E_avg")) < 1e-12
                    assert rel(p.mlqd_field("HO_E_avg"), a.mlqd_field("HO_E_avg")) < 1e-12
            Eg = a.mlqd_field("Eg_avg")
            for p, (g0, g1) in zip(parts, ranges):
                assert rel(p.mlqd_field("Eg_avg"), Eg[..., g0:g1]) < 1e-12
        finally:
            for p in parts:
                p.close()
