"""The transport-only time loop with the groups split over several handles (sharded.ShardedTimeLoop): the
group ranges of a multi-GPU run, or group slabs on one device.  The only exchange is the per-cell group
sums of the energy balance, added across the ranges every outer iteration.

CPU: the driver over oracle-backed members (each sweeps its group range with the oracle's TRANSPORT_SCB
restatement and forms its sums with the oracle's split energy balance) against the oracle's unsplit loop,
in one process and as two gloo ranks.  GPU: the driver over library handles, one handle against trt_tstep
bit for bit, two group-range handles on one device against one handle."""
import os
import tempfile

import numpy as np
import pytest

from common import C, CU, pkg, sweep_inputs

P = pkg.problems
S = pkg.sharded


def _problem():
    prob = P.random_small(51, 6, 5, 5, "S8")
    return prob, P.config_timestep_setup(prob)


class OracleMember:
    """A group range [g0, g1) of the time loop on the CPU oracle (test infrastructure)."""

    def __init__(self, prob, ts, g0, g1, law=1):
        from oracle import oracle as O
        self.O, self.prob, self.ts, self.g0, self.g1, self.law = O, prob, ts, g0, g1, law
        d = sweep_inputs(prob, random_old=False)
        sl = slice(g0, g1)
        self.st = {k: np.asfortranarray(d[k][..., sl]) for k in ("I_crn_old", "Ic_edgV", "Ic_edgH", "I_edgV", "I_edgH")}
        self.st["I_crn"] = self.st.pop("I_crn_old")
        self.d = d
        self.nu = ts.nu_eV[g0:g1 + 1]
        self.T = np.full((prob.nx, prob.ny), ts.Tini_eV, order="F")
        self._material()
        z = np.zeros((prob.nx, prob.ny), order="F")
        self.hist = [z.copy(), z.copy(), z.copy(), z.copy()]   # T_rt1, T_rt2, E_rt1, E_rt2

    def _material(self):
        mat = self.O.material_update_law if self.law == 1 else self.O.material_update
        self.KapE, self.src, _ = mat(self.T, self.nu, self.ts.kappa_mult, CU)

    def tstep_begin(self):
        self.Told = self.T.copy(order="F")
        self.I_old = self.st["I_crn"].copy(order="F")
        z = np.zeros_like(self.T)
        self.hist = [z.copy(), z.copy(), z.copy(), z.copy()]

    def tstep_sweep(self, its):
        O, d, nm = self.O, self.d, len(self.d["Omega_x"])
        Src_in = np.asfortranarray(np.repeat(np.repeat(self.src, 2, axis=0), 2, axis=1)[:, :, None, :].repeat(nm, axis=2))
        s = O.transport_scb(self.st["I_edgV"], self.st["I_edgH"], self.st["Ic_edgV"], self.st["Ic_edgH"], d["Omega_x"],
                            d["Omega_y"], d["Delx"], d["Dely"], d["A"], self.KapE, Src_in, self.I_old, C, self.ts.dt,
                            solver=1)
        for k in ("I_crn", "I_edgV", "I_edgH", "Ic_edgV", "Ic_edgH"):
            self.st[k] = s[k]
        self.m = O.collapse_intensities(s["I_avg"], s["I_edgV"], s["I_edgH"], d["Omega_x"], d["Omega_y"], d["w"], CU)

    def tstep_partials(self, buf):
        part = self.O.meb_partial(self.m["Eg_avg"], self.KapE, self.T, self.nu, CU, C, 0, self.g1 - self.g0, self.law)
        buf.numpy()[:] = part.ravel(order="F")

    def tstep_finish(self, total, its):
        nx, ny = self.T.shape
        sums = total.numpy().reshape((nx, ny, 3), order="F")
        self.T, E = self.O.meb_finish(sums, self.Told, self.ts.cv, self.ts.dt, self.ts.Kap0, CU, self.law)
        self._material()
        T1, T2, E1, E2 = self.hist
        tc, tn, _ = self.O.convergence(2, 0.0, self.T, T1, T2, its)
        ec, en, _ = self.O.convergence(2, 0.0, E, E1, E2, its)
        self.hist = [self.T.copy(order="F"), T1, E.copy(order="F"), E1]
        return tc and ec, tn, en

    def sync(self):
        pass


def _oracle_unsplit(prob, ts, steps, maxit):
    from oracle import oracle as O
    d = sweep_inputs(prob, random_old=False)
    st = dict(I_crn=d["I_crn_old"].copy(order="F"), Ic_edgV=d["Ic_edgV"], Ic_edgH=d["Ic_edgH"], I_edgV=d["I_edgV"],
              I_edgH=d["I_edgH"], Temp=np.full((prob.nx, prob.ny), ts.Tini_eV, order="F"))
    return O.tr_no_qd_steps(st, d["Omega_x"], d["Omega_y"], d["w"], d["Delx"], d["Dely"], ts.nu_eV, ts.kappa_mult,
                            ts.cv, ts.Kap0, CU, C, ts.dt, steps, conv_type=2, conv_ho=0.0, maxit=maxit, law=1)


def _rel(a, b):
    return float(np.max(np.abs(a - b) / np.abs(b)))


def test_group_ranges_cover_and_balance():
    for ng, parts in ((17, 1), (17, 2), (50, 8), (64, 3), (5, 5)):
        r = S.group_ranges(ng, parts)
        assert r[0][0] == 0 and r[-1][1] == ng and all(a[1] == b[0] for a, b in zip(r, r[1:]))
        sizes = [g1 - g0 for g0, g1 in r]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        S.group_ranges(4, 5)


def test_split_time_loop_on_oracle_members_matches_unsplit(oracle):
    prob, ts = _problem()
    ref = _oracle_unsplit(prob, ts, 3, 4)
    members = [OracleMember(prob, ts, g0, g1) for g0, g1 in S.group_ranges(prob.ng, 3)]
    loop = S.ShardedTimeLoop(members, prob.nx, prob.ny, maxit=4, device="cpu")
    for T_ref, _, its_ref, _, _ in ref:
        its, _, _ = loop.step()
        assert its == its_ref == 4
        for m in members:
            assert _rel(m.T, T_ref) < 1e-12


def _gloo_rank(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prob, ts = _problem()
        g0, g1 = S.group_ranges(prob.ng, world)[rank]
        member = OracleMember(prob, ts, g0, g1)
        loop = S.ShardedTimeLoop([member], prob.nx, prob.ny, maxit=4, allreduce=S.torch_allreduce(), device="cpu")
        Ts = []
        for _ in range(3):
            its, _, _ = loop.step()
            Ts.append(member.T.copy())
        np.save(os.path.join(out_dir, f"T{rank}.npy"), np.stack(Ts))
        np.save(os.path.join(out_dir, f"x{rank}.npy"), np.array([loop.exchanges, its]))
    finally:
        dist.destroy_process_group()


def test_split_time_loop_over_two_gloo_ranks(oracle):
    import socket

    import torch.multiprocessing as mp
    prob, ts = _problem()
    ref = _oracle_unsplit(prob, ts, 3, 4)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    with tempfile.TemporaryDirectory() as out:
        mp.start_processes(_gloo_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
        T = [np.load(os.path.join(out, f"T{r}.npy")) for r in range(2)]
        x = [np.load(os.path.join(out, f"x{r}.npy")) for r in range(2)]
    assert np.array_equal(T[0], T[1])            # every rank forms the same temperature
    assert x[0][0] == x[1][0] == 3 * 4           # one all-reduce per outer iteration
    for k, (T_ref, _, _, _, _) in enumerate(ref):
        assert _rel(T[0][k], T_ref) < 1e-12


# ------------------------------------------------------------------------------------------------ GPU

def _device(prob, ts, groups, law):
    g0, g1 = groups
    ox, oy, w = prob.directions()
    s = pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, g1 - g0)
    nu = ts.nu_eV[g0:g1 + 1]
    s.init_state(ts.Tini_eV, list(ts.bcT_eV), CU, nu)
    s.tstep_setup(nu, ts.kappa_mult, ts.cv, np.full((prob.nx, prob.ny), ts.Tini_eV), ts.Kap0, CU, C, ts.dt,
                  bcT=ts.bcT_eV, conv_type=2, conv_ho=0.0, maxit_rte=4, law=law)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("law", [0, 1])
def test_device_split_loop_one_handle_equals_tstep(law):
    prob = P.random_small(52, 9, 8, 4, "S8")
    ts = P.config_timestep_setup(prob) if law == 1 else P.fc_timestep_setup(prob)
    full = (0, prob.ng)
    a, b = _device(prob, ts, full, law), _device(prob, ts, full, law)
    try:
        loop = S.ShardedTimeLoop([b], prob.nx, prob.ny, maxit=4)
        for _ in range(3):
            assert a.tstep()[0] == loop.step()[0] == 4
            assert np.array_equal(a.temperature(), b.temperature())
        assert np.array_equal(a.get_state(), b.get_state())
    finally:
        a.close()
        b.close()


@pytest.mark.gpu
def test_device_group_slabs_on_one_device_match_one_handle():
    """Two handles, each with half the groups, their sums added on the device: the single-device form of
    the group-sharded run (and of the group slabs of an instance larger than the device)."""
    prob = P.random_small(53, 10, 7, 5, "S12")
    ts = P.config_timestep_setup(prob)
    one = _device(prob, ts, (0, prob.ng), 1)
    parts = [_device(prob, ts, r, 1) for r in S.group_ranges(prob.ng, 2)]
    try:
        loop = S.ShardedTimeLoop(parts, prob.nx, prob.ny, maxit=4)
        for _ in range(3):
            one.tstep()
            loop.step()
            for p in parts:
                assert _rel(p.temperature(), one.temperature()) < 1e-12
    finally:
        one.close()
        for p in parts:
            p.close()
