"""Batched instances (one sweep launch per tiling class over many handles) against the same handles
stepped one by one: bit-identical states, moments and temperatures, with mixed shapes, quadratures,
precisions and tilings in one batch."""
import numpy as np
import pytest

from common import CU, C, pkg, sweep_inputs

pytestmark = pytest.mark.gpu

SHAPES = [(9, 7, 2, "S8", "fp64"), (13, 11, 3, "S8", "fp64"), (6, 17, 2, "S12", "fp64"), (21, 5, 3, "S16", "fp64"),
          (9, 7, 2, "S8", "fp32"), (15, 12, 2, "S16", "fp32")]


def _resident(k, nx, ny, G, quad, prec):
    prob = pkg.problems.random_small(40 + k, nx, ny, G, quad)
    d = sweep_inputs(prob, seed=40 + k)
    s = pkg.TransportSweep(nx, ny, d["Omega_x"], d["Omega_y"], d["w"], d["Delx"], d["Dely"], G, precision=prec)
    s.put_state(d["I_crn_old"])
    s.set_boundary(d["Ic_edgV"], d["Ic_edgH"], (0, 0, 0, 0))
    s.set_material(d["KapE_in"], d["src_iso"], d["c"], d["dt"], CU)
    return s


@pytest.mark.parametrize("persistent", [True, False], ids=["queue", "grid"])
def test_batched_sweep_matches_single_sweeps(persistent):
    alone, batched = [], []
    for k, sh in enumerate(SHAPES):
        with _resident(k, *sh) as s:
            s.sweep(roll=True, moments=True)
            s.sweep(roll=False, moments=True)
            alone.append((s.get_state(), s.moments(["Eg_avg", "fg_edgV_xy", "Cg_T", "E_avg"])))
    hs = [_resident(k, *sh) for k, sh in enumerate(SHAPES)]
    hs[2].set_tiling(warps=3)                     # a tiling class of its own
    hs[2].put_state(_state_of(2))
    try:
        with pkg.Batch(hs) as b:
            b.set_persistent(persistent)
            b.sweep(roll=True)
            b.sweep(roll=False)
        for s in hs:
            batched.append((s.get_state(), s.moments(["Eg_avg", "fg_edgV_xy", "Cg_T", "E_avg"])))
    finally:
        for s in hs:
            s.close()
    for (Ia, ma), (Ib, mb) in zip(alone, batched):
        assert np.array_equal(Ia, Ib)
        for k in ma:
            assert np.array_equal(ma[k], mb[k]), k


def _state_of(k):
    nx, ny, G, quad, _ = SHAPES[k]
    return sweep_inputs(pkg.problems.random_small(40 + k, nx, ny, G, quad), seed=40 + k)["I_crn_old"]


def _tstep_handle(k, n, G, quad, prec):
    prob = pkg.problems.random_small(60 + k, n, n + 1, G, quad)
    ts = pkg.problems.fc_timestep_setup(prob)
    ox, oy, w = prob.directions()
    s = pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng, precision=prec)
    s.init_state(ts.Tini_eV, list(ts.bcT_eV), CU, ts.nu_eV)
    s.tstep_setup(ts.nu_eV, ts.kappa_mult, ts.cv, np.full((prob.nx, prob.ny), ts.Tini_eV), ts.Kap0, CU, C, ts.dt,
                  conv_type=2, conv_ho=1e-7, maxit_rte=12 + 3 * k)
    return s


def test_batched_time_steps_match_single_handles():
    cfg = [(6, 2, "S8", "fp64"), (9, 3, "S12", "fp64"), (5, 2, "S8", "fp32"), (11, 2, "S16", "fp64")]
    alone = []
    for k, c in enumerate(cfg):
        with _tstep_handle(k, *c) as s:
            alone.append([(s.tstep()[0], s.temperature()) for _ in range(3)])
    hs = [_tstep_handle(k, *c) for k, c in enumerate(cfg)]
    try:
        with pkg.Batch(hs) as b:
            for step in range(3):
                its, _, _ = b.tstep()
                for k, s in enumerate(hs):
                    assert its[k] == alone[k][step][0]
                    assert np.array_equal(s.temperature(), alone[k][step][1])
    finally:
        for s in hs:
            s.close()


def test_batch_rejects_duplicates_and_empty():
    with _resident(0, *SHAPES[0]) as s:
        with pytest.raises(pkg.TrtError):
            pkg.Batch([s, s])
    with pytest.raises(pkg.TrtError):
        pkg.Batch([])
