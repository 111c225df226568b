"""Pipelined stepping: trt_set_material_async / trt_moments_async (copies on the handle's two copy streams,
overlapping the neighbouring sweeps) give the same state and outputs, bit for bit, as the synchronous
trt_set_material / trt_moments, step after step, with a different material every step."""
import ctypes

import numpy as np
import pytest

from common import CU, pkg, sweep_inputs

pytestmark = pytest.mark.gpu

NAMES = ("fg_avg_xx", "fg_edgV_xy", "fg_edgH_yy", "Cg_L", "Cg_T", "Eg_avg", "E_avg", "Fx_edgV")


def materials(d, steps):
    rng = np.random.default_rng(7)
    out = []
    for _ in range(steps):
        f = rng.uniform(0.5, 2.0, d["KapE_in"].shape)
        out.append((np.asfortranarray(d["KapE_in"] * f), np.asfortranarray(d["src_iso"] * f ** 2)))
    return out


def make(d, precision):
    nx, ny, ng = len(d["Delx"]), len(d["Dely"]), d["KapE_in"].shape[2]
    s = pkg.TransportSweep(nx, ny, d["Omega_x"], d["Omega_y"], d["w"], d["Delx"], d["Dely"], ng, precision=precision)
    s.put_state(d["I_crn_old"])
    s.set_boundary(d["Ic_edgV"], d["Ic_edgH"], (0, 0, 0, 0))
    return s


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_async_stepping_matches_synchronous(precision):
    prob = pkg.problems.random_small(41, 23, 17, 3, "S12")
    d = sweep_inputs(prob, seed=4)
    mats = materials(d, 4)
    nx, ny, ng = prob.nx, prob.ny, prob.ng
    with make(d, precision) as s:
        ref = []
        for kap, src in mats:
            s.set_material(kap, src, d["c"], d["dt"], CU)
            s.sweep(roll=True, moments=True)
            ref.append(s.moments(list(NAMES)))
        ref_state = s.get_state()
    with make(d, precision) as s:
        outs, keep = [], []
        for kap, src in mats:
            s.set_material_async(kap, src, d["c"], d["dt"], CU)
            s.sweep(roll=True, moments=True, sync=False)
            o = {n: np.zeros(pkg._lib.moment_shape(n, nx, ny, ng), order="F") for n in NAMES}
            mh = pkg._lib.MomentsHost()
            for n, a in o.items():
                setattr(mh, n, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
            s.moments_async(mh)
            outs.append(o)
            keep.append(mh)
        s.sync()
        state = s.get_state()
    for o, r in zip(outs, ref):
        for n in NAMES:
            assert np.array_equal(o[n], r[n]), n
    assert np.array_equal(state, ref_state)


def test_async_and_snapshot_call_order():
    prob = pkg.problems.random_small(42, 5, 4, 2, "S8")
    d = sweep_inputs(prob, seed=5)
    with make(d, "fp64") as s:
        mh = pkg._lib.MomentsHost()
        with pytest.raises(pkg.TrtError):
            s.moments_async(mh)                                   # no moments yet
        dst = np.zeros(1)
        L = pkg.lib()
        assert L.trt_snapshot_output(s.handle, b"fg_avg_xx", ctypes.c_void_p(dst.ctypes.data)) == \
            pkg._lib.TRT_ERR_STATE
        s.set_material(d["KapE_in"], d["src_iso"], d["c"], d["dt"], CU)
        s.sweep(roll=True, moments=True)
        assert L.trt_snapshot_output(s.handle, b"no_such_output", ctypes.c_void_p(dst.ctypes.data)) == \
            pkg._lib.TRT_ERR_ARG
        assert L.trt_snapshot_angular(s.handle, None) == pkg._lib.TRT_ERR_ARG
        # a synchronous call after asynchronous ones sees their effect
        kap, src = materials(d, 1)[0]
        s.set_material_async(kap, src, d["c"], d["dt"], CU)
        s.sweep(roll=False, moments=True, sync=False)
        o = s.moments(["E_avg"])["E_avg"]
        with make(d, "fp64") as r:
            r.set_material(d["KapE_in"], d["src_iso"], d["c"], d["dt"], CU)
            r.sweep(roll=True, moments=True)
            r.set_material(kap, src, d["c"], d["dt"], CU)
            r.sweep(roll=False, moments=True)
            assert np.array_equal(o, r.moments(["E_avg"])["E_avg"])
