"""GPU test of trt_transport_residual_noalloc, the entry point that allocates no device memory.

Callers that cannot call cudaMalloc -- a host code that owns a fixed, pre-sized device arena, or a solver
loop that must not pay the device synchronisation of cudaMalloc/cudaFree -- get the residual norms of
TRANSPORT_SCB from device arrays they already hold, with the library's fixed scratch array instead of
allocated scratch.  Its results must equal those of the existing entry point (trt_transport_scb with
Res_Calc), on two calls in a row (the scratch keeps the first call's contents when the second runs).

This file is collected last so that a run stopping at its first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

from common import pkg, sweep_inputs

pytestmark = pytest.mark.gpu

LOC0 = -7   # initial RT_ResLoc values: kept where no norm exceeds zero, in both entry points


def existing_entry_point(d):
    nx, ny, nm, ng = len(d["Delx"]), len(d["Dely"]), len(d["Omega_x"]), d["KapE_in"].shape[2]
    out = dict(I_avg=np.zeros((nx, ny, nm, ng), order="F"), I_edgV=d["I_edgV"].copy(order="F"),
               I_edgH=d["I_edgH"].copy(order="F"), I_crn=np.zeros((2 * nx, 2 * ny, nm, ng), order="F"),
               Ic_edgV=d["Ic_edgV"].copy(order="F"), Ic_edgH=d["Ic_edgH"].copy(order="F"),
               RT_Residual=np.zeros((4, ng, 5), order="F"),
               RT_ResLoc_x=np.full((4, ng, 5), LOC0, dtype=np.int32, order="F"),
               RT_ResLoc_y=np.full((4, ng, 5), LOC0, dtype=np.int32, order="F"))
    pkg.TRANSPORT_SCB(out["I_avg"], out["I_edgV"], out["I_edgH"], out["I_crn"], out["Ic_edgV"], out["Ic_edgH"],
                      d["Omega_x"], d["Omega_y"], d["Delx"], d["Dely"], d["A"], d["KapE_in"], d["Src_in"],
                      d["I_crn_old"], d["c"], d["dt"], 1, out["RT_Residual"], out["RT_ResLoc_x"], out["RT_ResLoc_y"],
                      True)
    return out


def device_arrays(torch, d, sweep):
    """Device copies (allocated here, by the caller) of the arrays TRANSPORT_SCB used and produced, and the
    outputs (norms and their locations)."""
    ng = d["KapE_in"].shape[2]
    dev = lambda a, dt=torch.float64: torch.from_numpy(np.ascontiguousarray(np.asarray(a).ravel(order="F"))).to(
        device="cuda", dtype=dt)
    ins = [dev(sweep["I_crn"]), dev(sweep["Ic_edgV"]), dev(sweep["Ic_edgH"]), dev(d["Omega_x"]), dev(d["Omega_y"]),
           dev(d["Delx"]), dev(d["Dely"]), dev(d["A"]), dev(d["KapE_in"]), dev(d["Src_in"]), dev(d["I_crn_old"])]
    res = torch.zeros(4 * ng * 5, dtype=torch.float64, device="cuda")
    lx = torch.full((4 * ng * 5,), LOC0, dtype=torch.int32, device="cuda")
    ly = torch.full((4 * ng * 5,), LOC0, dtype=torch.int32, device="cuda")
    return ins, res, lx, ly


def call(torch, d, arrays):
    nx, ny, nm, ng = len(d["Delx"]), len(d["Dely"]), len(d["Omega_x"]), d["KapE_in"].shape[2]
    ins, res, lx, ly = arrays
    stream = torch.cuda.current_stream()
    rc = pkg.lib().trt_transport_residual_noalloc(nx, ny, nm, ng, *[ctypes.c_void_p(t.data_ptr()) for t in ins],
                                                  float(d["c"]), float(d["dt"]), ctypes.c_void_p(res.data_ptr()),
                                                  ctypes.c_void_p(lx.data_ptr()), ctypes.c_void_p(ly.data_ptr()),
                                                  ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, pkg.lib().trt_strerror(rc)
    torch.cuda.synchronize()


def no_alloc_entry_point(torch, d, sweep):
    ng = d["KapE_in"].shape[2]
    arrays = device_arrays(torch, d, sweep)
    call(torch, d, arrays)
    _, res, lx, ly = arrays
    shape = (4, ng, 5)
    return (res.cpu().numpy().reshape(shape, order="F"), lx.cpu().numpy().reshape(shape, order="F"),
            ly.cpu().numpy().reshape(shape, order="F"))


def test_no_alloc_residual_equals_existing_entry_point_on_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    # a larger problem first, then a smaller one: the second call runs over the first call's scratch
    cases = [sweep_inputs(pkg.problems.random_small(31, 9, 7, 4, "S12"), seed=5),
             sweep_inputs(pkg.problems.random_small(32, 5, 6, 2, "S8"), seed=6)]
    for d in cases:
        exp = existing_entry_point(d)
        res, lx, ly = no_alloc_entry_point(torch, d, exp)
        # same expression, same order, same inputs: the results are identical (tolerance 0)
        assert np.array_equal(res, exp["RT_Residual"])
        assert np.array_equal(lx, exp["RT_ResLoc_x"]) and np.array_equal(ly, exp["RT_ResLoc_y"])
        assert np.all(res[:, :, 0] > 0)


def test_no_alloc_rejects_problems_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    # n_m * n_g = 8 * 8193 > 65536: rejected before any launch
    rc = pkg.lib().trt_transport_residual_noalloc(2, 2, 8, 8193, *[p] * 11, 1.0, 1.0, p, p, p, None)
    assert rc == pkg._lib.TRT_ERR_SCRATCH
    assert "scratch" in pkg.lib().trt_strerror(rc).decode()


def test_no_alloc_call_takes_no_device_memory():
    """After a first call (which looks up the scratch array's device address), a call leaves the device's
    free memory exactly as it was: nothing is allocated, by the library or by any library it calls."""
    torch = pytest.importorskip("torch")
    d = sweep_inputs(pkg.problems.random_small(33, 7, 8, 3, "S8"), seed=7)
    arrays = device_arrays(torch, d, existing_entry_point(d))
    call(torch, d, arrays)
    free0 = torch.cuda.mem_get_info()[0]
    call(torch, d, arrays)
    call(torch, d, arrays)
    assert torch.cuda.mem_get_info()[0] == free0
