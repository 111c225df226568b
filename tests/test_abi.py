"""The C ABI library loads and exports every symbol include/trt_sweep.h declares (CPU only, no kernels)."""
import ctypes
import os
import re

import numpy as np
import pytest

from common import pkg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "trt_sweep.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(trt_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_reference_signatures():
    names = declared_functions()
    for n in ("trt_transport_scb", "trt_collapse_intensities", "trt_fg_calc", "trt_cg_calc", "trt_mgqd_in_calc",
              "trt_gqd_in_calc", "trt_rt_bc_update", "trt_create", "trt_sweep", "trt_moments", "trt_destroy",
              "trt_strerror", "trt_get_state", "trt_put_state", "trt_get_angular"):
        assert n in names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(pkg.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding declares a signature for each of them
    assert set(declared_functions()) <= set(pkg._lib.SIGNATURES)


def test_strerror_codes():
    L = pkg.lib()
    for code in range(0, -11, -1):
        msg = L.trt_strerror(code).decode()
        assert msg and msg != "unknown error"
    assert L.trt_strerror(-99).decode() == "unknown error"


def test_required_bytes_and_argument_checks():
    L = pkg.lib()
    assert L.trt_required_bytes(0, 4, 8, 1, 0) == 0           # invalid extent
    assert L.trt_required_bytes(4, 4, 6, 1, 0) == 0           # N_m not a multiple of 4
    b64 = L.trt_required_bytes(256, 256, 144, 50, 0)
    b32 = L.trt_required_bytes(256, 256, 144, 50, 1)
    # two FP64 corner states of config C1 are ~30 GB; FP32 halves them
    assert 29e9 < b64 < 40e9 and 14e9 < b32 < 22e9
    st = ctypes.c_int(0)
    d = np.zeros(8)
    h = L.trt_create(0, 4, 8, 1, *[d.ctypes.data_as(ctypes.POINTER(ctypes.c_double))] * 5, 0, 0, ctypes.byref(st))
    assert not h and st.value == pkg._lib.TRT_ERR_ARG


def test_no_device_is_reported_not_emulated():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    L = pkg.lib()
    st = ctypes.c_int(0)
    one = np.ones(8)
    p = one.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    h = L.trt_create(4, 4, 8, 1, p, p, p, p, p, 0, 0, ctypes.byref(st))
    assert not h and st.value == pkg._lib.TRT_ERR_NODEV


def test_rom_entry_points_need_a_device():
    """The POD / DMD entry points check their arguments, then report a missing device (no CPU path)."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    data = np.random.default_rng(0).standard_normal((6, 2, 5))
    with pytest.raises(pkg.TrtError) as e:
        pkg.POD_Calc(data, 5, 2, 6, 1)
    assert e.value.code == pkg._lib.TRT_ERR_NODEV
    with pytest.raises(pkg.TrtError) as e:
        pkg.POD_Calc(data, 5, 2, 6, 2)                      # block index out of range
    assert e.value.code == pkg._lib.TRT_ERR_ARG
    with pytest.raises(pkg.TrtError) as e:
        pkg.DMD_Calc(data, 5, 2, 6, 0, delt=0.1)
    assert e.value.code == pkg._lib.TRT_ERR_NODEV
    out = np.zeros(12)
    with pytest.raises(pkg.TrtError) as e:
        pkg.POD_RECONSTRUCT(out, np.zeros(12), np.ones(2), np.ones(12), np.ones(10), [1, 1], 12, 2, 5, 6, 0)
    assert e.value.code == pkg._lib.TRT_ERR_ARG            # t beyond N_t
    with pytest.raises(pkg.TrtError) as e:
        pkg.DMD_RECONSTRUCT(out, np.ones(2), np.ones(2), np.ones(12), np.zeros(12), [1, 1], 12, 2, 0, 0.5)
    assert e.value.code == pkg._lib.TRT_ERR_NODEV


def test_reconstruction_drivers_check_arguments_before_the_device():
    """The ROM drivers reject inconsistent calls on the host (group counts that differ, a simulation level or a
    time-map entry out of range, two bracketing data levels at one time) and only then look for a device."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    dN, N, ng, nt = 3, 4, 2, 3
    d = np.full(dN, 1.0 / dN)
    s = np.full(N, 1.0 / N)
    grids = pkg.GENERATE_GRIDS_XY(d, d, s, s, 1.0, 1.0, 1.0, 1.0)
    tgrids = pkg.GENERATE_GRIDS_T(1e-3, 1e-3, 0.0, 0.0, nt, nt)
    rank = np.ones(ng, dtype=np.int32)

    def dec(n):
        return (np.zeros(n), np.ones(ng), np.ones(n), np.ones(nt * ng), rank)

    la, lv, lh = dN * dN * ng, (dN + 1) * dN * ng, dN * (dN + 1) * ng
    fg = {k: dec(n) for k, n in zip(("avg_xx", "edgV_xx", "avg_yy", "edgH_yy", "edgV_xy", "edgH_xy"),
                                    (la, lv, la, lh, lv, lh))}
    bc = dec(ng * 4 * dN)

    def code(fn, *a):
        with pytest.raises(pkg.TrtError) as e:
            fn(*a)
        return e.value.code

    ARG, NODEV = pkg._lib.TRT_ERR_ARG, pkg._lib.TRT_ERR_NODEV
    assert code(pkg.POD_RECONSTRUCT_fg, fg, (dN, dN, ng, nt), (N, N, ng, nt), 2, 0, grids, tgrids) == NODEV
    assert code(pkg.POD_RECONSTRUCT_BCg, bc, (dN, dN, ng, nt), (N, N, ng, nt), 2, 0, grids, tgrids) == NODEV
    assert code(pkg.POD_RECONSTRUCT_fg, fg, (dN, dN, ng, nt), (N, N, ng + 1, nt), 2, 0, grids, tgrids) == ARG
    assert code(pkg.POD_RECONSTRUCT_BCg, bc, (dN, dN, ng, nt), (N, N, ng, nt), nt + 1, 0, grids, tgrids) == ARG
    bad_map = (tgrids[0], tgrids[1], np.array([1, 1, nt + 1, nt + 1, 3, 3], dtype=np.int32))
    assert code(pkg.POD_RECONSTRUCT_BCg, bc, (dN, dN, ng, nt), (N, N, ng, nt), 2, 0, grids, bad_map) == ARG
    same_time = (tgrids[0], np.array([1e-3, 1e-3, 3e-3]), np.array([1, 1, 2, 1, 3, 3], dtype=np.int32))
    assert code(pkg.POD_RECONSTRUCT_BCg, bc, (dN, dN, ng, nt), (N, N, ng, nt), 2, 0, grids, same_time) == ARG
    dmd = {k: (np.ones(ng, dtype=complex), np.ones(ng, dtype=complex), np.ones(v[0].size, dtype=complex), v[0], rank)
           for k, v in fg.items()}
    assert code(pkg.DMD_RECONSTRUCT_fg, dmd, (dN, dN, ng), (N, N, ng), 0.1, 0, grids) == NODEV
    assert code(pkg.DMD_RECONSTRUCT_fg, dmd, (dN, dN, ng), (N, N, ng), 0.1, 2, grids) == ARG
