"""In-place corner state (one buffer swept in place) and caller-bound state memory: the machinery that
lets the 1024^2 x 64-group x S16 instance fit (FP32) or stream through the device in group slabs (FP64).
Checked bit for bit against the default two-buffer handle."""
import numpy as np
import pytest

from common import CU, pkg, sweep_inputs

pytestmark = pytest.mark.gpu


def _handle(d, precision, inplace, bands=0):
    nx, ny, ng = len(d["Delx"]), len(d["Dely"]), d["KapE_in"].shape[2]
    s = pkg.TransportSweep(nx, ny, d["Omega_x"], d["Omega_y"], d["w"], d["Delx"], d["Dely"], ng, precision=precision)
    if inplace:
        s.set_inplace(True)
    if bands:
        s.set_tiling(warps=1, slices=8)
        s.set_bands(bands)
    s.put_state(d["I_crn_old"])
    s.set_boundary(d["Ic_edgV"], d["Ic_edgH"], (0, 0, 0, 0))
    s.set_material(d["KapE_in"], d["src_iso"], d["c"], d["dt"], CU)
    return s


@pytest.mark.parametrize("precision,bands", [("fp64", 0), ("fp32", 0), ("fp32", 3)])
def test_inplace_steps_bit_identical(precision, bands):
    prob = pkg.problems.random_small(12, 19, 23, 3, "S12")
    d = sweep_inputs(prob, seed=3)
    out = []
    for inplace in (False, True):
        with _handle(d, precision, inplace, bands) as s:
            for k in range(3):
                s.sweep(roll=k > 0, moments=True)
            out.append((s.get_state(), s.moments(["Eg_avg", "fg_edgH_xy", "Cg_R"])))
    assert np.array_equal(out[0][0], out[1][0])
    for k in out[0][1]:
        assert np.array_equal(out[0][1][k], out[1][1][k]), k


def test_inplace_from_creation_equals_switched_in_place():
    prob = pkg.problems.random_small(15, 8, 9, 2, "S8")
    d = sweep_inputs(prob, seed=8)
    nx, ny, ng = len(d["Delx"]), len(d["Dely"]), d["KapE_in"].shape[2]
    out = []
    for created in (False, True):
        s = pkg.TransportSweep(nx, ny, d["Omega_x"], d["Omega_y"], d["w"], d["Delx"], d["Dely"], ng, inplace=created)
        with s:
            if not created:
                s.set_inplace(True)
            s.put_state(d["I_crn_old"])
            s.set_boundary(d["Ic_edgV"], d["Ic_edgH"], (0, 0, 0, 0))
            s.set_material(d["KapE_in"], d["src_iso"], d["c"], d["dt"], CU)
            s.sweep(moments=True)
            s.sweep(roll=True, moments=True)
            out.append(s.get_state())
    assert np.array_equal(out[0], out[1])


def test_inplace_refuses_a_second_sweep_of_the_same_step():
    prob = pkg.problems.random_small(13, 6, 5, 2, "S8")
    d = sweep_inputs(prob, seed=4)
    with _handle(d, "fp64", True) as s:
        s.sweep(moments=True)
        with pytest.raises(pkg.TrtError):
            s.sweep(moments=True)                  # I_crn_old was overwritten
        with pytest.raises(pkg.TrtError):
            s.sweep(roll=True, res_calc=True)      # the residual needs I_crn_old
        s.sweep(roll=True, moments=True)


def test_bound_state_and_group_snapshots():
    import torch
    prob = pkg.problems.random_small(14, 11, 9, 4, "S8")
    d = sweep_inputs(prob, seed=6)
    nx, ny, nm, ng = prob.nx, prob.ny, prob.nm, prob.ng
    with _handle(d, "fp32", True) as s:
        s.sweep(moments=True)
        I_ref = s.get_state()
        full = torch.empty(nx * ny * nm * ng, dtype=torch.float32, device="cuda")
        s.snapshot_angular(full.data_ptr())
        s.sync()
        full = full.cpu().numpy()
    # the same step on caller-owned device memory, raw state bytes moved by the caller
    with _handle(d, "fp32", True) as s:
        raw = torch.empty(s.state_bytes(), dtype=torch.uint8, device="cuda")
        own = torch.empty_like(raw)
        s.sweep(moments=False)                       # fills the handle's own buffer (discarded)
        s.put_state(d["I_crn_old"])                  # the own buffer holds I_crn_old again
        s.bind_state(raw.data_ptr(), raw.numel())
        with pytest.raises(pkg.TrtError):
            s.bind_state(raw.data_ptr() + 1, raw.numel())   # misaligned
        s.put_state(d["I_crn_old"])
        torch.cuda.synchronize()
        own.copy_(raw)                               # raw bytes of I_crn_old in this layout
        raw.zero_()
        raw.copy_(own)
        torch.cuda.synchronize()
        s.state_written()
        s.sweep(moments=True)
        assert np.array_equal(s.get_state(), I_ref)
        part = torch.empty(nx * ny * nm * 2, dtype=torch.float32, device="cuda")
        s.snapshot_angular_groups(1, 2, part.data_ptr())
        s.sync()
        part = part.cpu().numpy()
    assert np.array_equal(part, full[nx * ny * nm * 1: nx * ny * nm * 3])
