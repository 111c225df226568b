"""Benchmark of the SCB transport sweep + QD-factor moments (the hot path of the 2D TRT solver).

Metric: cell-angle-group updates/s (one update = one (cell, direction, group) SCB corner solve).
Workload: config C1 -- 256x256 cells, 50 log-spaced groups, S16 (144 directions), 16 seeded material
rectangles; synthetic data (seeded materials at a fixed temperature field, Planck inflow on the left).
A step is one time step of the hot path: I_crn_old <- I_crn, one full sweep of all directions and
groups, and the combination of moments, QD factors (fg), boundary factors (Cg) and incoming E/F.
The corner state (15 GB FP64 / 7.5 GB FP32) is far larger than L2, so no flush is needed.

  value        plain FP64 throughout (the reference's precision), inputs resident in HBM
  e2e          the same step through the C ABI with host buffers: H2D of the step's material (KapE,
               KapB*Bg) from pinned memory, sweep + moments, D2H of fg, Cg, E and the group energies; the
               asynchronous calls let each step's copies overlap the neighbouring sweeps (e2e.sequential:
               the synchronous calls, one step after the other)
  mixed        the same step with the FP32 sweep and FP64 moment sums (value, e2e, roofline); its
               temperature error against FP64 comes from the time_steps and mlqd legs
  roofline     scb_sweep_kernel alone (CUDA events on the library's stream), algorithmic bytes
               B = 8*s + (8*8 + 48*8)/N_m per update (s = 8 FP64 / 4 FP32) over the measured HBM peak
  cpu_baseline the reference's CPU step as the oracle restates it (I_crn_old = I_crn, TRANSPORT_SCB,
               COLLAPSE_INTENSITIES, fg_Calc, Cg_Calc with the OpenMP team over groups, threads =
               min(cores, groups), g++ -O2 -fopenmp) on a sample of min(N_g, max(16, cores)) groups

Further legs on the same grid (single GPU), each with its own figures:
  time_steps   the transport-only time loop, mixed vs FP64 temperature error and step latency
  mlqd         the mlqd time step (sweeps + MGQD and grey Newton low-order iterations), mixed vs FP64
               errors in T, E and F, and where the step's time goes
  pod          the POD of fg-sized snapshots resident in HBM against the oracle's LAPACK restatement
  mgqd         the multigroup low-order solve alone, with its matrix-vector product roofline
  batched      config 2: 64 instances stepped as batches, mixed vs FP64 (HBM-budget admission)
  serving      config 3: a window of the Poisson request stream served with continuous batching,
               p50/p99 step and solve latency, mixed vs FP64

--impl reference times that CPU restatement alone (the reference Fortran cannot be built here).
Multi-GPU (torchrun, one rank per GPU): each rank sweeps its own C1 instance (independent instances,
no collective on the data path): weak scaling, time = max over ranks.
"""
import argparse
import importlib
import json
import os
import re
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="C1", choices=["C0", "C1"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision (FP32 sweep) leg")
    p.add_argument("--tiling", default="", help="warps,slices,stages[,splits] override for both precisions")
    p.add_argument("--profile", default="", choices=["", "fp64", "fp32"],
                   help="only run --warmup + --steps steps (roll + sweep + moments) of one precision, for ncu")
    p.add_argument("--n", type=int, default=0, help="grid size override (profiling small cases)")
    p.add_argument("--groups", type=int, default=0, help="group count override (profiling small cases)")
    p.add_argument("--tiling-sweep", action="store_true", help="time the sweep kernel over a set of tilings")
    p.add_argument("--sweep-prec", default="fp64,fp32", help="precisions of --tiling-sweep")
    p.add_argument("--serving", type=float, default=1.0,
                   help="arrival window (s) of a config-3 request stream served after the step timing; 0 = skip")
    p.add_argument("--batch", type=int, default=64,
                   help="instances of a config-2 batch, stepped as batches in mixed precision and in FP64; 0 = skip")
    p.add_argument("--no-autotune", dest="autotune", action="store_false",
                   help="use the library's default tiling instead of trt_autotune")
    p.add_argument("--mgqd", type=int, default=3,
                   help="timed low-order MGQD solves (MLOQD_FV) on the configuration's grid and groups; 0 skips")
    p.add_argument("--c4", type=int, default=0,
                   help="run only config 4 (1024^2, 64 groups, S16, in-place FP32 state) for this many time steps")
    p.add_argument("--config4-steps", type=int, default=2,
                   help="time steps of the config-4 leg (1024^2, 64 groups, S16, in-place FP32 state) in the default "
                        "run; 0 = skip")
    p.add_argument("--mgqd-only", action="store_true",
                   help="run only the low-order MGQD leg (--mgqd solves) and print its JSON object")
    p.add_argument("--mlqd-steps", type=int, default=2,
                   help="time steps of the mlqd algorithm (sweep + MGQD/grey low-order iterations) on the "
                        "configuration's grid, mixed vs FP64; 0 = skip")
    p.add_argument("--pod-snapshots", type=int, default=20,
                   help="time levels of the POD leg (per-group POD of fg-sized snapshots on the configuration's "
                        "grid and groups, device vs the oracle's LAPACK SVD); 0 = skip")
    p.add_argument("--time-steps", type=int, default=10,
                   help="time steps of the transport-only time loop (mixed vs FP64 temperature error); 0 = skip")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            P = json.load(f)
        return float(P["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def bytes_per_update(nm, prec):
    s = 8 if prec == "fp64" else 4
    return 8 * s + (8 * 8 + 48 * 8) / nm


def traffic_from_profile(prec):
    """Per-launch DRAM bytes of scb_sweep_kernel from the committed ncu summary, scaled to C1."""
    path = os.path.join(ROOT, "profiles", "scb_sweep_c1.md")
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(r"traffic_per_c1_launch_%s:\s*([0-9.eE+]+)" % prec, txt)
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index, period_ms=50):
        self.index = index
        self.period_ms = period_ms
        self.samples = []
        self._proc = None
        self._t = None
        self._first = threading.Event()

    def _read(self):
        for line in self._proc.stdout:
            parts = [x.strip() for x in line.strip().split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)
                self._first.set()

    def __enter__(self):
        """Start one nvidia-smi in loop mode; return once it has delivered its first sample."""
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                           "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self._proc = None
            return self
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        self._first.wait(10)
        self._n0 = len(self.samples)
        return self

    def __exit__(self, *a):
        if self._proc is None:
            return
        # keep only the samples taken while the timed region ran (plus the last one before it)
        n1 = len(self.samples)
        self._proc.terminate()
        try:
            self._proc.wait(5)
        except subprocess.TimeoutExpired:
            self._proc.kill()
            self._proc.wait(5)
        self._t.join(timeout=5)
        self.samples = self.samples[max(0, self._n0 - 1):max(n1, self._n0)]

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if len(s) > 3 + k and "Active" in s[3 + k]
                          and not s[3 + k].startswith("Not")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def build_problem(name, n=0, groups=0):
    pkg = importlib.import_module("2d_trt_rom_system_b200")
    if name == "C1":
        prob = pkg.problems.config1(n=n or 256, groups=groups or 50)
    else:
        prob = pkg.problems.config0()
    return pkg, prob


def run_profile(args):
    """Plain sweeps of one instance (the command ncu captures)."""
    import torch
    torch.cuda.set_device(0)
    pkg, prob = build_problem(args.config, args.n, args.groups)
    tiling = tuple(int(x) for x in args.tiling.split(",")) if args.tiling else None
    s, _, _ = setup_instance(pkg, prob, "mixed" if args.profile == "fp32" else "fp64", tiling)
    try:
        ms, n = time_resident(pkg, torch, s, args.steps, args.warmup, pkg._lib.TRT_ROLL_STATE | pkg._lib.TRT_MOMENTS)
        print(json.dumps({"profile": args.profile, "workload": f"{prob.nx}x{prob.ny} G={prob.ng} {prob.quad}",
                          "ms_per_sweep": ms, "tiling": s.tiling(), "launches": n}))
    finally:
        s.close()
    return 0


def run_tiling_sweep(args):
    import torch
    torch.cuda.set_device(0)
    pkg, prob = build_problem(args.config, args.n, args.groups)
    upd = prob.updates_per_sweep()
    peak, _ = peaks()
    for prec in args.sweep_prec.split(","):
        s, _, _ = setup_instance(pkg, prob, "mixed" if prec == "fp32" else "fp64", None)
        seen = set()
        try:
            for NH in (1, 2, 3, 4, 5, 6):
                for W in (2, 3, 4, 5, 6, 8, 12, 16):
                    for S in (0, 2, 4, 8, 16):
                        for st, NB in ((2, 1), (3, 1), (2, 2), (2, 4)):
                            try:
                                s.set_tiling(W, S, st, NH)
                                s.set_bands(NB)
                            except pkg.TrtError:
                                continue
                            tl = s.tiling()
                            key = tuple(sorted(tl.items()))
                            if key in seen:
                                continue
                            seen.add(key)
                            s.init_state(prob.T0 * 1e3, [t * 1e3 for t in prob.bcT], pkg.problems.COMP_UNIT,
                                         prob.nu_eV)
                            try:
                                ms, _ = time_resident(pkg, torch, s, 5, 1, 0)
                            except pkg.TrtError as e:
                                print(json.dumps({"prec": prec, "tiling": tl, "error": str(e)}), flush=True)
                                continue
                            B = bytes_per_update(prob.nm, prec)
                            print(json.dumps({"prec": prec, "tiling": tl, "kernel_ms": ms, "gupd_s": upd / ms / 1e6,
                                              "frac": upd * B / (ms * 1e-3) / 1e9 / peak}), flush=True)
        finally:
            s.close()
    return 0


def run_time_steps(pkg, torch, prob, steps, conv_type=2, conv_ho=0.0, maxit=8):
    """The reference's transport-only time loop (run_type 'tr_no_qd') on the device, FP64 and mixed from
    the same initial state, with the configuration's own material (the opacity law with its kappa0
    rectangles, c_v per cell, the T^4-linearised energy balance): per step `maxit` outer iterations of
    sweep + moments, energy balance, MATERIAL_UPDATE and CONVERGENCE.  The transport-only iteration is not
    accelerated (it moves a thick front a cell or so per iteration), so it does not reach a 1e-10 tolerance
    here; both runs take the same fixed count and the error is quoted at that count.  Reports the mixed
    run's temperature and energy error against FP64 after every step and the per-step latency (host wall
    clock, the loop synchronises per iteration)."""
    ts = pkg.problems.config_timestep_setup(prob)
    CU, C = pkg.problems.COMP_UNIT, pkg.problems.C_LIGHT
    ox, oy, w = prob.directions()
    res = {}
    for prec in ("fp64", "fp32"):
        s = pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng,
                               precision="mixed" if prec == "fp32" else "fp64")
        try:
            s.init_state(ts.Tini_eV, list(ts.bcT_eV), CU, ts.nu_eV)
            s.tstep_setup(ts.nu_eV, ts.kappa_mult, ts.cv, np.full((prob.nx, prob.ny), ts.Tini_eV), ts.Kap0, CU, C,
                          ts.dt, bcT=ts.bcT_eV, conv_type=conv_type, conv_ho=conv_ho, maxit_rte=maxit, law=1)
            Ts, Es, its, lat = [], [], [], []
            for _ in range(steps):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                n_it, _, _ = s.tstep()
                lat.append((time.perf_counter() - t0) * 1e3)
                its.append(n_it)
                Ts.append(s.temperature())
                Es.append(s.moments(["E_avg"])["E_avg"])
        finally:
            s.close()
        res[prec] = dict(T=Ts, E=Es, its=its, lat=lat)
    rel = lambda a, b: float(np.max(np.abs(a - b) / np.abs(b)))
    t_err = [rel(a, b) for a, b in zip(res["fp32"]["T"], res["fp64"]["T"])]
    e_err = [rel(a, b) for a, b in zip(res["fp32"]["E"], res["fp64"]["E"])]
    upd = prob.updates_per_sweep()
    out = {"algorithm": "tr_no_qd: (sweep + moments, MEB_SOLVE, MATERIAL_UPDATE, CONVERGENCE) per outer iteration, "
                        "on the device",
           "physics": "the configuration's opacity law kappa0 (1 - exp(-nu/T)) / (nu^3 sqrt(T)) on its rectangles, "
                      "c_v per cell, T^4-linearised energy balance; T in eV",
           "iterations": f"{maxit} outer iterations per step on both runs (unaccelerated, not converged)",
           "steps": steps, "conv_type": conv_type, "conv_ho": conv_ho, "maxit_rte": maxit,
           "T_rel_err_max": max(t_err), "E_rel_err_max": max(e_err), "T_rel_err_per_step": t_err}
    for prec in ("fp64", "fp32"):
        r = res[prec]
        lat = np.array(r["lat"])
        out[prec] = {"outer_its": r["its"], "step_ms_p50": float(np.percentile(lat, 50)),
                     "step_ms_p99": float(np.percentile(lat, 99)),
                     "updates_per_s": float(upd * sum(r["its"]) / (lat.sum() * 1e-3))}
    return out


def run_group_sharded(pkg, torch, prob, steps, maxit=4):
    """The transport-only time loop of the workload with its groups split over the ranks (one GPU each): every
    rank sweeps its group range and one all-reduce of the per-cell group sums per outer iteration gives every
    rank the same temperature (sharded.ShardedTimeLoop).  Strong scaling of one instance; step time is the
    maximum over ranks of the device-synchronised wall time."""
    ws, rank, _ = pkg.ranks.world()
    ts = pkg.problems.config_timestep_setup(prob)
    g0, g1 = pkg.sharded.group_ranges(prob.ng, ws)[rank]
    ox, oy, w = prob.directions()
    nu = ts.nu_eV[g0:g1 + 1]
    CU, C = pkg.problems.COMP_UNIT, pkg.problems.C_LIGHT
    s = pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, g1 - g0, precision="fp64")
    try:
        s.init_state(ts.Tini_eV, list(ts.bcT_eV), CU, nu)
        s.tstep_setup(nu, ts.kappa_mult, ts.cv, np.full((prob.nx, prob.ny), ts.Tini_eV), ts.Kap0, CU, C, ts.dt,
                      bcT=ts.bcT_eV, conv_type=2, conv_ho=0.0, maxit_rte=maxit, law=1)
        loop = pkg.sharded.ShardedTimeLoop([s], prob.nx, prob.ny, maxit=maxit,
                                           allreduce=pkg.sharded.torch_allreduce() if ws > 1 else None)
        loop.step()   # warm-up
        lat = []
        for _ in range(steps):
            torch.cuda.synchronize()
            pkg.ranks.barrier()
            t0 = time.perf_counter()
            loop.step()
            torch.cuda.synchronize()
            lat.append(pkg.ranks.reduce_max(time.perf_counter() - t0))
    finally:
        s.close()
    upd = prob.updates_per_sweep() * maxit
    return {"what": "transport-only time step (configuration's material, FP64), groups split over the ranks, "
                    "one all-reduce of 3 nx*ny doubles per outer iteration", "ranks": ws, "groups_per_rank": g1 - g0,
            "outer_its_per_step": maxit, "step_ms": [x * 1e3 for x in lat],
            "updates_per_s": upd * len(lat) / sum(lat), "scaling": "strong"}


def run_mlqd(pkg, torch, prob, steps, conv_ho=1e-8, conv_lo=1e-9, maxit_rte=10, maxit_mloqd=50):
    """The reference's mlqd algorithm (TRT_MLQD_ALGORITHM, run_type 'mlqd') on the device, FP64 and mixed from
    the same initial state: per outer iteration one sweep (from the second on), then MGQD iterations of
    MLOQD_FV + the grey EGP Newton solve + MATERIAL_UPDATE, all low-order work in FP64.  The material is
    the Fleck-Cummings opacity with Kappa_Mult = 1: the reference's grey emission (Q_bar with Kap0) leaves
    Kappa_Mult out, so only a uniform multiplier keeps the grey problem consistent with the multigroup one
    (with the configuration's rectangles the MGQD iteration does not converge, in the oracle as well).
    Reports the mixed run's temperature, energy density and flux error against FP64 after every step."""
    ts = pkg.problems.fc_timestep_setup(prob)
    CU, C = pkg.problems.COMP_UNIT, pkg.problems.C_LIGHT
    ox, oy, w = prob.directions()
    km = np.ones((prob.nx, prob.ny), order="F")
    fields = ("Temp", "E_avg", "HO_E_avg", "Fx_edgV", "Fy_edgH")
    res = {}
    for prec in ("fp64", "fp32"):
        s = pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng,
                               precision="mixed" if prec == "fp32" else "fp64")
        try:
            s.init_state(ts.Tini_eV, list(ts.bcT_eV), CU, ts.nu_eV)
            s.tstep_setup(ts.nu_eV, km, ts.cv, np.full((prob.nx, prob.ny), ts.Tini_eV), ts.Kap0, CU, C, ts.dt,
                          bcT=ts.bcT_eV, conv_type=2, conv_ho=conv_ho, maxit_rte=maxit_rte)
            s.mlqd_setup(ts.Tini_eV, conv_lo=conv_lo, maxit_mloqd=maxit_mloqd)
            out, stats, lat = {k: [] for k in fields}, [], []
            for _ in range(steps):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                st = s.mlqd_step()
                lat.append((time.perf_counter() - t0) * 1e3)
                stats.append(st)
                for k in fields:
                    out[k].append(s.mlqd_field(k))
        finally:
            s.close()
        res[prec] = dict(out=out, stats=stats, lat=lat)
    rel = lambda a, b: float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    r = {"algorithm": "mlqd: sweep + fused moments per outer iteration (none in the first), MGQD iterations of "
                      "MLOQD_FV (BiCGSTAB + multigrid), COLLAPSE_MG_EF, Cbar_Calc, GREY_COEFS, EGP_FV_NEWT, "
                      "MATERIAL_UPDATE; FP64 low-order in both runs",
         "problem": f"{prob.nx}x{prob.ny} cells, {prob.ng} groups, {prob.quad} ({prob.nm} directions); "
                    "Fleck-Cummings opacity, Kappa_Mult 1; T0 10 eV, left boundary 1 keV; dt 2e-3 sh",
         "steps": steps, "conv_ho": conv_ho, "conv_lo": conv_lo, "maxit_rte": maxit_rte, "maxit_mloqd": maxit_mloqd}
    for k in fields:
        r[k + "_rel_err_per_step"] = [rel(a, b) for a, b in zip(res["fp32"]["out"][k], res["fp64"]["out"][k])]
    r["T_rel_err_max"] = max(r["Temp_rel_err_per_step"])
    for prec in ("fp64", "fp32"):
        sts = res[prec]["stats"]
        lat = np.array(res[prec]["lat"])
        r[prec] = {"step_ms": [float(x) for x in lat], "rt_its": [x["rt_its"] for x in sts],
                   "sweeps": [x["sweeps"] for x in sts], "mgqd_its": [x["mgqd_its"] for x in sts],
                   "egp_its": [x["egp_its"] for x in sts], "sweep_ms": [x["sweep_ms"] for x in sts],
                   "low_order_ms": [x["low_order_ms"] for x in sts],
                   "mgqd_solve_ms": [x["mgqd_solve_ms"] for x in sts], "egp_ms": [x["egp_ms"] for x in sts],
                   "mgqd_krylov_sum": [x["mgqd_krylov_sum"] for x in sts],
                   "egp_krylov_sum": [x["egp_krylov_sum"] for x in sts],
                   "mgqd_nonconv": sum(x["mgqd_nonconv"] for x in sts),
                   "egp_nonconv": sum(x["egp_nonconv"] for x in sts),
                   "updates_per_s": float(prob.updates_per_sweep() * sum(x["sweeps"] for x in sts) / (lat.sum() * 1e-3))}
    return r


def run_pod(pkg, torch, prob, nt, cpu_groups=4):
    """The decomposer's POD (POD_Calc + SVD_Calc_Cntr) of fg-sized snapshots resident in HBM: data
    (nx*ny, n_g, n_t), every group decomposed by trt_pod_calc_device; the oracle (numpy/LAPACK SVD) on a
    few groups on the host for the CPU figure.  Synthetic snapshots: a mean field plus decaying modes."""
    import ctypes
    clen, ng = prob.nx * prob.ny, prob.ng
    gen = torch.Generator(device="cuda").manual_seed(5)
    k = min(clen, nt)
    modes = torch.randn(clen, 8, device="cuda", dtype=torch.float64, generator=gen)
    coef = torch.randn(8, ng * nt, device="cuda", dtype=torch.float64, generator=gen) * \
        (0.3 ** torch.arange(8, device="cuda", dtype=torch.float64))[:, None]
    # row g + ng * t of this (ng * nt, clen) row-major tensor is column (g, t) of data(clen, ng, nt)
    data = (1.0 / 3.0 + 1e-2 * (modes @ coef)).T.contiguous()
    outs = [torch.empty(n, dtype=torch.float64, device="cuda") for n in (clen, clen * k, k, k * nt)]
    L = pkg.lib()
    ptrs = [ctypes.c_void_p(o.data_ptr()) for o in outs]

    def one(g):
        assert L.trt_pod_calc_device(ctypes.c_void_p(data.data_ptr()), nt, ng, clen, g, *ptrs, None) == 0

    one(0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for g in range(ng):
        one(g)
    torch.cuda.synchronize()
    dev_s = (time.perf_counter() - t0) / ng
    r = {"workload": f"POD per group of {nt} snapshots of {prob.nx}x{prob.ny} values x {ng} groups (fg-sized), "
                     "resident in HBM", "metric": "group PODs/s", "value": 1.0 / dev_s, "ms_per_group": dev_s * 1e3,
         "path": "trt_pod_calc_device: centring kernel, then QR (cuSOLVER geqrf), SVD of the small triangle "
                 "(gesvd) and U = Q U_R (ormqr)"}
    try:
        sys.path.insert(0, ROOT)
        from oracle import oracle as O
        flat = data.cpu().numpy().reshape(-1)   # memory order = data(clen, ng, nt) in Fortran order
        O.pod_calc(flat, nt, ng, clen, 0)
        t0 = time.perf_counter()
        for g in range(cpu_groups):
            O.pod_calc(flat, nt, ng, clen, g)
        cpu_s = (time.perf_counter() - t0) / cpu_groups
        r["cpu_baseline"] = {"value": 1.0 / cpu_s, "unit": "group PODs/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"{cpu_groups} groups, numpy centring + LAPACK SVD (threaded BLAS)"}
    except Exception as exc:   # the CPU figure is context, not the measurement
        r["cpu_baseline"] = {"error": repr(exc)}
    return r


def run_config4(pkg, torch, steps, snapshots=True, n=1024):
    """Config 4: 1024^2 cells, 64 groups, S16 (9.66e9 updates per sweep), 8 material rectangles (seed 4),
    mixed precision.  The FP32 corner state alone is 155 GB, so the handle sweeps it in place (one state
    buffer); each time step is one sweep of the transport-only loop (trt_tstep with one outer iteration:
    sweep, moments, the configurations' energy balance, material update).  With `snapshots`, the FP32
    cell-average angular intensity of each group is derived from the state and streamed to pinned host
    memory (38.7 GB per step), the copies overlapping the next group's snapshot kernel."""
    prob = pkg.problems.config4(n=n)
    ts = pkg.problems.config_timestep_setup(prob)
    ox, oy, w = prob.directions()
    upd = prob.updates_per_sweep()
    out = {"workload": f"C4: {prob.nx}x{prob.ny} cells, {prob.ng} log-spaced groups, {prob.quad} ({prob.nm} "
                       f"directions), 8 seeded material rectangles", "updates_per_sweep": upd,
           "step": "one sweep of the transport-only loop per time step (trt_tstep, maxit_rte 1), in-place FP32 state"}
    free, total = torch.cuda.mem_get_info()
    out["device_gb_free_before"] = free / 1e9
    out["required_gb_two_buffers"] = pkg.required_bytes(prob.nx, prob.ny, prob.nm, prob.ng, "mixed") / 1e9
    s = pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng, precision="mixed",
                           inplace=True)
    try:
        s.init_state(ts.Tini_eV, list(ts.bcT_eV), pkg.problems.COMP_UNIT, ts.nu_eV)
        s.tstep_setup(ts.nu_eV, ts.kappa_mult, ts.cv, np.full((prob.nx, prob.ny), ts.Tini_eV), ts.Kap0,
                      pkg.problems.COMP_UNIT, pkg.problems.C_LIGHT, ts.dt, bcT=ts.bcT_eV, conv_type=2, conv_ho=0.0,
                      maxit_rte=1, law=1)
        free, total = torch.cuda.mem_get_info()
        out["state_gb"] = s.state_bytes() / 1e9
        out["device_gb_used"] = (total - free) / 1e9
        out["tiling"] = s.tiling()
        lat = []
        for _ in range(steps):
            s.sync()
            t0 = time.perf_counter()
            s.tstep()
            s.sync()
            lat.append(time.perf_counter() - t0)
        T = s.temperature()
        out["step_s"] = lat
        out["updates_per_s"] = upd * len(lat) / sum(lat)
        ms_k, _ = time_resident(pkg, torch, s, 3, 1, pkg._lib.TRT_ROLL_STATE)   # the sweep kernel alone
        peak, kind = peaks()
        B = bytes_per_update(prob.nm, "fp32")
        out["roofline"] = {"kernel": "scb_sweep_kernel<float>", "kernel_ms": ms_k, "bytes_per_update": B,
                           "achieved": upd * B / (ms_k * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                           "frac": upd * B / (ms_k * 1e-3) / 1e9 / peak, "peak_source": f"{kind} hbm_gbs"}
        out["T_min_max_eV"] = [float(T.min()), float(T.max())]
        if snapshots:
            try:
                # one group per slab: the in-place handle leaves a few GB of the device free, and a group's
                # snapshot (0.6 GB) is large enough for full-bandwidth copies
                slab = 1
                per = prob.nx * prob.ny * prob.nm * slab
                dev = [torch.empty(per, dtype=torch.float32, device="cuda") for _ in range(2)]
                host = [torch.empty(per, dtype=torch.float32, pin_memory=True) for _ in range(2)]
                copy = torch.cuda.Stream()
                hs = torch.cuda.ExternalStream(s.stream())
                ev = [torch.cuda.Event() for _ in range(2)]
                s.sync()
                t0 = time.perf_counter()
                for k, g0 in enumerate(range(0, prob.ng, slab)):
                    b = k % 2
                    if k >= 2:
                        ev[b].synchronize()   # the copy out of this buffer two slabs ago is done
                    s.snapshot_angular_groups(g0, slab, dev[b].data_ptr())
                    e = torch.cuda.Event()
                    e.record(hs)
                    copy.wait_event(e)
                    with torch.cuda.stream(copy):
                        host[b].copy_(dev[b], non_blocking=True)
                    ev[b].record(copy)
                copy.synchronize()
                snap_s = time.perf_counter() - t0
                nbytes = prob.nx * prob.ny * prob.nm * prob.ng * 4
                out["snapshot"] = {"bytes": nbytes, "seconds": snap_s, "gb_per_s": nbytes / snap_s / 1e9,
                                   "path": "trt_snapshot_angular_groups per group into two device buffers, "
                                           "copied to pinned host memory on a copy stream"}
                out["step_with_snapshot_s"] = float(np.median(lat)) + snap_s
            except RuntimeError as e:   # e.g. no room left for the two slab buffers
                out["snapshot"] = {"error": str(e).splitlines()[0][:300]}
    finally:
        s.close()
    return out


def run_serving(pkg, window_s, rate=200.0, budget_gb=120.0):
    """Config-3 request stream (Poisson arrivals at `rate`/s, seed 3) over a `window_s` arrival window,
    admitted against a `budget_gb` HBM budget; mixed and FP64 served separately."""
    out = {"rate_per_s": rate, "arrival_window_s": window_s, "hbm_budget_gb": budget_gb,
           "per_request": "10 backward-Euler steps of the transport-only loop, 4 outer iterations per step"}
    for prec in ("mixed", "fp64"):
        reqs = pkg.serving.config3_requests(rate=rate, duration=window_s, seed=3, precision=prec)
        srv = pkg.serving.BatchedServer(hbm_budget=int(budget_gb * 1e9))
        res, log = srv.run(reqs)
        summ = pkg.serving.latency_summary(res)
        summ["updates_per_s_stepping"] = srv.stepped_updates / max(srv.stepping_s, 1e-9)
        summ["max_concurrent_gb"] = max(e[2] for e in log) / 1e9
        out[prec] = summ
    return out


def run_batch(pkg, count, budget_gb=170.0):
    """Config 2: `count` independent instances (seed 2) submitted at once and stepped as batches
    (trt_batch_tstep: one sweep launch per tiling class over all admitted instances), in mixed precision
    and in plain FP64, each admitted against a `budget_gb` HBM budget (the FP64 states of all 64 do not fit
    at once: instances join as others finish)."""
    out = {"instances": count, "hbm_budget_gb": budget_gb,
           "per_instance": "10 backward-Euler steps of the transport-only loop, 4 outer iterations per step"}
    for name, prec in (("mixed_batched", "mixed"), ("fp64_batched", "fp64")):
        reqs = pkg.serving.config2_batch(count, precision=prec)
        t0 = time.perf_counter()
        srv = pkg.serving.BatchedServer(hbm_budget=int(budget_gb * 1e9))
        res, log = srv.run(reqs, realtime=False)
        wall = time.perf_counter() - t0
        summ = pkg.serving.latency_summary(res)
        summ["wall_s"] = wall
        summ["stepping_s"] = srv.stepping_s
        summ["updates_per_s_stepping"] = srv.stepped_updates / srv.stepping_s
        summ["max_concurrent_gb"] = max(e[2] for e in log) / 1e9
        out[name] = summ
    out["mixed_over_fp64_updates_per_s"] = (out["mixed_batched"]["updates_per_s"] /
                                            out["fp64_batched"]["updates_per_s"])
    return out


def mgqd_matvec_bytes(nx, ny, ng):
    """Algorithmic bytes of one matrix-vector product of the reduced MGQD system (matvec_kernel): the
    11 cell coefficient planes, the two edge diagonals, the operand, the product and rh, FP64."""
    nC, nV, nH = nx * ny, (nx + 1) * ny, nx * (ny + 1)
    nU = nC + nV + nH
    return 8 * ng * (11 * nC + nV + nH + 3 * nU)


def mgqd_cpu_baseline(pkg, n, ng, budget_s=30.0):
    """The reference's procedure for MLOQD_FV (its numbering, ILUT(3, 1e-6) + BiCGSTAB, OpenMP over
    groups) restated in the oracle, on a sample of the groups spread over the opacity range."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    gs = min(ng, max(16, cores))   # sample groups; threads = min(cores, groups), the reference's team
    d, c, dt, th = pkg.problems.mgqd_inputs(n, n, ng, seed=1, kap_range=(1e-4, 1e4), uniform=True)
    sel = np.linspace(0, ng - 1, gs).round().astype(int)
    ds = {}
    for k, v in d.items():
        v = np.asarray(v)
        ds[k] = np.asfortranarray(v[..., sel]) if v.ndim >= 2 and v.shape[-1] == ng else v
    ds.update(O.old_mgqd_coefs(ds, c, dt, th))
    times = []
    t_start = time.perf_counter()
    while len(times) < 3 and (time.perf_counter() - t_start) < budget_s:
        t0 = time.perf_counter()
        o = O.mloqd_fv(ds, c, dt, th, threads=min(cores, gs), solver=1)
        times.append(time.perf_counter() - t0)
    med = float(np.median(times))
    return {"value": n * n * gs / med, "unit": "cell*group/s", "cores": min(cores, gs), "kind": "port",
            "sample": f"{n}x{n} cells, {gs} of {ng} groups spread over the opacity range (matrix-vector products "
                      f"{int(o['MGQD_Kits'].min())}-{int(o['MGQD_Kits'].max())}), median of {len(times)} solves, "
                      f"{min(cores, gs)} threads (OpenMP over groups), g++ -O2 -fopenmp, host has {cores} logical CPUs"}


def run_mgqd(pkg, solves, n, ng, cpu=True):
    """MLOQD_FV through the reference-signature entry point (host arrays): device time of the solve
    (events inside the library, copies excluded) and the whole call."""
    P = pkg.problems
    d, c, dt, th = P.mgqd_inputs(n, n, ng, seed=1, kap_range=(1e-4, 1e4), uniform=True)
    old = {k: np.zeros((n, n, ng), order="F") for k in ("G_old", "Pold_L", "Pold_B", "Pold_R", "Pold_T")}
    pkg.OLD_MGQD_COEFS(*[d[k] for k in ("Eg_avg_old", "Eg_edgV_old", "Eg_edgH_old", "Fxg_edgV_old", "Fyg_edgH_old",
                                        "fg_avg_xx_old", "fg_avg_yy_old", "fg_edgV_xx_old", "fg_edgV_xy_old",
                                        "fg_edgH_yy_old", "fg_edgH_xy_old", "KapE_old", "KapR_old", "Src_old", "Delx",
                                        "Dely", "A")], c, dt, th, *old.values(), 1)
    d.update(old)
    ins = [d[k] for k in ("fg_avg_xx", "fg_avg_yy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy", "Cg_L",
                          "Cg_B", "Cg_R", "Cg_T", "Eg_in_L", "Eg_in_B", "Eg_in_R", "Eg_in_T", "Fg_in_L", "Fg_in_B",
                          "Fg_in_R", "Fg_in_T", "Src", "KapE", "KapR", "Delx", "Dely", "A")]
    olds = [d[k] for k in ("G_old", "Pold_L", "Pold_B", "Pold_R", "Pold_T", "Eg_avg_old", "Fxg_edgV_old",
                           "Fyg_edgH_old")]
    out = {"Fxg_edgV": np.zeros((n + 1, n, ng), order="F"), "Fyg_edgH": np.zeros((n, n + 1, ng), order="F"),
           "R": np.zeros((ng, 5, 5), order="F"), "RB": np.zeros((ng, 4), order="F"),
           "K": np.zeros(ng, dtype=np.int32)}
    rec = []
    launches0 = pkg.kernel_launches()
    for k in range(solves + 1):
        E = {q: d[q].copy(order="F") for q in ("Eg_avg", "Eg_edgV", "Eg_edgH")}
        t0 = time.perf_counter()
        pkg.MLOQD_FV(E["Eg_avg"], E["Eg_edgV"], E["Eg_edgH"], out["Fxg_edgV"], out["Fyg_edgH"], *ins, c, dt, th, 1, True,
                     out["R"], out["RB"], *olds, out["K"], 1.0, 1.0, 1.0)
        wall = time.perf_counter() - t0
        if k == 0:
            launches0 = pkg.kernel_launches()
            continue
        ms, its, mv = pkg.mgqd_last_stats()
        rec.append((ms, wall, its, mv))
    launches = (pkg.kernel_launches() - launches0) / max(1, solves)
    ms = float(np.median([r[0] for r in rec]))
    wall = float(np.median([r[1] for r in rec]))
    mv = float(np.median([r[3] for r in rec]))
    h2d = sum(np.asarray(a).nbytes for a in ins + olds) + sum(d[q].nbytes for q in ("Eg_avg", "Eg_edgV", "Eg_edgH"))
    d2h = sum(d[q].nbytes for q in ("Eg_avg", "Eg_edgV", "Eg_edgH")) + sum(v.nbytes for v in out.values())
    peak, kind = peaks()
    mvb = mgqd_matvec_bytes(n, n, ng)
    res = {"workload": f"MLOQD_FV: {n}x{n} cells, {ng} groups (the configuration's grid and groups), seeded synthetic "
                       f"QD factors, boundary factors and opacities log-spread over 1e-4..1e4 per group",
           "metric": "cell*group low-order solves/s", "value": n * n * ng / (ms * 1e-3), "unit": "cell*group/s",
           "device_ms": ms, "iterations_max": int(rec[-1][2]), "matvec_products": [int(out["K"].min()), int(out["K"].max())],
           "gpu_launches": launches, "dtype": "f64 (preconditioner f32)",
           "e2e": {"value": n * n * ng / wall, "unit": "cell*group/s", "ms": wall * 1e3, "h2d_bytes_per_step": int(h2d),
                   "d2h_bytes_per_step": int(d2h), "path": "trt_mloqd_fv with pageable host arrays (the Fortran call)"},
           "roofline": {"kernel": "matvec_kernel", "bound": "hbm", "bytes_per_launch": mvb,
                        "achieved": mvb / (mv * 1e-3) / 1e9 if mv > 0 else None, "peak": peak, "unit": "GB/s",
                        "frac": (mvb / (mv * 1e-3) / 1e9) / peak if mv > 0 else None, "kernel_ms": mv,
                        "peak_source": f"{kind} hbm_gbs"}}
    if cpu:
        res["cpu_baseline"] = mgqd_cpu_baseline(pkg, n, ng)
    return res


def setup_instance(pkg, prob, precision, tiling, autotune=False):
    ox, oy, w = prob.directions()
    s = pkg.TransportSweep(prob.nx, prob.ny, ox, oy, w, prob.delx, prob.dely, prob.ng, precision=precision)
    if tiling:
        s.set_tiling(*tiling)
    elif autotune:
        s.autotune()
    s.init_state(prob.T0 * 1e3, [t * 1e3 for t in prob.bcT], pkg.problems.COMP_UNIT, prob.nu_eV)
    # a temperature field between the cold initial state and the hot boundary
    x = (np.arange(prob.nx) + 0.5) / prob.nx
    T = np.asfortranarray(np.broadcast_to((prob.T0 + 0.5 * np.exp(-8 * x))[:, None], (prob.nx, prob.ny)))
    kap, src = prob.material(T)
    s.set_material(kap, src, pkg.problems.C_LIGHT, prob.dt, pkg.problems.COMP_UNIT)
    return s, kap, src


def time_resident(pkg, torch, s, steps, warmup, flags):
    L = pkg.lib()
    stream = torch.cuda.ExternalStream(s.stream())
    for _ in range(warmup):
        pkg.check(L.trt_sweep(s.handle, flags), "trt_sweep")
    # timed region bracketed by device synchronisation and a barrier over ranks on both sides
    s.sync()
    torch.cuda.synchronize()
    pkg.ranks.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    n0 = pkg.kernel_launches()
    e0.record(stream)
    for _ in range(steps):
        pkg.check(L.trt_sweep(s.handle, flags), "trt_sweep")
    e1.record(stream)
    s.sync()
    torch.cuda.synchronize()
    pkg.ranks.barrier()
    n1 = pkg.kernel_launches()
    return e0.elapsed_time(e1) / steps, n1 - n0


def time_e2e(pkg, torch, s, prob, kap, src, steps, warmup, pipelined=True):
    """Per step: H2D of the material from pinned memory, sweep + moments, D2H of the step's result.
    pipelined: through trt_set_material_async / trt_moments_async, so that step k+1's upload and step k's
    download run on copy streams while the sweeps run (every step still copies its own inputs and outputs);
    otherwise the synchronous calls, one step after the other."""
    import ctypes
    names = ["fg_avg_xx", "fg_avg_yy", "fg_avg_xy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy",
             "Cg_L", "Cg_B", "Cg_R", "Cg_T", "Eg_avg", "E_avg"]
    pin = lambda shape: torch.empty(int(np.prod(shape)), dtype=torch.float64, pin_memory=True).numpy()
    kp = pin(kap.shape)
    sp = pin(src.shape)
    kp[:] = kap.ravel(order="F")
    sp[:] = src.ravel(order="F")
    outs = {n: pin(pkg._lib.moment_shape(n, prob.nx, prob.ny, prob.ng)) for n in names}
    mh = pkg._lib.MomentsHost()
    for n, a in outs.items():
        setattr(mh, n, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    L = pkg.lib()
    D = ctypes.POINTER(ctypes.c_double)
    flags = pkg._lib.TRT_ROLL_STATE | pkg._lib.TRT_MOMENTS
    C, CU = pkg.problems.C_LIGHT, pkg.problems.COMP_UNIT

    if pipelined:
        def step():   # the step's copies overlap the neighbouring steps' sweeps (two copy streams)
            assert L.trt_set_material_async(s.handle, kp.ctypes.data_as(D), sp.ctypes.data_as(D), C, prob.dt,
                                            CU) == 0
            assert L.trt_sweep(s.handle, flags) == 0
            assert L.trt_moments_async(s.handle, ctypes.byref(mh)) == 0
    else:
        def step():
            assert L.trt_set_material(s.handle, kp.ctypes.data_as(D), sp.ctypes.data_as(D), C, prob.dt, CU) == 0
            assert L.trt_sweep(s.handle, flags) == 0
            assert L.trt_moments(s.handle, ctypes.byref(mh)) == 0

    for _ in range(warmup):
        step()
    assert L.trt_sync(s.handle) == 0
    # host wall clock: the region includes the host<->device copies the C ABI makes
    torch.cuda.synchronize()
    pkg.ranks.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    assert L.trt_sync(s.handle) == 0
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    pkg.ranks.barrier()
    h2d = kp.nbytes + sp.nbytes
    d2h = sum(a.nbytes for a in outs.values())
    return dt, h2d, d2h


def cpu_sample_groups(ng, cores):
    """Groups of the CPU sample: min(ng, max(16, cores)) groups spread evenly over the group range (the
    sweep's cost per update does not depend on the group, but thin and thick groups are both covered)."""
    gs = min(ng, max(16, cores))
    return [int(g) for g in np.linspace(0, ng - 1, gs).round()]


def cpu_step_inputs(prob, sel):
    """Reference-layout inputs of one hot-path step of `prob` restricted to the groups `sel`, in the
    benchmark's state (every corner at Bg(T0), Planck inflow on the left, material at the benchmark's
    temperature field)."""
    from oracle import oracle as O
    ox, oy, w = prob.directions()
    nx, ny, nm = prob.nx, prob.ny, len(ox)
    x = (np.arange(nx) + 0.5) / nx
    T = np.asfortranarray(np.broadcast_to((prob.T0 + 0.5 * np.exp(-8 * x))[:, None], (nx, ny)))
    kap, src = prob.material(T)
    nu = prob.nu_eV
    P = importlib.import_module("2d_trt_rom_system_b200").problems
    ns = len(sel)
    Bg0 = np.array([P.bg_planck(prob.T0 * 1e3, nu[g], nu[g + 1]) for g in sel])
    src_s = np.asfortranarray(src[:, :, sel])
    Src_in = np.asfortranarray(np.repeat(np.repeat(src_s, 2, axis=0), 2, axis=1)[:, :, None, :].repeat(nm, axis=2))
    faces = [np.empty((nx + 1, 2 * ny, nm, ns), order="F"), np.empty((2 * nx, ny + 1, nm, ns), order="F"),
             np.empty((nx + 1, ny, nm, ns), order="F"), np.empty((nx, ny + 1, nm, ns), order="F")]
    bT = [t * 1e3 for t in prob.bcT]
    for k, g in enumerate(sel):   # RT_INIT's boundary update, one group at a time
        b = Bg0[k]
        one = [np.full(f.shape[:3] + (1,), b, order="F") for f in faces]
        IV, IH, IcV, IcH = O.rt_bc_update((0, 0, 0, 0), bT[0], bT[1], bT[2], bT[3], P.COMP_UNIT, nu[g:g + 2], one[2],
                                          one[3], one[0], one[1])
        for f, v in zip(faces, (IcV, IcH, IV, IH)):
            f[..., k] = v[..., 0]
    I_crn = np.asfortranarray(np.broadcast_to(Bg0, (2 * nx, 2 * ny, nm, ns)).copy())
    return dict(Omega_x=ox, Omega_y=oy, w=w, Delx=prob.delx, Dely=prob.dely,
                A=np.asfortranarray(np.outer(prob.delx, prob.dely)), KapE_in=np.asfortranarray(kap[:, :, sel]),
                Src_in=Src_in, I_crn=I_crn, Ic_edgV=faces[0], Ic_edgH=faces[1], I_edgV=faces[2], I_edgH=faces[3])


def cpu_baseline(prob_full, reps=5, budget_s=90.0):
    """One step of the hot path on the host, in the reference's form: I_crn_old = I_crn
    (ALGORITHMS.f08:397), TRANSPORT_SCB, COLLAPSE_INTENSITIES, fg_Calc and Cg_Calc, each with the
    reference's OpenMP team over groups, threads = min(cores, groups) (TRANSPORT_SOLVES.f08:50-53), on a
    sample of min(ng, max(16, cores)) groups of the workload (the oracle's restatement, g++ -O2 -fopenmp:
    the reference's Fortran cannot be built here).  Median of `reps` steps after one warm-up step."""
    from oracle import oracle as O
    P = importlib.import_module("2d_trt_rom_system_b200").problems
    cores = os.cpu_count() or 1
    sel = cpu_sample_groups(prob_full.ng, cores)
    threads = min(cores, len(sel))
    d = cpu_step_inputs(prob_full, sel)
    upd = prob_full.nx * prob_full.ny * len(d["Omega_x"]) * len(sel)
    C, CU = P.C_LIGHT, P.COMP_UNIT

    def step():
        I_old = d["I_crn"].copy(order="F")   # I_crn_old = I_crn
        s = O.transport_scb(d["I_edgV"], d["I_edgH"], d["Ic_edgV"], d["Ic_edgH"], d["Omega_x"], d["Omega_y"],
                            d["Delx"], d["Dely"], d["A"], d["KapE_in"], d["Src_in"], I_old, C, prob_full.dt,
                            threads=threads)
        m = O.collapse_intensities(s["I_avg"], s["I_edgV"], s["I_edgH"], d["Omega_x"], d["Omega_y"], d["w"], CU,
                                   threads=threads)
        O.fg_calc(m, C, threads=threads)
        O.cg_calc(s["I_edgV"], s["I_edgH"], d["Omega_x"], d["Omega_y"], d["w"], CU, (0, 0, 0, 0), threads=threads)
        d["I_crn"] = s["I_crn"]

    step()
    times = []
    t_start = time.perf_counter()
    while len(times) < reps and (len(times) < 2 or (time.perf_counter() - t_start) < budget_s):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    med = float(np.median(times))
    return {"value": upd / med, "unit": "updates/s", "cores": threads, "kind": "port",
            "sample": f"{prob_full.name} grid and directions, {len(sel)} of {prob_full.ng} groups spread over the range "
                      f"({upd:.3g} updates per step); per step I_crn_old = I_crn, TRANSPORT_SCB, COLLAPSE_INTENSITIES, "
                      f"fg_Calc, Cg_Calc; median of {len(times)} steps; {threads} threads (OpenMP over groups, "
                      f"threads = min(cores, groups)) on a host with {cores} logical CPUs; g++ -O2 -fopenmp",
            "step_s": med}


def workload_config(prob):
    """The `config` object of both arms (identical words, so the two lines name the same workload)."""
    return {"workload": f"{prob.name}: {prob.nx}x{prob.ny} cells, {prob.ng} log-spaced groups, {prob.quad} "
                        f"({prob.nm} directions), seeded material rectangles",
            "updates_per_sweep": prob.updates_per_sweep(),
            "step": "one time step of the hot path: I_crn_old <- I_crn, full sweep, angular moments, QD factors fg, "
                    "boundary factors Cg",
            "precision": "f64 (the reference's REAL*8)",
            "l2": f"inputs larger than L2 (the corner state of the step: {8 * 4 * prob.updates_per_sweep() / 1e9:.3g} GB "
                  f"in FP64)"}


def run_reference(args):
    pkg, prob = build_problem(args.config)
    ws, rank, _ = pkg.ranks.world()
    if rank != 0:
        return 0
    cb = cpu_baseline(prob)
    line = {"metric": "cell-angle-group updates/s", "value": cb["value"], "unit": "updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "impl": "reference",
            "dtype": "f64", "data": "synthetic", "config": workload_config(prob),
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's CPU path as the oracle restates it (TRANSPORT_SOLVES.f08 with its OpenMP "
                    "decomposition); the reference's Fortran cannot be built here (no Fortran compiler, "
                    "un-vendored LA_TOOLS)"}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile:
        return run_profile(args)
    if args.tiling_sweep:
        return run_tiling_sweep(args)
    if args.c4:
        import torch
        torch.cuda.set_device(0)
        pkg, _ = build_problem(args.config)
        print(json.dumps({"config4": run_config4(pkg, torch, max(1, args.c4))}))
        return 0
    if args.mgqd_only:
        pkg, prob = build_problem(args.config, args.n, args.groups)
        print(json.dumps(run_mgqd(pkg, max(1, args.mgqd), prob.nx, prob.ng, cpu=not args.no_cpu_baseline)))
        return 0
    import torch
    pkg, prob = build_problem(args.config, args.n, args.groups)
    ranks = pkg.ranks
    ws, rank, local = ranks.init("nccl")
    torch.cuda.set_device(local)
    tiling = tuple(int(x) for x in args.tiling.split(",")) if args.tiling else None
    upd = prob.updates_per_sweep()
    peak, peak_kind = peaks()
    flags = pkg._lib.TRT_ROLL_STATE | pkg._lib.TRT_MOMENTS
    res = {}
    precs = ["fp64"] + ([] if args.no_mixed else ["fp32"])
    clocks = None
    for prec in precs:
        s, kap, src = setup_instance(pkg, prob, "mixed" if prec == "fp32" else "fp64", tiling, autotune=args.autotune)
        try:
            if prec == "fp64":
                with ClockSampler(local) as cs:
                    ms, launches = time_resident(pkg, torch, s, args.steps, args.warmup, flags)
                clocks = cs.summary()
            else:
                ms, launches = time_resident(pkg, torch, s, args.steps, args.warmup, flags)
            ms = ranks.reduce_max(ms)
            # sweep kernel alone (no moments, no roll): per-launch duration for the roofline
            ms_k, _ = time_resident(pkg, torch, s, max(3, args.steps // 2), 1, 0)
            ms_k = ranks.reduce_max(ms_k)
            # the pipelined run over the same K steps as the resident timing: its region still starts with the
            # first upload and ends with the last download, which overlap nothing
            e2e = (time_e2e(pkg, torch, s, prob, kap, src, max(3, args.steps), 3, pipelined=True),
                   time_e2e(pkg, torch, s, prob, kap, src, max(3, args.steps // 8), 3, pipelined=False))
            tl = s.tiling()
        finally:
            s.close()
        B = bytes_per_update(prob.nm, prec)
        ach = upd * B / (ms_k * 1e-3) / 1e9
        res[prec] = dict(ms=ms, launches=launches, ms_kernel=ms_k, achieved=ach, tiling=tl, e2e=e2e, B=B)

    def e2e_obj(r):
        (dt, h2d, d2h), (dt_seq, _, _) = r["e2e"]
        dt = ranks.reduce_max(dt)
        dt_seq = ranks.reduce_max(dt_seq)
        return {"value": ranks.whole_job_rate(upd, dt, ws), "unit": "updates/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": dt * 1e3, "timed_steps": max(3, args.steps),
                "path": "trt_set_material_async(pinned host) + trt_sweep + trt_moments_async(pinned host): each step "
                        "uploads its material and downloads its fg, Cg, Eg, E; the copies of neighbouring steps "
                        "overlap the sweeps on two copy streams; the region (host clock) runs from the first "
                        "upload to the last download",
                "sequential": {"value": ranks.whole_job_rate(upd, dt_seq, ws), "ms_per_step": dt_seq * 1e3,
                               "timed_steps": max(3, args.steps // 8),
                               "path": "trt_set_material + trt_sweep + trt_moments, one step after the other"}}

    def roofline_obj(r, prec):
        return {"bound": "hbm", "achieved": r["achieved"], "peak": peak, "unit": "GB/s", "frac": r["achieved"] / peak,
                "traffic": traffic_from_profile(prec),
                "kernel": "scb_sweep_kernel<%s>" % ("double" if prec == "fp64" else "float"),
                "bytes_per_update": r["B"], "peak_source": f"{peak_kind} hbm_gbs", "kernel_ms": r["ms_kernel"]}

    main_ = res["fp64"]
    cfg = workload_config(prob)
    line = {
        "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU",
        "metric": "cell-angle-group updates/s",
        "value": ranks.whole_job_rate(upd, main_["ms"] * 1e-3, ws),
        "unit": "updates/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": main_["ms"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": cfg,
        "tiling": main_["tiling"],
        "roofline": roofline_obj(main_, "fp64"),
        "gpu_launches": main_["launches"],
        "clocks": clocks,
        "e2e": e2e_obj(main_),
    }
    if "fp32" in res:
        r = res["fp32"]
        line["mixed"] = {"what": "the same step with the FP32 sweep and FP64 moment sums, QD factors, low-order "
                                 "fields and energy balance (the error against FP64 is reported by the time_steps "
                                 "and mlqd legs)",
                         "value": ranks.whole_job_rate(upd, r["ms"] * 1e-3, ws), "ms_per_step": r["ms"],
                         "dtype": "f32 sweep, f64 moments", "gpu_launches": r["launches"], "tiling": r["tiling"],
                         "roofline": roofline_obj(r, "fp32"), "e2e": e2e_obj(r)}
        line["mixed_over_fp64"] = line["mixed"]["value"] / line["value"]
        line["mixed_over_fp64_e2e"] = line["mixed"]["e2e"]["value"] / line["e2e"]["value"]
    if args.time_steps > 0:
        line["time_steps"] = run_time_steps(pkg, torch, prob, args.time_steps)
    if ws > 1:
        line["group_sharded"] = run_group_sharded(pkg, torch, prob, 3)
    if args.mlqd_steps > 0 and ws == 1:
        try:
            line["mlqd"] = run_mlqd(pkg, torch, prob, args.mlqd_steps)
        except Exception as exc:   # reported, not fatal to the headline line
            line["mlqd"] = {"error": repr(exc)}
    if args.pod_snapshots > 0 and ws == 1:
        try:
            line["pod"] = run_pod(pkg, torch, prob, args.pod_snapshots)
        except Exception as exc:
            line["pod"] = {"error": repr(exc)}
    if args.mgqd > 0 and ws == 1:
        line["mgqd"] = run_mgqd(pkg, args.mgqd, prob.nx, prob.ng, cpu=rank == 0 and not args.no_cpu_baseline)
    if args.serving > 0 and ws == 1:
        line["serving"] = run_serving(pkg, args.serving)
    if args.batch > 0 and ws == 1:
        line["batched"] = run_batch(pkg, args.batch)
    if args.config4_steps > 0 and ws == 1:
        torch.cuda.empty_cache()   # the leg needs ~171 of the device's ~178 GB
        try:
            line["config4"] = run_config4(pkg, torch, args.config4_steps)
        except Exception as exc:   # reported, not fatal to the headline line
            line["config4"] = {"error": repr(exc)[:300]}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(prob)
    if rank == 0:
        print(json.dumps(line))
    ranks.finalize()
    return 0


if __name__ == "__main__":
    sys.exit(main())
