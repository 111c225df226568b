"""Time steps of one instance whose groups are split over several handles.

The reference's only parallelism is over energy groups (the OpenMP loops of TRANSPORT_SOLVES.f08:50-53),
and in its transport-only time loop (run_type 'tr_no_qd', ALGORITHMS.f08:518-572, 662-668, 816-836) the
groups meet only in the energy balance (MEB_SOLVE, UPDATES.f08:185-230) and in the convergence test on the
transport E: both are per-cell sums over groups.  So the groups split into ranges, each range on its own
handle (a rank of a multi-GPU run, or a slab of a state too large for one device), and one outer iteration
becomes: every handle sweeps its groups and forms its group sums (trt_tstep_partials, 3 values per cell),
the sums are added over the handles (on the device, and with one all-reduce across ranks), and every handle
forms the same temperature from the totals (trt_tstep_finish).  The exchange is 3 n_x n_y doubles per outer
iteration (1.6 MB at 256^2).  ShardedMlqd does the same for the QD-accelerated (mlqd) time step.
"""
import numpy as np


def group_ranges(ng, parts):
    """`parts` contiguous ranges [(g0, g1), ...] covering groups 0..ng-1, sizes differing by at most one."""
    if not 1 <= parts <= ng:
        raise ValueError(f"cannot split {ng} groups into {parts} ranges")
    base, extra = divmod(ng, parts)
    out, g0 = [], 0
    for k in range(parts):
        g1 = g0 + base + (1 if k < extra else 0)
        out.append((g0, g1))
        g0 = g1
    return out


class ShardedTimeLoop:
    """Outer iterations of one time step over `members` (this process's handles, each holding a group range
    of the instance) with `allreduce(tensor)` adding the group sums across processes (None: one process).

    A member provides tstep_begin(), tstep_sweep(its), tstep_partials(buf), tstep_finish(total, its) ->
    (converged, T_norm, E_norm) and sync(); buffers are torch tensors of 3 n_x n_y doubles on the members'
    device.  Every member reaches the same temperature and the same convergence decision, so every process
    takes the same number of iterations (and the same collectives)."""

    def __init__(self, members, nx, ny, maxit, allreduce=None, device=None):
        import torch
        self.members = list(members)
        self.maxit = int(maxit)
        self.allreduce = allreduce
        dev = device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu")
        self.bufs = [torch.zeros(3 * nx * ny, dtype=torch.float64, device=dev) for _ in self.members]
        self.total = torch.zeros(3 * nx * ny, dtype=torch.float64, device=dev)
        self.exchanges = 0

    def step(self):
        """One backward-Euler step; returns (outer iterations, T norm, E norm)."""
        import torch
        for m in self.members:
            m.tstep_begin()
        its, conv, tn, en = 0, False, 0.0, 0.0
        while not conv and its < self.maxit:
            its += 1
            for m, b in zip(self.members, self.bufs):
                m.tstep_sweep(its)
                m.tstep_partials(b)
            for m in self.members:
                m.sync()
            self.total.copy_(self.bufs[0])
            for b in self.bufs[1:]:
                self.total.add_(b)
            if self.allreduce is not None:
                self.allreduce(self.total)
                self.exchanges += 1
            if self.total.is_cuda:
                torch.cuda.synchronize()
            flags = [m.tstep_finish(self.total, its) for m in self.members]
            conv, tn, en = flags[0]
            if any(f[0] != conv for f in flags):
                raise RuntimeError("group ranges disagree on convergence")
        return its, tn, en


class ShardedMlqd:
    """Time steps of the mlqd algorithm (run_type 'mlqd', ALGORITHMS.f08:389-416, 518-572, 670-836) with the
    groups split over `members` (this process's handles) and `allreduce(tensor)` adding the group sums across
    processes (None: one process).

    The groups meet only in group sums (the survey's exchange step): G_old's sum for OLD_GREY_COEFS once per
    step, the transport E of the outer convergence test once per outer iteration, and per MGQD iteration the
    sums behind COLLAPSE_MG_EF, Cbar_Calc and GREY_COEFS (MLOQD_SOLVES.f08:687-730, GLOQD_SOLVES.f08:89-229),
    16 n_x n_y + 2 (n_x+1) n_y + 2 n_x (n_y+1) + 4 (n_x + n_y) doubles (11 MB at 256^2): one all-reduce.  Every
    handle then solves the grey Newton problem with the same totals (replicated) and updates the material of
    its own groups, so every handle (and every process) takes the same iterations and the same collectives.

    A member provides the phases of include/trt_sweep.h: mlqd_exchange_size(), mlqd_step_begin(buf),
    mlqd_step_begin_finish(tot), mlqd_outer_begin(rt, buf), mlqd_outer_begin_finish(tot), mlqd_mgqd_local(buf),
    mlqd_mgqd_finish(mg, tot) -> converged, mlqd_outer_end(rt) -> converged, mlqd_step_end() -> stats;
    buffers are torch tensors on the members' device."""

    def __init__(self, members, maxit_rte, maxit_mloqd, allreduce=None, device=None):
        import torch
        self.members = list(members)
        self.maxit_rte, self.maxit_mloqd = int(maxit_rte), int(maxit_mloqd)
        self.allreduce = allreduce
        sizes = {m.mlqd_exchange_size() for m in self.members}
        if len(sizes) != 1:
            raise ValueError("members of one instance have one grid")
        n = sizes.pop()
        dev = device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu")
        self.bufs = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in self.members]
        self.total = torch.zeros(n, dtype=torch.float64, device=dev)
        self.exchanges = 0

    def _exchange(self, phase):
        import torch
        for m, b in zip(self.members, self.bufs):
            phase(m, b)
        self.total.copy_(self.bufs[0])
        for b in self.bufs[1:]:
            self.total.add_(b)
        if self.allreduce is not None:
            self.allreduce(self.total)
        self.exchanges += 1
        if self.total.is_cuda:
            torch.cuda.synchronize()

    def _agree(self, flags):
        if any(f != flags[0] for f in flags):
            raise RuntimeError("group ranges disagree on convergence")
        return flags[0]

    def step(self):
        """One time step; returns the members' statistics (one dict each: iteration counts, timings)."""
        self._exchange(lambda m, b: m.mlqd_step_begin(b))
        for m in self.members:
            m.mlqd_step_begin_finish(self.total)
        rt, rt_conv = 0, False
        while not rt_conv and rt < self.maxit_rte:
            rt += 1
            self._exchange(lambda m, b: m.mlqd_outer_begin(rt, b))
            for m in self.members:
                m.mlqd_outer_begin_finish(self.total)
            mg, mg_conv = 0, False
            while not mg_conv and mg < self.maxit_mloqd:
                mg += 1
                self._exchange(lambda m, b: m.mlqd_mgqd_local(b))
                mg_conv = self._agree([m.mlqd_mgqd_finish(mg, self.total) for m in self.members])
            rt_conv = self._agree([m.mlqd_outer_end(rt) for m in self.members])
        return [m.mlqd_step_end() for m in self.members]


def torch_allreduce(group=None):
    """All-reduce (sum) across the ranks of torch.distributed's default (or given) process group."""
    import torch.distributed as dist

    def f(t):
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return f
