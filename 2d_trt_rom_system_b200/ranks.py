"""One process per GPU for replica runs: rank setup, barrier and max-over-ranks timing.

The sweep shards by independent instance (or group) with no exchange on the data path, so a run on N
GPUs is N replicas: each rank times its own work on the device, the job time is the maximum over ranks,
and whole-job throughput is N x (units per rank) / that time.  The backend is NCCL on GPUs; the same
code runs with gloo on CPU (tests).
"""
import datetime
import os


def world():
    """(world_size, rank, local_rank) from the torchrun environment (1, 0, 0 when absent)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=600):
    """Join the process group when world_size > 1; bind the local GPU for NCCL."""
    ws, rank, local = world()
    if ws > 1:
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank, local


def _device():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def reduce_max(val):
    """Maximum of a float over all ranks (every rank gets it)."""
    ws, _, _ = world()
    if ws == 1:
        return float(val)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(val)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    ws, _, _ = world()
    if ws > 1:
        import torch.distributed as dist
        if dist.get_backend() == "nccl":
            import torch
            dist.barrier(device_ids=[torch.cuda.current_device()])
        else:
            dist.barrier()


def finalize():
    ws, _, _ = world()
    if ws > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()


def whole_job_rate(units_per_rank, seconds_max, ws):
    """Aggregate throughput of ws replicas that each processed units_per_rank in at most seconds_max."""
    return ws * units_per_rank / seconds_max
