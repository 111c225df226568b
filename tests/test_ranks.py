"""Replica runs over several ranks (one process per GPU on the bench's N>1 path), exercised on CPU with
the gloo backend: max-over-ranks timing, whole-job throughput, barriers, and the reference arm's
rank-0-only rule."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import importlib, json, os, sys, time
sys.path.insert(0, {root!r})
ranks = importlib.import_module("2d_trt_rom_system_b200.ranks")
ws, rank, local = ranks.init("gloo", timeout_s=60)
assert ws == 2 and local == rank
ranks.barrier()
# each rank times different work; the job time is the slower rank's
ms = [3.0, 5.0][rank]
ms_max = ranks.reduce_max(ms)
rate = ranks.whole_job_rate(1000.0, ms_max * 1e-3, ws)
ranks.barrier()
ranks.finalize()
print(json.dumps({{"rank": rank, "ms_max": ms_max, "rate": rate}}))
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch(code, nproc=2, timeout=120):
    port = free_port()
    procs = []
    for r in range(nproc):
        env = dict(os.environ, WORLD_SIZE=str(nproc), RANK=str(r), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            out, err = p.communicate()
        outs.append((p.returncode, out, err))
    return outs


def test_max_over_ranks_and_whole_job_rate_gloo():
    import json
    outs = launch(WORKER.format(root=ROOT))
    for rc, out, err in outs:
        assert rc == 0, err
    res = [json.loads(o[1].strip().splitlines()[-1]) for o in outs]
    for r in res:
        assert r["ms_max"] == 5.0                       # the slower rank sets the job time
        assert r["rate"] == pytest.approx(2 * 1000.0 / 5e-3)


def test_reference_arm_runs_on_rank_zero_only():
    """bench.py --impl reference: ranks other than 0 exit 0 at once without work."""
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1", CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


def test_single_rank_defaults():
    import importlib
    sys.path.insert(0, ROOT)
    ranks = importlib.import_module("2d_trt_rom_system_b200.ranks")
    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        assert ranks.world() == (1, 0, 0)
        assert ranks.reduce_max(2.5) == 2.5
        ranks.barrier()
        assert ranks.whole_job_rate(10.0, 2.0, 1) == 5.0
    finally:
        os.environ.update(env)
