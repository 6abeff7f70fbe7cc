"""The multi-rank path of bench.py on CPU (gloo, world size 2): ranks run
independent replicas, the timed region's duration is the maximum over ranks
and throughput aggregates over ranks; under torchrun the reference arm runs
on rank 0 only and every rank exits cleanly."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # rank r "took" 10 * (r + 1) ms for 4 steps of 2^10 elements
    t = bench.max_over_ranks(0.010 * (rank + 1), dist, "cpu")
    rate = bench.aggregate_rate(4 * 1024, world, t)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, t, rate))


def test_max_over_ranks_and_aggregate_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    for _, t, rate in got:
        assert t == pytest.approx(0.020)
        assert rate == pytest.approx(2 * 4 * 1024 / 0.020)


def test_reference_arm_under_torchrun_rank0_only():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--log-n", "10"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["impl"] == "reference" and lines[0]["value"] > 0


def test_summary_digests_every_configuration():
    """bench.py ends its line with a short digest of every configuration; the digest reads the
    keys the configurations write (a renamed key would break the default run on the GPU)."""
    import bench
    cfg = {"ms_per_batch": 3.0, "plain_ms_per_batch": 15.0, "speedup_vs_plain": 5.0, "bit_exact_vs_plain": True}
    served = {"p50_ms": 0.12, "p99_ms": 3.0, "throughput_req_s": 2000.0, "mismatches": 0, "failures": 0}
    line = {"ms_per_step": 3.54, "roofline": {"frac": 0.845},
            "e2e": {"value": 1.4e9, "pcie": {"e2e_frac_of_bound": 0.94}},
            "sizes": {"bn254_fr 2^24 forward": {"ms": 3.54, "frac": 0.845}},
            "batched": cfg, "coset_lde": cfg,
            "serve": {"continuous_batching": served, "serial_plain": dict(served, p50_ms=0.13)},
            "poly_mul": {"ms": 11.4}, "small_fields": {"fields": {"goldilocks": {"ms": 0.52}}}}
    s = bench.summarize(line)
    assert s["headline"]["frac"] == 0.845 and s["batched"]["speedup_vs_plain"] == 5.0
    assert s["serve"]["serial_p50_ms"] == 0.13 and s["serve"]["mismatches"] == 0
    assert s["sizes_ms_frac"]["bn254_fr 2^24 forward"] == [3.54, 0.845]
    assert len(json.dumps(s)) < 1400  # it must fit the end of the line that readers keep
