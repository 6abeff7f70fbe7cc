"""The continuously batching server: every result equals the same request
computed alone, batching and overlap happen, admission respects the HBM
budget, and oversized requests are rejected.  Needs a B200."""
from __future__ import annotations

import importlib
import sys

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def z(zntt):
    zntt.init(0)
    return zntt


@pytest.fixture(scope="module")
def serving(z):
    return importlib.import_module("zig_algebra_b200.serving")


def test_trace_in_the_mix_equals_alone(z, serving):
    import torch
    F = z.BN254_FR
    trace = serving.make_trace(300, rate=2000.0, seed=7, log_min=10, log_max=16)
    work = serving.Workload(z, torch, F, trace)
    try:
        batched = serving.replay(z, torch, F, trace, work, hbm_budget=8 << 30, serial=False)
        serial = serving.replay(z, torch, F, trace, work, hbm_budget=8 << 30, serial=True)
    finally:
        work.close()
    for r in (batched, serial):
        assert r["failures"] == 0 and r["mismatches"] == 0, r
        assert r["requests"] == 300
    assert serial["batches"] == 300 + serial["warmup_requests"]


def test_bursts_are_batched_and_overlap(z, serving):
    import torch
    F = z.BLS12_381_FR
    trace = serving.make_trace(200, rate=200000.0, seed=9, log_min=10, log_max=14)
    work = serving.Workload(z, torch, F, trace)
    try:
        r = serving.replay(z, torch, F, trace, work, hbm_budget=8 << 30, serial=False, slots=3)
    finally:
        work.close()
    assert r["failures"] == 0 and r["mismatches"] == 0, r
    assert r["batches"] < r["requests"]
    assert r["max_batch_jobs"] > 1


def test_admission_stays_within_budget(z, serving):
    import torch
    F = z.BN254_FR
    trace = serving.make_trace(60, rate=1e6, seed=3, log_min=14, log_max=16)
    budget = 3 * (2 * 32 << 16) + 1  # room for three of the largest transforms at once
    work = serving.Workload(z, torch, F, trace)
    try:
        r = serving.replay(z, torch, F, trace, work, hbm_budget=budget, serial=False, slots=4)
    finally:
        work.close()
    assert r["failures"] == 0 and r["mismatches"] == 0, r
    assert 0 < r["peak_device_bytes"] <= budget


def test_oversized_request_is_rejected(z):
    import torch
    F = z.BN254_FR
    buf = torch.empty(4 * (1 << 12), dtype=torch.int64, pin_memory=True)
    with z.Server(F, hbm_budget_bytes=1 << 16) as s:
        req = z.Request()
        req.kind, req.mode, req.log_n, req.log_in = z.JOB_NTT, z.FORWARD, 12, 12
        req.h_in = buf.data_ptr()
        req.h_out = buf.data_ptr()
        with pytest.raises(z.Rejected):
            s.submit(req)
        assert s.stats()["rejected"] == 1
