"""The continuously batching server: every result equals the same request
computed alone, batching and overlap happen, admission respects the HBM
budget, and oversized requests are rejected.  Needs a B200."""
from __future__ import annotations

import importlib
import os
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


def test_trace_in_the_mix_equals_alone_and_oracle(z, serving):
    """A mixed trace reaching 2^20 with coset extensions, every request with its own input:
    every output served by continuous batching equals the same request served alone (the
    serial replay, one request per plain launch sequence) and the oracle's result
    (nttWithTwiddles / inttWithTwiddles, libs/ntt/src/root.zig:148-212, or the coset
    composition with libs/poly/src/vector.zig:24-32,68-73), word for word."""
    import numpy as np
    import torch
    from concurrent.futures import ThreadPoolExecutor

    import oracle as O
    F, fid = z.BN254_FR, O.BN254_FR
    trace = serving.make_trace(300, rate=2000.0, seed=7, log_min=10, log_max=20, p=0.25)
    # the largest size in every kind, spread through the trace
    for i, k in zip((40, 120, 200, 260), (0, 1, 2, 2)):
        a, _, _, v = trace[i]
        trace[i] = (a, k, 20, v)
    assert {k for _, k, _, _ in trace} == {0, 1, 2} and max(L for _, _, L, _ in trace) == 20
    work = serving.Workload(z, torch, F, trace)
    got_b, got_s = {}, {}
    try:
        batched = serving.replay(z, torch, F, trace, work, hbm_budget=8 << 30, serial=False, keep_outputs=got_b)
        serial = serving.replay(z, torch, F, trace, work, hbm_budget=8 << 30, serial=True, keep_outputs=got_s)
        inputs = [work.input_host(serving.input_log(k, L), v) for _, k, L, v in trace]
    finally:
        work.close()
    for r in (batched, serial):
        assert r["failures"] == 0 and r["mismatches"] == 0, r
        assert r["requests"] == 300
    assert serial["batches"] == 300 + serial["warmup_requests"]
    assert batched["batches"] < serial["batches"]

    tables = {}
    for L in sorted({L for _, k, L, _ in trace if k != 2}):
        st, root = O.primitive_root(fid, L)
        tables[L] = O.precompute_twiddles(fid, L, root)[1]
    shift = O.from_int(fid, 5)

    def oracle(i):
        _, k, L, _ = trace[i]
        x = inputs[i]
        if k == 2:
            return O.coset_lde(fid, x, L - 2, 2, shift)
        assert O.ntt_with_twiddles(fid, x, L, tables[L], inverse=k == 1, inplace4=True) == O.OK
        return x

    with ThreadPoolExecutor(max_workers=min(os.cpu_count() or 1, 64)) as ex:
        wants = list(ex.map(oracle, range(len(trace))))
    for i, want in enumerate(wants):
        _, k, L, _ = trace[i]
        np.testing.assert_array_equal(got_b[i], want, err_msg=f"request {i}: kind {k} 2^{L} (batched)")
        np.testing.assert_array_equal(got_s[i], want, err_msg=f"request {i}: kind {k} 2^{L} (alone)")


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
