"""Batches (one persistent launch over many jobs), coset low-degree extensions
and the autotuner, checked bit-exactly against the plain per-job path and the
oracle.  Needs a B200."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
WORKERS = min(os.cpu_count() or 1, 64)


@pytest.fixture(scope="module")
def z(zntt):
    zntt.init(0)
    return zntt


def _torch():
    import torch
    return torch


def _vec(z, F, seed, n):
    torch = _torch()
    x = torch.empty(n * 4, dtype=torch.int64, device="cuda")
    z.random_elements(F, seed, x.data_ptr(), n)
    return x


def _host(t):
    return t.cpu().numpy().view(np.uint64).reshape(-1, 4).copy()


class Tables:
    """Device twiddle tables per log n, closed at the end."""

    def __init__(self, z, F):
        self.z, self.F, self.t = z, F, {}

    def __call__(self, log_n):
        if log_n not in self.t:
            self.t[log_n] = self.z.DeviceTwiddles(self.F, log_n, self.z.primitiveRootOfUnity(self.F, log_n))
        return self.t[log_n]

    def close(self):
        for t in self.t.values():
            t.close()


@pytest.mark.parametrize("shape", [-1, 0, 1, 2, 3, 4])
def test_mixed_batch_matches_per_job_launches(z, shape):
    torch = _torch()
    rng = np.random.default_rng(11)
    for F in z.FIELDS:
        tabs = Tables(z, F)
        logs = [int(v) for v in rng.integers(1, 17, 40)] + [0, 11, 12, 20]
        jobs, refs, outs = [], [], []
        for i, L in enumerate(logs):
            n = 1 << L
            x = _vec(z, F, 500 + i, n)
            mode = z.INVERSE if rng.random() < 0.5 else z.FORWARD
            want = torch.empty_like(x)
            z.ntt_device(tabs(L), x.data_ptr(), want.data_ptr(), mode)
            if i % 3 == 0:  # in place
                dst = x
            else:
                dst = torch.empty_like(x)
            jobs.append({"kind": z.JOB_NTT, "tw": tabs(L), "mode": mode, "src": x.data_ptr(),
                         "dst": dst.data_ptr()})
            refs.append(want)
            outs.append((x, dst))
        torch.cuda.synchronize()
        keep = [x.clone() for x, _ in outs]
        with z.Batch(F, jobs, shape=shape) as b:
            info = b.info()
            assert info["items"] > 0 and info["passes"] >= len(jobs)
            for rep, graph in enumerate([False, True, True]):
                if rep:  # restore in-place inputs between replays
                    for (x, dst), k in zip(outs, keep):
                        x.copy_(k)
                torch.cuda.synchronize()
                b.run(graph=graph)
                torch.cuda.synchronize()
                b.status()
                for i, ((x, dst), want) in enumerate(zip(outs, refs)):
                    assert torch.equal(dst, want), f"{F} job {i} 2^{logs[i]} replay {rep}"
        tabs.close()


def test_coset_lde_matches_oracle_and_fixture(z):
    torch = _torch()
    c = json.load(open(os.path.join(GOLDEN, "coset_lde.json")))
    F = z.BLS12_381_FR
    fid = O.BLS12_381_FR
    shift = O.from_int(fid, c["shift"])
    tabs = Tables(z, F)
    for log_in, blow in [(c["log_in"], c["log_blowup"]), (1, 2), (10, 2), (12, 1), (14, 2)]:
        seed = c["seed"] if log_in == c["log_in"] else 900 + log_in
        ev = _vec(z, F, seed, 1 << log_in)
        out = torch.empty((1 << (log_in + blow)) * 4, dtype=torch.int64, device="cuda")
        z.coset_lde_device(tabs(log_in), tabs(log_in + blow), shift, ev.data_ptr(), out.data_ptr())
        torch.cuda.synchronize()
        want = O.coset_lde(fid, _host(ev), log_in, blow, shift, workers=WORKERS)
        np.testing.assert_array_equal(_host(out), want)
        if log_in == c["log_in"]:
            got = O.to_ints(O.from_mont(fid, _host(out)))
            assert got == [int(v, 16) for v in c["output"]]
    tabs.close()


def test_coset_lde_full_size_against_oracle(z):
    """One extension of the C4 size: 2^18 evaluations to 2^20 over BLS12-381-Fr."""
    torch = _torch()
    F, fid = z.BLS12_381_FR, O.BLS12_381_FR
    shift = O.from_int(fid, 5)
    tabs = Tables(z, F)
    ev = _vec(z, F, 4040, 1 << 18)
    out = torch.empty((1 << 20) * 4, dtype=torch.int64, device="cuda")
    z.coset_lde_device(tabs(18), tabs(20), shift, ev.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    want = O.coset_lde(fid, _host(ev), 18, 2, shift, workers=WORKERS)
    np.testing.assert_array_equal(_host(out), want)
    tabs.close()


def test_batched_coset_extensions_and_mixed_kinds(z):
    torch = _torch()
    F, fid = z.BLS12_381_FR, O.BLS12_381_FR
    shift = O.from_int(fid, 5)
    tabs = Tables(z, F)
    jobs, refs = [], []
    for i, (li, lo) in enumerate([(10, 12), (12, 14), (8, 10), (13, 15), (6, 8)]):
        ev = _vec(z, F, 70 + i, 1 << li)
        out = torch.empty((1 << lo) * 4, dtype=torch.int64, device="cuda")
        want = torch.empty_like(out)
        z.coset_lde_device(tabs(li), tabs(lo), shift, ev.data_ptr(), want.data_ptr())
        jobs.append({"kind": z.JOB_COSET_LDE, "tw": tabs(lo), "tw_in": tabs(li), "shift": shift,
                     "src": ev.data_ptr(), "dst": out.data_ptr(), "_keep": (ev, out)})
        refs.append((out, want))
    for i, L in enumerate([9, 13, 16]):
        x = _vec(z, F, 80 + i, 1 << L)
        y = torch.empty_like(x)
        want = torch.empty_like(x)
        z.ntt_device(tabs(L), x.data_ptr(), want.data_ptr(), z.INVERSE)
        jobs.append({"kind": z.JOB_NTT, "tw": tabs(L), "mode": z.INVERSE, "src": x.data_ptr(), "dst": y.data_ptr(),
                     "_keep": (x, y)})
        refs.append((y, want))
    torch.cuda.synchronize()
    with z.Batch(F, jobs) as b:
        b.run(graph=True)
        torch.cuda.synchronize()
        b.status()
    for i, (got, want) in enumerate(refs):
        assert torch.equal(got, want), f"job {i}"
    tabs.close()


def test_autotune_persists_and_keeps_results(z, tmp_path):
    torch = _torch()
    F = z.BN254_FR
    z.autotune(F, 10, 13)
    path = str(tmp_path / "tune.json")
    z.tune_save(path)
    text = open(path).read()
    assert '"log_n": 12' in text and '"kmax"' in text
    z.tune_clear()
    z.tune_load(path)
    # transforms under the tuned plans still equal the oracle
    for L in (10, 12, 13):
        x = _vec(z, F, 3000 + L, 1 << L)
        y = torch.empty_like(x)
        root = z.primitiveRootOfUnity(F, L)
        with z.DeviceTwiddles(F, L, root) as tw:
            z.ntt_device(tw, x.data_ptr(), y.data_ptr(), z.FORWARD)
        torch.cuda.synchronize()
        want = _host(x)
        O.ntt(O.BN254_FR, want, L, root)
        np.testing.assert_array_equal(_host(y), want)
    z.tune_clear()


@pytest.mark.parametrize("shape", [0, 1, 2, 3, 4])
def test_every_pass_shape_matches_oracle(z, tmp_path, shape):
    """Plans forced to one pass shape (through a tuning file) stay bit-exact."""
    torch = _torch()
    name = torch.cuda.get_device_name(0)
    path = tmp_path / "tune.json"
    lt = {0: 11, 1: 10, 2: 9, 3: 8, 4: 9}[shape]  # the shape's tile (kShapes in csrc/kernels.cuh)
    lines = [f' {{"gpu": "{name}", "field": {f}, "log_n": {L}, "shape": {shape}, "kmax": {k}, "us": 1.0}}'
             for f in (0, 1) for L in range(1, 23) for k in [lt - 1 if L % 2 else lt - 3]]
    path.write_text("[\n" + ",\n".join(lines) + "\n]\n")
    z.tune_clear()
    z.tune_load(str(path))
    try:
        for F in z.FIELDS:
            fid = F.id
            for L in (5, 11, 12, 15, 18, 21):
                root = z.primitiveRootOfUnity(F, L)
                x = _vec(z, F, 8000 + L, 1 << L)
                with z.DeviceTwiddles(F, L, root) as tw:
                    for mode in (z.FORWARD, z.INVERSE):
                        y = torch.empty_like(x)
                        z.ntt_device(tw, x.data_ptr(), y.data_ptr(), mode)
                        torch.cuda.synchronize()
                        want = _host(x)
                        st, otw = O.precompute_twiddles(fid, L, root)
                        O.ntt_with_twiddles(fid, want, L, otw, inverse=mode == z.INVERSE, workers=WORKERS,
                                            inplace4=True)
                        np.testing.assert_array_equal(_host(y), want, err_msg=f"{F} 2^{L} mode {mode}")
    finally:
        z.tune_clear()


# --- the batched configurations against the oracle directly ---------------------------------

def _oracle_jobs(fn, args_list):
    """Runs oracle calls (each single-threaded) on all host cores; ctypes releases the GIL."""
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=WORKERS) as ex:
        return list(ex.map(lambda a: fn(*a), args_list))


class OracleTables:
    """The oracle's precomputeTwiddles stages of the primitive 2^log_n-th root, per log n."""

    def __init__(self, fid):
        self.fid, self.t = fid, {}

    def __call__(self, log_n):
        if log_n not in self.t:
            st, root = O.primitive_root(self.fid, log_n)
            assert st == O.OK
            st, stages = O.precompute_twiddles(self.fid, log_n, root)
            assert st == O.OK
            self.t[log_n] = stages
        return self.t[log_n]


def test_mixed_batch_of_the_benchmark_matches_oracle(z):
    """The batched configuration itself -- 512 BN254-Fr transforms of 2^U{10..16} plus 8 of 2^20,
    directions 50/50 by seed, in one persistent launch (plain and through the CUDA graph) --
    equals the oracle's nttWithTwiddles / inttWithTwiddles (libs/ntt/src/root.zig:148-212) for
    every job."""
    torch = _torch()
    F, fid = z.BN254_FR, O.BN254_FR
    rng = np.random.default_rng(33)
    logs = [int(v) for v in rng.integers(10, 17, 512)] + [20] * 8
    modes = [z.INVERSE if v < 0.5 else z.FORWARD for v in rng.random(len(logs))]
    total = sum(1 << L for L in logs)
    pool = torch.empty(total * 4, dtype=torch.int64, device="cuda")
    z.random_elements(F, 33, pool.data_ptr(), total)
    host = _host(pool)
    tabs, otabs = Tables(z, F), OracleTables(fid)
    jobs, outs, offs = [], [], []
    off = 0
    for L, m in zip(logs, modes):
        y = torch.empty((1 << L) * 4, dtype=torch.int64, device="cuda")
        jobs.append({"kind": z.JOB_NTT, "tw": tabs(L), "mode": m, "src": pool.data_ptr() + off * 32,
                     "dst": y.data_ptr()})
        outs.append(y)
        offs.append(off)
        off += 1 << L

    def oracle_job(i):
        L = logs[i]
        want = np.ascontiguousarray(host[offs[i]:offs[i] + (1 << L)])
        assert O.ntt_with_twiddles(fid, want, L, otabs(L), inverse=modes[i] == z.INVERSE, inplace4=True) == O.OK
        return want

    for L in sorted(set(logs)):
        otabs(L)  # tables built once, before the threads share them
    wants = _oracle_jobs(oracle_job, [(i,) for i in range(len(logs))])
    with z.Batch(F, jobs) as b:
        assert b.info()["items"] > 10000  # 16,827 tiles of 2^11 elements under the default plan
        for graph in (False, True, True):
            for y in outs:
                y.zero_()
            torch.cuda.synchronize()
            b.run(graph=graph)
            torch.cuda.synchronize()
            b.status()
            for i, (y, want) in enumerate(zip(outs, wants)):
                np.testing.assert_array_equal(_host(y), want, err_msg=f"job {i}: 2^{logs[i]} mode {modes[i]} "
                                                                      f"graph {graph}")
    tabs.close()


def test_batched_coset_extensions_of_the_benchmark_match_oracle(z):
    """The batched coset-extension configuration: 64 BLS12-381-Fr extensions 2^18 -> 2^20 with
    g = 5 in one persistent launch, every one equal to the oracle's composition of
    inttWithTwiddles, zero padding, powers/hadamard (libs/poly/src/vector.zig:24-32,68-73) and
    nttWithTwiddles."""
    torch = _torch()
    F, fid = z.BLS12_381_FR, O.BLS12_381_FR
    shift = O.from_int(fid, 5)
    tabs = Tables(z, F)
    pool = torch.empty(64 * (1 << 18) * 4, dtype=torch.int64, device="cuda")
    z.random_elements(F, 44, pool.data_ptr(), 64 << 18)
    host = _host(pool)
    outs = [torch.empty((1 << 20) * 4, dtype=torch.int64, device="cuda") for _ in range(64)]
    jobs = [{"kind": z.JOB_COSET_LDE, "tw": tabs(20), "tw_in": tabs(18), "shift": shift,
             "src": pool.data_ptr() + i * (32 << 18), "dst": outs[i].data_ptr()} for i in range(64)]
    wants = _oracle_jobs(lambda i: O.coset_lde(fid, np.ascontiguousarray(host[i << 18:(i + 1) << 18]), 18, 2, shift),
                         [(i,) for i in range(64)])
    with z.Batch(F, jobs) as b:
        for graph in (False, True):
            for y in outs:
                y.zero_()
            torch.cuda.synchronize()
            b.run(graph=graph)
            torch.cuda.synchronize()
            b.status()
            for i, (y, want) in enumerate(zip(outs, wants)):
                np.testing.assert_array_equal(_host(y), want, err_msg=f"extension {i} graph {graph}")
    tabs.close()


def test_bounded_wait_times_out_then_batch_recovers(z):
    """The persistent kernel's dependency wait is bounded.  With a limit of zero rounds the
    first tile that finds its previous pass unfinished raises the batch's error flag: the
    launch still completes, every CTA stops at its next item, and status() reports Timeout.
    With the default limit restored the same batch (plain and graph) is bit-exact again."""
    torch = _torch()
    F, fid = z.BN254_FR, O.BN254_FR
    tabs, otabs = Tables(z, F), OracleTables(fid)
    # One multi-pass job: its second pass's first tile is taken while the first pass's last
    # wave of tiles is still running on the other CTAs, so that wait cannot find it done.
    logs = [21]
    xs = [_vec(z, F, 6100 + i, 1 << L) for i, L in enumerate(logs)]
    ys = [torch.empty_like(x) for x in xs]
    jobs = [{"kind": z.JOB_NTT, "tw": tabs(L), "mode": z.FORWARD, "src": x.data_ptr(), "dst": y.data_ptr()}
            for L, x, y in zip(logs, xs, ys)]

    def oracle_job(i):
        want = _host(xs[i])
        assert O.ntt_with_twiddles(fid, want, logs[i], otabs(logs[i]), inplace4=True) == O.OK
        return want

    for L in set(logs):
        otabs(L)
    wants = _oracle_jobs(oracle_job, [(i,) for i in range(len(logs))])
    with z.Batch(F, jobs) as b:
        assert b.info()["passes"] > len(jobs) and b.info()["items"] > 2 * b.info()["grid"]
        for graph in (False, True):
            b.set_spin_limit(0)
            torch.cuda.synchronize()
            b.run(graph=graph)
            torch.cuda.synchronize()  # the launch ends: no CTA waits without a bound
            with pytest.raises(z.Timeout):
                b.status()
            b.set_spin_limit(z.BATCH_SPIN_LIMIT)
            for y in ys:
                y.zero_()
            b.run(graph=graph)
            torch.cuda.synchronize()
            b.status()
            for i, (y, want) in enumerate(zip(ys, wants)):
                np.testing.assert_array_equal(_host(y), want, err_msg=f"job {i} after the timeout, graph {graph}")
    tabs.close()
