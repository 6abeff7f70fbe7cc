"""Replays a request trace through the transform server and reports latency.

The trace is the serving workload of the benchmark: Poisson arrivals at a
seeded rate, log2 sizes from a truncated geometric distribution, a mix of
forward transforms, inverse transforms and blowup-4 coset extensions.  Every
request has its own input: a distinct slice of one seeded pool of field
elements, generated on the device and held in pinned host memory.  Every
output is checked against the same request computed alone with the plain
entry points, by a consumer thread while the replay runs: both sides are
reduced to a 64-bit weighted checksum (sum of word_i * w_i mod 2^64 with seeded
odd weights w_i), so the check needs no second copy of every output; callers
that want the outputs themselves (the tests compare each with the oracle) ask
replay() to keep them.
"""
from __future__ import annotations

import gc
import sys
import threading
import time

import numpy as np

_OFFSET_STEP = 8191  # prime: distinct input ids map to distinct pool offsets


def make_trace(n: int, rate: float, seed: int, log_min: int = 10, log_max: int = 22, p: float = 0.35,
               mix=(0.7, 0.2, 0.1)):
    """(arrival_s, kind, log_n, input_id) per request; kind 0 forward, 1 inverse, 2 coset
    extension (output 2^log_n from 2^(log_n - 2) evaluations).  input_id is the request's
    index, so every request transforms its own input."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    ks = np.arange(log_min, log_max + 1)
    probs = p * (1 - p) ** (ks - log_min)
    probs /= probs.sum()
    logs = rng.choice(ks, size=n, p=probs)
    u = rng.random(n)
    kinds = np.where(u < mix[0], 0, np.where(u < mix[0] + mix[1], 1, 2))  # 0 fwd, 1 inv, 2 lde
    return [(float(a), int(k), int(L), i) for i, (a, k, L) in enumerate(zip(arrivals, kinds, logs))]


def input_log(kind: int, log_n: int) -> int:
    return log_n - 2 if kind == 2 else log_n


class Workload:
    """Every request's pinned input and the checksum of its result computed alone."""

    def __init__(self, z, torch, F, trace, seed: int = 5):
        self.z, self.torch, self.F = z, torch, F
        self.shift = z.to_montgomery(F, 5)
        self.tabs = {}
        max_in = max(1 << input_log(k, L) for _, k, L, _ in trace)
        max_out = max(1 << L for _, _, L, _ in trace)
        self.pool_elems = 2 * max_in
        # One stream orders the library's launches and the torch reductions after them.
        stream = torch.cuda.Stream()
        sptr = stream.cuda_stream
        with torch.cuda.stream(stream):
            self.d_pool = torch.empty(self.pool_elems * 4, dtype=torch.int64, device="cuda")
            z.random_elements(F, seed, self.d_pool.data_ptr(), self.pool_elems, stream=sptr)
            self.h_pool = torch.empty(self.d_pool.numel(), dtype=torch.int64, pin_memory=True)
            self.h_pool.copy_(self.d_pool)
            # Checksum weights: seeded odd 64-bit words, one per output word.
            w = np.random.default_rng(seed + 1).integers(0, 1 << 63, 4 * max_out, dtype=np.uint64) * \
                np.uint64(2) + np.uint64(1)
            self.w_host = w
            self.w_dev = torch.from_numpy(w.view(np.int64)).cuda()
            seen: dict[int, set] = {}
            for _, k, L, v in trace:
                lin = input_log(k, L)
                o = self.offset(lin, v)
                assert o not in seen.setdefault(lin, set()), "two requests share an input"
                seen[lin].add(o)
            # The result of every request computed alone, reduced to its checksum on the device
            # (int64 products and sums wrap modulo 2^64 like the host's uint64 ones).
            dig = torch.empty(len(trace), dtype=torch.int64, device="cuda")
            outs = {}
            for tag, (_, k, L, v) in enumerate(trace):
                if L not in outs:
                    outs[L] = torch.empty((1 << L) * 4, dtype=torch.int64, device="cuda")
                out = outs[L]
                src = self.d_pool.data_ptr() + self.offset(input_log(k, L), v) * 32
                if k == 2:
                    z.coset_lde_device(self.table(L - 2), self.table(L), self.shift, src, out.data_ptr(),
                                       stream=sptr)
                else:
                    z.ntt_device(self.table(L), src, out.data_ptr(), z.FORWARD if k == 0 else z.INVERSE,
                                 stream=sptr)
                dig[tag] = (out * self.w_dev[:out.numel()]).sum()
            self.digests = dig.cpu().numpy().view(np.uint64).copy()
            del outs, dig
        torch.cuda.synchronize()

    def offset(self, lin: int, input_id: int) -> int:
        """Element offset of an input in the pool: distinct for distinct ids of one size."""
        return (input_id * _OFFSET_STEP) % (self.pool_elems - (1 << lin) + 1)

    def input_ptr(self, lin: int, input_id: int) -> int:
        return self.h_pool.data_ptr() + self.offset(lin, input_id) * 32

    def input_host(self, lin: int, input_id: int) -> np.ndarray:
        """The request's input as (2^lin, 4) Montgomery limbs (a copy)."""
        o = self.offset(lin, input_id)
        return self.h_pool.numpy().view(np.uint64).reshape(-1, 4)[o:o + (1 << lin)].copy()

    def checksum(self, out_words: np.ndarray) -> int:
        """The weighted checksum of a result given as uint64 words."""
        return int((out_words * self.w_host[:len(out_words)]).sum())

    def table(self, L):
        if L not in self.tabs:
            self.tabs[L] = self.z.DeviceTwiddles(self.F, L, self.z.primitiveRootOfUnity(self.F, L))
        return self.tabs[L]

    def close(self):
        for t in self.tabs.values():
            t.close()
        self.tabs = {}


def replay(z, torch, F, trace, work: Workload, hbm_budget: int, serial: bool, slots: int = 4,
           max_batch_jobs: int = 256, warmup: bool = True, keep_outputs: dict | None = None) -> dict:
    """Submits each request at its arrival time; returns latency and throughput figures.
    With `keep_outputs` (a dict), every served result is also stored there by request index,
    as (2^log_n, 4) Montgomery limbs."""
    pools: dict[int, list] = {}
    lock = threading.Lock()
    inflight: dict[int, tuple] = {}
    lat, mismatches, failures = [], [], []
    records = []  # (tag, kind, log_n, arrival, submit, admit, done)
    submit_ns: dict[int, int] = {}
    done_count = [0]
    total = len(trace)
    first_done = [None]
    last_done = [0]

    diag = {"pinned_allocs": 0, "pinned_alloc_ms": 0.0, "max_verify_ms": 0.0, "gc_pause_ms": 0.0,
            "max_gc_pause_ms": 0.0, "pinned_alloc_events": []}
    t_start = [time.perf_counter()]

    def out_buf(L):
        with lock:
            lst = pools.setdefault(L, [])
            if lst:
                return lst.pop()
        t = time.perf_counter()
        b = torch.empty((1 << L) * 4, dtype=torch.int64, pin_memory=True)
        dt = 1e3 * (time.perf_counter() - t)
        diag["pinned_allocs"] += 1
        diag["pinned_alloc_ms"] += dt
        if len(diag["pinned_alloc_events"]) < 16:
            diag["pinned_alloc_events"].append((round(t - t_start[0], 4), L, round(dt, 3)))
        return b

    gc_t = [0.0]

    def gc_cb(phase, info):
        if phase == "start":
            gc_t[0] = time.perf_counter()
        else:
            d = 1e3 * (time.perf_counter() - gc_t[0])
            diag["gc_pause_ms"] += d
            diag["max_gc_pause_ms"] = max(diag["max_gc_pause_ms"], d)

    server = z.Server(F, hbm_budget, slots=slots, max_batch_jobs=max_batch_jobs, serial=serial)

    def make_request(tag, k, L, v, buf, arrival):
        lin = L - 2 if k == 2 else L
        req = z.Request()
        req.kind = z.JOB_COSET_LDE if k == 2 else z.JOB_NTT
        req.mode = z.INVERSE if k == 1 else z.FORWARD
        req.log_n = L
        req.log_in = lin
        req.h_in = work.input_ptr(lin, v)
        req.h_out = buf.data_ptr()
        for i in range(4):
            req.shift[i] = int(work.shift[i])
        req.user_tag = tag
        req.arrival_ns = arrival
        return req

    n_warm = 0
    if warmup:
        # One request per (kind, size) before the timed trace: the server builds
        # its resident tables and buffers, the way it would before taking traffic.
        # Three concurrent copies per class, so the buffer pool holds more
        # than one buffer of each size.
        classes = sorted({(k, L): v for _, k, L, v in trace}.items()) * 3
        bufs = [torch.empty((1 << L) * 4, dtype=torch.int64, pin_memory=True) for (_, L), _ in classes]
        for i, (((k, L), v), b) in enumerate(zip(classes, bufs)):
            server.submit(make_request((1 << 62) + i, k, L, v, b, z.now_ns()))
        got = 0
        while got < len(classes):
            got += len(server.poll(wait_ms=100))
        n_warm = len(classes)

    def consume():
        while done_count[0] < total:
            for tag, status, arr, adm, dn in server.poll(wait_ms=50):
                with lock:
                    k, L, v, buf = inflight.pop(tag)
                tv = time.perf_counter()
                if status != 0:
                    failures.append((tag, status))
                else:
                    words = buf.numpy().view(np.uint64)
                    if work.checksum(words) != int(work.digests[tag]):
                        mismatches.append(tag)
                    if keep_outputs is not None:
                        keep_outputs[tag] = words.reshape(-1, 4).copy()
                diag["max_verify_ms"] = max(diag["max_verify_ms"], 1e3 * (time.perf_counter() - tv))
                lat.append((dn - arr) / 1e6)
                records.append((tag, k, L, arr, submit_ns.get(tag, arr), adm, dn))
                last_done[0] = max(last_done[0], dn)
                with lock:
                    pools.setdefault(L, []).append(buf)
                done_count[0] += 1

    # Pinned output buffers are allocated before the replay (a pinned
    # allocation can take milliseconds): as many per size as may be in flight.
    counts: dict[int, int] = {}
    for _, _, L, _ in trace:
        counts[L] = counts.get(L, 0) + 1
    # Up to 256 MB per size (at least 16 buffers): a pinned allocation during the replay
    # stalls the submitting thread for milliseconds to hundreds of milliseconds.
    for L, c in counts.items():
        cap = max(16, (256 << 20) // (32 << L))
        pools[L] = [torch.empty((1 << L) * 4, dtype=torch.int64, pin_memory=True) for _ in range(min(c, cap))]
    th = threading.Thread(target=consume, daemon=True)
    pool0 = z.pool_stats()
    gc.callbacks.append(gc_cb)
    old_switch = sys.getswitchinterval()
    sys.setswitchinterval(5e-5)  # hand the interpreter over quickly between submitter and consumer
    th.start()
    t0 = z.now_ns() + 20_000_000
    t_start[0] = time.perf_counter() + 0.02
    late = 0
    for tag, (a, k, L, v) in enumerate(trace):
        arrival = t0 + int(a * 1e9)
        while True:
            now = z.now_ns()
            if now >= arrival:
                break
            if arrival - now > 200_000:
                time.sleep((arrival - now - 150_000) / 1e9)
        if z.now_ns() - arrival > 1_000_000:
            late += 1
        buf = out_buf(L)
        with lock:
            inflight[tag] = (k, L, v, buf)
        req = make_request(tag, k, L, v, buf, arrival)
        submit_ns[tag] = z.now_ns()
        server.submit(req)
    th.join()
    sys.setswitchinterval(old_switch)
    gc.callbacks.remove(gc_cb)
    stats = server.stats()
    server.close()
    pool1 = z.pool_stats()
    diag["pool_device_mallocs"] = pool1["device_mallocs"] - pool0["device_mallocs"]
    lat_a = np.array(lat)
    rec = np.array(records, dtype=np.float64)
    worst = rec[np.argsort(rec[:, 6] - rec[:, 3])[-8:]] if len(rec) else rec
    lateness = (rec[:, 4] - rec[:, 3]) / 1e6 if len(rec) else np.zeros(1)
    queueing = (rec[:, 5] - rec[:, 4]) / 1e6 if len(rec) else np.zeros(1)
    service = (rec[:, 6] - rec[:, 5]) / 1e6 if len(rec) else np.zeros(1)
    span_s = (last_done[0] - t0) / 1e9
    elements = sum(1 << L for _, _, L, _ in trace)
    return {
        "mode": "serial plain launches" if serial else "continuous batching",
        "requests": total, "warmup_requests": n_warm, "failures": len(failures), "mismatches": len(mismatches),
        "p50_ms": float(np.percentile(lat_a, 50)), "p99_ms": float(np.percentile(lat_a, 99)),
        "mean_ms": float(lat_a.mean()), "max_ms": float(lat_a.max()),
        "throughput_req_s": total / span_s, "elements_per_s": elements / span_s, "span_s": span_s,
        "late_submits": late, "batches": stats["batches"], "max_batch_jobs": stats["max_batch_jobs"],
        "max_inflight_jobs": stats["max_inflight_jobs"], "peak_device_bytes": stats["peak_bytes"],
        "max_launch_ms": stats["max_launch_ns"] / 1e6, "max_batch_ms": stats["max_batch_ns"] / 1e6,
        "driver": diag,
        "p99_submit_lateness_ms": float(np.percentile(lateness, 99)),
        "p99_queueing_ms": float(np.percentile(queueing, 99)), "p99_service_ms": float(np.percentile(service, 99)),
        "worst": [{"tag": int(r[0]), "kind": int(r[1]), "log_n": int(r[2]), "at_s": (r[3] - t0) / 1e9,
                   "late_ms": (r[4] - r[3]) / 1e6, "queue_ms": (r[5] - r[4]) / 1e6, "service_ms": (r[6] - r[5]) / 1e6}
                  for r in worst],
    }
