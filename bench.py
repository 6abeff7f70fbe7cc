"""Benchmark: BN254-Fr forward NTT of 2^24 elements on B200, one JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl zntt|reference] [--log-n L]
                    [--headline-only] [--workload ntt|batched|lde|poly|small|fri|serve]

A step is one forward transform (zig-ntt nttWithTwiddles semantics,
libs/ntt/src/root.zig:148-175) of 2^24 seeded uniform BN254-Fr elements with
the twiddle table resident on the device.  `value` is elements/s over all
ranks with the input already in HBM (512 MiB per vector, larger than the
126 MB L2, so no flush is needed between steps).  `e2e` is the same metric
through the C ABI's host-buffer entry points: zntt_ntt_host_many over pinned
host vectors, whose timed region includes every step's host->device copy of
the input and device->host copy of the result (overlapped across vectors), and
beside it one synchronous zntt_ntt_with_twiddles call.  Under torchrun every
rank transforms its own vector (independent objects: weak scaling, no
collective on the data path); the time is the max over ranks.  `e2e.pcie`
measures the host link's duplex bound beside it.  The default run adds, on
a single-GPU run, one key per configuration beside the headline (a multi-GPU run prints the
headline and e2e only): sizes (BN254-Fr 2^20,
2^22, 2^24 and BLS12-381-Fr 2^24, forward and inverse, each with its fraction of
the multiply-pipe roofline), batched, coset_lde, poly_mul, small_fields --
transforms, an extension, a 64-column trace extension and row commitment --,
fri_fold -- folds, layer and row commitments against the BLAKE3 probe, the
prover loop and its openings, for BN254-Fr, Goldilocks and BabyBear -- and serve
(the 20,000-request trace, continuous batching against serial plain launches;
--no-serve leaves it out).  The line ends with `summary`, a short digest of
every configuration.  --workload prints one configuration alone as its own line
(`serve` adds a capacity sweep).

`--impl reference` times the CPU restatement of zig-ntt (oracle/) on all host
cores instead: zig-ntt has no GPU path and its toolchain (Zig 0.16) is not
available, so the reference arm is the oracle port with the reference's
fork-join pool semantics (libs/parallel/src/root.zig:45-79).
"""
from __future__ import annotations

import argparse
import ctypes
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
# Multiply-pipe issue slots per 8x32-bit CIOS field product: 2N^2 + N = 136
# full 32x32->64 products, each two 32-bit IMAD slots (lo and hi).
IMAD_PER_MODMUL = 272
METRIC = "BN254-Fr NTT elems/s at 2^24"


def metric_name(log_n: int) -> str:
    """The headline metric's name for a transform of 2^log_n (2^24 by default)."""
    return METRIC if log_n == 24 else f"BN254-Fr NTT elems/s at 2^{log_n}"


def l2_note(n: int) -> str:
    mib = n * 32 / 2**20
    if mib * 2**20 > 126e6:
        return f"inputs ({mib:g} MiB per vector) larger than L2; no flush"
    return f"inputs ({mib:g} MiB per vector) fit in L2 (126 MB); no flush"


def load_package():
    name = "zig_algebra_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = os.path.join(ROOT, "zig-algebra_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The maximum of `value` over all ranks (the value itself without a process group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(per_rank_units: float, world: int, seconds_max: float) -> float:
    """Whole-job throughput: every rank processed per_rank_units; time is the slowest rank's."""
    return world * per_rank_units / seconds_max


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def read_traffic(log_n: int):
    """DRAM bytes (read + write) per pass launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"ntt_pass_bn254_fr_2p{log_n}_dram.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch_mean:"):
            return float(line.split(":", 1)[1].split()[0])
    return None


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return json.load(open(path)), "measured"
    return {"hbm_gbs": 6650.0}, "fallback"


# --- CPU baseline (the oracle port) ------------------------------------------------------

def cpu_oracle(native: bool = True):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    lib = None
    if native:
        try:
            lib = O.load(O.build(native=True))
        except Exception:  # noqa: BLE001 -- fall back to the portable build of the checker
            lib = None
    if lib is None:
        O.load()
        lib = O.load(os.path.join(ROOT, "oracle", "liboracle.so"))
    return O, lib


def cpu_transform_seconds(O, lib, data, log_n, stages, workers, field=None):
    """One in-place oracle nttWithTwiddles over `data` (BN254-Fr 4-u64 slots, or one u64 per
    element for a 64-bit `field`), fork-join over `workers` threads."""
    ptrs = (O._U64P * len(stages))()
    lens = (ctypes.c_size_t * len(stages))()
    for s, a in enumerate(stages):
        ptrs[s] = a.ctypes.data_as(O._U64P)
        lens[s] = len(a)
    t0 = time.perf_counter()
    if field is None:
        st = lib.zo_ntt_with_twiddles_inplace4(O.BN254_FR, O._p(data), len(data), log_n, ptrs, lens, len(stages), 0,
                                               workers)
    else:
        st = lib.zo_ntt_with_twiddles_inplace1(field, data.ctypes.data_as(O._U64P), len(data), log_n, ptrs, lens,
                                               len(stages), 0, workers)
    dt = time.perf_counter() - t0
    assert st == 0
    return dt


def cpu_reference_setup(log_n, seed, host_data=None):
    O, lib = cpu_oracle(native=True)
    n = 1 << log_n
    data = host_data.copy() if host_data is not None else O.random_elements(O.BN254_FR, seed, n)
    st, root = O.primitive_root(O.BN254_FR, log_n)
    st, stages = O.precompute_twiddles(O.BN254_FR, log_n, root)
    return O, lib, data, stages


def run_reference(args, rank):
    """The reference arm: zig-ntt's algorithm (oracle port) on every host core.

    A step is one forward transform of the workload's size when all K steps
    fit in about three minutes; otherwise each step is a 2^(log_n - 2)
    transform (the sample is named in the line).  Only rank 0 runs."""
    if rank != 0:
        return
    workers = min(os.cpu_count() or 1, 64)
    log_n = args.log_n
    O, lib, data, stages = cpu_reference_setup(log_n, args.seed)
    t_one = cpu_transform_seconds(O, lib, data, log_n, stages, workers)  # first warm-up step
    if (args.steps + args.warmup) * t_one > 180.0 and log_n > 12:
        log_n -= 2
        O, lib, data, stages = cpu_reference_setup(log_n, args.seed)
    n = 1 << log_n
    for _ in range(max(0, args.warmup - 1)):
        cpu_transform_seconds(O, lib, data, log_n, stages, workers)
    times = [cpu_transform_seconds(O, lib, data, log_n, stages, workers) for _ in range(args.steps)]
    total = sum(times)
    value = n * args.steps / total
    sample = (f"{args.steps} full 2^{log_n} forward transforms, oracle nttWithTwiddles, fork-join over the "
              f"butterflies of each stage on {workers} threads")
    if log_n != args.log_n:
        sample += f" (2^{log_n} per step: 2^{args.log_n} steps would not fit the time budget)"
    line = {
        "impl": "reference", "metric": metric_name(args.log_n), "value": value, "unit": "elements/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u256-mod-r (BN254-Fr)",
        "data": "synthetic: seeded ChaCha20 randomFieldElement draws",
        "config": {"workload": f"bn254_fr_ntt_forward_2^{args.log_n}", "log_n": args.log_n, "sample_log_n": log_n,
                   "field": "bn254_fr", "direction": "forward", "twiddles": "precomputed", "threads": workers},
        "cpu_baseline": {"value": value, "unit": "elements/s", "cores": workers, "kind": "port", "sample": sample,
                         "note": "zig-ntt has no parallel path: the fork-join over each stage's butterflies is a "
                                 "harness construction; single_thread is the reference's own serial loop",
                         "single_thread": cpu_single_thread_sample()},
        "e2e": {"value": value, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --- the GPU arm -------------------------------------------------------------------------

TUNE_FILE = os.path.join(ROOT, "zig-algebra_b200", "tune", "b200.json")


def load_tuning(z):
    """The persisted autotuner table for this GPU; tunes and saves a fresh one
    (under ~/.cache/zntt) when the committed table has no entries for it."""
    try:
        z.tune_load(TUNE_FILE)
        return TUNE_FILE
    except z.ZnttError:
        path = os.path.join(os.path.expanduser("~"), ".cache", "zntt", "tune.json")
        os.makedirs(os.path.dirname(path), exist_ok=True)
        for F in z.FIELDS:
            z.autotune(F, 10, 24)
        z.tune_save(path)
        return path


def run_zntt(args, rank, world, local):
    import torch
    z = load_package()
    torch.cuda.set_device(local)
    z.init(local)
    tuning = load_tuning(z)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = dist
    F = z.BN254_FR
    log_n = args.log_n
    n = 1 << log_n
    # A dedicated stream: the library runs on it and the CUDA events see it.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream

    x = torch.empty(n * 4, dtype=torch.int64, device="cuda")
    y = torch.empty_like(x)
    z.random_elements(F, args.seed + rank, x.data_ptr(), n, stream=sptr)
    root = z.primitiveRootOfUnity(F, log_n)
    tw = z.DeviceTwiddles(F, log_n, root)

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    # Warm-up, then exactly K timed steps bracketed by barrier + synchronize.
    for _ in range(args.warmup):
        z.ntt_device(tw, x.data_ptr(), y.data_ptr(), z.FORWARD, stream=sptr)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        z.ntt_device(tw, x.data_ptr(), y.data_ptr(), z.FORWARD, stream=sptr)
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    ms_max = max_over_ranks(e0.elapsed_time(e1), pg, "cuda")
    ms_step = ms_max / args.steps
    value = aggregate_rate(n * args.steps, world, ms_max * 1e-3)

    # e2e through the public host-buffer API: every step uploads its input from
    # pinned host memory, transforms, and downloads its result.
    # (a) zntt_ntt_host_many: the steps' copies overlap their neighbours' transforms;
    # (b) one synchronous zntt_ntt_with_twiddles call per step, for reference.
    hbufs = [torch.empty(n * 4, dtype=torch.int64, pin_memory=True) for _ in range(3)]
    for hb in hbufs:
        hb.copy_(x.cpu())
    e2e_steps = max(8, args.steps)  # enough vectors that the pipeline's fill and drain are a small share
    ptrs = [hbufs[i % 3].data_ptr() for i in range(e2e_steps)]
    z.ntt_host_many(tw, ptrs[:3], z.FORWARD)  # warm-up (buffers, streams)
    for hb in hbufs:
        hb.copy_(x.cpu())
    barrier()
    t0 = time.perf_counter()
    z.ntt_host_many(tw, ptrs, z.FORWARD)
    e2e_s = max_over_ranks(time.perf_counter() - t0, pg, "cuda")
    e2e_value = aggregate_rate(n * e2e_steps, world, e2e_s)
    pcie = measure_pcie(torch, hbufs[1], hbufs[2], y, n, e2e_value / world)
    # correctness of the pipelined path: a fresh input through it equals the device result
    hbufs[0].copy_(x.cpu())
    z.ntt_host_many(tw, [hbufs[0].data_ptr()], z.FORWARD)
    ok = bool(torch.equal(hbufs[0].cuda(), y))
    host = hbufs[1].numpy().view("uint64").reshape(n, 4)
    orig = x.cpu().numpy().view("uint64").reshape(n, 4).copy()
    htw = z.precomputeTwiddles(F, log_n, root)
    host[:] = orig
    z.nttWithTwiddles(F, host, log_n, htw)
    single = []
    for _ in range(3):
        host[:] = orig
        t1 = time.perf_counter()
        z.nttWithTwiddles(F, host, log_n, htw)
        single.append(time.perf_counter() - t1)
    e2e_single = n / min(single)
    z.freeTwiddles(F, htw)

    # Roofline: the pass kernel is the only kernel in the timed region.
    imad = z.probe_imad()
    peak_modmul = imad / IMAD_PER_MODMUL
    modmuls = n / 2 * log_n
    achieved = modmuls / (ms_step * 1e-3)
    peaks, peaks_kind = measured_peaks()
    alg_bytes = 2 * n * 32
    passes = __import__("math").ceil(log_n / 10) if log_n > 11 else 1
    traffic = read_traffic(log_n)
    tw.close()
    extra = {}
    # The configurations beside the headline run once, in a single-GPU run: they describe the
    # library, not the scaling, and under torchrun the other ranks would wait for them at the
    # closing barrier for longer than the process group's timeout.
    if not args.headline_only and world == 1:
        with torch.cuda.stream(stream):
            extra["sizes"] = run_size_sweep(z, torch, stream, steps=10, warmup=3, peak_modmul=peak_modmul)
            extra["batched"] = run_batched_config(z, torch, stream, steps=20, warmup=3)
            extra["coset_lde"] = run_lde_config(z, torch, stream, steps=5, warmup=2)
            extra["poly_mul"] = run_poly_config(z, torch, stream, steps=5, warmup=2,
                                                cpu_sample=not args.no_cpu_baseline)
            extra["small_fields"] = run_small_config(z, torch, stream, steps=20, warmup=3,
                                                     cpu_sample=not args.no_cpu_baseline)
            extra["fri_fold"] = run_fri_config(z, torch, stream, steps=20, warmup=3,
                                               cpu_sample=not args.no_cpu_baseline)
        if not args.no_serve:
            extra["serve"] = serve_trace(z, torch, args.serve_requests, args.seed)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": metric_name(log_n), "value": value, "unit": "elements/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u256-mod-r (BN254-Fr, 8x32-bit Montgomery)",
        "data": "synthetic: seeded ChaCha20 randomFieldElement draws generated on the device",
        "config": {"workload": f"bn254_fr_ntt_forward_2^{log_n}", "log_n": log_n, "field": "bn254_fr",
                   "direction": "forward", "twiddles": "precomputed, device-resident",
                   "l2": l2_note(n), "passes": passes,
                   "parallelism": f"replicas x{world} (independent vectors, no collective)",
                   "tuning": os.path.relpath(tuning, ROOT) if tuning.startswith(ROOT) else tuning},
        "e2e": {"value": e2e_value, "unit": "elements/s", "h2d_bytes_per_step": n * 32, "d2h_bytes_per_step": n * 32,
                "steps": e2e_steps, "api": "zntt_ntt_host_many (pinned host vectors, copies overlapped across steps)",
                "matches_device_result": ok,
                "single_call_value": e2e_single, "single_call_api": "zntt_ntt_with_twiddles, one synchronous call",
                "pcie": pcie},
        "gpu_launches": args.steps * passes,
        "roofline": {"bound": "imad", "achieved": achieved, "peak": peak_modmul, "unit": "modmul/s",
                     "frac": achieved / peak_modmul, "traffic": traffic,
                     "peak_source": f"measured live: dependent mad.lo.u32 probe {imad:.4g} IMAD/s / "
                                    f"{IMAD_PER_MODMUL} IMAD slots per 8x32-bit CIOS modmul",
                     "hbm": {"achieved": alg_bytes / (ms_step * 1e-3) / 1e9, "peak": peaks["hbm_gbs"],
                             "unit": "GB/s", "frac": alg_bytes / (ms_step * 1e-3) / 1e9 / peaks["hbm_gbs"],
                             "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peaks_kind})"}},
        "clocks": clk,
    }
    if world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline_sample(orig, log_n)
        except Exception as e:  # noqa: BLE001 -- report, never fail the GPU line
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    # the detailed configuration keys, then a short summary of every configuration last, so
    # that a reader of the line's end sees all of them
    line.update(extra)
    if extra:
        line["summary"] = summarize(line)
    print(json.dumps(line), flush=True)


class TableCache:
    """Device twiddle tables per log n for one field."""

    def __init__(self, z, F):
        self.z, self.F, self.t = z, F, {}

    def __call__(self, log_n):
        if log_n not in self.t:
            self.t[log_n] = self.z.DeviceTwiddles(self.F, log_n, self.z.primitiveRootOfUnity(self.F, log_n))
        return self.t[log_n]

    def close(self):
        for t in self.t.values():
            t.close()


def measure_pcie(torch, h_in, h_out, d_src, n, e2e_per_gpu):
    """Pinned host <-> device copy bandwidth of one step's vectors (n x 32 bytes), alone and with
    both directions at once on two streams: the bound that the e2e path, which moves one
    vector each way per step, cannot beat on this GPU.  Returns the GB/s figures, the duplex
    bound in elements/s per GPU and the e2e fraction of it."""
    d_dst = torch.empty_like(d_src)
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    nbytes = n * 32

    def timed(copy_in, copy_out, reps=4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for st in (s_in, s_out):
            st.wait_event(e0)
        for _ in range(reps):
            if copy_in:
                with torch.cuda.stream(s_in):
                    d_dst.copy_(h_in, non_blocking=True)
            if copy_out:
                with torch.cuda.stream(s_out):
                    h_out.copy_(d_src, non_blocking=True)
        for st in (s_in, s_out):
            torch.cuda.current_stream().wait_stream(st)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3 / reps

    timed(True, True, 1)  # warm-up
    # best of three runs each: the link is shared with nothing else here, so the fastest run
    # is the closest to its capacity
    t_in = min(timed(True, False) for _ in range(3))
    t_out = min(timed(False, True) for _ in range(3))
    t_both = min(timed(True, True) for _ in range(3))
    del d_dst
    bound = n / t_both
    return {"h2d_gbs": nbytes / t_in / 1e9, "d2h_gbs": nbytes / t_out / 1e9,
            "duplex_gbs_each_way": nbytes / t_both / 1e9, "bound_elements_per_s": bound,
            "e2e_frac_of_bound": e2e_per_gpu / bound,
            "note": "torch copies of one n x 32-byte vector each way, pinned host memory, CUDA events"}


def time_region(torch, stream, fn, steps):
    """CUDA-event time of `steps` calls of fn() on `stream`, in ms."""
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def run_size_sweep(z, torch, stream, steps, warmup, peak_modmul, seed=66):
    """The single-transform configuration across sizes and directions: BN254-Fr 2^20, 2^22 and
    2^24, forward and inverse (nttWithTwiddles / inttWithTwiddles, libs/ntt/src/root.zig:148-212),
    and BLS12-381-Fr 2^24, with the tables resident.  Each entry: ms per transform, elements/s,
    the modmul rate ((n/2) log n products, plus n for the inverse's 1/n) over the live
    multiply-pipe peak, and the algorithmic HBM rate (the vector read and written once,
    2 n 32 bytes) over the measured copy bandwidth."""
    sptr = stream.cuda_stream
    peaks, _ = measured_peaks()
    hbm_peak = float(peaks["hbm_gbs"])
    out = {}
    for F, sizes in ((z.BN254_FR, (20, 22, 24)), (z.BLS12_381_FR, (24,))):
        x = torch.empty((1 << max(sizes)) * 4, dtype=torch.int64, device="cuda")
        y = torch.empty_like(x)
        z.random_elements(F, seed, x.data_ptr(), 1 << max(sizes), stream=sptr)
        for L in sizes:
            n = 1 << L
            with z.DeviceTwiddles(F, L, z.primitiveRootOfUnity(F, L)) as tw:
                for mode, name in ((z.FORWARD, "forward"), (z.INVERSE, "inverse")):
                    run = lambda: z.ntt_device(tw, x.data_ptr(), y.data_ptr(), mode, stream=sptr)  # noqa: E731
                    for _ in range(warmup):
                        run()
                    ms = time_region(torch, stream, run, steps) / steps
                    modmuls = n // 2 * L + (n if mode == z.INVERSE else 0)
                    hbm_gbs = 2 * n * 32 / (ms * 1e-3) / 1e9
                    out[f"{F.name} 2^{L} {name}"] = {
                        "ms": ms, "elements_per_s": n / (ms * 1e-3), "modmul_per_s": modmuls / (ms * 1e-3),
                        "frac": modmuls / (ms * 1e-3) / peak_modmul, "hbm_gbs": hbm_gbs,
                        "hbm_frac": hbm_gbs / hbm_peak}
        del x, y
    return out


def serve_trace(z, torch, requests, seed, keep_worst=False):
    """The serving configuration in the default run: the whole trace replayed with continuous
    batching and with serial plain launches (no capacity sweep; --workload serve adds it).
    Device memory cached by the configurations before it is handed back first, so that the
    server's buffers come from a device in the state a serving process starts in."""
    serving = importlib.import_module("zig_algebra_b200.serving")
    F = z.BN254_FR
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    free0, total = torch.cuda.mem_get_info()
    trace = serving.make_trace(requests, rate=2000.0, seed=seed)
    work = serving.Workload(z, torch, F, trace)
    try:
        batched = serving.replay(z, torch, F, trace, work, hbm_budget=120 << 30, serial=False)
        serial = serving.replay(z, torch, F, trace, work, hbm_budget=120 << 30, serial=True)
    finally:
        work.close()
    if not keep_worst:
        for r in (batched, serial):
            r.pop("worst", None)
    return {"workload": f"{requests} BN254-Fr requests, Poisson 2000/s, log n in 10..22 geometric(0.35), "
                        "70/20/10 fwd/inv/LDE x4, 120 GB budget, every request its own input",
            "device_free_gb_at_start": free0 / 1e9,
            "continuous_batching": batched, "serial_plain": serial,
            "p99_speedup_vs_serial": serial["p99_ms"] / batched["p99_ms"],
            "p50_speedup_vs_serial": serial["p50_ms"] / batched["p50_ms"]}


def _r(v, digits=4):
    return None if v is None else float(f"{v:.{digits}g}")


def summarize(line):
    """A short digest of every configuration in the line, for readers of its end."""
    out = {"headline": {"ms": _r(line["ms_per_step"]), "frac": _r(line["roofline"]["frac"], 3),
                        "e2e_elements_per_s": _r(line["e2e"]["value"]),
                        "e2e_frac_of_pcie_bound": _r(line["e2e"]["pcie"]["e2e_frac_of_bound"], 3)}}
    if "sizes" in line:
        out["sizes_ms_frac"] = {k: [_r(v["ms"]), _r(v["frac"], 3)] for k, v in line["sizes"].items()}
    if "batched" in line:
        b = line["batched"]
        out["batched"] = {"ms": _r(b["ms_per_batch"]), "plain_ms": _r(b["plain_ms_per_batch"]),
                          "speedup_vs_plain": _r(b["speedup_vs_plain"], 3), "bit_exact": b["bit_exact_vs_plain"]}
    if "coset_lde" in line:
        c = line["coset_lde"]
        out["coset_lde"] = {"ms": _r(c["ms_per_batch"]), "plain_ms": _r(c["plain_ms_per_batch"]),
                            "speedup_vs_plain": _r(c["speedup_vs_plain"], 3), "bit_exact": c["bit_exact_vs_plain"]}
    if "serve" in line:
        sv = line["serve"]
        cb, sp = sv["continuous_batching"], sv["serial_plain"]
        out["serve"] = {"p50_ms": _r(cb["p50_ms"]), "p99_ms": _r(cb["p99_ms"]),
                        "req_per_s": _r(cb["throughput_req_s"]), "serial_p50_ms": _r(sp["p50_ms"]),
                        "serial_p99_ms": _r(sp["p99_ms"]), "mismatches": cb["mismatches"] + sp["mismatches"],
                        "failures": cb["failures"] + sp["failures"]}
    if "poly_mul" in line:
        out["poly_mul_2^23_ms"] = _r(line["poly_mul"]["ms"])
    if "small_fields" in line:
        out["small_2^24_ms"] = {k: _r(v["ms"]) for k, v in line["small_fields"]["fields"].items()}
    return out


def run_batched_config(z, torch, stream, steps, warmup, seed=33):
    """512 BN254-Fr transforms of 2^10..2^16 (log size uniform) plus 8 of 2^20,
    directions 50/50 by seed: one persistent launch (CUDA graph) against one
    plain launch sequence per polynomial; both must agree bit for bit."""
    import numpy as np
    F = z.BN254_FR
    rng = np.random.default_rng(seed)
    logs = [int(v) for v in rng.integers(10, 17, 512)] + [20] * 8
    modes = [z.INVERSE if v < 0.5 else z.FORWARD for v in rng.random(len(logs))]
    tabs = TableCache(z, F)
    sptr = stream.cuda_stream
    xs, ys, ps, jobs = [], [], [], []
    # All inputs are consecutive slices of one seeded stream (one generator call).
    total = sum(1 << L for L in logs)
    pool = torch.empty(total * 4, dtype=torch.int64, device="cuda")
    z.random_elements(F, seed, pool.data_ptr(), total, stream=sptr)
    off = 0
    for i, (L, m) in enumerate(zip(logs, modes)):
        x = pool[off * 4:(off + (1 << L)) * 4]
        off += 1 << L
        y, pl = torch.empty_like(x), torch.empty_like(x)
        xs.append(x); ys.append(y); ps.append(pl)
        jobs.append({"kind": z.JOB_NTT, "tw": tabs(L), "mode": m, "src": x.data_ptr(), "dst": y.data_ptr()})
    elements = sum(1 << L for L in logs)
    butterflies = sum((1 << L) // 2 * L for L in logs)

    def plain():
        for L, m, x, pl in zip(logs, modes, xs, ps):
            z.ntt_device(tabs(L), x.data_ptr(), pl.data_ptr(), m, stream=sptr)

    with z.Batch(F, jobs) as b:
        info = b.info()
        run = lambda: b.run(stream=sptr, graph=True)  # noqa: E731
        for _ in range(warmup):
            run()
            plain()
        ms_b = time_region(torch, stream, run, steps)
        ms_p = time_region(torch, stream, plain, steps)
        b.status()
    exact = all(torch.equal(y, pl) for y, pl in zip(ys, ps))
    tabs.close()
    return {
        "workload": "512 x 2^U{10..16} + 8 x 2^20 BN254-Fr, fwd/inv 50/50, one persistent launch (CUDA graph)",
        "elements": elements, "jobs": len(logs), "items": info["items"], "grid": info["grid"],
        "shape": info["shape"], "ms_per_batch": ms_b / steps, "value": elements * steps / (ms_b * 1e-3),
        "plain_ms_per_batch": ms_p / steps, "plain_value": elements * steps / (ms_p * 1e-3),
        "speedup_vs_plain": ms_p / ms_b, "modmul_per_s": butterflies * steps / (ms_b * 1e-3),
        "unit": "elements/s", "bit_exact_vs_plain": exact,
    }


def run_lde_config(z, torch, stream, steps, warmup, seed=44, count=64):
    """64 BLS12-381-Fr coset extensions 2^18 -> 2^20 (inverse, zero-pad, g^i with
    g = 5, forward): one persistent launch against plain per-polynomial passes."""
    F = z.BLS12_381_FR
    shift = z.to_montgomery(F, 5)
    tabs = TableCache(z, F)
    sptr = stream.cuda_stream
    evs, outs, pls, jobs = [], [], [], []
    pool = torch.empty(count * (1 << 18) * 4, dtype=torch.int64, device="cuda")
    z.random_elements(F, seed, pool.data_ptr(), count << 18, stream=sptr)
    for i in range(count):
        ev = pool[i * (1 << 18) * 4:(i + 1) * (1 << 18) * 4]
        out = torch.empty((1 << 20) * 4, dtype=torch.int64, device="cuda")
        pl = torch.empty_like(out)
        evs.append(ev); outs.append(out); pls.append(pl)
        jobs.append({"kind": z.JOB_COSET_LDE, "tw": tabs(20), "tw_in": tabs(18), "shift": shift,
                     "src": ev.data_ptr(), "dst": out.data_ptr()})

    def plain():
        for ev, pl in zip(evs, pls):
            z.coset_lde_device(tabs(18), tabs(20), shift, ev.data_ptr(), pl.data_ptr(), stream=sptr)

    with z.Batch(F, jobs) as b:
        run = lambda: b.run(stream=sptr, graph=True)  # noqa: E731
        for _ in range(warmup):
            run()
            plain()
        ms_b = time_region(torch, stream, run, steps)
        ms_p = time_region(torch, stream, plain, steps)
        b.status()
    exact = all(torch.equal(o, p) for o, p in zip(outs, pls))
    tabs.close()
    modmuls = count * ((1 << 17) * 18 + (1 << 18) + (1 << 19) * 20)
    return {
        "workload": f"{count} x coset LDE 2^18 -> 2^20 BLS12-381-Fr (g = 5), one persistent launch (CUDA graph)",
        "ms_per_batch": ms_b / steps, "value": count * (1 << 20) * steps / (ms_b * 1e-3), "unit": "output elements/s",
        "plain_ms_per_batch": ms_p / steps, "speedup_vs_plain": ms_p / ms_b,
        "modmul_per_s": modmuls * steps / (ms_b * 1e-3), "bit_exact_vs_plain": exact,
    }


def run_poly_config(z, torch, stream, steps, warmup, seed=55, cpu_sample=True):
    """Polynomial.mul (libs/poly/src/poly.zig:197-212) on the device: one BN254-Fr product of
    two 2^23-coefficient polynomials (three 2^24-point transforms, the pointwise product fused
    into the second), and 64 products of two 2^14-coefficient polynomials in one persistent
    launch against plain per-product launches.  The CPU figure is the reference's schoolbook
    loop (the oracle port) on a bounded sample, extrapolated by its O(n^2) count."""
    F = z.BN254_FR
    sptr = stream.cuda_stream
    tabs = TableCache(z, F)
    n = 1 << 23
    a = torch.empty(n * 4, dtype=torch.int64, device="cuda")
    b = torch.empty_like(a)
    z.random_elements(F, seed, a.data_ptr(), n, stream=sptr)
    z.random_elements(F, seed + 1, b.data_ptr(), n, stream=sptr)
    out = torch.empty((2 * n - 1) * 4, dtype=torch.int64, device="cuda")
    one = lambda: z.poly_mul_device(tabs(24), a.data_ptr(), n, b.data_ptr(), n, out.data_ptr(), stream=sptr)  # noqa: E731
    for _ in range(warmup):
        one()
    ms_one = time_region(torch, stream, one, steps) / steps
    N = 1 << 24
    modmuls = 3 * (N // 2) * 24 + 2 * N  # three transforms, the pointwise product, n^-1

    m, count = 1 << 14, 64
    pa = torch.empty(count * m * 4, dtype=torch.int64, device="cuda")
    pb = torch.empty_like(pa)
    z.random_elements(F, seed + 2, pa.data_ptr(), count * m, stream=sptr)
    z.random_elements(F, seed + 3, pb.data_ptr(), count * m, stream=sptr)
    outs = [torch.empty((2 * m - 1) * 4, dtype=torch.int64, device="cuda") for _ in range(count)]
    pls = [torch.empty_like(o) for o in outs]
    ptr = lambda t, i: t.data_ptr() + i * m * 32  # noqa: E731
    jobs = [{"kind": z.JOB_POLY_MUL, "tw": tabs(15), "src": ptr(pa, i), "len": m, "src2": ptr(pb, i), "len2": m,
             "dst": outs[i].data_ptr()} for i in range(count)]

    def plain():
        for i in range(count):
            z.poly_mul_device(tabs(15), ptr(pa, i), m, ptr(pb, i), m, pls[i].data_ptr(), stream=sptr)

    with z.Batch(F, jobs) as bt:
        run = lambda: bt.run(stream=sptr, graph=True)  # noqa: E731
        for _ in range(warmup):
            run()
            plain()
        ms_b = time_region(torch, stream, run, steps) / steps
        ms_p = time_region(torch, stream, plain, steps) / steps
        bt.status()
    exact = all(torch.equal(o, q) for o, q in zip(outs, pls))
    tabs.close()
    r = {
        "workload": "BN254-Fr product of two 2^23-coefficient polynomials (three 2^24-point transforms)",
        "ms": ms_one, "value": (2 * n - 1) / (ms_one * 1e-3), "unit": "product coefficients/s",
        "modmul_per_s": modmuls / (ms_one * 1e-3),
        "batched": {"workload": "64 products of two 2^14-coefficient BN254-Fr polynomials (2^15 points), one "
                                "persistent launch (CUDA graph)",
                    "ms_per_batch": ms_b, "plain_ms_per_batch": ms_p, "speedup_vs_plain": ms_p / ms_b,
                    "bit_exact_vs_plain": exact},
    }
    if cpu_sample:
        r["cpu_schoolbook"] = cpu_schoolbook_sample(n)
    return r


def cpu_schoolbook_sample(n_full, log_sample=12):
    """Polynomial.mul's double loop (the oracle port, all host cores) on two 2^log_sample-
    coefficient polynomials; its product rate extrapolates the full size's n^2 products."""
    workers = min(os.cpu_count() or 1, 64)
    O, lib = cpu_oracle(native=True)
    k = 1 << log_sample
    a = O.random_elements(O.BN254_FR, 1, k)
    b = O.random_elements(O.BN254_FR, 2, k)
    out = O.elems(2 * k - 1)
    deg = ctypes.c_int64(0)
    best = None
    for _ in range(3):
        t0 = time.perf_counter()
        st = lib.zo_poly_mul(O.BN254_FR, O._p(a), k, O._p(b), k, 2 * k - 2, O._p(out), ctypes.byref(deg), workers)
        dt = time.perf_counter() - t0
        assert st == 0
        best = dt if best is None else min(best, dt)
    rate = k * k / best
    return {"sample": f"2^{log_sample} x 2^{log_sample} coefficients, schoolbook on {workers} threads (best of 3)",
            "products_per_s": rate, "cores": workers, "kind": "port",
            "extrapolated_ms_full": n_full * n_full / rate * 1e3}


def run_small_config(z, torch, stream, steps, warmup, log_n=24, cpu_sample=True):
    """Goldilocks and BabyBear (zig-field's SmallField, 8-byte canonical elements) forward
    transforms of 2^log_n with the device-resident API.  These are memory- and issue-bound,
    not multiply-bound: the roofline is HBM bytes moved by the passes against the measured
    copy bandwidth."""
    import numpy as np
    sptr = stream.cuda_stream
    n = 1 << log_n
    peaks, hbm_src = measured_peaks()
    hbm_peak = float(peaks["hbm_gbs"])
    out = {"workload": f"forward transform of 2^{log_n} canonical u64 elements per field", "fields": {}}
    for F in (z.GOLDILOCKS, z.BABYBEAR):
        xs = np.random.default_rng(77).integers(0, F.modulus, n, dtype=np.uint64)
        x = torch.from_numpy(xs.view(np.int64)).cuda()
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        with z.DeviceTwiddles(F, log_n, z.primitiveRootOfUnity(F, log_n)) as tw:
            run = lambda: z.ntt_device(tw, x.data_ptr(), y.data_ptr(), z.FORWARD, stream=sptr)  # noqa: E731
            for _ in range(warmup):
                run()
            ms = time_region(torch, stream, run, steps) / steps
        passes = 1 if log_n <= 12 else -(-log_n // 10)
        moved = passes * 2 * 8 * n
        r = {"ms": ms, "value": n / (ms * 1e-3), "unit": "elements/s", "passes": passes,
             "hbm": {"achieved": moved / (ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                     "frac": moved / (ms * 1e-3) / 1e9 / hbm_peak, "bytes_per_transform": moved,
                     "peak_source": hbm_src}}
        # Coset extension 2^(log_n - 2) -> 2^log_n (blowup 4, shift 7): inverse transform,
        # coset scaling, zero tail, forward transform.
        lin = log_n - 2
        with z.DeviceTwiddles(F, lin, z.primitiveRootOfUnity(F, lin)) as ti, \
                z.DeviceTwiddles(F, log_n, z.primitiveRootOfUnity(F, log_n)) as to:
            shift = np.array([7, 0, 0, 0], dtype=np.uint64)
            lde = lambda: z.coset_lde_device(ti, to, shift, x.data_ptr(), y.data_ptr(), stream=sptr)  # noqa: E731
            for _ in range(warmup):
                lde()
            r["lde_ms"] = time_region(torch, stream, lde, steps) / steps
        r["lde_note"] = (f"coset extension 2^{lin} -> 2^{log_n} (zntt_coset_lde_device; the call waits for "
                         f"its stream)")
        # A STARK trace commitment: 64 columns of 2^18 rows extended to 2^20 (zntt_coset_lde_columns),
        # then the 2^20 rows committed (zntt_merkle_commit_rows).
        m, t_in, t_out = 64, 18, 20
        tcols = [torch.from_numpy(np.random.default_rng(300 + k).integers(0, F.modulus, 1 << t_in, dtype=np.uint64)
                                  .view(np.int64)).cuda() for k in range(m)]
        touts = [torch.empty(1 << t_out, dtype=torch.int64, device="cuda") for _ in range(m)]
        tnodes = torch.empty((2 << t_out) * 4, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        with z.DeviceTwiddles(F, t_in, z.primitiveRootOfUnity(F, t_in)) as ti, \
                z.DeviceTwiddles(F, t_out, z.primitiveRootOfUnity(F, t_out)) as to:
            shift = np.array([7, 0, 0, 0], dtype=np.uint64)
            ins, outs_p = [c_.data_ptr() for c_ in tcols], [o.data_ptr() for o in touts]
            ext = lambda: z.coset_lde_columns(ti, to, shift, ins, outs_p, stream=sptr)  # noqa: E731
            com = lambda: z.merkle_commit_rows(F, outs_p, t_out, tnodes.data_ptr(), stream=sptr)  # noqa: E731
            for _ in range(2):
                ext()
                com()
            k_t = max(steps // 4, 2)
            r["trace"] = {"columns": m, "rows_in": 1 << t_in, "rows_out": 1 << t_out,
                          "extend_ms": time_region(torch, stream, ext, k_t) / k_t,
                          "commit_ms": time_region(torch, stream, com, k_t) / k_t,
                          "note": "a STARK trace commitment: zntt_coset_lde_columns then zntt_merkle_commit_rows"}
        del tcols, touts, tnodes
        if cpu_sample:
            r["cpu_baseline"] = cpu_small_sample(F, xs, log_n)
        out["fields"][F.name] = r
        del x, y
    return out


def cpu_fri_sample(fid_name, log_sample=20):
    """The oracle port's fold (the reference's literal loop: an inverse per element) and layer
    commitment (hashPair + BLAKE3 Merkle tree) on one 2^log_sample layer, all host cores."""
    workers = min(os.cpu_count() or 1, 64)
    O, _ = cpu_oracle(native=True)
    fid = {"bn254_fr": O.BN254_FR, "goldilocks": O.GOLDILOCKS, "babybear": O.BABYBEAR}[fid_name]
    n = 1 << log_sample
    layer = O.random_elements(fid, 5, n)
    alpha = O.random_elements(fid, 6, 1)[0]
    t0 = time.perf_counter()
    O.fri_fold(fid, layer, log_sample, alpha, workers=workers)
    t_fold = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.fri_commit_layer(fid, layer, log_sample, workers=workers)
    t_commit = time.perf_counter() - t0
    return {"sample": f"one 2^{log_sample} layer: fold and commitment, oracle port on {workers} threads",
            "fold_value": (n // 2) / t_fold, "fold_unit": "output elements/s",
            "commit_hashes_per_s": (n - 1) / t_commit, "cores": workers, "kind": "port"}


def run_fri_config(z, torch, stream, steps, warmup, log_n=24, cpu_sample=True):
    """FRI fold rounds (libs/fri/src/root.zig:396-403) on resident evaluations: one fold of a
    2^log_n layer, and the whole chain 2^log_n -> 2^10 sharing one table, for BN254-Fr and
    Goldilocks.  A fold reads the layer and the 1/(2x) table and writes half a layer."""
    import numpy as np
    sptr = stream.cuda_stream
    peaks, hbm_src = measured_peaks()
    hbm_peak = float(peaks["hbm_gbs"])
    b3_peak = z.probe_blake3()
    out = {"workload": f"FRI fold of a 2^{log_n}-evaluation layer, the chain 2^{log_n} -> 2^10, and the "
                       f"layer's BLAKE3 Merkle commitment",
           "fields": {}}
    for F in (z.BN254_FR, z.GOLDILOCKS, z.BABYBEAR):
        ew = 8 * F.limbs  # bytes per element in device memory
        n = 1 << log_n
        layer = torch.empty(n * F.limbs, dtype=torch.int64, device="cuda")
        if F.limbs == 4:
            z.random_elements(F, 91, layer.data_ptr(), n, stream=sptr)
        else:
            xs = np.random.default_rng(91).integers(0, F.modulus, n, dtype=np.uint64)
            layer.copy_(torch.from_numpy(xs.view(np.int64)))
        bufs = [torch.empty((n >> (r + 1)) * F.limbs, dtype=torch.int64, device="cuda") for r in range(log_n - 10)]
        alpha = z.to_montgomery(F, 987654321) if F.limbs == 4 else np.array([987654321, 0, 0, 0], dtype=np.uint64)
        torch.cuda.synchronize()
        one = lambda: z.fri_fold(F, layer.data_ptr(), log_n, alpha, bufs[0].data_ptr(), log_table=log_n,  # noqa: E731
                                 stream=sptr)

        def chain():
            src = layer
            for r, dst in enumerate(bufs):
                z.fri_fold(F, src.data_ptr(), log_n - r, alpha, dst.data_ptr(), log_table=log_n, stream=sptr)
                src = dst

        nodes = torch.empty(n * 4, dtype=torch.int64, device="cuda")  # 2^log_n digests of 32 bytes
        commit = lambda: z.fri_commit_layer(F, layer.data_ptr(), log_n, nodes.data_ptr(), stream=sptr)  # noqa: E731
        # proveOn's commit loop over the same buffers (a fixed alpha stands in for the caller's
        # transcript) and 64 query openings from the resident layers and trees.
        rounds = log_n - 10
        players = [layer.data_ptr()] + [b.data_ptr() for b in bufs]
        ptrees = [nodes] + [torch.empty((n >> r) * 4, dtype=torch.int64, device="cuda") for r in range(1, rounds)]
        ptree_ptrs = [t.data_ptr() for t in ptrees]
        positions = np.random.default_rng(7).integers(0, n, 64, dtype=np.uint64)
        prove = lambda: z.fri_commit_phase(F, log_n, 10, players, ptree_ptrs, lambda r, root: alpha,  # noqa: E731
                                           stream=sptr)
        # The openings through the C ABI into preallocated host buffers (the Python wrapper's
        # unpacking into per-query lists is not library time).
        import ctypes
        nb = z._num_bytes(F)  # toBytes length
        per_query = sum(log_n - r - 1 for r in range(rounds))
        q_vals = ctypes.create_string_buffer(64 * rounds * 2 * nb)
        q_paths = ctypes.create_string_buffer(64 * per_query * 32)
        q_layers = (ctypes.c_void_p * rounds)(*players[:rounds])
        q_trees = (ctypes.c_void_p * rounds)(*ptree_ptrs)
        q_pos = positions.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))

        def queries():
            z._check(z.lib().zntt_fri_query_extract(F.id, log_n, rounds, q_layers, q_trees, q_pos, 64, q_vals,
                                                    q_paths, sptr))
        for _ in range(warmup):
            one()
            chain()
            commit()
        ms_one = time_region(torch, stream, one, steps) / steps
        ms_chain = time_region(torch, stream, chain, steps) / steps
        ms_commit = time_region(torch, stream, commit, steps) / steps
        # Row commitment of 8 columns of 2^(log_n - 2) rows (MerkleTree.init over rows, a trace
        # commitment): ceil(8 * NB / 64) compressions per row plus the tree's rows - 1.
        rows_log, ncol = log_n - 2, 8
        rows = 1 << rows_log
        cols = [torch.empty(rows * F.limbs, dtype=torch.int64, device="cuda") for _ in range(ncol)]
        for c_i, col in enumerate(cols):
            if F.limbs == 4:
                z.random_elements(F, 200 + c_i, col.data_ptr(), rows, stream=sptr)
            else:
                col.copy_(torch.from_numpy(np.random.default_rng(200 + c_i).integers(
                    0, F.modulus, rows, dtype=np.uint64).view(np.int64)))
        rnodes = torch.empty((2 * rows) * 4, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        col_ptrs = [c_.data_ptr() for c_ in cols]
        rcommit = lambda: z.merkle_commit_rows(F, col_ptrs, rows_log, rnodes.data_ptr(), stream=sptr)  # noqa: E731
        for _ in range(warmup):
            rcommit()
        ms_rows = time_region(torch, stream, rcommit, steps) / steps
        rows_compressions = rows * -(-ncol * z._num_bytes(F) // 64) + rows - 1
        del cols, rnodes
        layer_copy = layer.clone()  # the commit phase folds into bufs; layer 0 is only read
        for _ in range(2):
            prove()
            queries()
        # the loop makes one host round trip per round (root copy, Python callback): take the best
        # of three timed regions so a host-side pause does not stand for the library
        k_prove = max(steps // 4, 2)
        ms_prove = min(time_region(torch, stream, prove, k_prove) / k_prove for _ in range(3))
        ms_queries = time_region(torch, stream, queries, steps) / steps
        assert torch.equal(layer, layer_copy)
        del layer_copy, ptrees
        moved = (n + n // 2 + n // 2) * ew  # layer read, table read, half layer written
        out["fields"][F.name] = {
            "fold_ms": ms_one, "fold_value": (n // 2) / (ms_one * 1e-3), "unit": "output elements/s",
            "hbm": {"achieved": moved / (ms_one * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                    "frac": moved / (ms_one * 1e-3) / 1e9 / hbm_peak, "peak_source": hbm_src},
            "chain_rounds": log_n - 10, "chain_ms": ms_chain,
            "commit_ms": ms_commit, "commit_hashes_per_s": (n - 1) / (ms_commit * 1e-3),
            "commit_roofline": {"bound": "alu", "achieved": (n - 1) / (ms_commit * 1e-3), "peak": b3_peak,
                                "unit": "compressions/s", "frac": (n - 1) / (ms_commit * 1e-3) / b3_peak,
                                "peak_source": "zntt_probe_blake3: chained compressions in registers"},
            "commit_note": "hashPair leaves + BLAKE3 Merkle tree, n - 1 single-block compressions; "
                           "the call copies the root to the host, inside the timed region",
            "prove_commit_ms": ms_prove, "prove_queries_ms": ms_queries,
            "cpu_baseline": cpu_fri_sample(F.name) if cpu_sample else None,
            "rows_commit": {"columns": ncol, "rows": rows, "ms": ms_rows, "compressions": rows_compressions,
                            "compressions_per_s": rows_compressions / (ms_rows * 1e-3),
                            "frac_of_probe": rows_compressions / (ms_rows * 1e-3) / b3_peak,
                            "note": "zntt_merkle_commit_rows: MerkleTree.init over the rows of the columns"},
            "prove_note": f"zntt_fri_commit_phase: {rounds} rounds of commit, root to the host, challenge "
                          f"callback, fold (2^{log_n} -> 2^10); zntt_fri_query_extract: 64 openings "
                          f"(pairs and Merkle paths of every round) to the host",
        }
        del layer, bufs, nodes
    return out


def cpu_small_sample(F, xs, log_n):
    """The oracle's nttWithTwiddles on all host cores for one full transform (Montgomery form
    inside the oracle; conversion excluded from the time)."""
    import numpy as np
    O, lib = cpu_oracle(native=True)
    fid = {"goldilocks": O.GOLDILOCKS, "babybear": O.BABYBEAR}[F.name]
    workers = min(os.cpu_count() or 1, 64)
    slots = O.elems(len(xs))
    slots[:, 0] = xs
    data = np.ascontiguousarray(O.to_mont(fid, slots)[:, 0])  # one u64 per element, Montgomery form
    st, root = O.primitive_root(fid, log_n)
    st, stages = O.precompute_twiddles(fid, log_n, root)
    dt = cpu_transform_seconds(O, lib, data, log_n, stages, workers, field=fid)
    return {"value": len(xs) / dt, "unit": "elements/s", "cores": workers, "kind": "port",
            "sample": f"one full 2^{log_n} forward transform, oracle nttWithTwiddles, fork-join over butterflies"}


def cpu_baseline_sample(host_data, log_n):
    """The oracle port on all host cores, on the same input, for one full transform."""
    workers = min(os.cpu_count() or 1, 64)
    O, lib, data, stages = cpu_reference_setup(log_n, 0, host_data)
    dt = cpu_transform_seconds(O, lib, data, log_n, stages, workers)
    reps = [dt]
    while sum(reps) < 30.0 and len(reps) < 7:
        data[:] = host_data
        reps.append(cpu_transform_seconds(O, lib, data, log_n, stages, workers))
    best = min(reps)
    return {"value": (1 << log_n) / best, "unit": "elements/s", "cores": workers, "kind": "port",
            "min_ms": 1e3 * best, "median_ms": 1e3 * statistics.median(reps),
            "sample": f"{len(reps)} full 2^{log_n} forward transforms (value: the fastest), oracle "
                      f"nttWithTwiddles, fork-join over butterflies per stage",
            "note": "zig-ntt has no parallel path: the fork-join over each stage's butterflies is a harness "
                    "construction; single_thread is the reference's own serial loop",
            "single_thread": cpu_single_thread_sample()}


def cpu_single_thread_sample(log_n=20, seed=7):
    """zig-ntt's serial nttWithTwiddles (the oracle port on one thread) on one 2^log_n
    transform, the size of the reference's own published figure (1113.9 ms at 2^20)."""
    O, lib, data, stages = cpu_reference_setup(log_n, seed)
    orig = data.copy()
    reps = []
    while len(reps) < 3 and sum(reps) < 6.0:
        data[:] = orig
        reps.append(cpu_transform_seconds(O, lib, data, log_n, stages, 1))
    best = min(reps)
    return {"value": (1 << log_n) / best, "unit": "elements/s", "cores": 1, "ms": round(best * 1e3, 1),
            "sample": f"best of {len(reps)} 2^{log_n} forward transforms, oracle nttWithTwiddles on 1 thread"}


def run_serve(args):
    """The serving trace: 20,000 BN254-Fr requests, Poisson arrivals at 2,000/s,
    log2 size truncated-geometric on {10..22} (p = 0.35), 70% forward / 20%
    inverse / 10% blowup-4 coset extensions, 120 GB HBM budget; continuous
    batching against serial plain execution, every output checked against the
    request computed alone; then a capacity sweep at higher arrival rates."""
    import torch
    z = load_package()
    torch.cuda.set_device(0)
    z.init(0)
    load_tuning(z)
    serving = importlib.import_module("zig_algebra_b200.serving")
    F = z.BN254_FR
    n = args.serve_requests
    main = serve_trace(z, torch, n, args.seed, keep_worst=True)
    # Capacity: the same request mix at higher arrival rates (shorter traces).
    sweep = []
    for rate in args.serve_sweep:
        tr = serving.make_trace(args.serve_sweep_requests, rate=rate, seed=args.seed + 1)
        wk = serving.Workload(z, torch, F, tr)
        try:
            rb = serving.replay(z, torch, F, tr, wk, hbm_budget=120 << 30, serial=False)
            rs = serving.replay(z, torch, F, tr, wk, hbm_budget=120 << 30, serial=True)
        finally:
            wk.close()
        pick = ("p50_ms", "p99_ms", "throughput_req_s", "mismatches", "failures", "batches", "max_batch_jobs")
        sweep.append({"rate_req_s": rate, "requests": len(tr),
                      "continuous_batching": {k: rb[k] for k in pick}, "serial_plain": {k: rs[k] for k in pick}})
    line = {
        "metric": "serve p50/p99 ms (BN254-Fr NTT/LDE trace)", "value": main["continuous_batching"]["p99_ms"],
        "unit": "ms (p99)", "higher_is_better": False, "n_gpus": 1,
        "data": "synthetic: seeded Poisson trace, seeded inputs (every request its own)",
        "config": {"workload": f"serve {n} requests, Poisson 2000/s, log n in 10..22 geometric(0.35), "
                               "70/20/10 fwd/inv/LDE x4, 120 GB budget"},
        "capacity_sweep": sweep,
    }
    line.update(main)
    print(json.dumps(line), flush=True)


def run_single_config(args):
    """One of the batched configurations alone (for profiling): its JSON line."""
    import torch
    z = load_package()
    torch.cuda.set_device(0)
    z.init(0)
    load_tuning(z)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    with torch.cuda.stream(stream):
        if args.workload == "batched":
            r = run_batched_config(z, torch, stream, steps=args.steps, warmup=args.warmup)
            metric = "batched BN254-Fr NTT elems/s (512 x 2^U{10..16} + 8 x 2^20)"
        elif args.workload == "small":
            r = run_small_config(z, torch, stream, steps=args.steps, warmup=args.warmup,
                                 cpu_sample=not args.no_cpu_baseline)
            r["value"] = r["fields"]["goldilocks"]["value"]
            r["unit"] = "elements/s"
            metric = "Goldilocks NTT elems/s at 2^24 (BabyBear beside it)"
        elif args.workload == "fri":
            r = run_fri_config(z, torch, stream, steps=args.steps, warmup=args.warmup,
                               cpu_sample=not args.no_cpu_baseline)
            r["value"] = r["fields"]["bn254_fr"]["fold_value"]
            r["unit"] = "output elements/s"
            metric = "BN254-Fr FRI fold output elems/s (2^24 -> 2^23; Goldilocks and BabyBear beside it)"
        elif args.workload == "poly":
            r = run_poly_config(z, torch, stream, steps=args.steps, warmup=args.warmup,
                                cpu_sample=not args.no_cpu_baseline)
            metric = "BN254-Fr polynomial product coefficients/s (2^23 x 2^23 coefficients)"
        else:
            r = run_lde_config(z, torch, stream, steps=args.steps, warmup=args.warmup, count=args.lde_jobs)
            metric = f"batched coset LDE output elems/s ({args.lde_jobs} x 2^18 -> 2^20, BLS12-381-Fr)"
    line = {"metric": metric, "value": r["value"], "unit": r["unit"], "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "data": "synthetic: seeded inputs",
            "config": {"workload": r["workload"]}, "detail": r}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="zntt", choices=["zntt", "reference"])
    ap.add_argument("--log-n", type=int, default=24)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the batched, coset-extension, polynomial-product, small-field and FRI lines")
    ap.add_argument("--workload", default="ntt", choices=["ntt", "serve", "batched", "lde", "poly", "small", "fri"])
    ap.add_argument("--no-serve", action="store_true", help="leave the serving trace out of the default run")
    ap.add_argument("--lde-jobs", type=int, default=64, help="extensions in the --workload lde batch (profiling)")
    ap.add_argument("--serve-requests", type=int, default=20000)
    ap.add_argument("--serve-sweep", type=float, nargs="*", default=[8000.0, 32000.0])
    ap.add_argument("--serve-sweep-requests", type=int, default=6000)
    args = ap.parse_args()
    rank, world, local = dist_env()
    if args.workload == "serve":
        if rank == 0:
            run_serve(args)
        return
    if args.workload in ("batched", "lde", "poly", "small", "fri"):
        if rank == 0:
            run_single_config(args)
        return
    if args.impl == "reference":
        run_reference(args, rank)
    else:
        run_zntt(args, rank, world, local)


if __name__ == "__main__":
    main()
