"""Host-side mirror of zig-ntt over the B200 library libzntt_cuda.so.

zig-ntt (libs/ntt/src/root.zig) is a Zig module whose functions take the field
type as a `comptime F` argument; here the field is a `Field` object and the
data is a numpy uint64 array of shape (n, 4) holding the reference's [4]u64
Montgomery limbs per element (C-contiguous, transformed in place).  Names,
argument meaning and error behaviour follow zig-ntt:

    bitReverse(F, data)                       root.zig:38-58
    ntt(F, data, log_n, root)                 root.zig:65-90
    intt(F, data, log_n, root)                root.zig:95-107
    precomputeTwiddles(F, log_n, root)        root.zig:112-134
    freeTwiddles(F, twiddles)                 root.zig:136-141
    nttWithTwiddles(F, data, log_n, tw)       root.zig:148-175
    inttWithTwiddles(F, data, log_n, tw)      root.zig:180-212

Each zig-ntt error is an exception class of the same name.  Every transform
runs on the GPU; if the CUDA library or a device is missing the calls raise,
there is no CPU fallback.  The device-resident API (`DeviceTwiddles`,
`ntt_device`, `random_elements`) works on raw device pointers, e.g. from
`torch.Tensor.data_ptr()`.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("ZNTT_LIB") or os.path.join(HERE, "libzntt_cuda.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "zntt.h")


# --- errors (zig-ntt's error set plus device failures) ------------------------

class ZnttError(Exception):
    code = -1


class LogTooLarge(ZnttError):
    code = 1


class LengthMismatch(ZnttError):
    code = 2


class InvalidTwiddles(ZnttError):
    code = 3


class InvalidLength(ZnttError):
    code = 4


class OutOfMemory(ZnttError):
    code = 5


class OrderTooLarge(ZnttError):
    code = 6


class UnsupportedField(ZnttError):
    code = 7


class DeviceError(ZnttError):
    code = 8


class Timeout(ZnttError):
    code = 9


class InvalidArgument(ZnttError):
    code = 10


class NotInitialized(ZnttError):
    code = 11


class Rejected(ZnttError):
    code = 12


class DegreeTooLarge(ZnttError):
    """error.DegreeTooLarge of libs/poly/src/poly.zig:77, 200."""
    code = 13


_ERRORS = {c.code: c for c in (LogTooLarge, LengthMismatch, InvalidTwiddles, InvalidLength, OutOfMemory,
                               OrderTooLarge, UnsupportedField, DeviceError, Timeout, InvalidArgument,
                               NotInitialized, Rejected, DegreeTooLarge)}


# --- fields ----------------------------------------------------------------------

class Field:
    """A scalar field served by the library (the `comptime F` of zig-ntt).  `limbs` is the
    element's width in u64 words: 4 Montgomery limbs for the 256-bit fields, 1 canonical
    value for zig-field's SmallField (Goldilocks, BabyBear)."""

    def __init__(self, fid: int, name: str, modulus: int, two_adicity: int, limbs: int = 4):
        self.id, self.name, self.modulus, self.two_adicity, self.limbs = fid, name, modulus, two_adicity, limbs

    def __repr__(self):
        return f"Field({self.name})"


BN254_FR = Field(0, "bn254_fr", 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001, 28)
BLS12_381_FR = Field(1, "bls12_381_fr", 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001, 32)
FIELDS = (BN254_FR, BLS12_381_FR)
GOLDILOCKS = Field(2, "goldilocks", 0xFFFFFFFF00000001, 32, limbs=1)
BABYBEAR = Field(3, "babybear", 0x78000001, 27, limbs=1)
SMALL_FIELDS = (GOLDILOCKS, BABYBEAR)

FORWARD = 0
INVERSE = 1


# --- library loading ------------------------------------------------------------------

class _Stage(ctypes.Structure):
    _fields_ = [("ptr", ctypes.POINTER(ctypes.c_uint64)), ("len", ctypes.c_size_t)]


_U64P = ctypes.POINTER(ctypes.c_uint64)
_lib = None

JOB_NTT = 0
BATCH_SPIN_LIMIT = 4194304  # ZNTT_BATCH_SPIN_LIMIT: sleep rounds a batch tile waits for its previous pass
JOB_COSET_LDE = 1
JOB_POLY_MUL = 2


class ServerConfig(ctypes.Structure):
    """zntt_server_config (include/zntt.h)."""
    _fields_ = [("field", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_size_t), ("slots", ctypes.c_int),
                ("max_batch_jobs", ctypes.c_int), ("max_items", ctypes.c_uint32), ("serial", ctypes.c_int),
                ("max_batch_bytes", ctypes.c_size_t)]


class Request(ctypes.Structure):
    """zntt_request (include/zntt.h)."""
    _fields_ = [("kind", ctypes.c_int), ("mode", ctypes.c_int), ("log_n", ctypes.c_uint32),
                ("log_in", ctypes.c_uint32), ("h_in", ctypes.c_void_p), ("h_out", ctypes.c_void_p),
                ("shift", ctypes.c_uint64 * 4), ("user_tag", ctypes.c_uint64), ("arrival_ns", ctypes.c_uint64)]


class Completion(ctypes.Structure):
    """zntt_completion (include/zntt.h)."""
    _fields_ = [("user_tag", ctypes.c_uint64), ("status", ctypes.c_int), ("arrival_ns", ctypes.c_uint64),
                ("admit_ns", ctypes.c_uint64), ("done_ns", ctypes.c_uint64)]


class ServerStats(ctypes.Structure):
    """zntt_server_stats (include/zntt.h)."""
    _fields_ = [(k, ctypes.c_uint64) for k in ("submitted", "completed", "rejected", "batches", "max_batch_jobs",
                                               "max_inflight_jobs", "peak_bytes", "pending", "max_launch_ns",
                                               "max_batch_ns")]


# zntt_fri_challenge_fn: (user, round, root[32], alpha_out[4]) -> status.
FRI_CHALLENGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32,
                                    ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64))


class Job(ctypes.Structure):
    """zntt_job (include/zntt.h)."""
    _fields_ = [("kind", ctypes.c_int), ("mode", ctypes.c_int), ("tw", ctypes.c_void_p),
                ("tw_in", ctypes.c_void_p), ("d_src", ctypes.c_void_p), ("d_dst", ctypes.c_void_p),
                ("shift", ctypes.c_uint64 * 4), ("d_src2", ctypes.c_void_p), ("len", ctypes.c_uint64),
                ("len2", ctypes.c_uint64)]
_device = None


def lib():
    """The loaded CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run zig-algebra_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        sz, i, vp = ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p
        L.zntt_init.argtypes = [i]
        L.zntt_last_error.restype = ctypes.c_char_p
        L.zntt_field_info.argtypes = [i, _U64P, ctypes.POINTER(ctypes.c_uint32)]
        L.zntt_primitive_root.argtypes = [i, ctypes.c_uint32, _U64P]
        L.zntt_bit_reverse.argtypes = [_U64P, sz]
        L.zntt_bit_reverse_small.argtypes = [_U64P, sz]
        L.zntt_ntt.argtypes = [i, _U64P, sz, sz, _U64P]
        L.zntt_intt.argtypes = [i, _U64P, sz, sz, _U64P]
        L.zntt_precompute_twiddles.argtypes = [i, sz, _U64P, ctypes.POINTER(_U64P)]
        L.zntt_free_twiddles.argtypes = [i, ctypes.POINTER(_Stage), sz]
        L.zntt_free_twiddles.restype = None
        L.zntt_ntt_with_twiddles.argtypes = [i, _U64P, sz, sz, ctypes.POINTER(_Stage), sz]
        L.zntt_intt_with_twiddles.argtypes = [i, _U64P, sz, sz, ctypes.POINTER(_Stage), sz]
        L.zntt_twiddles_acquire.argtypes = [i, ctypes.c_uint32, _U64P, ctypes.POINTER(vp)]
        L.zntt_twiddles_release.argtypes = [vp]
        L.zntt_ntt_device.argtypes = [vp, vp, vp, vp, i, vp]
        L.zntt_ntt_device_columns.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_uint32, i, vp]
        L.zntt_random_elements.argtypes = [i, ctypes.c_char_p, vp, sz, vp]
        L.zntt_elementwise_device.argtypes = [i, i, vp, vp, vp, sz, vp]
        L.zntt_probe_imad.argtypes = [ctypes.POINTER(ctypes.c_double)]
        L.zntt_probe_modmul.argtypes = [i, ctypes.POINTER(ctypes.c_double)]
        L.zntt_probe_mul_wide.argtypes = [ctypes.POINTER(ctypes.c_double)]
        L.zntt_probe_blake3.argtypes = [ctypes.POINTER(ctypes.c_double)]
        L.zntt_ntt_device_inplace_noalloc.argtypes = [vp, vp, i, vp]
        L.zntt_batch_create.argtypes = [i, ctypes.POINTER(Job), sz, i, ctypes.POINTER(vp)]
        L.zntt_batch_run.argtypes = [vp, vp]
        L.zntt_batch_run_graph.argtypes = [vp, vp]
        L.zntt_batch_status.argtypes = [vp]
        L.zntt_batch_set_spin_limit.argtypes = [vp, ctypes.c_uint32]
        L.zntt_pool_stats.argtypes = [ctypes.POINTER(ctypes.c_uint64)] * 3
        L.zntt_batch_info.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                                      ctypes.POINTER(i), ctypes.POINTER(i)]
        L.zntt_batch_destroy.argtypes = [vp]
        L.zntt_coset_lde_device.argtypes = [vp, vp, _U64P, vp, vp, vp]
        L.zntt_coset_lde_columns.argtypes = [vp, vp, _U64P, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_uint32,
                                             vp]
        L.zntt_poly_mul_device.argtypes = [vp, vp, sz, vp, sz, vp, vp]
        L.zntt_fri_domain_fill.argtypes = [i, ctypes.c_uint32, vp, vp]
        L.zntt_fri_fold_device.argtypes = [i, vp, ctypes.c_uint32, _U64P, vp, ctypes.c_uint32, vp]
        L.zntt_merkle_commit_rows.argtypes = [i, ctypes.POINTER(vp), ctypes.c_uint32, ctypes.c_uint32, vp,
                                              ctypes.c_char_p, vp]
        L.zntt_merkle_open_rows.argtypes = [i, ctypes.POINTER(vp), ctypes.c_uint32, ctypes.c_uint32, vp, _U64P, sz,
                                            ctypes.c_char_p, ctypes.c_char_p, vp]
        L.zntt_fri_fold_commit.argtypes = [i, vp, ctypes.c_uint32, _U64P, vp, ctypes.c_uint32, vp, ctypes.c_char_p,
                                           vp]
        L.zntt_fri_commit_phase.argtypes = [i, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(vp),
                                            ctypes.POINTER(vp), ctypes.c_char_p, FRI_CHALLENGE_FN, vp, vp]
        L.zntt_fri_query_extract.argtypes = [i, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(vp),
                                             ctypes.POINTER(vp), _U64P, sz, ctypes.c_char_p, ctypes.c_char_p, vp]
        L.zntt_fri_commit_layer.argtypes = [i, vp, ctypes.c_uint32, vp, ctypes.c_char_p, vp]
        L.zntt_poly_mul.argtypes = [i, _U64P, sz, _U64P, sz, sz, _U64P, ctypes.POINTER(ctypes.c_int64)]
        L.zntt_autotune.argtypes = [i, ctypes.c_uint32, ctypes.c_uint32]
        L.zntt_tune_save.argtypes = [ctypes.c_char_p]
        L.zntt_tune_load.argtypes = [ctypes.c_char_p]
        L.zntt_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
        L.zntt_server_submit.argtypes = [vp, ctypes.POINTER(Request)]
        L.zntt_server_poll.argtypes = [vp, ctypes.POINTER(Completion), sz, ctypes.POINTER(sz), i]
        L.zntt_server_stats_get.argtypes = [vp, ctypes.POINTER(ServerStats)]
        L.zntt_server_destroy.argtypes = [vp]
        L.zntt_now_ns.restype = ctypes.c_uint64
        L.zntt_ntt_host_many.argtypes = [vp, ctypes.POINTER(vp), sz, i]
        _lib = L
    return _lib


def _check(status: int) -> None:
    if status != 0:
        msg = lib().zntt_last_error().decode(errors="replace")
        if status == NotInitialized.code and _init_failure is not None:
            msg = f"{msg}; device initialisation failed: {_init_failure}"
        raise _ERRORS.get(status, ZnttError)(msg or f"status {status}")


def init(device: int = 0) -> None:
    """Binds the library to a CUDA device (idempotent)."""
    global _device, _init_failure
    _check(lib().zntt_init(device))
    _device = device
    _init_failure = None


_init_failure = None


def _ensure_init() -> None:
    """Binds the default device once.  A failure is remembered, not raised, so
    argument errors still surface first (the library validates before it
    touches the device) and a device-needing call then raises NotInitialized."""
    global _init_failure
    if _device is None and _init_failure is None:
        try:
            init(int(os.environ.get("LOCAL_RANK", "0")))
        except ZnttError as e:
            _init_failure = e


def shutdown() -> None:
    global _device
    lib().zntt_shutdown()
    _device = None


def declared_symbols() -> list[str]:
    """Entry points declared in include/zntt.h."""
    import re
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const char\*|int|void)\s+(zntt_\w+)\(", text, re.M)))


# --- element helpers ---------------------------------------------------------------

def _p(a: np.ndarray, F: Field | None = None):
    """The array's data pointer, after checking that its shape is F's element layout:
    (n, 4) Montgomery limbs, or (n,) canonical values for a small field."""
    if F is not None and F.limbs == 1:
        if a.dtype != np.uint64 or not a.flags["C_CONTIGUOUS"] or a.ndim != 1:
            raise InvalidArgument(f"{F.name} data must be a C-contiguous uint64 array of shape (n,)")
        return a.ctypes.data_as(_U64P)
    if a.dtype != np.uint64 or not a.flags["C_CONTIGUOUS"] or a.ndim != 2 or a.shape[1] != 4:
        raise InvalidArgument("data must be a C-contiguous uint64 array of shape (n, 4)")
    return a.ctypes.data_as(_U64P)


def _root(root) -> ctypes.Array:
    r = np.ascontiguousarray(np.asarray(root, dtype=np.uint64).reshape(4))
    return (ctypes.c_uint64 * 4)(*[int(v) for v in r])


def to_montgomery(F: Field, x: int) -> np.ndarray:
    """fromInt (libs/field/src/field.zig:911-921): x mod p in Montgomery limbs."""
    v = (int(x) % F.modulus) * (1 << 256) % F.modulus
    return np.array([(v >> (64 * k)) & 0xFFFFFFFFFFFFFFFF for k in range(4)], dtype=np.uint64)


def primitiveRootOfUnity(F: Field, log_n: int) -> np.ndarray:
    """F.primitiveRootOfUnity(log_n) (libs/field/src/roots.zig:149-158), Montgomery limbs."""
    out = (ctypes.c_uint64 * 4)()
    _check(lib().zntt_primitive_root(F.id, log_n, out))
    return np.array(list(out), dtype=np.uint64)


# --- zig-ntt mirror --------------------------------------------------------------------

def bitReverse(F: Field, data: np.ndarray) -> None:
    _ensure_init()
    fn = lib().zntt_bit_reverse_small if F.limbs == 1 else lib().zntt_bit_reverse
    _check(fn(_p(data, F), len(data)))


def ntt(F: Field, data: np.ndarray, log_n: int, root) -> None:
    _ensure_init()
    _check(lib().zntt_ntt(F.id, _p(data, F), len(data), log_n, _root(root)))


def intt(F: Field, data: np.ndarray, log_n: int, root) -> None:
    _ensure_init()
    _check(lib().zntt_intt(F.id, _p(data, F), len(data), log_n, _root(root)))


class Twiddles(list):
    """zig-ntt's `[]const []const F`: stage s is a (2^s, 4) uint64 array (a (2^s,) array for
    the small fields)."""

    def __init__(self, F: Field, stages):
        super().__init__(stages)
        self.field = F
        self.registered = False

    def stage_array(self):
        arr = (_Stage * max(len(self), 1))()
        wide = self.field.limbs == 4
        for s, a in enumerate(self):
            if a.dtype != np.uint64 or not a.flags["C_CONTIGUOUS"]:
                raise InvalidTwiddles("stage arrays must be C-contiguous uint64")
            if (a.ndim != 2 or a.shape[1] != 4) if wide else a.ndim != 1:
                raise InvalidTwiddles(f"stage arrays of {self.field.name} must have shape "
                                      f"{'(len, 4)' if wide else '(len,)'}")
            arr[s].ptr = a.ctypes.data_as(_U64P)
            arr[s].len = len(a)
        return arr


def precomputeTwiddles(F: Field, log_n: int, root) -> Twiddles:
    if log_n >= 64:
        _check(1)
    stages = [np.zeros((1 << s, 4) if F.limbs == 4 else (1 << s,), dtype=np.uint64) for s in range(log_n)]
    ptrs = (_U64P * max(log_n, 1))()
    for s, a in enumerate(stages):
        ptrs[s] = a.ctypes.data_as(_U64P)
    _ensure_init()
    _check(lib().zntt_precompute_twiddles(F.id, log_n, _root(root), ptrs))
    tw = Twiddles(F, stages)
    tw.registered = True
    return tw


def freeTwiddles(F: Field, twiddles: Twiddles) -> None:
    if getattr(twiddles, "registered", False) and len(twiddles):
        lib().zntt_free_twiddles(F.id, twiddles.stage_array(), len(twiddles))
        twiddles.registered = False


def _as_stages(F: Field, twiddles) -> Twiddles:
    return twiddles if isinstance(twiddles, Twiddles) else Twiddles(F, list(twiddles))


def nttWithTwiddles(F: Field, data: np.ndarray, log_n: int, twiddles) -> None:
    tw = _as_stages(F, twiddles)
    _ensure_init()
    _check(lib().zntt_ntt_with_twiddles(F.id, _p(data, F), len(data), log_n, tw.stage_array(), len(tw)))


def inttWithTwiddles(F: Field, data: np.ndarray, log_n: int, twiddles) -> None:
    tw = _as_stages(F, twiddles)
    _ensure_init()
    _check(lib().zntt_intt_with_twiddles(F.id, _p(data, F), len(data), log_n, tw.stage_array(), len(tw)))


# snake_case aliases
bit_reverse = bitReverse
precompute_twiddles = precomputeTwiddles
free_twiddles = freeTwiddles
ntt_with_twiddles = nttWithTwiddles
intt_with_twiddles = inttWithTwiddles
primitive_root_of_unity = primitiveRootOfUnity


# --- device-resident API -------------------------------------------------------------------

class DeviceTwiddles:
    """A device twiddle table for (field, log_n, root), released on close()."""

    def __init__(self, F: Field, log_n: int, root):
        _ensure_init()
        h = ctypes.c_void_p()
        _check(lib().zntt_twiddles_acquire(F.id, log_n, _root(root), ctypes.byref(h)))
        self.field, self.log_n, self.handle = F, log_n, h

    def close(self) -> None:
        if self.handle:
            _check(lib().zntt_twiddles_release(self.handle))
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def ntt_device(tw: DeviceTwiddles, d_src: int, d_dst: int, mode: int = FORWARD, d_scratch: int = 0,
               stream: int = 0) -> None:
    """Transforms 2^tw.log_n device elements (pointers as ints) on `stream`."""
    _check(lib().zntt_ntt_device(tw.handle, d_src, d_dst, d_scratch or None, mode, stream or None))


def ntt_device_columns(tw: DeviceTwiddles, d_srcs, d_dsts, mode: int = FORWARD, stream: int = 0) -> None:
    """Transforms of several device columns of the table's size, out of place
    (zntt_ntt_device_columns)."""
    m = len(d_srcs)
    src = (ctypes.c_void_p * max(m, 1))(*d_srcs)
    dst = (ctypes.c_void_p * max(len(d_dsts), 1))(*d_dsts)
    _check(lib().zntt_ntt_device_columns(tw.handle, src, dst, m, mode, stream or None))


def ntt_device_inplace_noalloc(tw: DeviceTwiddles, d_data: int, mode: int = FORWARD, stream: int = 0) -> None:
    """In-place transform of up to 2^18 device elements that allocates no memory.

    For callers that must not allocate device memory while they transform
    (a fixed up-front memory budget, memory owned by another allocator, or a
    latency-critical path).  Its scratch is an 8 MiB array inside the library;
    calls that overlap on the GPU share it and race."""
    _check(lib().zntt_ntt_device_inplace_noalloc(tw.handle, d_data, mode, stream or None))


def ntt_host_many(tw: DeviceTwiddles, host_ptrs, mode: int = FORWARD) -> None:
    """Transforms host vectors (addresses of 2^tw.log_n-element buffers) in place,
    pipelining each vector's copies with its neighbours' transforms."""
    arr = (ctypes.c_void_p * max(len(host_ptrs), 1))(*host_ptrs)
    _check(lib().zntt_ntt_host_many(tw.handle, arr, len(host_ptrs), mode))


def seed_bytes(seed: int) -> bytes:
    """The 32-byte ChaCha20 key for an integer seed: u64 little-endian, then zeros."""
    return int(seed).to_bytes(8, "little") + b"\x00" * 24


def random_elements(F: Field, seed: int, d_out: int, count: int, stream: int = 0) -> None:
    """Seeded randomFieldElement draws written to device memory (Montgomery form)."""
    _ensure_init()
    _check(lib().zntt_random_elements(F.id, seed_bytes(seed), d_out, count, stream or None))


def elementwise_device(F: Field, op: str, d_a: int, d_b: int, d_out: int, count: int, stream: int = 0) -> None:
    code = {"mul": 0, "add": 1, "sub": 2, "neg": 3}[op]
    _ensure_init()
    _check(lib().zntt_elementwise_device(F.id, code, d_a, d_b or None, d_out, count, stream or None))


def pool_stats() -> dict:
    """The device buffer pool's counters: acquires, cudaMalloc calls and cached idle bytes."""
    a, m, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    _check(lib().zntt_pool_stats(ctypes.byref(a), ctypes.byref(m), ctypes.byref(c)))
    return {"acquires": a.value, "device_mallocs": m.value, "cached_bytes": c.value}


def probe_imad() -> float:
    _ensure_init()
    v = ctypes.c_double()
    _check(lib().zntt_probe_imad(ctypes.byref(v)))
    return v.value


def probe_mul_wide() -> float:
    """32x32->64 multiply-adds per second (the modmul ceiling is this / 136)."""
    _ensure_init()
    v = ctypes.c_double()
    _check(lib().zntt_probe_mul_wide(ctypes.byref(v)))
    return v.value


def probe_blake3() -> float:
    """Single-block BLAKE3 compressions per second in registers (the commitment's roofline)."""
    _ensure_init()
    v = ctypes.c_double()
    _check(lib().zntt_probe_blake3(ctypes.byref(v)))
    return v.value


def probe_modmul(F: Field) -> float:
    _ensure_init()
    v = ctypes.c_double()
    _check(lib().zntt_probe_modmul(F.id, ctypes.byref(v)))
    return v.value


# --- batches, coset extensions, autotuner ----------------------------------------------------

class Batch:
    """Many jobs (transforms and coset extensions) run by one persistent launch.

    `jobs` is a list of dicts: {"kind": JOB_NTT, "tw": DeviceTwiddles, "mode": FORWARD,
    "src": ptr, "dst": ptr} or {"kind": JOB_COSET_LDE, "tw": out table, "tw_in": in table,
    "shift": 4 Montgomery limbs, "src": ptr, "dst": ptr} or {"kind": JOB_POLY_MUL, "tw": table of
    2^log_n >= len + len2 - 1 points, "src": ptr, "len": n, "src2": ptr, "len2": m, "dst": ptr to
    len + len2 - 1 elements}.  Device buffers stay owned by the caller and must outlive the batch."""

    def __init__(self, F: Field, jobs, shape: int = -1):
        _ensure_init()
        arr = (Job * max(len(jobs), 1))()
        for i, j in enumerate(jobs):
            arr[i].kind = j.get("kind", JOB_NTT)
            arr[i].mode = j.get("mode", FORWARD)
            arr[i].tw = j["tw"].handle
            arr[i].tw_in = j["tw_in"].handle if j.get("tw_in") is not None else None
            arr[i].d_src = j["src"]
            arr[i].d_dst = j["dst"]
            if "shift" in j:
                for k, v in enumerate(np.asarray(j["shift"], dtype=np.uint64).reshape(4)):
                    arr[i].shift[k] = int(v)
            arr[i].d_src2 = j.get("src2")
            arr[i].len = j.get("len", 0)
            arr[i].len2 = j.get("len2", 0)
        h = ctypes.c_void_p()
        _check(lib().zntt_batch_create(F.id, arr, len(jobs), shape, ctypes.byref(h)))
        self.handle = h

    def run(self, stream: int = 0, graph: bool = False) -> None:
        fn = lib().zntt_batch_run_graph if graph else lib().zntt_batch_run
        _check(fn(self.handle, stream or None))

    def status(self) -> None:
        _check(lib().zntt_batch_status(self.handle))

    def set_spin_limit(self, spin_limit: int = BATCH_SPIN_LIMIT) -> None:
        """Rounds a tile waits for its job's previous pass before the batch gives up
        (Timeout from status()); 0 gives up at the first wait."""
        _check(lib().zntt_batch_set_spin_limit(self.handle, spin_limit))

    def info(self) -> dict:
        ni, npp = ctypes.c_uint32(), ctypes.c_uint32()
        g, sh = ctypes.c_int(), ctypes.c_int()
        _check(lib().zntt_batch_info(self.handle, ctypes.byref(ni), ctypes.byref(npp), ctypes.byref(g),
                                     ctypes.byref(sh)))
        return {"items": ni.value, "passes": npp.value, "grid": g.value, "shape": sh.value}

    def close(self) -> None:
        if self.handle:
            lib().zntt_batch_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def coset_lde_device(tw_in: DeviceTwiddles, tw_out: DeviceTwiddles, shift, d_evals: int, d_out: int,
                     stream: int = 0) -> None:
    """One coset low-degree extension with plain per-pass launches."""
    _check(lib().zntt_coset_lde_device(tw_in.handle, tw_out.handle, _root(shift), d_evals, d_out, stream or None))


def coset_lde_columns(tw_in: DeviceTwiddles, tw_out: DeviceTwiddles, shift, d_evals, d_outs,
                      stream: int = 0) -> None:
    """The coset extension of several columns (zntt_coset_lde_columns): column k from d_evals[k]
    into d_outs[k]."""
    m = len(d_evals)
    ev = (ctypes.c_void_p * max(m, 1))(*d_evals)
    out = (ctypes.c_void_p * max(len(d_outs), 1))(*d_outs)
    _check(lib().zntt_coset_lde_columns(tw_in.handle, tw_out.handle, _root(shift), ev, out, m, stream or None))


def poly_mul_device(tw: DeviceTwiddles, d_a: int, len_a: int, d_b: int, len_b: int, d_out: int,
                    stream: int = 0) -> None:
    """d_out[0 .. len_a + len_b - 2] = the product of two device coefficient vectors
    (zntt_poly_mul_device); tw is the table of a primitive 2^log_n-th root with
    2^log_n >= len_a + len_b - 1."""
    _check(lib().zntt_poly_mul_device(tw.handle, d_a, len_a, d_b, len_b, d_out, stream or None))


def poly_mul(F: Field, a: np.ndarray, b: np.ndarray, max_degree: int):
    """Polynomial(F, max_degree).fromCoeffs(a).mul(fromCoeffs(b)) (libs/poly/src/poly.zig:76-84,
    197-212) on the device: returns (coefficients, an (max_degree + 1, 4) uint64 array of
    Montgomery limbs -- (max_degree + 1,) canonical values for Goldilocks and BabyBear -- zero
    beyond the degree; degree, -1 for the zero polynomial).  Raises DegreeTooLarge as the
    reference does."""
    _ensure_init()
    shape = (-1, 4) if F.limbs == 4 else (-1,)  # small fields: one canonical u64 per coefficient
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint64).reshape(shape))
    b = np.ascontiguousarray(np.asarray(b, dtype=np.uint64).reshape(shape))
    out = np.zeros((max_degree + 1, 4) if F.limbs == 4 else (max_degree + 1,), dtype=np.uint64)
    deg = ctypes.c_int64(0)
    pa = a.ctypes.data_as(_U64P) if len(a) else None
    pb = b.ctypes.data_as(_U64P) if len(b) else None
    _check(lib().zntt_poly_mul(F.id, pa, len(a), pb, len(b), max_degree, out.ctypes.data_as(_U64P),
                               ctypes.byref(deg)))
    return out, deg.value


def fri_domain_fill(F: Field, log_n: int, d_out: int, stream: int = 0) -> None:
    """Domain(F).fill (libs/fri/src/root.zig:155-166) into a device buffer of 2^log_n elements."""
    _ensure_init()
    _check(lib().zntt_fri_domain_fill(F.id, log_n, d_out, stream or None))


def fri_fold(F: Field, d_layer: int, log_n: int, alpha, d_out: int, log_table: int = 0, stream: int = 0) -> None:
    """One FRI fold round (libs/fri/src/root.zig:396-403) of a device layer of 2^log_n evaluations
    into 2^(log_n - 1); `alpha` in the field's scalar form (4 Montgomery limbs, or [value, 0, 0, 0])."""
    _ensure_init()
    _check(lib().zntt_fri_fold_device(F.id, d_layer, log_n, _root(alpha), d_out, log_table, stream or None))


def fri_fold_commit(F: Field, d_layer: int, log_n: int, alpha, d_out: int, d_nodes: int, log_table: int = 0,
                    stream: int = 0) -> bytes:
    """One fold round of a device layer of 2^log_n evaluations into d_out and the commitment of
    that new layer into d_nodes, in one pass (zntt_fri_fold_commit); returns the new layer's root."""
    _ensure_init()
    root = ctypes.create_string_buffer(32)
    _check(lib().zntt_fri_fold_commit(F.id, d_layer, log_n, _root(alpha), d_out, log_table, d_nodes, root,
                                      stream or None))
    return root.raw


def fri_commit_phase(F: Field, log_domain: int, log_final: int, d_layers, d_nodes, challenge,
                     stream: int = 0) -> list:
    """The commit phase of proveOn (libs/fri/src/root.zig:372-403) on device layers: d_layers
    holds rounds + 1 device pointers (d_layers[0] the evaluations), d_nodes rounds node arrays;
    challenge(round, root: bytes) returns alpha in the field's scalar form (4 Montgomery limbs,
    or [value, 0, 0, 0]).  Returns the rounds' roots.  An exception in the callback stops the
    phase and is raised again here."""
    _ensure_init()
    rounds = log_domain - log_final
    raised = []

    def cb(_user, rnd, root, alpha_out):
        try:
            a = _root(challenge(int(rnd), bytes(root[:32])))
            for k in range(4):
                alpha_out[k] = int(a[k])
            return 0
        except BaseException as e:  # noqa: BLE001 -- reported after the C call returns
            raised.append(e)
            return 1

    fn = FRI_CHALLENGE_FN(cb)
    layers = (ctypes.c_void_p * len(d_layers))(*d_layers)
    nodes = (ctypes.c_void_p * max(len(d_nodes), 1))(*d_nodes)
    roots = ctypes.create_string_buffer(32 * max(rounds, 1))
    status = lib().zntt_fri_commit_phase(F.id, log_domain, log_final, layers, nodes, roots, fn, None, stream or None)
    if raised:
        raise raised[0]
    _check(status)
    return [roots.raw[32 * r:32 * (r + 1)] for r in range(rounds)]


def fri_query_extract(F: Field, log_domain: int, rounds: int, d_layers, d_nodes, positions, stream: int = 0):
    """The openings of buildQueries (libs/fri/src/root.zig:551-571) from resident layers and
    trees: returns (values, paths) with values[q][r] = serializePair bytes of round r's pair and
    paths[q][r] = the list of sibling digests of MerkleTree.prove, leaf level first."""
    _ensure_init()
    nb = 32 if F.limbs == 4 else (8 if F.id == GOLDILOCKS.id else 4)
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.uint64))
    nq = len(pos)
    per_query = sum(log_domain - r - 1 for r in range(rounds))
    vals = ctypes.create_string_buffer(max(nq * rounds * 2 * nb, 1))
    paths = ctypes.create_string_buffer(max(nq * per_query * 32, 1))
    layers = (ctypes.c_void_p * max(len(d_layers), 1))(*d_layers)
    nodes = (ctypes.c_void_p * max(len(d_nodes), 1))(*d_nodes)
    _check(lib().zntt_fri_query_extract(F.id, log_domain, rounds, layers, nodes,
                                        pos.ctypes.data_as(_U64P) if nq else None, nq, vals, paths, stream or None))
    vraw, praw = vals.raw, paths.raw  # one copy each (.raw copies the whole buffer)
    values, out_paths, off = [], [], 0
    for q in range(nq):
        values.append([vraw[(q * rounds + r) * 2 * nb:(q * rounds + r + 1) * 2 * nb] for r in range(rounds)])
        per_round = []
        for r in range(rounds):
            depth = log_domain - r - 1
            per_round.append([praw[(off + k) * 32:(off + k + 1) * 32] for k in range(depth)])
            off += depth
        out_paths.append(per_round)
    return values, out_paths


class FriConfig:
    """zig-fri's Config (libs/fri/src/root.zig:171-203)."""

    def __init__(self, log_domain: int, log_initial_degree: int, log_final: int, log_residual_degree: int,
                 num_queries: int):
        self.log_domain, self.log_initial_degree = log_domain, log_initial_degree
        self.log_final, self.log_residual_degree, self.num_queries = log_final, log_residual_degree, num_queries

    def rounds(self) -> int:
        """Config.rounds (root.zig:188-195); InvalidArgument for the reference's InvalidParameters."""
        if self.log_domain == 0 or self.log_domain > 63 or self.log_final >= self.log_domain \
                or self.log_residual_degree >= self.log_final or self.log_final > 12 \
                or self.log_residual_degree > 12 or self.num_queries == 0:
            raise InvalidArgument("invalid FRI parameters (Config.rounds)")
        return self.log_domain - self.log_final

    def validate(self) -> None:
        """Config.validate (root.zig:197-202)."""
        r = self.rounds()
        if self.log_initial_degree > self.log_domain or self.log_initial_degree < r \
                or self.log_initial_degree - r != self.log_residual_degree:
            raise InvalidArgument("invalid FRI parameters (Config.validate)")


class FriProof:
    """zig-fri's Proof (libs/fri/src/root.zig:209-240): per round the Merkle root, the residual
    coefficients' toBytes, and per query the pair index with each round's serializePair bytes
    and Merkle siblings (leaf level first)."""

    def __init__(self, roots, residual, queries, log_domain, log_final, log_residual_degree):
        self.roots, self.residual, self.queries = roots, residual, queries
        self.log_domain, self.log_final, self.log_residual_degree = log_domain, log_final, log_residual_degree


def _num_bytes(F: Field) -> int:
    return 32 if F.limbs == 4 else (8 if F.id == GOLDILOCKS.id else 4)


def _canonical(F: Field, limbs) -> int:
    v = sum(int(x) << (64 * k) for k, x in enumerate(limbs))
    return v * pow(1 << 256, -1, F.modulus) % F.modulus if F.limbs == 4 else v


def fri_prove(F: Field, transcript, d_evals: int, config: FriConfig, stream: int = 0) -> FriProof:
    """zig-fri's prove (proveOn over Domain(F), libs/fri/src/root.zig:311-503) with the
    evaluations resident on the device at d_evals (2^log_domain elements in F's layout, left
    unchanged).  The transcript is the caller's, as in the reference: it needs
    absorb_bytes(bytes), challenge_field_checked(modulus, num_bytes) -> int in [0, p) and
    challenge_u64() -> int.  Layers, trees and folds stay on the device; the final layer's
    interpolant comes from the library's inverse transform; only roots, the residual and the
    openings cross to the host.  Device buffers are allocated with torch."""
    import torch  # device allocation only
    config.validate()
    rounds = config.rounds()
    if config.log_domain > F.two_adicity:
        raise InvalidArgument("log_domain exceeds the field's two-adicity (proveOn)")
    _ensure_init()
    nb = _num_bytes(F)
    n = 1 << config.log_domain
    layers = [torch.empty((n >> r) * F.limbs, dtype=torch.int64, device="cuda") for r in range(1, rounds + 1)]
    trees = [torch.empty((n >> r) * 4, dtype=torch.int64, device="cuda") for r in range(rounds)]
    layer_ptrs = [d_evals] + [t.data_ptr() for t in layers]
    tree_ptrs = [t.data_ptr() for t in trees]

    def challenge(_r, root):
        transcript.absorb_bytes(root)
        a = transcript.challenge_field_checked(F.modulus, nb)
        return to_montgomery(F, a) if F.limbs == 4 else np.array([a, 0, 0, 0], dtype=np.uint64)

    roots = fri_commit_phase(F, config.log_domain, config.log_final, layer_ptrs, tree_ptrs, challenge, stream)
    final = layers[-1].cpu().numpy().view(np.uint64)
    final = final.reshape(-1, 4).copy() if F.limbs == 4 else final.copy()
    intt(F, final, config.log_final, primitiveRootOfUnity(F, config.log_final))  # interpolateToCoeffs
    residual = [_canonical(F, final[i] if F.limbs == 4 else [final[i]]).to_bytes(nb, "little")
                for i in range(1 << config.log_residual_degree)]
    for cb in residual:
        transcript.absorb_bytes(cb)  # absorbField of the deserialized coefficient: the same bytes
    positions = [transcript.challenge_u64() % n for _ in range(config.num_queries)]
    values, paths = fri_query_extract(F, config.log_domain, rounds, layer_ptrs[:rounds], tree_ptrs, positions,
                                      stream)
    queries = [{"pair_index": e0, "values": values[q], "paths": paths[q]} for q, e0 in enumerate(positions)]
    return FriProof(roots, residual, queries, config.log_domain, config.log_final, config.log_residual_degree)


def merkle_commit_rows(F: Field, d_columns, log_n: int, d_nodes: int, stream: int = 0) -> bytes:
    """MerkleTree.init over the 2^log_n rows of device columns (zntt_merkle_commit_rows): leaf i
    hashes the row's toBytes values in column order; d_nodes receives 2^(log_n+1) digests of 32
    bytes in heap order.  Returns the root."""
    _ensure_init()
    cols = (ctypes.c_void_p * max(len(d_columns), 1))(*d_columns)
    root = ctypes.create_string_buffer(32)
    _check(lib().zntt_merkle_commit_rows(F.id, cols, len(d_columns), log_n, d_nodes, root, stream or None))
    return root.raw


def merkle_open_rows(F: Field, d_columns, log_n: int, d_nodes: int, positions, stream: int = 0):
    """Openings of a row commitment (zntt_merkle_open_rows): returns (rows, paths) with rows[q]
    the toBytes values of row positions[q] in column order and paths[q] its sibling digests,
    leaf level first."""
    _ensure_init()
    nb = _num_bytes(F)
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.uint64))
    nq, m = len(pos), len(d_columns)
    cols = (ctypes.c_void_p * max(m, 1))(*d_columns)
    vals = ctypes.create_string_buffer(max(nq * m * nb, 1))
    paths = ctypes.create_string_buffer(max(nq * log_n * 32, 1))
    _check(lib().zntt_merkle_open_rows(F.id, cols, m, log_n, d_nodes, pos.ctypes.data_as(_U64P) if nq else None, nq,
                                       vals, paths, stream or None))
    vraw, praw = vals.raw, paths.raw
    rows = [vraw[q * m * nb:(q + 1) * m * nb] for q in range(nq)]
    out = [[praw[(q * log_n + k) * 32:(q * log_n + k + 1) * 32] for k in range(log_n)] for q in range(nq)]
    return rows, out


def fri_commit_layer(F: Field, d_layer: int, log_n: int, d_nodes: int, stream: int = 0) -> bytes:
    """The FRI layer commitment (hashPair leaves, heap-ordered BLAKE3 Merkle tree) of a device
    layer of 2^log_n evaluations into d_nodes (2^log_n x 32 bytes); returns the root."""
    _ensure_init()
    root = ctypes.create_string_buffer(32)
    _check(lib().zntt_fri_commit_layer(F.id, d_layer, log_n, d_nodes, root, stream or None))
    return root.raw


def autotune(F: Field, log_n_min: int, log_n_max: int) -> None:
    _ensure_init()
    _check(lib().zntt_autotune(F.id, log_n_min, log_n_max))


def tune_save(path: str) -> None:
    _check(lib().zntt_tune_save(path.encode()))


def tune_load(path: str) -> None:
    _ensure_init()
    _check(lib().zntt_tune_load(path.encode()))


def tune_clear() -> None:
    lib().zntt_tune_clear()


class Server:
    """The continuously batching request server (zntt_server_*)."""

    def __init__(self, F: Field, hbm_budget_bytes: int, slots: int = 4, max_batch_jobs: int = 256,
                 max_items: int = 1 << 20, serial: bool = False, max_batch_bytes: int = 0):
        _ensure_init()
        cfg = ServerConfig(F.id, hbm_budget_bytes, slots, max_batch_jobs, max_items, int(serial), max_batch_bytes)
        h = ctypes.c_void_p()
        _check(lib().zntt_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.handle, self.field = h, F
        self._buf = (Completion * 1024)()

    def submit(self, req: Request) -> None:
        _check(lib().zntt_server_submit(self.handle, ctypes.byref(req)))

    def poll(self, wait_ms: int = 0):
        n = ctypes.c_size_t()
        _check(lib().zntt_server_poll(self.handle, self._buf, len(self._buf), ctypes.byref(n), wait_ms))
        return [(c.user_tag, c.status, c.arrival_ns, c.admit_ns, c.done_ns) for c in self._buf[:n.value]]

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().zntt_server_stats_get(self.handle, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self) -> None:
        if self.handle:
            lib().zntt_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def now_ns() -> int:
    return int(lib().zntt_now_ns())
