"""ctypes wrapper over oracle/liboracle.so -- TEST INFRASTRUCTURE ONLY.

The CPU restatement of zig-ntt (libs/ntt/src/root.zig:33-212) and its field
arithmetic lives in zntt_oracle.cpp.  Only the test suite, the smoke check and
the CPU-baseline leg of the benchmark may load this module; the product library
never does.

Elements are numpy uint64 arrays of shape (n, 4): little-endian limbs, in
Montgomery form unless a function says "canonical".  Single-limb fields
(Goldilocks, BabyBear) use column 0.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

BN254_FR = 0
BLS12_381_FR = 1
GOLDILOCKS = 2
BABYBEAR = 3
BN254_FP = 4

OK = 0
LOG_TOO_LARGE = 1
LENGTH_MISMATCH = 2
INVALID_TWIDDLES = 3
INVALID_LENGTH = 4
OUT_OF_MEMORY = 5
ORDER_TOO_LARGE = 6
DEGREE_TOO_LARGE = 13

MODULI = {
    BN254_FR: 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001,
    BLS12_381_FR: 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001,
    GOLDILOCKS: 0xFFFFFFFF00000001,
    BABYBEAR: 0x78000001,
    BN254_FP: 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47,
}
NLIMBS = {BN254_FR: 4, BLS12_381_FR: 4, GOLDILOCKS: 1, BABYBEAR: 1, BN254_FP: 4}

_U64P = ctypes.POINTER(ctypes.c_uint64)
_lib = None


def build(native: bool = False) -> str:
    """Compile the oracle with its Makefile; returns the library path."""
    target = "native" if native else "liboracle.so"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)
    return os.path.join(HERE, "liboracle_native.so" if native else "liboracle.so")


def load(path: str | None = None):
    global _lib
    if _lib is not None and path is None:
        return _lib
    if path is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
    lib = ctypes.CDLL(path)
    sz = ctypes.c_size_t
    i = ctypes.c_int
    lib.zo_field_info.argtypes = [i, _U64P, ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(i)]
    lib.zo_to_mont.argtypes = [i, _U64P, _U64P, sz]
    lib.zo_from_mont.argtypes = [i, _U64P, _U64P, sz]
    lib.zo_elementwise.argtypes = [i, i, _U64P, _U64P, _U64P, sz]
    lib.zo_from_int.argtypes = [i, ctypes.c_uint64, _U64P]
    lib.zo_pow.argtypes = [i, _U64P, _U64P, _U64P]
    lib.zo_primitive_root.argtypes = [i, sz, _U64P]
    lib.zo_qnr.argtypes = [i, _U64P]
    lib.zo_bit_reverse.argtypes = [i, _U64P, sz]
    lib.zo_ntt.argtypes = [i, _U64P, sz, sz, _U64P, i]
    lib.zo_precompute_twiddles.argtypes = [i, sz, _U64P, _U64P]
    lib.zo_ntt_with_twiddles.argtypes = [i, _U64P, sz, sz, ctypes.POINTER(_U64P),
                                         ctypes.POINTER(sz), sz, i, i]
    lib.zo_ntt_with_twiddles_inplace4.argtypes = lib.zo_ntt_with_twiddles.argtypes
    lib.zo_ntt_with_twiddles_inplace1.argtypes = lib.zo_ntt_with_twiddles.argtypes
    lib.zo_chacha20_stream.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p, sz]
    lib.zo_random_elements.argtypes = [i, ctypes.c_char_p, _U64P, sz]
    lib.zo_powers.argtypes = [i, _U64P, _U64P, sz]
    lib.zo_coset_lde.argtypes = [i, _U64P, sz, sz, _U64P, _U64P, i]
    lib.zo_merkle_commit_rows.argtypes = [i, ctypes.POINTER(_U64P), sz, sz, ctypes.c_void_p, i]
    lib.zo_dft_points.argtypes = [i, _U64P, sz, _U64P, _U64P, sz, _U64P, i]
    lib.zo_poly_mul.argtypes = [i, _U64P, sz, _U64P, sz, sz, _U64P, ctypes.POINTER(ctypes.c_int64), i]
    lib.zo_poly_eval.argtypes = [i, _U64P, sz, _U64P, sz, _U64P, i]
    lib.zo_fri_domain_fill.argtypes = [i, sz, _U64P]
    lib.zo_fri_fold.argtypes = [i, _U64P, sz, _U64P, _U64P, i]
    lib.zo_blake3.argtypes = [ctypes.c_char_p, sz, ctypes.c_char_p]
    lib.zo_fri_commit_layer.argtypes = [i, _U64P, sz, ctypes.c_void_p, i]
    if path.endswith("liboracle.so"):
        _lib = lib
    return lib


def _p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_U64P)


def elems(n: int) -> np.ndarray:
    return np.zeros((n, 4), dtype=np.uint64)


def int_to_limbs(x: int) -> list[int]:
    return [(x >> (64 * k)) & 0xFFFFFFFFFFFFFFFF for k in range(4)]


def limbs_to_int(row) -> int:
    return sum(int(row[k]) << (64 * k) for k in range(4))


def from_ints(values) -> np.ndarray:
    out = elems(len(values))
    for i, v in enumerate(values):
        out[i] = int_to_limbs(v)
    return out


def to_ints(a: np.ndarray) -> list[int]:
    return [limbs_to_int(r) for r in a]


def to_mont(field: int, canon: np.ndarray) -> np.ndarray:
    out = elems(len(canon))
    st = load().zo_to_mont(field, _p(np.ascontiguousarray(canon)), _p(out), len(canon))
    assert st == OK
    return out


def from_mont(field: int, mont: np.ndarray) -> np.ndarray:
    out = elems(len(mont))
    st = load().zo_from_mont(field, _p(np.ascontiguousarray(mont)), _p(out), len(mont))
    assert st == OK
    return out


def elementwise(field: int, op: str, a: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
    code = {"mul": 0, "add": 1, "sub": 2, "neg": 3, "inv": 4}[op]
    out = elems(len(a))
    bp = _p(np.ascontiguousarray(b)) if b is not None else None
    st = load().zo_elementwise(field, code, _p(np.ascontiguousarray(a)), bp, _p(out), len(a))
    assert st == OK
    return out


def from_int(field: int, x: int) -> np.ndarray:
    out = elems(1)
    load().zo_from_int(field, x, _p(out))
    return out[0]


def pow_(field: int, base: np.ndarray, exp: int) -> np.ndarray:
    e = np.array([(exp >> (64 * k)) & 0xFFFFFFFFFFFFFFFF for k in range(8)], dtype=np.uint64)
    out = elems(1)
    b = np.ascontiguousarray(base.reshape(1, 4))
    load().zo_pow(field, _p(b), _p(e), _p(out))
    return out[0]


def primitive_root(field: int, log_n: int):
    """Montgomery-form primitive 2^log_n-th root (roots.zig:149-158), or an error code."""
    out = elems(1)
    st = load().zo_primitive_root(field, log_n, _p(out))
    return (st, out[0])


def qnr(field: int) -> np.ndarray:
    out = elems(1)
    load().zo_qnr(field, _p(out))
    return out[0]


def bit_reverse(field: int, data: np.ndarray) -> int:
    return load().zo_bit_reverse(field, _p(data), len(data))


def ntt(field: int, data: np.ndarray, log_n: int, root: np.ndarray) -> int:
    r = np.ascontiguousarray(root.reshape(1, 4))
    return load().zo_ntt(field, _p(data), len(data), log_n, _p(r), 0)


def intt(field: int, data: np.ndarray, log_n: int, root: np.ndarray) -> int:
    r = np.ascontiguousarray(root.reshape(1, 4))
    return load().zo_ntt(field, _p(data), len(data), log_n, _p(r), 1)


def precompute_twiddles(field: int, log_n: int, root: np.ndarray):
    """Returns (status, [stage arrays]) in zig-ntt's layout: stage s has 2^s entries."""
    n = 1 << log_n if log_n < 64 else 0
    if log_n >= 64:
        return (LOG_TOO_LARGE, None)
    flat = elems(max(n - 1, 1))
    r = np.ascontiguousarray(root.reshape(1, 4))
    st = load().zo_precompute_twiddles(field, log_n, _p(r), _p(flat))
    if st != OK:
        return (st, None)
    return (OK, [flat[(1 << s) - 1:(1 << (s + 1)) - 1].copy() for s in range(log_n)])


def ntt_with_twiddles(field: int, data: np.ndarray, log_n: int, stages, inverse: bool = False,
                      workers: int = 1, inplace4: bool = False) -> int:
    ptrs = (_U64P * max(len(stages), 1))()
    lens = (ctypes.c_size_t * max(len(stages), 1))()
    for s, a in enumerate(stages):
        assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
        ptrs[s] = a.ctypes.data_as(_U64P)
        lens[s] = len(a)
    fn = load().zo_ntt_with_twiddles_inplace4 if inplace4 else load().zo_ntt_with_twiddles
    return fn(field, _p(data), len(data), log_n, ptrs, lens, len(stages), int(inverse), workers)


def chacha20_stream(seed32: bytes, nbytes: int, nonce12: bytes | None = None) -> bytes:
    buf = ctypes.create_string_buffer(nbytes)
    st = load().zo_chacha20_stream(seed32, nonce12, buf, nbytes)
    assert st == OK
    return buf.raw


def seed_bytes(seed: int) -> bytes:
    """The 32-byte ChaCha20 key for an integer seed: u64 little-endian, then zeros."""
    return int(seed).to_bytes(8, "little") + b"\x00" * 24


def random_elements(field: int, seed: int, count: int) -> np.ndarray:
    out = elems(count)
    st = load().zo_random_elements(field, seed_bytes(seed), _p(out), count)
    assert st == OK
    return out


def powers(field: int, base: np.ndarray, n: int) -> np.ndarray:
    out = elems(n)
    b = np.ascontiguousarray(base.reshape(1, 4))
    load().zo_powers(field, _p(b), _p(out), n)
    return out


def coset_lde(field: int, evals: np.ndarray, log_in: int, log_blowup: int, shift: np.ndarray,
              workers: int = 1) -> np.ndarray:
    out = elems(1 << (log_in + log_blowup))
    s = np.ascontiguousarray(shift.reshape(1, 4))
    st = load().zo_coset_lde(field, _p(np.ascontiguousarray(evals)), log_in, log_blowup, _p(s), _p(out),
                             workers)
    assert st == OK, st
    return out


def dft_points(field: int, x: np.ndarray, root: np.ndarray, ks, workers: int = 1) -> np.ndarray:
    """X_k = sum_j x_j root^(jk) for each k in ks, by Horner evaluation (Montgomery form)."""
    kk = np.ascontiguousarray(np.asarray(ks, dtype=np.uint64))
    out = elems(len(kk))
    r = np.ascontiguousarray(root.reshape(1, 4))
    st = load().zo_dft_points(field, _p(np.ascontiguousarray(x)), len(x), _p(r), kk.ctypes.data_as(_U64P),
                              len(kk), _p(out), workers)
    assert st == OK
    return out


def poly_mul(field: int, a: np.ndarray, b: np.ndarray, max_degree: int, workers: int = 1):
    """Polynomial(F, max_degree).fromCoeffs(a).mul(fromCoeffs(b)) by the schoolbook loops of
    libs/poly/src/poly.zig:197-212: (status, coefficients[max_degree + 1], degree)."""
    out = elems(max_degree + 1)
    deg = ctypes.c_int64(0)
    na, nb = len(a), len(b)
    a = np.ascontiguousarray(a.reshape(-1, 4)) if na else elems(1)
    b = np.ascontiguousarray(b.reshape(-1, 4)) if nb else elems(1)
    st = load().zo_poly_mul(field, _p(a), na, _p(b), nb, max_degree, _p(out), ctypes.byref(deg), workers)
    return st, out, deg.value


def poly_eval(field: int, c: np.ndarray, xs: np.ndarray, workers: int = 1) -> np.ndarray:
    """Horner evaluation of the coefficients c at each point of xs (poly.zig:214-224)."""
    out = elems(len(xs))
    st = load().zo_poly_eval(field, _p(np.ascontiguousarray(c)), len(c), _p(np.ascontiguousarray(xs)), len(xs),
                             _p(out), workers)
    assert st == OK, st
    return out


def fri_domain_fill(field: int, log_n: int) -> np.ndarray:
    """Domain(F).fill (libs/fri/src/root.zig:155-166): g^i for i < 2^log_n (Montgomery slots)."""
    out = elems(1 << log_n)
    st = load().zo_fri_domain_fill(field, log_n, _p(out))
    assert st == OK, st
    return out


def fri_fold(field: int, layer: np.ndarray, log_n: int, alpha: np.ndarray, workers: int = 1) -> np.ndarray:
    """One fold round of proveOn (libs/fri/src/root.zig:396-403) on 2^log_n slots."""
    out = elems(1 << (log_n - 1))
    a = np.ascontiguousarray(np.asarray(alpha, dtype=np.uint64).reshape(1, 4))
    st = load().zo_fri_fold(field, _p(np.ascontiguousarray(layer)), log_n, _p(a), _p(out), workers)
    assert st == OK, st
    return out


def blake3(msg: bytes) -> bytes:
    """BLAKE3-256 of a message of at most 1024 bytes."""
    out = ctypes.create_string_buffer(32)
    st = load().zo_blake3(msg, len(msg), out)
    assert st == OK, st
    return out.raw


def fri_commit_layer(field: int, layer: np.ndarray, log_n: int, workers: int = 1) -> np.ndarray:
    """The FRI layer commitment (hashPair leaves, heap-ordered BLAKE3 Merkle tree): a
    (2^log_n, 32) uint8 array of node digests, row 1 the root, row 0 zero."""
    nodes = np.zeros((1 << log_n, 32), dtype=np.uint8)
    st = load().zo_fri_commit_layer(field, _p(np.ascontiguousarray(layer)), log_n, nodes.ctypes.data, workers)
    assert st == OK, st
    return nodes


def element_bytes(field: int) -> int:
    """F.NUM_BYTES: ceil(bits / 8) of the modulus (32, 32, 8, 4)."""
    return {BN254_FR: 32, BLS12_381_FR: 32, GOLDILOCKS: 8, BABYBEAR: 4}[field]


def to_bytes(field: int, slots: np.ndarray) -> list:
    """toBytes of each Montgomery slot: the canonical value, NUM_BYTES little-endian bytes."""
    canon = from_mont(field, np.ascontiguousarray(slots))
    nb = element_bytes(field)
    return [row.tobytes()[:nb] for row in canon]


def fri_commit_phase(field: int, evals: np.ndarray, log_domain: int, log_final: int, challenge,
                     workers: int = 1):
    """The commit loop of proveOn (libs/fri/src/root.zig:372-403): per round, commit the
    layer (hashPair leaves, BLAKE3 Merkle tree), take alpha = challenge(round, root) (a
    Montgomery slot), fold.  Returns (roots, layers 0..rounds, node arrays 0..rounds-1)."""
    layers, trees, roots = [np.ascontiguousarray(evals)], [], []
    for r in range(log_domain - log_final):
        log_n = log_domain - r
        nodes = fri_commit_layer(field, layers[r], log_n, workers=workers)
        trees.append(nodes)
        roots.append(nodes[1].tobytes())
        alpha = np.asarray(challenge(r, roots[r]), dtype=np.uint64)
        layers.append(fri_fold(field, layers[r], log_n, alpha, workers=workers))
    return roots, layers, trees


def fri_query_extract(field: int, layers: list, trees: list, log_domain: int, rounds: int, positions) -> tuple:
    """The openings of buildQueries (libs/fri/src/root.zig:551-571): per query and round,
    serializePair(f_r[j], f_r[j + half]) with j = e mod half, e carried from round to round
    (e = j), and MerkleTree.prove(j)'s siblings (libs/merkle/src/merkle_tree.zig:206-233):
    node pos ^ 1 for pos = half + j, half + j >> 1, ... while pos > 1."""
    values, paths = [], []
    for e0 in positions:
        e, vq, pq = int(e0), [], []
        for r in range(rounds):
            half = 1 << (log_domain - r - 1)
            j = e % half
            pair = to_bytes(field, layers[r][[j, j + half]])
            vq.append(pair[0] + pair[1])
            sib, pos = [], half + j
            while pos > 1:
                sib.append(trees[r][pos + 1 if pos % 2 == 0 else pos - 1].tobytes())
                pos >>= 1
            pq.append(sib)
            e = j
        values.append(vq)
        paths.append(pq)
    return values, paths


def fri_prove(field: int, evals: np.ndarray, log_domain: int, log_final: int, log_residual: int, num_queries: int,
              transcript, workers: int = 1) -> dict:
    """proveOn over Domain(F) (libs/fri/src/root.zig:335-503) on the oracle's commitment, fold
    and inverse transform: the commit loop above with alpha = transcript.absorb_bytes(root),
    challenge_field_checked (root.zig:386-388); the residual = the first 2^log_residual
    coefficients of the final layer's interpolant (interpolateToCoeffs, the unique polynomial
    of degree < 2^log_final: its inverse transform), absorbed as toBytes; then num_queries
    positions challengeU64() % 2^log_domain and their openings.  `transcript` is the caller's
    (absorb_bytes, challenge_field_checked(p, num_bytes), challenge_u64)."""
    p, nb = MODULI[field], element_bytes(field)

    def challenge(_r, root):
        transcript.absorb_bytes(root)
        return to_mont(field, from_ints([transcript.challenge_field_checked(p, nb)]))[0]

    rounds = log_domain - log_final
    roots, layers, trees = fri_commit_phase(field, evals, log_domain, log_final, challenge, workers=workers)
    coeffs = np.ascontiguousarray(layers[rounds].copy())
    st, g = primitive_root(field, log_final)
    assert st == OK and intt(field, coeffs, log_final, g) == OK
    residual = to_bytes(field, coeffs[:1 << log_residual])
    for cb in residual:
        transcript.absorb_bytes(cb)
    positions = [transcript.challenge_u64() % (1 << log_domain) for _ in range(num_queries)]
    values, paths = fri_query_extract(field, layers, trees, log_domain, rounds, positions)
    return {"roots": roots, "residual": residual,
            "queries": [{"pair_index": e0, "values": values[q], "paths": paths[q]} for q, e0 in enumerate(positions)],
            "log_domain": log_domain, "log_final": log_final, "log_residual_degree": log_residual}


def merkle_commit_rows(field: int, columns: list, log_n: int, workers: int = 1) -> np.ndarray:
    """MerkleTree.init (libs/merkle/src/merkle_tree.zig:70-103) over the 2^log_n rows of the
    columns (Montgomery slots): leaf i = BLAKE3 of the row's toBytes concatenated in column
    order.  A (2^(log_n+1), 32) uint8 array of node digests, row 1 the root, row 0 zero."""
    cols = [np.ascontiguousarray(c) for c in columns]
    ptrs = (_U64P * len(cols))(*[c.ctypes.data_as(_U64P) for c in cols])
    nodes = np.zeros((2 << log_n, 32), dtype=np.uint8)
    st = load().zo_merkle_commit_rows(field, ptrs, len(cols), log_n, nodes.ctypes.data, workers)
    assert st == OK, st
    return nodes
