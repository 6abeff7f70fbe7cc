"""Independent pure-Python restatement used to make and check golden fixtures.

It shares no code with the C++ oracle or the CUDA library, so agreement between
the three is evidence rather than self-consistency:

* ChaCha20 keystream (RFC 8439; the reference's libs/rng/src/chacha20.zig:36-160)
  and randomFieldElement (libs/rng/src/rng.zig:32-65: NUM_BYTES bytes read
  big-endian, rejected when >= p).
* The transform by its definition X_k = sum_j x_j * w^(j*k) (the convention the
  reference's known-answer test pins, libs/ntt/src/root.zig:399-453), plus a
  recursive radix-2 FFT over Python integers for sizes where the O(n^2) sum is
  too slow; the FFT is checked against the definition at small sizes.
* Polynomial products by the schoolbook sum c_k = sum_{i+j=k} a_i b_j over
  Python integers (what Polynomial.mul of libs/poly/src/poly.zig:197-212
  computes), with the reference's degree convention (-1 for zero).
* BLAKE3 (the published specification; single-chunk messages, up to 1024 bytes)
  for the FRI layer commitment: hashPair (libs/fri/src/root.zig:286-295) and the
  heap-ordered Merkle tree of libs/merkle/src/merkle_tree.zig:146-180.
* Roots of unity as the reference derives them (libs/field/src/roots.zig:149-158):
  z = the first quadratic non-residue counting up from 2, raised to
  odd_part << (two_adicity - log_n).
* The Fiat-Shamir transcript of libs/transcript/src/root.zig:38-170 (length-
  prefixed absorbs into one BLAKE3 message, squeeze = the digest, re-keyed with
  it) and zig-fri's prove / verify (libs/fri/src/root.zig:335-503, 606-720) over
  it, in field integers, for proofs whose transcript messages fit one chunk.
"""
from __future__ import annotations

BN254_FR_P = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
BLS12_381_FR_P = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
MASK32 = 0xFFFFFFFF


def _rotl(x: int, r: int) -> int:
    return ((x << r) | (x >> (32 - r))) & MASK32


def chacha20_block(key: bytes, counter: int, nonce: bytes) -> bytes:
    st = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574]
    st += [int.from_bytes(key[4 * i:4 * i + 4], "little") for i in range(8)]
    st += [counter & MASK32]
    st += [int.from_bytes(nonce[4 * i:4 * i + 4], "little") for i in range(3)]
    x = list(st)

    def qr(a, b, c, d):
        x[a] = (x[a] + x[b]) & MASK32; x[d] = _rotl(x[d] ^ x[a], 16)
        x[c] = (x[c] + x[d]) & MASK32; x[b] = _rotl(x[b] ^ x[c], 12)
        x[a] = (x[a] + x[b]) & MASK32; x[d] = _rotl(x[d] ^ x[a], 8)
        x[c] = (x[c] + x[d]) & MASK32; x[b] = _rotl(x[b] ^ x[c], 7)

    for _ in range(10):
        qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15)
        qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14)
    return b"".join(((x[i] + st[i]) & MASK32).to_bytes(4, "little") for i in range(16))


class ChaChaStream:
    """Keystream from counter 0, consumed in order."""

    def __init__(self, key: bytes, nonce: bytes = b"\x00" * 12):
        self.key, self.nonce, self.counter, self.buf = key, nonce, 0, b""

    def read(self, n: int) -> bytes:
        while len(self.buf) < n:
            self.buf += chacha20_block(self.key, self.counter, self.nonce)
            self.counter += 1
        out, self.buf = self.buf[:n], self.buf[n:]
        return out


def seed_key(seed: int) -> bytes:
    """Integer seed -> 32-byte ChaCha20 key: u64 little-endian, then zeros."""
    return int(seed).to_bytes(8, "little") + b"\x00" * 24


def random_field_values(p: int, seed: int, count: int) -> list[int]:
    """Canonical values of `count` randomFieldElement draws."""
    nbytes = (p.bit_length() + 7) // 8
    s = ChaChaStream(seed_key(seed))
    out = []
    while len(out) < count:
        for _ in range(1024):
            v = int.from_bytes(s.read(nbytes), "big")
            if v < p:
                out.append(v)
                break
        else:
            raise RuntimeError("rejection sampling failed")
    return out


def two_adicity(p: int) -> tuple[int, int]:
    q, s = p - 1, 0
    while q % 2 == 0:
        q //= 2
        s += 1
    return s, q


def first_qnr(p: int) -> int:
    z = 2
    while pow(z, (p - 1) // 2, p) != p - 1:
        z += 1
    return z


def primitive_root(p: int, log_n: int) -> int:
    s, q = two_adicity(p)
    assert log_n <= s
    return pow(first_qnr(p), q << (s - log_n), p)


def dft(x: list[int], w: int, p: int) -> list[int]:
    n = len(x)
    return [sum(x[j] * pow(w, (j * k) % n, p) for j in range(n)) % p for k in range(n)]


def fft(x: list[int], w: int, p: int) -> list[int]:
    n = len(x)
    if n == 1:
        return [x[0] % p]
    even = fft(x[0::2], w * w % p, p)
    odd = fft(x[1::2], w * w % p, p)
    out = [0] * n
    wk = 1
    h = n // 2
    for k in range(h):
        t = wk * odd[k] % p
        out[k] = (even[k] + t) % p
        out[k + h] = (even[k] - t) % p
        wk = wk * w % p
    return out


def inverse_transform(x: list[int], w: int, p: int) -> list[int]:
    n = len(x)
    y = fft(x, pow(w, -1, p), p)
    ninv = pow(n, -1, p)
    return [v * ninv % p for v in y]


def coset_lde(evals: list[int], log_blowup: int, shift: int, p: int) -> list[int]:
    """inverse transform -> zero-pad -> scale c_i by shift^i -> forward transform."""
    n_in = len(evals)
    log_in = n_in.bit_length() - 1
    coeffs = inverse_transform(evals, primitive_root(p, log_in), p)
    n_out = n_in << log_blowup
    padded = coeffs + [0] * (n_out - n_in)
    g = 1
    for i in range(n_out):
        padded[i] = padded[i] * g % p
        g = g * shift % p
    return fft(padded, primitive_root(p, log_in + log_blowup), p)


def degree(c: list[int]) -> int:
    d = len(c) - 1
    while d >= 0 and c[d] == 0:
        d -= 1
    return d


def poly_mul(a: list[int], b: list[int], p: int) -> list[int]:
    """The product's coefficients (degree deg a + deg b), [] when a factor is zero."""
    da, db = degree(a), degree(b)
    if da < 0 or db < 0:
        return []
    c = [0] * (da + db + 1)
    for i in range(da + 1):
        for j in range(db + 1):
            c[i + j] = (c[i + j] + a[i] * b[j]) % p
    return c


# ---- BLAKE3, single chunk ---------------------------------------------------------
B3_IV = [0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A, 0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19]
B3_PERM = [2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8]
B3_CHUNK_START, B3_CHUNK_END, B3_ROOT = 1, 2, 8


def _rotr(x: int, r: int) -> int:
    return ((x >> r) | (x << (32 - r))) & MASK32


def _b3_compress(cv, block_words, counter, block_len, flags):
    v = list(cv) + B3_IV[:4] + [counter & MASK32, counter >> 32, block_len, flags]
    m = list(block_words)

    def g(a, b, c, d, x, y):
        v[a] = (v[a] + v[b] + x) & MASK32
        v[d] = _rotr(v[d] ^ v[a], 16)
        v[c] = (v[c] + v[d]) & MASK32
        v[b] = _rotr(v[b] ^ v[c], 12)
        v[a] = (v[a] + v[b] + y) & MASK32
        v[d] = _rotr(v[d] ^ v[a], 8)
        v[c] = (v[c] + v[d]) & MASK32
        v[b] = _rotr(v[b] ^ v[c], 7)

    for rnd in range(7):
        g(0, 4, 8, 12, m[0], m[1])
        g(1, 5, 9, 13, m[2], m[3])
        g(2, 6, 10, 14, m[4], m[5])
        g(3, 7, 11, 15, m[6], m[7])
        g(0, 5, 10, 15, m[8], m[9])
        g(1, 6, 11, 12, m[10], m[11])
        g(2, 7, 8, 13, m[12], m[13])
        g(3, 4, 9, 14, m[14], m[15])
        if rnd < 6:
            m = [m[i] for i in B3_PERM]
    return [v[i] ^ v[i + 8] for i in range(8)]


def blake3(msg: bytes) -> bytes:
    """BLAKE3-256 of a message of at most one chunk (1024 bytes): its 64-byte blocks are
    compressed in order from the IV, the first flagged CHUNK_START, the last CHUNK_END | ROOT."""
    assert len(msg) <= 1024
    blocks = [msg[i:i + 64] for i in range(0, len(msg), 64)] or [b""]
    cv = B3_IV
    for i, blk in enumerate(blocks):
        words = [int.from_bytes((blk + bytes(64 - len(blk)))[4 * k:4 * k + 4], "little") for k in range(16)]
        flags = (B3_CHUNK_START if i == 0 else 0) | (B3_CHUNK_END | B3_ROOT if i == len(blocks) - 1 else 0)
        cv = _b3_compress(cv, words, 0, len(blk), flags)
    return b"".join(w.to_bytes(4, "little") for w in cv)


def to_bytes(value: int, num_bytes: int) -> bytes:
    """Field.toBytes: the canonical value, little-endian, NUM_BYTES = ceil(bits / 8) bytes."""
    return value.to_bytes(num_bytes, "little")


def fri_commit_layer(values: list[int], num_bytes: int) -> list[bytes]:
    """The FRI layer commitment of proveOn: leaf j = BLAKE3(toBytes(f_j) || toBytes(f_{j+n/2}))
    (hashPair), then MerkleTree.initFromHashes: nodes[1] is the root, nodes[h + j] leaf j,
    nodes[i] = BLAKE3(nodes[2i] || nodes[2i+1]); leaf counts are padded to a power of two with
    BLAKE3 of the empty string.  Returns nodes[0 .. 2h) with nodes[0] all zero."""
    half = len(values) // 2
    h = 1
    while h < half:
        h *= 2
    nodes = [bytes(32)] * (2 * h)
    for j in range(half):
        nodes[h + j] = blake3(to_bytes(values[j], num_bytes) + to_bytes(values[j + half], num_bytes))
    for j in range(half, h):
        nodes[h + j] = blake3(b"")
    for i in range(h - 1, 0, -1):
        nodes[i] = blake3(nodes[2 * i] + nodes[2 * i + 1])
    return nodes


class Transcript:
    """zig-transcript's Transcript (libs/transcript/src/root.zig:38-170).  The hasher state is
    the message absorbed since the last re-key; a squeeze hashes it."""

    def __init__(self, label: bytes):
        self.msg = len(label).to_bytes(8, "little") + label

    def absorb_bytes(self, data: bytes) -> None:
        self.msg += len(data).to_bytes(8, "little") + data

    def absorb_u64(self, v: int) -> None:
        self.absorb_bytes(v.to_bytes(8, "little"))

    def challenge_bytes(self, n: int) -> bytes:
        digest = blake3(self.msg)
        out = b""
        while len(out) < n:
            out += digest[:min(32, n - len(out))]
            if len(out) < n:
                digest = blake3(digest)
        self.msg = digest  # re-key with the (last) digest
        return out

    def challenge_u64(self) -> int:
        return int.from_bytes(self.challenge_bytes(8), "little")

    def challenge_field_checked(self, p: int, num_bytes: int) -> int:
        """challengeFieldChecked: NUM_BYTES little-endian bytes, rejected (and re-drawn) when >= p."""
        while True:
            v = int.from_bytes(self.challenge_bytes(num_bytes), "little")
            if v < p:
                return v


def fri_fold_values(f: list[int], alpha: int, p: int) -> list[int]:
    """One fold round (libs/fri/src/root.zig:396-403) on the natural-order subgroup of order len(f)."""
    n = len(f)
    h = n // 2
    g = primitive_root(p, n.bit_length() - 1)
    inv2 = pow(2, -1, p)
    out = []
    for j in range(h):
        x = pow(g, j, p)
        even = (f[j] + f[j + h]) * inv2 % p
        odd = (f[j] - f[j + h]) * pow(x, -1, p) * inv2 % p
        out.append((even + alpha * odd) % p)
    return out


def merkle_siblings(nodes: list[bytes], leaf_count: int, index: int) -> list[bytes]:
    """MerkleTree.prove's siblings (libs/merkle/src/merkle_tree.zig:206-233), leaf level first."""
    out, pos = [], leaf_count + index
    while pos > 1:
        out.append(nodes[pos ^ 1])
        pos >>= 1
    return out


def fri_prove(p: int, num_bytes: int, transcript: Transcript, evals: list[int], log_domain: int, log_final: int,
              log_residual: int, num_queries: int) -> dict:
    """proveOn (libs/fri/src/root.zig:335-503) over Domain(F): commit, absorb the root, draw
    alpha, fold, per round; the residual = the first 2^log_residual coefficients of the final
    layer's interpolant (interpolateToCoeffs), absorbed; then per query e0 = challengeU64 % n
    and, per round, the pair at j = e mod half and its Merkle path (buildQueries)."""
    rounds = log_domain - log_final
    layers, trees, roots = [list(evals)], [], []
    for r in range(rounds):
        nodes = fri_commit_layer(layers[r], num_bytes)
        trees.append(nodes)
        roots.append(nodes[1])
        transcript.absorb_bytes(nodes[1])
        alpha = transcript.challenge_field_checked(p, num_bytes)
        layers.append(fri_fold_values(layers[r], alpha, p))
    coeffs = inverse_transform(layers[rounds], primitive_root(p, log_final), p)
    residual = [to_bytes(c, num_bytes) for c in coeffs[:1 << log_residual]]
    for cb in residual:
        transcript.absorb_bytes(cb)
    queries = []
    for _ in range(num_queries):
        e0 = transcript.challenge_u64() % (1 << log_domain)
        e, values, paths = e0, [], []
        for r in range(rounds):
            half = len(layers[r]) // 2
            j = e % half
            values.append(to_bytes(layers[r][j], num_bytes) + to_bytes(layers[r][j + half], num_bytes))
            paths.append(merkle_siblings(trees[r], half, j))
            e = j
        queries.append({"pair_index": e0, "values": values, "paths": paths})
    return {"roots": roots, "residual": residual, "queries": queries, "log_domain": log_domain,
            "log_final": log_final, "log_residual_degree": log_residual}


def fri_verify(p: int, num_bytes: int, transcript: Transcript, proof: dict, log_domain: int, log_final: int,
               log_residual: int, num_queries: int) -> bool:
    """verifyOn (libs/fri/src/root.zig:606-720) over Domain(F): replay the challenges, evaluate
    the residual on the final domain, and per query check the pair index, every Merkle path
    (MerkleTree.verifyPath: the sibling's side from the index), the fold into the next round's
    pair and, in the last round, into the residual's evaluation."""
    rounds = log_domain - log_final
    if (proof["log_domain"], proof["log_final"], proof["log_residual_degree"]) != (log_domain, log_final,
                                                                                 log_residual):
        return False
    if len(proof["roots"]) != rounds or len(proof["residual"]) != 1 << log_residual:
        return False
    if len(proof["queries"]) != num_queries:
        return False
    alphas = []
    for root in proof["roots"]:
        transcript.absorb_bytes(root)
        alphas.append(transcript.challenge_field_checked(p, num_bytes))
    residual = []
    for cb in proof["residual"]:
        c = int.from_bytes(cb, "little")
        if len(cb) != num_bytes or c >= p:
            return False
        residual.append(c)
        transcript.absorb_bytes(cb)
    gf = primitive_root(p, log_final)
    final = [sum(c * pow(gf, i * k, p) for k, c in enumerate(residual)) % p for i in range(1 << log_final)]
    inv2 = pow(2, -1, p)
    for q in proof["queries"]:
        if q["pair_index"] != transcript.challenge_u64() % (1 << log_domain):
            return False
        if len(q["values"]) != rounds or len(q["paths"]) != rounds:
            return False
        e = q["pair_index"]
        for r in range(rounds):
            layer_log = log_domain - r
            half = (1 << layer_log) // 2
            j = e % half
            vb = q["values"][r]
            x, negx = int.from_bytes(vb[:num_bytes], "little"), int.from_bytes(vb[num_bytes:], "little")
            if len(vb) != 2 * num_bytes or x >= p or negx >= p:
                return False
            cur, idx = blake3(vb), j
            if len(q["paths"][r]) != layer_log - 1:
                return False
            for sib in q["paths"][r]:
                cur = blake3(cur + sib if idx % 2 == 0 else sib + cur)
                idx >>= 1
            if cur != proof["roots"][r]:
                return False
            xv = pow(primitive_root(p, layer_log), j, p)
            expected = ((x + negx) * inv2 + alphas[r] * (x - negx) * pow(xv, -1, p) * inv2) % p
            if r + 1 < rounds:
                nb = q["values"][r + 1]
                slot = 0 if j < half // 2 else 1
                if expected != int.from_bytes(nb[slot * num_bytes:(slot + 1) * num_bytes], "little"):
                    return False
            elif expected != final[j]:
                return False
            e = j
    return True


def merkle_commit_rows(columns: list[list[int]], num_bytes: int) -> list[bytes]:
    """MerkleTree.init (libs/merkle/src/merkle_tree.zig:70-103) over the rows of equal-length
    columns: leaf i = BLAKE3 of toBytes(col_0[i]) || ... || toBytes(col_{m-1}[i]), leaf count
    padded to a power of two with BLAKE3 of the empty string, nodes[i] = BLAKE3(nodes[2i] ||
    nodes[2i+1]).  Returns nodes[0 .. 2 * leaf_count) with nodes[0] all zero."""
    n = len(columns[0])
    count = 1
    while count < n:
        count *= 2
    nodes = [bytes(32)] * (2 * count)
    for i in range(n):
        nodes[count + i] = blake3(b"".join(to_bytes(col[i], num_bytes) for col in columns))
    for i in range(n, count):
        nodes[count + i] = blake3(b"")
    for i in range(count - 1, 0, -1):
        nodes[i] = blake3(nodes[2 * i] + nodes[2 * i + 1])
    return nodes
