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
* Roots of unity as the reference derives them (libs/field/src/roots.zig:149-158):
  z = the first quadratic non-residue counting up from 2, raised to
  odd_part << (two_adicity - log_n).
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
