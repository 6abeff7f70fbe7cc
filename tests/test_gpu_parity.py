"""Parity of the CUDA path with the oracle, through the C ABI (needs a B200).

Every comparison is bit-exact: all arithmetic is exact modular arithmetic and
both sides reduce fully, so equal inputs must give equal limbs.  Mirrors the
reference's NTT tests (libs/ntt/src/root.zig:290-738) and adds sizes, fields
and device-level checks the reference cannot reach.
"""
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


def _fields(z):
    return [(z.BN254_FR, O.BN254_FR), (z.BLS12_381_FR, O.BLS12_381_FR)]


def _torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _to_dev(a: np.ndarray):
    torch = _torch()
    return torch.from_numpy(a.view(np.int64).copy()).cuda()


def _to_host(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64).reshape(-1, 4).copy()


# --- device arithmetic ---------------------------------------------------------

def test_device_field_arithmetic_matches_oracle(z):
    for F, fid in _fields(z):
        p = O.MODULI[fid]
        edge = [0, 1, 2, p - 1, p - 2, (p - 1) // 2, (p + 1) // 2, (1 << 255) % p, (1 << 128) % p, 0xFFFFFFFF]
        xs = [a for a in edge for _ in edge]
        ys = [b for _ in edge for b in edge]
        a = np.concatenate([O.to_mont(fid, O.from_ints(xs)), O.random_elements(fid, 1, 20000)])
        b = np.concatenate([O.to_mont(fid, O.from_ints(ys)), O.random_elements(fid, 2, 20000)])
        da, db = _to_dev(a), _to_dev(b)
        out = _torch().empty_like(da)
        for op in ("mul", "add", "sub", "neg"):
            z.elementwise_device(F, op, da.data_ptr(), db.data_ptr(), out.data_ptr(), len(a))
            _torch().cuda.synchronize()
            want = O.elementwise(fid, op, a, None if op == "neg" else b)
            np.testing.assert_array_equal(_to_host(out), want, err_msg=f"{F} {op}")


def test_random_elements_match_sequential_draw(z):
    torch = _torch()
    for F, fid in _fields(z):
        for seed, count in [(0, 1), (7, 33), (12, 4096), (99, 150001)]:
            out = torch.empty(count * 4, dtype=torch.int64, device="cuda")
            z.random_elements(F, seed, out.data_ptr(), count)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(_to_host(out), O.random_elements(fid, seed, count))


# --- known answers and the definition ---------------------------------------------

def test_fr_golden_transforms(z):
    import make_golden
    for c in json.load(open(os.path.join(GOLDEN, "fr_transforms.json"))):
        F = z.BN254_FR if c["field"] == "bn254_fr" else z.BLS12_381_FR
        fid = F.id
        log_n = c["log_n"]
        x = O.random_elements(fid, c["seed"], 1 << log_n)
        root = z.primitiveRootOfUnity(F, log_n)
        fwd, inv = x.copy(), x.copy()
        z.ntt(F, fwd, log_n, root)
        z.intt(F, inv, log_n, root)
        tw = z.precomputeTwiddles(F, log_n, root)
        fwd2, inv2 = x.copy(), x.copy()
        z.nttWithTwiddles(F, fwd2, log_n, tw)
        z.inttWithTwiddles(F, inv2, log_n, tw)
        z.freeTwiddles(F, tw)
        canon = lambda a: O.to_ints(O.from_mont(fid, a))
        if "forward" in c:
            assert canon(fwd) == [int(v, 16) for v in c["forward"]]
            assert canon(inv) == [int(v, 16) for v in c["inverse"]]
        else:
            assert make_golden.vec_digest(canon(fwd)) == c["forward_sha256"]
            assert make_golden.vec_digest(canon(inv)) == c["inverse_sha256"]
        np.testing.assert_array_equal(fwd, fwd2)
        np.testing.assert_array_equal(inv, inv2)


# --- parity with the oracle at every size up to 2^16 ------------------------------------

@pytest.mark.parametrize("log_n", list(range(0, 17)))
def test_transforms_match_oracle(z, log_n):
    for F, fid in _fields(z):
        n = 1 << log_n
        x = O.random_elements(fid, 1000 + log_n, n)
        root = z.primitiveRootOfUnity(F, log_n)
        # ntt / intt
        got, want = x.copy(), x.copy()
        z.ntt(F, got, log_n, root)
        assert O.ntt(fid, want, log_n, root) == 0
        np.testing.assert_array_equal(got, want)
        got_i, want_i = x.copy(), x.copy()
        z.intt(F, got_i, log_n, root)
        assert O.intt(fid, want_i, log_n, root) == 0
        np.testing.assert_array_equal(got_i, want_i)
        # precomputeTwiddles: same table as the reference's layout
        tw = z.precomputeTwiddles(F, log_n, root)
        st, otw = O.precompute_twiddles(fid, log_n, root)
        assert len(tw) == log_n
        for s in range(log_n):
            np.testing.assert_array_equal(tw[s], otw[s])
        got2 = x.copy()
        z.nttWithTwiddles(F, got2, log_n, tw)
        np.testing.assert_array_equal(got2, want)
        got3 = x.copy()
        z.inttWithTwiddles(F, got3, log_n, tw)
        want3 = x.copy()
        assert O.ntt_with_twiddles(fid, want3, log_n, otw, inverse=True) == 0
        np.testing.assert_array_equal(got3, want3)
        # round trip
        z.inttWithTwiddles(F, got2, log_n, tw)
        np.testing.assert_array_equal(got2, x)
        z.freeTwiddles(F, tw)


def test_bit_reverse_matches_oracle(z):
    for log_n in [0, 1, 2, 5, 12, 17]:
        x = O.random_elements(O.BN254_FR, log_n, 1 << log_n)
        got, want = x.copy(), x.copy()
        z.bitReverse(z.BN254_FR, got)
        O.bit_reverse(O.BN254_FR, want)
        np.testing.assert_array_equal(got, want)


def test_foreign_and_non_root_tables(z):
    """root is not validated (libs/ntt/README.md): a non-root and a caller-built table
    must give exactly the reference network's output, including tw[s][0] != 1."""
    for F, fid in _fields(z):
        log_n = 13
        x = O.random_elements(fid, 5, 1 << log_n)
        w = O.from_int(fid, 7)
        got, want = x.copy(), x.copy()
        z.ntt(F, got, log_n, w)
        O.ntt(fid, want, log_n, w)
        np.testing.assert_array_equal(got, want)
        got, want = x.copy(), x.copy()
        z.intt(F, got, log_n, w)
        O.intt(fid, want, log_n, w)
        np.testing.assert_array_equal(got, want)
        # A table the library never made: random stages.
        table = [O.random_elements(fid, 50 + s, 1 << s) for s in range(log_n)]
        for inverse in (False, True):
            got, want = x.copy(), x.copy()
            (z.inttWithTwiddles if inverse else z.nttWithTwiddles)(F, got, log_n, table)
            assert O.ntt_with_twiddles(fid, want, log_n, table, inverse=inverse) == 0
            np.testing.assert_array_equal(got, want)


def test_registered_table_is_recognised_and_rechecked(z):
    F, fid = z.BN254_FR, O.BN254_FR
    log_n = 12
    root = z.primitiveRootOfUnity(F, log_n)
    tw = z.precomputeTwiddles(F, log_n, root)
    x = O.random_elements(fid, 77, 1 << log_n)
    want = x.copy()
    O.ntt(fid, want, log_n, root)
    got = x.copy()
    z.nttWithTwiddles(F, got, log_n, tw)
    np.testing.assert_array_equal(got, want)
    # Rewrite the table in place (through the const-less numpy view): the
    # library must notice the changed pinning entries and use the new contents.
    other = O.from_int(fid, 3)
    st, otw = O.precompute_twiddles(fid, log_n, other)
    for s in range(log_n):
        tw[s][:] = otw[s]
    got = x.copy()
    z.nttWithTwiddles(F, got, log_n, tw)
    want = x.copy()
    O.ntt_with_twiddles(fid, want, log_n, otw)
    np.testing.assert_array_equal(got, want)
    z.freeTwiddles(F, tw)


def test_errors_leave_data_untouched(z):
    F, fid = z.BN254_FR, O.BN254_FR
    root = z.primitiveRootOfUnity(F, 3)
    tw = z.precomputeTwiddles(F, 3, root)
    d = O.random_elements(fid, 1, 8)
    before = d.copy()
    with pytest.raises(z.InvalidTwiddles):
        z.nttWithTwiddles(F, d, 3, [tw[0], tw[1][:1], tw[2]])
    np.testing.assert_array_equal(d, before)  # zig-ntt would have mutated it
    with pytest.raises(z.InvalidTwiddles):
        z.inttWithTwiddles(F, d, 3, tw[:2])
    np.testing.assert_array_equal(d, before)
    z.freeTwiddles(F, tw)


@pytest.mark.parametrize("log_n", [10, 11, 16, 21])
def test_lazy_reduction_bounds(z, log_n):
    """Inputs and caller tables that push every butterfly to its bounds.  BN254-Fr keeps values in
    [0, 2p) inside a pass and skips each product's final subtraction; with every element and
    every twiddle at p - 1 (raw limbs, so tw[s][0] != 1 and every butterfly multiplies) the sums
    and differences meet 2p - 2 and the products their largest inputs.  Also alternating 0 / p - 1
    data, and p - 1 data against tables of 1, of Montgomery one and of 0 (the inverse multiplies
    by p - tw, which is p for a zero entry: still a valid factor).  Under the default plan
    (2^11-element tiles, at most 10 stages per pass) 2^10 and 2^11 run one pass, 2^16 two and
    2^21 three, so every pass boundary's reduction to [0, p) is crossed.  Both directions,
    nttWithTwiddles / inttWithTwiddles (libs/ntt/src/root.zig:148-212; the arithmetic is
    libs/field/src/montgomery.zig:197-297), against the oracle bit for bit."""
    n = 1 << log_n
    for F, fid in _fields(z):
        p = O.MODULI[fid]
        pm1 = np.array(O.int_to_limbs(p - 1), dtype=np.uint64)
        one = np.array(O.int_to_limbs(1), dtype=np.uint64)
        mont_one = O.from_int(fid, 1)
        zero = np.zeros(4, dtype=np.uint64)

        def filled(v, count):
            return np.ascontiguousarray(np.tile(v, (count, 1)))

        alternating = np.ascontiguousarray(np.where((np.arange(n) % 2 == 0)[:, None], zero, pm1))
        cases = [("p-1 data, p-1 table", filled(pm1, n), pm1),
                 ("alternating 0/p-1 data, p-1 table", alternating, pm1),
                 ("p-1 data, table of 1", filled(pm1, n), one),
                 ("p-1 data, table of Montgomery one", filled(pm1, n), mont_one),
                 ("p-1 data, table of 0", filled(pm1, n), zero)]
        for name, x, tv in cases:
            table = [filled(tv, 1 << s) for s in range(log_n)]
            for inverse in (False, True):
                got, want = x.copy(), x.copy()
                (z.inttWithTwiddles if inverse else z.nttWithTwiddles)(F, got, log_n, table)
                assert O.ntt_with_twiddles(fid, want, log_n, table, inverse=inverse, workers=WORKERS,
                                           inplace4=True) == 0
                np.testing.assert_array_equal(got, want, err_msg=f"{F} 2^{log_n} {name} inverse={inverse}")


def test_convolution_property(z):
    F, fid = z.BLS12_381_FR, O.BLS12_381_FR
    p = O.MODULI[fid]
    log_n, n = 10, 1 << 10
    rng = np.random.default_rng(3)
    fv = [int(v) for v in rng.integers(0, 1 << 62, n // 2)] + [0] * (n // 2)
    gv = [int(v) for v in rng.integers(0, 1 << 62, n // 2)] + [0] * (n // 2)
    root = z.primitiveRootOfUnity(F, log_n)
    a = O.to_mont(fid, O.from_ints(fv))
    b = O.to_mont(fid, O.from_ints(gv))
    z.ntt(F, a, log_n, root)
    z.ntt(F, b, log_n, root)
    c = O.elementwise(fid, "mul", a, b)
    z.intt(F, c, log_n, root)
    conv = [0] * n
    for i, fi in enumerate(fv[: n // 2]):
        for j, gj in enumerate(gv[: n // 2]):
            conv[(i + j) % n] = (conv[(i + j) % n] + fi * gj) % p
    assert O.to_ints(O.from_mont(fid, c)) == conv


# --- device-resident API ------------------------------------------------------------------

@pytest.mark.parametrize("log_n", [1, 11, 12, 18])
def test_device_api_in_and_out_of_place(z, log_n):
    torch = _torch()
    for F, fid in _fields(z):
        n = 1 << log_n
        x = torch.empty(n * 4, dtype=torch.int64, device="cuda")
        z.random_elements(F, 31 + log_n, x.data_ptr(), n)
        root = z.primitiveRootOfUnity(F, log_n)
        host = _to_host(x)
        want = host.copy()
        O.ntt(fid, want, log_n, root)
        with z.DeviceTwiddles(F, log_n, root) as tw:
            y = torch.empty_like(x)
            z.ntt_device(tw, x.data_ptr(), y.data_ptr(), z.FORWARD)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(_to_host(y), want)
            # in place with an explicit scratch, then in place borrowing one
            xi = x.clone()
            s = torch.empty_like(x)
            torch.cuda.synchronize()  # the clone runs on torch's stream, the library on its own
            z.ntt_device(tw, xi.data_ptr(), xi.data_ptr(), z.FORWARD, d_scratch=s.data_ptr())
            torch.cuda.synchronize()
            np.testing.assert_array_equal(_to_host(xi), want)
            z.ntt_device(tw, xi.data_ptr(), xi.data_ptr(), z.INVERSE)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(_to_host(xi), host)


# --- large sizes -------------------------------------------------------------------------

@pytest.mark.parametrize("log_n", [20, 22])
def test_large_transforms_match_oracle(z, log_n):
    F, fid = z.BN254_FR, O.BN254_FR
    n = 1 << log_n
    torch = _torch()
    x = torch.empty(n * 4, dtype=torch.int64, device="cuda")
    z.random_elements(F, 2024 + log_n, x.data_ptr(), n)
    host = _to_host(x)
    root = z.primitiveRootOfUnity(F, log_n)
    st, otw = O.precompute_twiddles(fid, log_n, root)
    want = host.copy()
    assert O.ntt_with_twiddles(fid, want, log_n, otw, workers=WORKERS, inplace4=True) == 0
    got = host.copy()
    tw = z.precomputeTwiddles(F, log_n, root)
    z.nttWithTwiddles(F, got, log_n, tw)
    np.testing.assert_array_equal(got, want)
    z.inttWithTwiddles(F, got, log_n, tw)
    np.testing.assert_array_equal(got, host)
    z.freeTwiddles(F, tw)


@pytest.mark.parametrize("fname,log_n", [("BN254_FR", 24), ("BLS12_381_FR", 23)])
def test_full_size_properties(z, fname, log_n):
    """At the benchmark size: inverse(forward(x)) == x, linearity, and outputs
    at spread indices equal to the definition sum_j x_j w^(jk)."""
    F = getattr(z, fname)
    fid = F.id
    torch = _torch()
    n = 1 << log_n
    x = torch.empty(n * 4, dtype=torch.int64, device="cuda")
    y = torch.empty_like(x)
    z.random_elements(F, 4242, x.data_ptr(), n)
    z.random_elements(F, 4343, y.data_ptr(), n)
    root = z.primitiveRootOfUnity(F, log_n)
    with z.DeviceTwiddles(F, log_n, root) as tw:
        X = torch.empty_like(x)
        z.ntt_device(tw, x.data_ptr(), X.data_ptr(), z.FORWARD)
        back = torch.empty_like(x)
        z.ntt_device(tw, X.data_ptr(), back.data_ptr(), z.INVERSE)
        torch.cuda.synchronize()
        assert torch.equal(back, x)
        # linearity: NTT(x + y) == NTT(x) + NTT(y)
        s = torch.empty_like(x)
        z.elementwise_device(F, "add", x.data_ptr(), y.data_ptr(), s.data_ptr(), n)
        S = torch.empty_like(x)
        z.ntt_device(tw, s.data_ptr(), S.data_ptr(), z.FORWARD)
        Y = torch.empty_like(x)
        z.ntt_device(tw, y.data_ptr(), Y.data_ptr(), z.FORWARD)
        XY = torch.empty_like(x)
        z.elementwise_device(F, "add", X.data_ptr(), Y.data_ptr(), XY.data_ptr(), n)
        torch.cuda.synchronize()
        assert torch.equal(S, XY)
    ks = [0, 1, 2, 3, n // 2, n // 2 + 1, n - 1, 12345, 987654 % n]
    pts = O.dft_points(fid, _to_host(x), root, ks, workers=WORKERS)
    Xh = _to_host(X)
    np.testing.assert_array_equal(Xh[ks], pts)


@pytest.mark.parametrize("log_n", [3, 16, 20])
def test_pipelined_host_vectors_match_single_calls(z, log_n):
    torch = _torch()
    for F, fid in _fields(z):
        n = 1 << log_n
        root = z.primitiveRootOfUnity(F, log_n)
        tw_host = z.precomputeTwiddles(F, log_n, root)
        bufs, wants = [], []
        for i in range(5):
            x = O.random_elements(fid, 700 + i, n) if log_n < 20 else None
            if x is None:
                d = torch.empty(n * 4, dtype=torch.int64, device="cuda")
                z.random_elements(F, 700 + i, d.data_ptr(), n)
                x = _to_host(d)
            pinned = torch.empty(n * 4, dtype=torch.int64, pin_memory=True)
            pinned.numpy().view(np.uint64)[:] = x.reshape(-1)
            w = x.copy()
            z.inttWithTwiddles(F, w, log_n, tw_host) if i % 2 else z.nttWithTwiddles(F, w, log_n, tw_host)
            bufs.append(pinned)
            wants.append(w)
        with z.DeviceTwiddles(F, log_n, root) as tw:
            fw = [b.data_ptr() for i, b in enumerate(bufs) if i % 2 == 0]
            iv = [b.data_ptr() for i, b in enumerate(bufs) if i % 2 == 1]
            z.ntt_host_many(tw, fw, z.FORWARD)
            z.ntt_host_many(tw, iv, z.INVERSE)
        for b, w in zip(bufs, wants):
            np.testing.assert_array_equal(b.numpy().view(np.uint64).reshape(-1, 4), w)
        z.freeTwiddles(F, tw_host)


def test_largest_order_transform(z):
    """BN254-Fr at its two-adicity, 2^28 (8 GiB per vector; the plan's later passes have tile
    rows of one element): inverse(forward(x)) == x, and forward outputs at sampled indices equal
    the definition sum_j x_j w^(jk)."""
    torch = _torch()
    F = z.BN254_FR
    log_n = F.two_adicity
    n = 1 << log_n
    x = torch.empty(n * 4, dtype=torch.int64, device="cuda")
    z.random_elements(F, 2828, x.data_ptr(), n)
    root = z.primitiveRootOfUnity(F, log_n)
    X = torch.empty_like(x)
    with z.DeviceTwiddles(F, log_n, root) as tw:
        z.ntt_device(tw, x.data_ptr(), X.data_ptr(), z.FORWARD)
        back = torch.empty_like(x)
        z.ntt_device(tw, X.data_ptr(), back.data_ptr(), z.INVERSE)
        torch.cuda.synchronize()
        assert torch.equal(back, x)
        del back
    ks = [0, 1, n // 2 + 7, n - 1]
    pts = O.dft_points(F.id, _to_host(x), root, ks, workers=WORKERS)
    np.testing.assert_array_equal(_to_host(X)[ks], pts)


def test_init_is_idempotent_and_keeps_its_device(z):
    """The Zig shim calls zntt_init(0) on every entry point: a repeated call on the same device
    returns OK at once, and a call naming another device is refused without disturbing the
    library."""
    L = z.lib()
    assert L.zntt_init(0) == 0
    assert L.zntt_init(0) == 0
    with pytest.raises(z.ZnttError):
        z._check(L.zntt_init(1))
    assert L.zntt_init(0) == 0
    root = z.primitiveRootOfUnity(z.BN254_FR, 10)
    x = O.random_elements(O.BN254_FR, 91, 1 << 10)
    want = x.copy()
    st, tw = O.precompute_twiddles(O.BN254_FR, 10, root)
    O.ntt_with_twiddles(O.BN254_FR, want, 10, tw, inverse=False, workers=1, inplace4=True)
    got = x.copy()
    z.ntt(z.BN254_FR, got, 10, root)
    np.testing.assert_array_equal(got, want)
