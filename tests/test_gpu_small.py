"""Goldilocks and BabyBear (zig-field's SmallField backend) through the zig-ntt entry
points on the device: the reference's own known-answer transform test
(libs/ntt/src/root.zig:399-453, vectors in tests/golden/ntt_kat.json), the oracle
at sizes across the pass boundaries, caller-made tables with zig-ntt's per-stage
semantics, and a full-size device round trip.  Needs a B200."""
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
    return [(z.GOLDILOCKS, O.GOLDILOCKS), (z.BABYBEAR, O.BABYBEAR)]


def _canon(fid, slots):
    """Oracle Montgomery slots (limb 0 used by the 64-bit fields) -> canonical u64 vector
    (the device layout)."""
    return np.ascontiguousarray(O.from_mont(fid, np.ascontiguousarray(slots))[:, 0])


def _slots(fid, values):
    s = O.elems(len(values))
    s[:, 0] = np.asarray(values, dtype=np.uint64)
    return O.to_mont(fid, s)


def _random(fid, seed, n):
    return _canon(fid, O.random_elements(fid, seed, n))


def _oracle_transform(fid, x, log_n, stages_canon, inverse):
    """nttWithTwiddles / inttWithTwiddles of the oracle on canonical data and a canonical table."""
    data = _slots(fid, x)
    stages = [_slots(fid, s) for s in stages_canon]
    st = O.ntt_with_twiddles(fid, data, log_n, stages, inverse=inverse, workers=WORKERS)
    assert st == O.OK
    return _canon(fid, data)


def test_reference_known_answer_transforms(z):
    """The reference's KAT: ntt with the given root gives `expect`, intt returns the input;
    the same through precomputeTwiddles / nttWithTwiddles / inttWithTwiddles."""
    cases = json.load(open(os.path.join(GOLDEN, "ntt_kat.json")))
    by_name = {"goldilocks": z.GOLDILOCKS, "babybear": z.BABYBEAR}
    assert len(cases) == 8
    for c in cases:
        F = by_name[c["field"]]
        L = c["log_n"]
        inp = np.array([int(v, 16) for v in c["input"]], dtype=np.uint64)
        exp = np.array([int(v, 16) for v in c["expect"]], dtype=np.uint64)
        root = np.array([int(c["root"], 16), 0, 0, 0], dtype=np.uint64)
        np.testing.assert_array_equal(z.primitiveRootOfUnity(F, L), root, err_msg=c["source"])
        data = inp.copy()
        z.ntt(F, data, L, root)
        np.testing.assert_array_equal(data, exp, err_msg=c["source"])
        z.intt(F, data, L, root)
        np.testing.assert_array_equal(data, inp, err_msg=c["source"])
        tw = z.precomputeTwiddles(F, L, root)
        data = inp.copy()
        z.nttWithTwiddles(F, data, L, tw)
        np.testing.assert_array_equal(data, exp, err_msg=c["source"])
        z.inttWithTwiddles(F, data, L, tw)
        np.testing.assert_array_equal(data, inp, err_msg=c["source"])
        z.freeTwiddles(F, tw)


@pytest.mark.parametrize("log_n", [1, 2, 5, 11, 12, 13, 16, 20, 23])
def test_transforms_match_oracle(z, log_n):
    """Forward and inverse through the registered table, a caller's copy of it (uploaded
    with zig-ntt's semantics) and ntt(root), against the oracle: one pass up to 2^12,
    two or three passes beyond."""
    for F, fid in _fields(z):
        n = 1 << log_n
        x = _random(fid, 600 + log_n, n)
        root = z.primitiveRootOfUnity(F, log_n)
        tw = z.precomputeTwiddles(F, log_n, root)
        st, ostages = O.precompute_twiddles(fid, log_n, _slots(fid, [int(root[0])])[0])
        assert st == O.OK
        for s in range(log_n):
            np.testing.assert_array_equal(tw[s], _canon(fid, ostages[s]), err_msg=f"{F.name} stage {s}")
        copy = [np.array(t) for t in tw]
        for inverse in (False, True):
            want = _oracle_transform(fid, x, log_n, copy, inverse)
            for table in (tw, copy):
                data = x.copy()
                (z.inttWithTwiddles if inverse else z.nttWithTwiddles)(F, data, log_n, table)
                np.testing.assert_array_equal(data, want, err_msg=f"{F.name} 2^{log_n} inverse={inverse}")
        data = x.copy()
        z.ntt(F, data, log_n, root)
        np.testing.assert_array_equal(data, _oracle_transform(fid, x, log_n, copy, False))
        z.intt(F, data, log_n, root)
        np.testing.assert_array_equal(data, x)
        z.freeTwiddles(F, tw)


@pytest.mark.parametrize("log_n", [3, 12, 14])
def test_caller_tables_with_arbitrary_entries(z, log_n):
    """A caller's table of arbitrary values (entry 0 of a stage not one) runs zig-ntt's exact
    per-stage arithmetic (root.zig:148-212), as the oracle does."""
    for F, fid in _fields(z):
        rng = np.random.default_rng(log_n)
        stages = [np.ascontiguousarray(rng.integers(0, F.modulus, 1 << s, dtype=np.uint64)) for s in range(log_n)]
        x = _random(fid, 700 + log_n, 1 << log_n)
        for inverse in (False, True):
            want = _oracle_transform(fid, x, log_n, stages, inverse)
            data = x.copy()
            (z.inttWithTwiddles if inverse else z.nttWithTwiddles)(F, data, log_n, stages)
            np.testing.assert_array_equal(data, want, err_msg=f"{F.name} 2^{log_n} inverse={inverse}")


def test_bit_reverse_small(z):
    for F, _ in _fields(z):
        for log_n in (0, 1, 4, 13):
            n = 1 << log_n
            x = np.arange(n, dtype=np.uint64) * 7 + 1
            data = x.copy()
            z.bitReverse(F, data)
            rev = [int(format(i, f"0{log_n}b")[::-1], 2) if log_n else 0 for i in range(n)]
            np.testing.assert_array_equal(data[rev], x)


def test_device_api_full_size(z):
    """Device-resident transforms: 2^24 Goldilocks and 2^22 BabyBear forward outputs at
    sampled indices equal the DFT by definition (Horner in the oracle); 2^24 and 2^27
    (BabyBear's two-adicity) round trips, out of place and in place, return the input."""
    torch = pytest.importorskip("torch")
    for (F, fid), log_check, log_trip in zip(_fields(z), (24, 22), (24, 27)):
        for log_n in sorted({log_check, log_trip}):
            n = 1 << log_n
            rng = np.random.default_rng(900 + log_n)
            xs = rng.integers(0, F.modulus, n, dtype=np.uint64)
            x = torch.from_numpy(xs.view(np.int64)).cuda()
            y = torch.empty_like(x)
            back = torch.empty_like(x)
            root = z.primitiveRootOfUnity(F, log_n)
            with z.DeviceTwiddles(F, log_n, root) as t:
                z.ntt_device(t, x.data_ptr(), y.data_ptr(), z.FORWARD)
                torch.cuda.synchronize()  # the library runs on its own stream, not torch's
                fwd = y.clone()
                torch.cuda.synchronize()
                z.ntt_device(t, y.data_ptr(), back.data_ptr(), z.INVERSE)
                z.ntt_device(t, y.data_ptr(), y.data_ptr(), z.INVERSE)  # in place (pooled scratch)
            torch.cuda.synchronize()
            assert torch.equal(back, x) and torch.equal(y, x), f"{F.name} 2^{log_n}"
            if log_n == log_check:
                ks = [0, 1, 2, 12345, n // 2, n - 1]
                want = _canon(fid, O.dft_points(fid, _slots(fid, xs), _slots(fid, [int(root[0])])[0], ks,
                                                workers=WORKERS))
                np.testing.assert_array_equal(fwd.cpu().numpy().view(np.uint64)[ks], want)
            del x, y, back, fwd
            torch.cuda.empty_cache()


@pytest.mark.parametrize("log_in,log_blowup", [(0, 1), (4, 2), (10, 1), (13, 2), (18, 2)])
def test_coset_lde_matches_oracle(z, log_in, log_blowup):
    """zntt_coset_lde_device with small-field tables against the oracle's composition
    (inttWithTwiddles, zero padding, powers(shift) hadamard, nttWithTwiddles; the oracle's
    zo_coset_lde), shift 7, one and several passes on either side."""
    torch = pytest.importorskip("torch")
    for F, fid in _fields(z):
        log_out = log_in + log_blowup
        x = _random(fid, 800 + log_in, 1 << log_in)
        want = _canon(fid, O.coset_lde(fid, _slots(fid, x), log_in, log_blowup, _slots(fid, [7])[0], workers=WORKERS))
        src = torch.from_numpy(x.view(np.int64).copy()).cuda()
        out = torch.empty(1 << log_out, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        with z.DeviceTwiddles(F, log_in, z.primitiveRootOfUnity(F, log_in)) as ti, \
                z.DeviceTwiddles(F, log_out, z.primitiveRootOfUnity(F, log_out)) as to:
            z.coset_lde_device(ti, to, np.array([7, 0, 0, 0], dtype=np.uint64), src.data_ptr(), out.data_ptr())
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy().view(np.uint64), want, err_msg=f"{F.name} 2^{log_in}")


def test_coset_lde_argument_checks(z):
    """A shift that is not a nonzero canonical element, tables of two fields, and an output
    overlapping the input are refused."""
    torch = pytest.importorskip("torch")
    F = z.GOLDILOCKS
    buf = torch.zeros(1 << 12, dtype=torch.int64, device="cuda")
    with z.DeviceTwiddles(F, 4, z.primitiveRootOfUnity(F, 4)) as t, \
            z.DeviceTwiddles(F, 6, z.primitiveRootOfUnity(F, 6)) as t6, \
            z.DeviceTwiddles(z.BABYBEAR, 6, z.primitiveRootOfUnity(z.BABYBEAR, 6)) as b6, \
            z.DeviceTwiddles(z.BN254_FR, 6, z.primitiveRootOfUnity(z.BN254_FR, 6)) as w6:
        for shift in ([0, 0, 0, 0], [F.modulus, 0, 0, 0], [5, 1, 0, 0]):
            with pytest.raises(z.InvalidArgument):
                z.coset_lde_device(t, t6, np.array(shift, dtype=np.uint64), buf.data_ptr(), buf[2048:].data_ptr())
        for other in (b6, w6):
            with pytest.raises(z.InvalidArgument):
                z.coset_lde_device(t, other, np.array([7, 0, 0, 0], dtype=np.uint64), buf.data_ptr(),
                                   buf[2048:].data_ptr())
        with pytest.raises(z.InvalidArgument):
            z.coset_lde_device(t, t6, np.array([7, 0, 0, 0], dtype=np.uint64), buf.data_ptr(), buf[8:].data_ptr())


def test_small_tables_are_refused_by_256_bit_entry_points(z):
    torch = pytest.importorskip("torch")
    F = z.GOLDILOCKS
    buf = torch.zeros(1 << 12, dtype=torch.int64, device="cuda")
    with z.DeviceTwiddles(F, 4, z.primitiveRootOfUnity(F, 4)) as t, \
            z.DeviceTwiddles(F, 6, z.primitiveRootOfUnity(F, 6)) as t6:
        with pytest.raises(z.UnsupportedField):
            z.poly_mul_device(t6, buf.data_ptr(), 3, buf[1024:].data_ptr(), 3, buf[2048:].data_ptr())
        with pytest.raises(z.UnsupportedField):
            z._check(z.lib().zntt_ntt_device_inplace_noalloc(t.handle, buf.data_ptr(), z.FORWARD, None))
        with pytest.raises((z.UnsupportedField, z.InvalidArgument)):
            z.Batch(z.BN254_FR, [{"kind": z.JOB_NTT, "tw": t, "mode": z.FORWARD, "src": buf.data_ptr(),
                                  "dst": buf[1024:].data_ptr()}])


@pytest.mark.parametrize("la,lb", [(1, 1), (5, 3), (300, 200), (1 << 12, 1 << 12), ((1 << 15) + 3, 1 << 14)])
def test_poly_mul_matches_oracle(z, la, lb):
    """zntt_poly_mul over Goldilocks and BabyBear against the oracle's schoolbook product
    (Polynomial.mul, libs/poly/src/poly.zig:197-212): coefficients, degree and the zero tail."""
    for F, fid in _fields(z):
        a = _random(fid, 2000 + la, la)
        b = _random(fid, 3000 + lb, lb)
        a[-1] = a[-1] or 1  # keep the leading coefficients non-zero
        b[-1] = b[-1] or 1
        max_degree = la + lb + 5
        got, deg = z.poly_mul(F, a, b, max_degree)
        workers = WORKERS if la * lb > 1 << 20 else 1
        st, want, wdeg = O.poly_mul(fid, _slots(fid, a), _slots(fid, b), max_degree, workers=workers)
        assert st == O.OK and deg == wdeg == la + lb - 2
        np.testing.assert_array_equal(got, _canon(fid, want), err_msg=f"{F.name} {la} x {lb}")


def test_coset_lde_columns_equal_single_extensions(z):
    """zntt_coset_lde_columns (the columns back to back on one stream) equals one
    zntt_coset_lde_device call per column, for the small fields and BN254-Fr."""
    torch = pytest.importorskip("torch")
    cases = [(z.GOLDILOCKS, O.GOLDILOCKS, 5), (z.BABYBEAR, O.BABYBEAR, 3), (z.BN254_FR, O.BN254_FR, 2)]
    for F, fid, m in cases:
        log_in, log_out = 10, 12
        if F.limbs == 4:
            cols = [torch.from_numpy(O.random_elements(fid, 50 + k, 1 << log_in).view(np.int64).reshape(-1).copy()).cuda()
                    for k in range(m)]
            shift = z.to_montgomery(F, 5)
        else:
            cols = [torch.from_numpy(_random(fid, 50 + k, 1 << log_in).view(np.int64).copy()).cuda() for k in range(m)]
            shift = np.array([7, 0, 0, 0], dtype=np.uint64)
        outs = [torch.empty((1 << log_out) * F.limbs, dtype=torch.int64, device="cuda") for _ in range(m)]
        wants = [torch.empty_like(o) for o in outs]
        torch.cuda.synchronize()
        with z.DeviceTwiddles(F, log_in, z.primitiveRootOfUnity(F, log_in)) as ti, \
                z.DeviceTwiddles(F, log_out, z.primitiveRootOfUnity(F, log_out)) as to:
            z.coset_lde_columns(ti, to, shift, [c.data_ptr() for c in cols], [o.data_ptr() for o in outs])
            for c, w in zip(cols, wants):
                z.coset_lde_device(ti, to, shift, c.data_ptr(), w.data_ptr())
        torch.cuda.synchronize()
        for k, (o, w) in enumerate(zip(outs, wants)):
            assert torch.equal(o, w), (F.name, k)


@pytest.mark.parametrize("log_n", [0, 1, 10, 13, 20])
def test_ntt_device_columns_equal_single_transforms(z, log_n):
    """zntt_ntt_device_columns (every launch over all columns) equals one zntt_ntt_device call
    per column, forward and inverse, for the small fields and BN254-Fr; in place is refused."""
    torch = pytest.importorskip("torch")
    for F, fid, m in [(z.GOLDILOCKS, O.GOLDILOCKS, 5), (z.BABYBEAR, O.BABYBEAR, 3), (z.BN254_FR, O.BN254_FR, 2)]:
        n = 1 << log_n
        if F.limbs == 4 and log_n == 0:
            continue  # the 256-bit path is one zntt_ntt_device call per column, covered elsewhere
        if F.limbs == 4:
            cols = [torch.from_numpy(O.random_elements(fid, 70 + k, n).view(np.int64).reshape(-1).copy()).cuda()
                    for k in range(m)]
        else:
            cols = [torch.from_numpy(_random(fid, 70 + k, n).view(np.int64).copy()).cuda() for k in range(m)]
        torch.cuda.synchronize()
        with z.DeviceTwiddles(F, log_n, z.primitiveRootOfUnity(F, log_n)) as t:
            for mode in (z.FORWARD, z.INVERSE):
                outs = [torch.empty_like(c) for c in cols]
                wants = [torch.empty_like(c) for c in cols]
                torch.cuda.synchronize()
                z.ntt_device_columns(t, [c.data_ptr() for c in cols], [o.data_ptr() for o in outs], mode)
                for c, w in zip(cols, wants):
                    z.ntt_device(t, c.data_ptr(), w.data_ptr(), mode)
                torch.cuda.synchronize()
                for k, (o, w) in enumerate(zip(outs, wants)):
                    assert torch.equal(o, w), (F.name, log_n, mode, k)
            if F.limbs == 1 and log_n > 0:
                with pytest.raises(z.InvalidArgument):
                    z.ntt_device_columns(t, [cols[0].data_ptr()], [cols[0].data_ptr()])
