"""Polynomial products on the device (zntt_poly_mul, zntt_poly_mul_device and the
ZNTT_JOB_POLY_MUL batch job) against the schoolbook oracle of Polynomial.mul
(libs/poly/src/poly.zig:197-212), the independent pure-Python fixture, and at
full size the evaluation property c(x) = a(x) b(x).  Needs a B200."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
WORKERS = min(os.cpu_count() or 1, 64)
FIELD_IDS = {"bn254_fr": O.BN254_FR, "bls12_381_fr": O.BLS12_381_FR}


@pytest.fixture(scope="module")
def z(zntt):
    zntt.init(0)
    return zntt


def _torch():
    import torch
    return torch


def _dev(a):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64).reshape(-1)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64).reshape(-1, 4).copy()


def _field(z, fid):
    return z.BN254_FR if fid == O.BN254_FR else z.BLS12_381_FR


def _mont(fid, hexes):
    if not hexes:
        return O.elems(0)
    return O.to_mont(fid, O.from_ints([int(v, 16) for v in hexes]))


def test_poly_mul_matches_fixture(z):
    for c in json.load(open(os.path.join(GOLDEN, "poly_mul.json"))):
        fid = FIELD_IDS[c["field"]]
        F = _field(z, fid)
        a, b = _mont(fid, c["a"]), _mont(fid, c["b"])
        if "error" in c:
            with pytest.raises(z.DegreeTooLarge):
                z.poly_mul(F, a, b, c["max_degree"])
            continue
        out, deg = z.poly_mul(F, a, b, c["max_degree"])
        assert deg == c["degree"]
        got = O.to_ints(O.from_mont(fid, out))
        want = [int(v, 16) for v in c["product"]]
        assert got[:len(want)] == want and not any(got[len(want):])


@pytest.mark.parametrize("la,lb", [(1, 1), (1, 300), (1024, 1025), (1025, 1024), (1500, 900), (2048, 2049),
                                   (3000, 2500)])
def test_poly_mul_matches_schoolbook_oracle(z, la, lb):
    """Sizes around the transform-size boundaries (len_a + len_b - 1 = 2^k and 2^k + 1) and
    across the one-pass / several-pass plans."""
    for fid in (O.BN254_FR, O.BLS12_381_FR):
        F = _field(z, fid)
        a = O.random_elements(fid, 1000 + la, la)
        b = O.random_elements(fid, 2000 + lb, lb)
        md = la + lb + 5
        out, deg = z.poly_mul(F, a, b, md)
        st, want, wdeg = O.poly_mul(fid, a, b, md, workers=WORKERS)
        assert st == O.OK and deg == wdeg == la + lb - 2
        np.testing.assert_array_equal(out, want)


def test_poly_mul_device_and_batch_jobs(z):
    """The device entry point and the batch job kind give the oracle's coefficients, with
    transform sizes larger than needed, mixed in one persistent launch with plain transforms."""
    torch = _torch()
    fid = O.BLS12_381_FR
    F = _field(z, fid)
    tabs = {}

    def tw(L):
        if L not in tabs:
            tabs[L] = z.DeviceTwiddles(F, L, z.primitiveRootOfUnity(F, L))
        return tabs[L]

    cases = [(1, 1, 0), (1, 1, 3), (3, 2, 2), (100, 29, 7), (700, 350, 11), (700, 350, 12), (2000, 2000, 12),
             (5000, 3000, 14)]
    jobs, refs, keep = [], [], []
    for q, (la, lb, L) in enumerate(cases):
        a = O.random_elements(fid, 300 + q, la)
        b = O.random_elements(fid, 400 + q, lb)
        st, want, _ = O.poly_mul(fid, a, b, la + lb - 1, workers=WORKERS)
        want = want[:la + lb - 1]
        da, db = _dev(a), _dev(b)
        out = torch.empty((la + lb - 1) * 4, dtype=torch.int64, device="cuda")
        z.poly_mul_device(tw(L), da.data_ptr(), la, db.data_ptr(), lb, out.data_ptr())
        torch.cuda.synchronize()
        np.testing.assert_array_equal(_host(out), want, err_msg=f"device {la}x{lb} on 2^{L}")
        out2 = torch.full(((la + lb - 1) * 4 + 8,), 7, dtype=torch.int64, device="cuda")
        jobs.append({"kind": z.JOB_POLY_MUL, "tw": tw(L), "src": da.data_ptr(), "len": la, "src2": db.data_ptr(),
                     "len2": lb, "dst": out2.data_ptr()})
        refs.append((out2, want))
        keep += [da, db]
    x = _dev(O.random_elements(fid, 77, 1 << 13))
    y = torch.empty_like(x)
    want_y = torch.empty_like(x)
    z.ntt_device(tw(13), x.data_ptr(), want_y.data_ptr(), z.FORWARD)
    jobs.append({"kind": z.JOB_NTT, "tw": tw(13), "mode": z.FORWARD, "src": x.data_ptr(), "dst": y.data_ptr()})
    torch.cuda.synchronize()
    with z.Batch(F, jobs) as bt:
        for graph in (False, True):
            bt.run(graph=graph)
            torch.cuda.synchronize()
            bt.status()
            for i, (out2, want) in enumerate(refs):
                got = _host(out2)
                np.testing.assert_array_equal(got[:len(want)], want, err_msg=f"batch job {i}")
                # Nothing is stored past the product (the guard words keep their value).
                assert (out2[len(want) * 4:] == 7).all()
            assert torch.equal(y, want_y)
    for t in tabs.values():
        t.close()


def test_poly_mul_device_rejects_bad_arguments(z):
    torch = _torch()
    F = z.BN254_FR
    with z.DeviceTwiddles(F, 4, z.primitiveRootOfUnity(F, 4)) as t:
        a = torch.zeros(40 * 4, dtype=torch.int64, device="cuda")
        with pytest.raises(z.InvalidArgument):  # 9 + 9 - 1 > 16 points
            z.poly_mul_device(t, a.data_ptr(), 9, a[36 * 4:].data_ptr(), 9, a[10 * 4:].data_ptr())
        with pytest.raises(z.InvalidArgument):  # the output overlaps a factor
            z.poly_mul_device(t, a.data_ptr(), 4, a[20 * 4:].data_ptr(), 4, a[2 * 4:].data_ptr())
        with pytest.raises(z.InvalidArgument):
            z.poly_mul_device(t, a.data_ptr(), 0, a[20 * 4:].data_ptr(), 4, a[30 * 4:].data_ptr())


def test_poly_mul_full_size_evaluation_property(z):
    """Two 2^23-coefficient BN254-Fr factors (a 2^24-point product): c(x) = a(x) b(x) at
    random points, the leading and constant coefficients exactly."""
    torch = _torch()
    fid = O.BN254_FR
    F = z.BN254_FR
    n = 1 << 23
    da = torch.empty(n * 4, dtype=torch.int64, device="cuda")
    db = torch.empty_like(da)
    z.random_elements(F, 31, da.data_ptr(), n)
    z.random_elements(F, 32, db.data_ptr(), n)
    out = torch.empty((2 * n - 1) * 4, dtype=torch.int64, device="cuda")
    with z.DeviceTwiddles(F, 24, z.primitiveRootOfUnity(F, 24)) as t:
        z.poly_mul_device(t, da.data_ptr(), n, db.data_ptr(), n, out.data_ptr())
    torch.cuda.synchronize()
    a, b, c = _host(da), _host(db), _host(out)
    xs = O.random_elements(fid, 33, 8)
    lhs = O.poly_eval(fid, c, xs, workers=WORKERS)
    rhs = O.elementwise(fid, "mul", O.poly_eval(fid, a, xs, workers=WORKERS), O.poly_eval(fid, b, xs, workers=WORKERS))
    np.testing.assert_array_equal(lhs, rhs)
    np.testing.assert_array_equal(c[0], O.elementwise(fid, "mul", a[:1], b[:1])[0])
    np.testing.assert_array_equal(c[-1], O.elementwise(fid, "mul", a[-1:], b[-1:])[0])
