"""FRI's data-parallel prover steps on the device (zntt_fri_domain_fill, zntt_fri_fold_device)
against the oracle's restatement of Domain.fill and the proveOn fold round
(libs/fri/src/root.zig:133-166, 396-403) on all four fields, fold chains sharing one table, and
at full size the fold identity fold(evals of p) = evals of p_even + alpha p_odd.  Needs a B200."""
from __future__ import annotations

import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
WORKERS = min(os.cpu_count() or 1, 64)


@pytest.fixture(scope="module")
def z(zntt):
    zntt.init(0)
    return zntt


def _torch():
    import torch
    return torch


def _all(z):
    return [(z.BN254_FR, O.BN254_FR), (z.BLS12_381_FR, O.BLS12_381_FR), (z.GOLDILOCKS, O.GOLDILOCKS),
            (z.BABYBEAR, O.BABYBEAR)]


def _to_dev(F, slots):
    """Oracle Montgomery slots -> the device layout of F (slots as they are, or canonical u64)."""
    torch = _torch()
    a = np.ascontiguousarray(slots) if F.limbs == 4 else np.ascontiguousarray(O.from_mont(_fid(F), slots)[:, 0])
    t = torch.from_numpy(a.view(np.int64).reshape(-1).copy()).cuda()
    torch.cuda.synchronize()
    return t


def _from_dev(F, t):
    """Device layout -> oracle Montgomery slots."""
    a = t.cpu().numpy().view(np.uint64)
    if F.limbs == 4:
        return a.reshape(-1, 4).copy()
    s = O.elems(len(a))
    s[:, 0] = a
    return O.to_mont(_fid(F), s)


def _fid(F):
    return {"bn254_fr": O.BN254_FR, "bls12_381_fr": O.BLS12_381_FR, "goldilocks": O.GOLDILOCKS,
            "babybear": O.BABYBEAR}[F.name]


def _scalar(F, slot):
    """An oracle Montgomery slot as the C ABI's scalar for F."""
    if F.limbs == 4:
        return np.asarray(slot, dtype=np.uint64)
    v = O.from_mont(_fid(F), np.asarray(slot, dtype=np.uint64).reshape(1, 4))[0, 0]
    return np.array([v, 0, 0, 0], dtype=np.uint64)


def test_domain_fill_matches_oracle(z):
    torch = _torch()
    for F, fid in _all(z):
        for log_n in (0, 1, 5, 12, 17):
            out = torch.empty((1 << log_n) * F.limbs, dtype=torch.int64, device="cuda")
            z.fri_domain_fill(F, log_n, out.data_ptr())
            torch.cuda.synchronize()
            np.testing.assert_array_equal(_from_dev(F, out), O.fri_domain_fill(fid, log_n), err_msg=f"{F.name} {log_n}")
        with pytest.raises(z.OrderTooLarge):
            z.fri_domain_fill(F, F.two_adicity + 1, out.data_ptr())


@pytest.mark.parametrize("log_n", [1, 2, 7, 12, 14])
def test_fold_matches_oracle(z, log_n):
    torch = _torch()
    for F, fid in _all(z):
        layer = O.random_elements(fid, 40 + log_n, 1 << log_n)
        alpha = O.random_elements(fid, 50 + log_n, 1)[0]
        want = O.fri_fold(fid, layer, log_n, alpha, workers=WORKERS)
        d = _to_dev(F, layer)
        out = torch.empty((1 << (log_n - 1)) * F.limbs, dtype=torch.int64, device="cuda")
        z.fri_fold(F, d.data_ptr(), log_n, _scalar(F, alpha), out.data_ptr())
        torch.cuda.synchronize()
        np.testing.assert_array_equal(_from_dev(F, out), want, err_msg=f"{F.name} 2^{log_n}")


def test_fold_chain_shares_one_table(z):
    """Rounds 13 -> 3 of one proof, every round with the first layer's table (log_table 13)."""
    torch = _torch()
    for F, fid in _all(z):
        layer = O.random_elements(fid, 61, 1 << 13)
        d = _to_dev(F, layer)
        for log_n in range(13, 3, -1):
            alpha = O.random_elements(fid, 70 + log_n, 1)[0]
            layer = O.fri_fold(fid, layer, log_n, alpha, workers=WORKERS)
            out = torch.empty((1 << (log_n - 1)) * F.limbs, dtype=torch.int64, device="cuda")
            z.fri_fold(F, d.data_ptr(), log_n, _scalar(F, alpha), out.data_ptr(), log_table=13)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(_from_dev(F, out), layer, err_msg=f"{F.name} round at 2^{log_n}")
            d = out


def test_fold_of_extension_is_the_folded_polynomial_full_size(z):
    """BN254-Fr at 2^24: evaluations of a degree < 2^23 polynomial c on the domain (a forward
    transform of c zero-padded), folded with alpha, equal the 2^23-point forward transform of
    c_even + alpha c_odd -- two different kernels, one identity."""
    torch = _torch()
    F, fid = z.BN254_FR, O.BN254_FR
    n = 1 << 24
    c = torch.zeros(n * 4, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()  # the zero fill (torch's stream) before the library writes (its own)
    z.random_elements(F, 5, c.data_ptr(), n // 2)
    alpha = z.to_montgomery(F, 123456789)
    evals = torch.empty_like(c)
    half = torch.empty(n // 2 * 4, dtype=torch.int64, device="cuda")
    with z.DeviceTwiddles(F, 24, z.primitiveRootOfUnity(F, 24)) as t24:
        z.ntt_device(t24, c.data_ptr(), evals.data_ptr(), z.FORWARD)
        z.fri_fold(F, evals.data_ptr(), 24, alpha, half.data_ptr())
    torch.cuda.synchronize()
    cv = c[: n // 2 * 4].view(-1, 4)
    ce = cv[0::2].contiguous()
    co = cv[1::2].contiguous()
    al = torch.from_numpy(np.tile(alpha.view(np.int64), n // 4)).cuda()
    torch.cuda.synchronize()
    t = torch.empty_like(ce)
    z.elementwise_device(F, "mul", co.data_ptr(), al.data_ptr(), t.data_ptr(), n // 4)
    folded_c = torch.zeros(n // 2 * 4, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    z.elementwise_device(F, "add", ce.data_ptr(), t.data_ptr(), folded_c.data_ptr(), n // 4)
    want = torch.empty_like(folded_c)
    with z.DeviceTwiddles(F, 23, z.primitiveRootOfUnity(F, 23)) as t23:
        z.ntt_device(t23, folded_c.data_ptr(), want.data_ptr(), z.FORWARD)
    torch.cuda.synchronize()
    assert torch.equal(half, want)


def test_fold_argument_errors(z):
    torch = _torch()
    F = z.GOLDILOCKS
    buf = torch.zeros(64, dtype=torch.int64, device="cuda")
    one = np.array([1, 0, 0, 0], dtype=np.uint64)
    with pytest.raises(z.InvalidArgument):  # output overlaps the layer
        z.fri_fold(F, buf.data_ptr(), 5, one, buf[8:].data_ptr())
    with pytest.raises(z.InvalidArgument):  # log_n beyond the table
        z.fri_fold(F, buf.data_ptr(), 5, one, buf[32:].data_ptr(), log_table=4)
    with pytest.raises(z.InvalidArgument):
        z.fri_fold(F, buf.data_ptr(), 0, one, buf[32:].data_ptr())


def test_layer_commitment_matches_fixture_and_oracle(z):
    """zntt_fri_commit_layer against the pure-Python fixture (roots and whole node arrays) and
    the oracle's whole node arrays at sizes on both sides of each launch boundary: leaves alone
    below 2^10 evaluations, one subtree launch, chained subtree launches, and the one-CTA top
    levels."""
    import json
    torch = _torch()
    d = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fri_commit.json")))
    names = {F.name: (F, fid) for F, fid in _all(z)}
    for c in d["cases"]:
        F, fid = names[c["field"]]
        slots = O.to_mont(fid, O.from_ints([int(v, 16) for v in c["values"]]))
        dev = _to_dev(F, slots)
        nodes = torch.zeros((1 << c["log_n"]) * 4, dtype=torch.int64, device="cuda")
        root = z.fri_commit_layer(F, dev.data_ptr(), c["log_n"], nodes.data_ptr())
        assert root.hex() == c["root"], (c["field"], c["log_n"])
        if "nodes" in c:
            got = nodes.cpu().numpy().view(np.uint8).reshape(-1, 32)
            assert [x.tobytes().hex() for x in got[1:]] == c["nodes"]
    for F, fid in _all(z):
        for log_n in (9, 10, 12, 13, 14, 16, 18):
            layer = O.random_elements(fid, 300 + log_n, 1 << log_n)
            want = O.fri_commit_layer(fid, layer, log_n, workers=WORKERS)
            nodes = torch.zeros((1 << log_n) * 4, dtype=torch.int64, device="cuda")
            z.fri_commit_layer(F, _to_dev(F, layer).data_ptr(), log_n, nodes.data_ptr())
            np.testing.assert_array_equal(nodes.cpu().numpy().view(np.uint8).reshape(-1, 32), want,
                                          err_msg=f"{F.name} 2^{log_n}")


def test_layer_commitment_full_size(z):
    """A 2^24 Goldilocks layer and a 2^22 BN254-Fr layer against the oracle's root."""
    torch = _torch()
    for (F, fid), log_n in ((_all(z)[2], 24), (_all(z)[0], 22)):
        layer = O.random_elements(fid, 400 + log_n, 1 << log_n)
        want = O.fri_commit_layer(fid, layer, log_n, workers=WORKERS)
        nodes = torch.empty((1 << log_n) * 4, dtype=torch.int64, device="cuda")
        root = z.fri_commit_layer(F, _to_dev(F, layer).data_ptr(), log_n, nodes.data_ptr())
        assert root == want[1].tobytes(), f"{F.name} 2^{log_n}"


def test_blake3_probe(z):
    """The commitment's roofline probe runs and gives a plausible compression rate."""
    rate = z.probe_blake3()
    assert 1e9 < rate < 1e13
