"""FRI's data-parallel prover steps on the device (zntt_fri_domain_fill, zntt_fri_fold_device,
zntt_fri_commit_layer, zntt_fri_commit_phase, zntt_fri_query_extract) against the oracle's
restatement of Domain.fill, the proveOn fold round and commit loop, and buildQueries
(libs/fri/src/root.zig:133-166, 372-403, 551-571) on all four fields; fold chains sharing one
table; at full size the fold identity fold(evals of p) = evals of p_even + alpha p_odd; and
every opened path authenticates against its round's root.  Needs a B200."""
from __future__ import annotations

import ctypes
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


def _transcript(fid):
    """A stand-in for the caller's transcript: alpha_r = 1 + the root's first three bytes
    (little-endian) + 2^24 r, a field element of every field, as an oracle slot."""
    def alpha(r, root):
        return O.to_mont(fid, O.from_ints([1 + int.from_bytes(root[:3], "little") + (r << 24)]))[0]
    return alpha


def _prover_buffers(F, log_domain, log_final):
    torch = _torch()
    rounds = log_domain - log_final
    layers = [torch.empty((1 << (log_domain - r)) * F.limbs, dtype=torch.int64, device="cuda")
              for r in range(rounds + 1)]
    trees = [torch.empty((1 << (log_domain - r)) * 4, dtype=torch.int64, device="cuda") for r in range(rounds)]
    return layers, trees


def _verify_path(root, index, leaf_bytes, siblings):
    """MerkleTree.verify (libs/merkle/src/merkle_tree.zig:236-260) over BLAKE3: the side of each
    sibling comes from the index."""
    cur = O.blake3(leaf_bytes)
    for sib in siblings:
        cur = O.blake3(cur + sib if index % 2 == 0 else sib + cur)
        index >>= 1
    return cur == root


def _check_prover(z, F, fid, log_domain, log_final, seed, num_queries):
    torch = _torch()
    rounds = log_domain - log_final
    evals = O.random_elements(fid, seed, 1 << log_domain)
    layers, trees = _prover_buffers(F, log_domain, log_final)
    layers[0].copy_(_to_dev(F, evals))
    torch.cuda.synchronize()
    transcript = _transcript(fid)
    roots = z.fri_commit_phase(F, log_domain, log_final, [t.data_ptr() for t in layers],
                               [t.data_ptr() for t in trees], lambda r, root: _scalar(F, transcript(r, root)))
    want_roots, want_layers, want_trees = O.fri_commit_phase(fid, evals, log_domain, log_final, transcript,
                                                             workers=WORKERS)
    assert roots == want_roots, F.name
    for r in range(rounds + 1):
        np.testing.assert_array_equal(_from_dev(F, layers[r]), want_layers[r], err_msg=f"{F.name} layer {r}")
    for r in range(rounds):
        np.testing.assert_array_equal(trees[r].cpu().numpy().view(np.uint8).reshape(-1, 32)[1:],
                                      want_trees[r][1:], err_msg=f"{F.name} tree {r}")
    positions = np.random.default_rng(seed).integers(0, 1 << log_domain, num_queries, dtype=np.uint64)
    values, paths = z.fri_query_extract(F, log_domain, rounds, [t.data_ptr() for t in layers[:rounds]],
                                        [t.data_ptr() for t in trees], positions)
    want_values, want_paths = O.fri_query_extract(fid, want_layers, want_trees, log_domain, rounds, positions)
    assert values == want_values and paths == want_paths, F.name
    for q, e0 in enumerate(positions):
        for r in range(rounds):
            j = int(e0) % (1 << (log_domain - r - 1))
            assert _verify_path(roots[r], j, values[q][r], paths[q][r]), (F.name, q, r)


def test_commit_phase_and_queries_match_oracle(z):
    """proveOn's commit loop (root.zig:372-403) and buildQueries' openings (root.zig:551-571) on
    the device equal the oracle's, layer by layer and tree by tree, down to a final layer of 2^0
    and 2^3 evaluations; every opened path authenticates against its round's root."""
    for F, fid in _all(z):
        _check_prover(z, F, fid, 11, 3, 500 + F.id, 16)
        _check_prover(z, F, fid, 6, 0, 520 + F.id, 5)


def test_commit_phase_full_size(z):
    """2^20 BN254-Fr and 2^22 Goldilocks evaluations folded to 2^8 / 2^10 with 32 queries."""
    everything = _all(z)
    for (F, fid), log_domain, log_final in ((everything[0], 20, 8), (everything[2], 22, 10)):
        _check_prover(z, F, fid, log_domain, log_final, 540 + F.id, 32)


def test_commit_phase_errors(z):
    """A callback error stops the phase with the caller's exception; an alpha outside the field
    is InvalidArgument; a domain beyond the two-adicity is OrderTooLarge (proveOn's check,
    root.zig:347)."""
    F, fid = _all(z)[0]
    layers, trees = _prover_buffers(F, 8, 4)
    lp, tp = [t.data_ptr() for t in layers], [t.data_ptr() for t in trees]

    def boom(r, root):
        raise KeyError("transcript failed")
    with pytest.raises(KeyError):
        z.fri_commit_phase(F, 8, 4, lp, tp, boom)
    with pytest.raises(z.InvalidArgument):
        z.fri_commit_phase(F, 8, 4, lp, tp, lambda r, root: [2**64 - 1] * 4)
    with pytest.raises(z.InvalidArgument):
        z.fri_commit_phase(z.GOLDILOCKS, 8, 4, lp, tp, lambda r, root: [z.GOLDILOCKS.modulus, 0, 0, 0])
    with pytest.raises(z.OrderTooLarge):
        z.fri_commit_phase(z.BABYBEAR, 28, 12, [1] * 17, [16] * 16, lambda r, root: [1, 0, 0, 0])


def _proof_dict(proof):
    return {"roots": proof.roots, "residual": proof.residual, "queries": proof.queries,
            "log_domain": proof.log_domain, "log_final": proof.log_final,
            "log_residual_degree": proof.log_residual_degree}


def test_device_prove_matches_fixture(z):
    """zig-fri's prove on the device (fri_prove: commit phase, residual, openings) over the
    reference's transcript equals the pure-Python proofs of fri_proof.json byte for byte, on
    all four fields."""
    import json
    import pyref
    d = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fri_proof.json")))
    cfg = d["config"]
    config = z.FriConfig(cfg["log_domain"], cfg["log_initial_degree"], cfg["log_final"], cfg["log_residual_degree"],
                         cfg["num_queries"])
    names = {F.name: (F, fid) for F, fid in _all(z)}
    for c in d["cases"]:
        F, fid = names[c["field"]]
        dev = _to_dev(F, O.to_mont(fid, O.from_ints([int(v, 16) for v in c["evals"]])))
        proof = z.fri_prove(F, pyref.Transcript(cfg["label"].encode()), dev.data_ptr(), config)
        assert [r.hex() for r in proof.roots] == c["roots"], F.name
        assert [x.hex() for x in proof.residual] == c["residual"], F.name
        got_q = [{"pair_index": int(q["pair_index"]), "values": [v.hex() for v in q["values"]],
                  "paths": [[x.hex() for x in path] for path in q["paths"]]} for q in proof.queries]
        assert got_q == c["queries"], F.name


def test_device_prove_full_size_verifies(z):
    """Honest proofs of low-degree evaluations made on the device (the evaluations themselves a
    device transform of 2^16 coefficients): 2^20 BN254-Fr and 2^22 Goldilocks, final layers of
    2^8 and 2^10, a residual of 2^4 coefficients and 32 queries.  Each equals the oracle's
    proof and passes the restated verifier; random (not low-degree) evaluations are rejected
    (the reference's regression test, libs/fri/src/root.zig:775)."""
    import pyref
    torch = _torch()
    everything = _all(z)
    for (F, fid), log_domain, log_final in ((everything[0], 20, 8), (everything[2], 22, 10)):
        rounds = log_domain - log_final
        config = z.FriConfig(log_domain, rounds + 4, log_final, 4, 32)
        n = 1 << log_domain
        coeffs = np.zeros((n, 4), dtype=np.uint64)
        coeffs[:1 << (rounds + 4)] = O.random_elements(fid, 600 + log_domain, 1 << (rounds + 4))
        src = _to_dev(F, coeffs)
        evals = torch.empty_like(src)
        with z.DeviceTwiddles(F, log_domain, z.primitiveRootOfUnity(F, log_domain)) as tw:
            z.ntt_device(tw, src.data_ptr(), evals.data_ptr(), z.FORWARD)
        torch.cuda.synchronize()
        label = b"fri full size"
        proof = z.fri_prove(F, pyref.Transcript(label), evals.data_ptr(), config)
        want = O.fri_prove(fid, _from_dev(F, evals), log_domain, log_final, 4, 32, pyref.Transcript(label),
                           workers=WORKERS)
        assert _proof_dict(proof) == want, F.name
        p, nb = O.MODULI[fid], O.element_bytes(fid)
        assert pyref.fri_verify(p, nb, pyref.Transcript(label), want, log_domain, log_final, 4, 32), F.name
        noise = _to_dev(F, O.random_elements(fid, 700 + log_domain, n))
        bad = z.fri_prove(F, pyref.Transcript(label), noise.data_ptr(), config)
        assert not pyref.fri_verify(p, nb, pyref.Transcript(label), _proof_dict(bad), log_domain, log_final, 4, 32)
        del src, evals, noise
        torch.cuda.empty_cache()


def test_prove_config_checks(z):
    """Config.rounds / Config.validate (libs/fri/src/root.zig:188-202) and proveOn's
    two-adicity check refuse bad parameters before any device work."""
    import pyref
    for args in ((10, 6, 4, 2, 0), (10, 6, 4, 4, 3), (10, 6, 13, 2, 3), (10, 5, 4, 2, 3), (10, 11, 4, 2, 3)):
        with pytest.raises(z.InvalidArgument):
            z.fri_prove(z.BN254_FR, pyref.Transcript(b"x"), 1, z.FriConfig(*args))
    with pytest.raises(z.InvalidArgument):
        z.fri_prove(z.BABYBEAR, pyref.Transcript(b"x"), 1, z.FriConfig(28, 20, 10, 2, 3))


def test_extension_then_prove_goldilocks(z):
    """A STARK prover's path over Goldilocks kept on the device: 2^16 evaluations extended to
    2^20 (zntt_coset_lde_device, shift 1, so the result is the same polynomial on the larger
    subgroup), then zig-fri's prove on the extension; the proof equals the oracle's (prove on
    the oracle's own extension) and passes the restated verifier."""
    import pyref
    torch = _torch()
    F, fid = _all(z)[2]
    log_in, log_domain, log_final = 16, 20, 8
    x = np.random.default_rng(990).integers(0, F.modulus, 1 << log_in, dtype=np.uint64)
    src = torch.from_numpy(x.view(np.int64).copy()).cuda()
    ext = torch.empty(1 << log_domain, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    with z.DeviceTwiddles(F, log_in, z.primitiveRootOfUnity(F, log_in)) as ti, \
            z.DeviceTwiddles(F, log_domain, z.primitiveRootOfUnity(F, log_domain)) as to:
        z.coset_lde_device(ti, to, np.array([1, 0, 0, 0], dtype=np.uint64), src.data_ptr(), ext.data_ptr())
    torch.cuda.synchronize()
    slots = O.elems(len(x))
    slots[:, 0] = x
    want_ext = O.coset_lde(fid, O.to_mont(fid, slots), log_in, log_domain - log_in, O.to_mont(fid, O.from_ints([1]))[0],
                           workers=WORKERS)
    np.testing.assert_array_equal(_from_dev(F, ext), want_ext)
    rounds = log_domain - log_final
    config = z.FriConfig(log_domain, log_in, log_final, log_in - rounds, 16)
    label = b"lde then fri"
    proof = z.fri_prove(F, pyref.Transcript(label), ext.data_ptr(), config)
    want = O.fri_prove(fid, want_ext, log_domain, log_final, log_in - rounds, 16, pyref.Transcript(label),
                       workers=WORKERS)
    assert _proof_dict(proof) == want
    assert pyref.fri_verify(O.MODULI[fid], O.element_bytes(fid), pyref.Transcript(label), want, log_domain,
                            log_final, log_in - rounds, 16)


@pytest.mark.parametrize("log_n", [2, 3, 9, 10, 11, 14, 20])
def test_fold_commit_equals_fold_then_commit(z, log_n):
    """zntt_fri_fold_commit (a fold fused with the commitment of the layer it makes) equals
    zntt_fri_fold_device followed by zntt_fri_commit_layer -- new layer, whole node array and
    root -- on all four fields, on both sides of every launch boundary of the tree, with a
    table shared with a larger first layer (log_table = log_n + 2)."""
    torch = _torch()
    for F, fid in _all(z):
        n = 1 << log_n
        layer = _to_dev(F, O.random_elements(fid, 1200 + log_n, n))
        alpha = _scalar(F, O.random_elements(fid, 1300 + log_n, 1)[0])
        half = (n // 2) * F.limbs
        out_a, out_b = (torch.empty(half, dtype=torch.int64, device="cuda") for _ in range(2))
        nodes_a, nodes_b = (torch.empty((n // 2) * 4, dtype=torch.int64, device="cuda") for _ in range(2))
        torch.cuda.synchronize()
        root_a = z.fri_fold_commit(F, layer.data_ptr(), log_n, alpha, out_a.data_ptr(), nodes_a.data_ptr(),
                                   log_table=log_n + 2)
        z.fri_fold(F, layer.data_ptr(), log_n, alpha, out_b.data_ptr(), log_table=log_n + 2)
        root_b = z.fri_commit_layer(F, out_b.data_ptr(), log_n - 1, nodes_b.data_ptr())
        torch.cuda.synchronize()
        assert root_a == root_b, F.name
        assert torch.equal(out_a, out_b), F.name
        assert torch.equal(nodes_a, nodes_b), F.name


def test_fold_commit_argument_checks(z):
    torch = _torch()
    F = z.BN254_FR
    buf = torch.empty(1 << 14, dtype=torch.int64, device="cuda")
    one = z.to_montgomery(F, 1)
    with pytest.raises(z.InvalidArgument):  # the new layer overlaps the old one
        z.fri_fold_commit(F, buf.data_ptr(), 6, one, buf[64:].data_ptr(), buf[8192:].data_ptr())
    with pytest.raises(z.InvalidArgument):  # the nodes overlap the new layer
        z.fri_fold_commit(F, buf.data_ptr(), 6, one, buf[4096:].data_ptr(), buf[4100:].data_ptr())
    with pytest.raises(z.InvalidArgument):  # log_table below log_n
        z.fri_fold_commit(F, buf.data_ptr(), 6, one, buf[4096:].data_ptr(), buf[8192:].data_ptr(), log_table=5)


def test_row_commitment_matches_fixture_and_oracle(z):
    """zntt_merkle_commit_rows (MerkleTree.init over the rows of device columns) against the
    pure-Python fixture and the oracle's whole node arrays: all four fields, 1 to the maximum
    number of columns (one 1024-byte chunk per row), on both sides of the launch boundaries."""
    import json
    torch = _torch()
    d = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "merkle_rows.json")))
    names = {F.name: (F, fid) for F, fid in _all(z)}
    for c in d["cases"]:
        F, fid = names[c["field"]]
        cols = [_to_dev(F, O.to_mont(fid, O.from_ints([int(v, 16) for v in col]))) for col in c["values"]]
        nodes = torch.zeros((2 << c["log_n"]) * 4, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        root = z.merkle_commit_rows(F, [t.data_ptr() for t in cols], c["log_n"], nodes.data_ptr())
        assert root.hex() == c["root"], (c["field"], c["columns"], c["log_n"])
        if "nodes" in c:
            got = nodes.cpu().numpy().view(np.uint8).reshape(-1, 32)
            assert [x.tobytes().hex() for x in got[1:]] == c["nodes"]
    for F, fid in _all(z):
        nb = O.element_bytes(fid)
        for m, log_n in ((1, 0), (1, 9), (3, 10), (8, 13), (1024 // nb, 12), (2, 16)):
            host = [O.random_elements(fid, 1700 + 13 * m + c, 1 << log_n) for c in range(m)]
            want = O.merkle_commit_rows(fid, host, log_n, workers=WORKERS)
            cols = [_to_dev(F, h) for h in host]
            nodes = torch.zeros((2 << log_n) * 4, dtype=torch.int64, device="cuda")
            torch.cuda.synchronize()
            z.merkle_commit_rows(F, [t.data_ptr() for t in cols], log_n, nodes.data_ptr())
            torch.cuda.synchronize()
            np.testing.assert_array_equal(nodes.cpu().numpy().view(np.uint8).reshape(-1, 32)[1:], want[1:],
                                          err_msg=f"{F.name} {m} columns 2^{log_n}")


def test_row_commitment_argument_checks(z):
    torch = _torch()
    F = z.BN254_FR
    buf = torch.empty(1 << 14, dtype=torch.int64, device="cuda")
    col = buf.data_ptr()
    nodes = buf[8192:].data_ptr()
    with pytest.raises(z.InvalidArgument):  # 33 columns of 32 bytes exceed one chunk
        z.merkle_commit_rows(F, [col] * 33, 4, nodes)
    with pytest.raises(z.InvalidArgument):
        z.merkle_commit_rows(F, [col, 0], 4, nodes)
    with pytest.raises(z.InvalidArgument):  # a column count whose byte size wraps 32 bits
        z._check(z.lib().zntt_merkle_commit_rows(F.id, (ctypes.c_void_p * 1)(col), 1 << 27, 4, nodes, None, None))
    with pytest.raises(z.InvalidArgument):
        z.merkle_commit_rows(F, [], 4, nodes)
    with pytest.raises(z.InvalidArgument):  # the nodes overlap the column
        z.merkle_commit_rows(F, [col], 6, buf[64:].data_ptr())


def test_row_openings_match_oracle_and_verify(z):
    """zntt_merkle_open_rows: each opened row equals the columns' toBytes at that row, each path
    equals the oracle tree's siblings (MerkleTree.prove, libs/merkle/src/merkle_tree.zig:206-233)
    and authenticates the row's hash against the root; all four fields."""
    torch = _torch()
    for F, fid in _all(z):
        for m, log_n in ((1, 0), (3, 11), (8, 14)):
            host = [O.random_elements(fid, 1900 + 7 * m + c, 1 << log_n) for c in range(m)]
            tree = O.merkle_commit_rows(fid, host, log_n, workers=WORKERS)
            cols = [_to_dev(F, h) for h in host]
            nodes = torch.empty((2 << log_n) * 4, dtype=torch.int64, device="cuda")
            torch.cuda.synchronize()
            root = z.merkle_commit_rows(F, [t.data_ptr() for t in cols], log_n, nodes.data_ptr())
            positions = np.random.default_rng(log_n + m).integers(0, 1 << log_n, 9, dtype=np.uint64)
            rows, paths = z.merkle_open_rows(F, [t.data_ptr() for t in cols], log_n, nodes.data_ptr(), positions)
            byte_cols = [O.to_bytes(fid, h) for h in host]
            for q, i in enumerate(int(p) for p in positions):
                assert rows[q] == b"".join(bc[i] for bc in byte_cols), (F.name, m, q)
                assert paths[q] == [tree[((1 << log_n) + i >> k) ^ 1].tobytes() for k in range(log_n)]
                assert _verify_path(root, i, rows[q], paths[q]), (F.name, m, q)
    with pytest.raises(z.InvalidArgument):  # a row outside the commitment
        z.merkle_open_rows(z.GOLDILOCKS, [1], 4, 16, [16])
