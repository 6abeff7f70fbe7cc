"""Pins the CPU oracle to the reference's own vectors and to an independent DFT.

Mirrors the reference's NTT tests (libs/ntt/src/root.zig:290-738), its
Montgomery tests (libs/field/src/montgomery.zig:409-471) and its RFC 8439
ChaCha20 test (libs/rng/src/root.zig:182-228).  CPU only.
"""
from __future__ import annotations

import json
import os
import random

import numpy as np
import pytest

import oracle as O
import pyref

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELD_IDS = {"goldilocks": O.GOLDILOCKS, "babybear": O.BABYBEAR, "bn254_fr": O.BN254_FR,
             "bls12_381_fr": O.BLS12_381_FR}


def _canon_ints(field, mont):
    return O.to_ints(O.from_mont(field, mont))


def _mont_of(field, values):
    return O.to_mont(field, O.from_ints([v % O.MODULI[field] for v in values]))


@pytest.fixture(scope="module", autouse=True)
def _lib():
    O.load()


# --- known answers -------------------------------------------------------

def test_ntt_matches_reference_dft_kats():
    """root.zig:405-453: 8 Python-DFT cases over Goldilocks and BabyBear, and their inverse."""
    cases = json.load(open(os.path.join(GOLDEN, "ntt_kat.json")))
    assert len(cases) == 8
    for c in cases:
        f = FIELD_IDS[c["field"]]
        log_n = c["log_n"]
        inp = [int(v, 16) for v in c["input"]]
        exp = [int(v, 16) for v in c["expect"]]
        data = _mont_of(f, inp)
        root = _mont_of(f, [int(c["root"], 16)])[0]
        assert O.ntt(f, data, log_n, root) == O.OK
        assert _canon_ints(f, data) == exp, c["source"]
        assert O.intt(f, data, log_n, root) == O.OK
        assert _canon_ints(f, data) == inp, c["source"]
        # The KAT roots are the library's own primitiveRootOfUnity(log_n) values.
        st, r = O.primitive_root(f, log_n)
        assert st == O.OK and _canon_ints(f, r.reshape(1, 4)) == [int(c["root"], 16)]


def test_chacha20_rfc8439_vectors():
    v = json.load(open(os.path.join(GOLDEN, "chacha20_rfc8439.json")))
    key = bytes.fromhex(v["key"])
    s = O.chacha20_stream(key, 128, bytes.fromhex(v["block_nonce"]))
    assert s[64:128].hex() == v["block_counter1"]
    s = O.chacha20_stream(key, 64 + 114, bytes.fromhex(v["cipher_nonce"]))
    ks = s[64:]
    assert ks.hex() == v["keystream_counter1"]
    ct = bytes(a ^ b for a, b in zip(v["plaintext"].encode(), ks))
    assert ct.hex() == v["ciphertext"]
    # The independent Python keystream agrees too.
    blk = pyref.chacha20_block(key, 1, bytes.fromhex(v["block_nonce"]))
    assert blk.hex() == v["block_counter1"]


def test_fr_transforms_match_independent_definition():
    """BN254-Fr / BLS12-381-Fr: seeded inputs, roots, forward and inverse vs the Python DFT/FFT."""
    for c in json.load(open(os.path.join(GOLDEN, "fr_transforms.json"))):
        f = FIELD_IDS[c["field"]]
        log_n, n = c["log_n"], 1 << c["log_n"]
        x = O.random_elements(f, c["seed"], n)
        xs = _canon_ints(f, x)
        if "input" in c:
            assert xs == [int(v, 16) for v in c["input"]]
        else:
            assert pyref_digest(xs) == c["input_sha256"]
        st, root = O.primitive_root(f, log_n)
        assert st == O.OK and _canon_ints(f, root.reshape(1, 4)) == [int(c["root"], 16)]
        fwd = x.copy()
        assert O.ntt(f, fwd, log_n, root) == O.OK
        inv = x.copy()
        assert O.intt(f, inv, log_n, root) == O.OK
        st, tw = O.precompute_twiddles(f, log_n, root)
        fwd_tw = x.copy()
        assert O.ntt_with_twiddles(f, fwd_tw, log_n, tw) == O.OK
        inv_tw = x.copy()
        assert O.ntt_with_twiddles(f, inv_tw, log_n, tw, inverse=True) == O.OK
        np.testing.assert_array_equal(fwd, fwd_tw)
        np.testing.assert_array_equal(inv, inv_tw)
        if "forward" in c:
            assert _canon_ints(f, fwd) == [int(v, 16) for v in c["forward"]]
            assert _canon_ints(f, inv) == [int(v, 16) for v in c["inverse"]]
        else:
            assert pyref_digest(_canon_ints(f, fwd)) == c["forward_sha256"]
            assert pyref_digest(_canon_ints(f, inv)) == c["inverse_sha256"]


def pyref_digest(values):
    import make_golden
    return make_golden.vec_digest(values)


def test_coset_lde_fixture():
    c = json.load(open(os.path.join(GOLDEN, "coset_lde.json")))
    f = FIELD_IDS[c["field"]]
    ev = O.random_elements(f, c["seed"], 1 << c["log_in"])
    assert _canon_ints(f, ev) == [int(v, 16) for v in c["evals"]]
    shift = O.from_int(f, c["shift"])
    out = O.coset_lde(f, ev, c["log_in"], c["log_blowup"], shift)
    assert _canon_ints(f, out) == [int(v, 16) for v in c["output"]]


# --- roots and field constants --------------------------------------------

@pytest.mark.parametrize("field,adicity", [(O.BN254_FR, 28), (O.BLS12_381_FR, 32)])
def test_fr_roots(field, adicity):
    p = O.MODULI[field]
    assert pyref.two_adicity(p)[0] == adicity
    assert _canon_ints(field, O.qnr(field).reshape(1, 4)) == [5]
    st, _ = O.primitive_root(field, adicity + 1)
    assert st == O.ORDER_TOO_LARGE
    for log_n in (0, 1, 12, 20, adicity):
        st, r = O.primitive_root(field, log_n)
        assert st == O.OK
        assert _canon_ints(field, r.reshape(1, 4)) == [pyref.primitive_root(p, log_n)]


# --- Montgomery arithmetic -------------------------------------------------

@pytest.mark.parametrize("field", [O.BN254_FP, O.BN254_FR, O.BLS12_381_FR, O.GOLDILOCKS, O.BABYBEAR])
def test_montgomery_ops_vs_bigint(field):
    """montgomery.zig:409-439 (add/sub/neg vs u512) extended to mul and inv."""
    p = O.MODULI[field]
    rnd = random.Random(11 + field)
    xs = [0, 1, 2, p - 1, p - 2, (p + 1) // 2] + [rnd.randrange(p) for _ in range(200)]
    ys = [p - 1, 0, p - 1, p - 1, 3, (p - 1) // 2] + [rnd.randrange(p) for _ in range(200)]
    a, b = _mont_of(field, xs), _mont_of(field, ys)
    assert _canon_ints(field, O.elementwise(field, "add", a, b)) == [(x + y) % p for x, y in zip(xs, ys)]
    assert _canon_ints(field, O.elementwise(field, "sub", a, b)) == [(x - y) % p for x, y in zip(xs, ys)]
    assert _canon_ints(field, O.elementwise(field, "neg", a)) == [(-x) % p for x in xs]
    assert _canon_ints(field, O.elementwise(field, "mul", a, b)) == [x * y % p for x, y in zip(xs, ys)]
    inv = _canon_ints(field, O.elementwise(field, "inv", a))
    assert inv == [pow(x, -1, p) if x else 0 for x in xs]


# --- bitReverse -------------------------------------------------------------

def test_bit_reverse_order_and_involution():
    d = _mont_of(O.BN254_FR, [0, 1, 2, 3])
    assert O.bit_reverse(O.BN254_FR, d) == O.OK
    assert _canon_ints(O.BN254_FR, d) == [0, 2, 1, 3]
    d = _mont_of(O.BN254_FR, [0, 1, 2, 3, 4, 5, 6, 0])
    orig = d.copy()
    O.bit_reverse(O.BN254_FR, d)
    O.bit_reverse(O.BN254_FR, d)
    np.testing.assert_array_equal(d, orig)
    assert O.bit_reverse(O.BN254_FR, O.elems(0)) == O.INVALID_LENGTH
    assert O.bit_reverse(O.BN254_FR, O.elems(3)) == O.INVALID_LENGTH


# --- error contracts (root.zig:675-738) -------------------------------------

def test_error_contracts():
    f = O.BN254_FR
    one = O.from_int(f, 1)
    short = O.elems(3)
    assert O.ntt(f, short, 2, one) == O.LENGTH_MISMATCH
    assert O.intt(f, short, 2, one) == O.LENGTH_MISMATCH
    two = O.elems(2)
    assert O.ntt(f, two, 64, one) == O.LOG_TOO_LARGE
    assert O.intt(f, two, 200, one) == O.LOG_TOO_LARGE
    assert O.precompute_twiddles(f, 64, one)[0] == O.LOG_TOO_LARGE
    # twiddle table shape
    st, root = O.primitive_root(f, 3)
    st, tw = O.precompute_twiddles(f, 3, root)
    data = _mont_of(f, [1] * 8)
    assert O.ntt_with_twiddles(f, data.copy(), 3, tw[:2]) == O.INVALID_TWIDDLES
    assert O.ntt_with_twiddles(f, data.copy(), 3, tw[:2], inverse=True) == O.INVALID_TWIDDLES
    assert O.ntt_with_twiddles(f, data.copy(), 3, [tw[0][:1]]) == O.INVALID_TWIDDLES
    # A bad stage length is found inside the stage loop, after the data moved.
    bad = [tw[0], tw[1][:1], tw[2]]
    d = _mont_of(f, list(range(8)))
    assert O.ntt_with_twiddles(f, d, 3, bad) == O.INVALID_TWIDDLES
    assert _canon_ints(f, d) != list(range(8))
    # LogTooLarge is reported before LengthMismatch, LengthMismatch before InvalidTwiddles.
    assert O.ntt_with_twiddles(f, O.elems(3), 64, []) == O.LOG_TOO_LARGE
    assert O.ntt_with_twiddles(f, O.elems(3), 3, []) == O.LENGTH_MISMATCH
    # The correct table round-trips.
    d = data.copy()
    assert O.ntt_with_twiddles(f, d, 3, tw) == O.OK
    assert O.ntt_with_twiddles(f, d, 3, tw, inverse=True) == O.OK
    np.testing.assert_array_equal(d, data)


def test_twiddle_layout():
    """root.zig:605-636: tw[s][j] == (root^(2^(log_n-1-s)))^j, and log_n = 0 gives no stages."""
    f = O.BLS12_381_FR
    p = O.MODULI[f]
    for log_n in range(0, 7):
        st, root = O.primitive_root(f, log_n)
        st, tw = O.precompute_twiddles(f, log_n, root)
        assert st == O.OK and len(tw) == log_n
        r = _canon_ints(f, root.reshape(1, 4))[0]
        for s in range(log_n):
            wm = pow(r, 1 << (log_n - 1 - s), p)
            assert _canon_ints(f, tw[s]) == [pow(wm, j, p) for j in range(1 << s)]


def test_length_one_transform():
    f = O.BN254_FR
    d = _mont_of(f, [42])
    assert O.ntt(f, d, 0, O.from_int(f, 1)) == O.OK
    assert O.intt(f, d, 0, O.from_int(f, 1)) == O.OK
    assert _canon_ints(f, d) == [42]
    assert O.ntt_with_twiddles(f, d, 0, []) == O.OK
    assert O.ntt_with_twiddles(f, d, 0, [], inverse=True) == O.OK
    assert _canon_ints(f, d) == [42]


def test_convolution_property():
    """root.zig:539-603 over BN254-Fr: NTT(f) . NTT(g) -> intt == cyclic convolution."""
    f = O.BN254_FR
    p = O.MODULI[f]
    n, log_n = 16, 4
    fv = [1, 2, 3] + [0] * 13
    gv = [2, 3] + [0] * 14
    conv = [sum(fv[j] * gv[(i - j) % n] for j in range(n)) % p for i in range(n)]
    st, root = O.primitive_root(f, log_n)
    a, b = _mont_of(f, fv), _mont_of(f, gv)
    O.ntt(f, a, log_n, root)
    O.ntt(f, b, log_n, root)
    c = O.elementwise(f, "mul", a, b)
    O.intt(f, c, log_n, root)
    assert _canon_ints(f, c) == conv


def test_non_root_table_semantics():
    """root is not validated: ntt(w) for a non-root w still equals nttWithTwiddles(table(w))."""
    f = O.BN254_FR
    w = O.from_int(f, 7)
    x = O.random_elements(f, 9, 32)
    a = x.copy()
    O.ntt(f, a, 5, w)
    st, tw = O.precompute_twiddles(f, 5, w)
    b = x.copy()
    O.ntt_with_twiddles(f, b, 5, tw)
    np.testing.assert_array_equal(a, b)


def test_parallel_harness_matches_single_thread():
    f = O.BN254_FR
    log_n = 10
    x = O.random_elements(f, 5, 1 << log_n)
    st, root = O.primitive_root(f, log_n)
    st, tw = O.precompute_twiddles(f, log_n, root)
    a, b = x.copy(), x.copy()
    O.ntt_with_twiddles(f, a, log_n, tw, workers=1)
    O.ntt_with_twiddles(f, b, log_n, tw, workers=4, inplace4=True)
    np.testing.assert_array_equal(a, b)
    O.ntt_with_twiddles(f, b, log_n, tw, inverse=True, workers=3, inplace4=True)
    np.testing.assert_array_equal(b, x)


def _poly_fixture_inputs(c):
    f = FIELD_IDS[c["field"]]
    a = _mont_of(f, [int(v, 16) for v in c["a"]]) if c["a"] else O.elems(0)
    b = _mont_of(f, [int(v, 16) for v in c["b"]]) if c["b"] else O.elems(0)
    return f, a, b


def test_poly_mul_fixture():
    """The schoolbook product (libs/poly/src/poly.zig:197-212) against the independent
    pure-Python sum, with the reference's normalisation, zero and DegreeTooLarge cases."""
    for c in json.load(open(os.path.join(GOLDEN, "poly_mul.json"))):
        f, a, b = _poly_fixture_inputs(c)
        st, out, deg = O.poly_mul(f, a, b, c["max_degree"], workers=4)
        if "error" in c:
            assert st == O.DEGREE_TOO_LARGE, c
            continue
        assert st == O.OK and deg == c["degree"], (st, deg, c["degree"])
        got = _canon_ints(f, out)
        want = [int(v, 16) for v in c["product"]]
        assert got[:len(want)] == want
        assert all(v == 0 for v in got[len(want):])


def test_poly_mul_evaluates_to_the_product_of_evaluations():
    """c(x) = a(x) b(x) at random points (Polynomial.eval, poly.zig:214-224), for sizes the
    fixture does not reach, and one thread vs several give the same coefficients."""
    for f in (O.BN254_FR, O.BLS12_381_FR):
        a = O.random_elements(f, 71, 700)
        b = O.random_elements(f, 72, 333)
        st, c1, d = O.poly_mul(f, a, b, 1100, workers=1)
        st4, c4, d4 = O.poly_mul(f, a, b, 1100, workers=8)
        assert st == st4 == O.OK and d == d4 == 1031
        np.testing.assert_array_equal(c1, c4)
        x = O.random_elements(f, 73, 8)
        lhs = O.poly_eval(f, c1[:d + 1], x)
        rhs = O.elementwise(f, "mul", O.poly_eval(f, a, x), O.poly_eval(f, b, x))
        np.testing.assert_array_equal(lhs, rhs)


def test_blake3_and_fri_commitment_fixture():
    """BLAKE3 against the reference's own known answer (libs/hash/src/root.zig, kat) and the
    FRI layer commitment (hashPair + MerkleTree.initFromHashes) against the pure-Python one,
    on all four fields."""
    d = json.load(open(os.path.join(GOLDEN, "fri_commit.json")))
    assert O.blake3(d["kat"]["message"].encode()).hex() == d["kat"]["blake3"], d["kat"]["source"]
    assert pyref.blake3(d["kat"]["message"].encode()).hex() == d["kat"]["blake3"]
    assert O.blake3(b"").hex() == d["empty"]
    for m in (b"a" * 63, b"b" * 64, b"c" * 65, b"d" * 200, bytes(range(256)) * 4):
        assert O.blake3(m) == pyref.blake3(m), len(m)
    for c in d["cases"]:
        f = FIELD_IDS[c["field"]]
        layer = _mont_of(f, [int(v, 16) for v in c["values"]])
        nodes = O.fri_commit_layer(f, layer, c["log_n"], workers=4)
        assert nodes[1].tobytes().hex() == c["root"], (c["field"], c["log_n"])
        if "nodes" in c:
            assert [x.tobytes().hex() for x in nodes[1:]] == c["nodes"]


def _proof_hex(proof):
    return {"roots": [r.hex() for r in proof["roots"]], "residual": [c.hex() for c in proof["residual"]],
            "queries": [{"pair_index": int(q["pair_index"]), "values": [v.hex() for v in q["values"]],
                         "paths": [[x.hex() for x in path] for path in q["paths"]]} for q in proof["queries"]]}


def _proof_bytes(c, cfg):
    return {"roots": [bytes.fromhex(r) for r in c["roots"]], "residual": [bytes.fromhex(x) for x in c["residual"]],
            "queries": [{"pair_index": q["pair_index"], "values": [bytes.fromhex(v) for v in q["values"]],
                         "paths": [[bytes.fromhex(x) for x in path] for path in q["paths"]]} for q in c["queries"]],
            "log_domain": cfg["log_domain"], "log_final": cfg["log_final"],
            "log_residual_degree": cfg["log_residual_degree"]}


def test_transcript_known_answer():
    """pyref.Transcript (libs/transcript/src/root.zig:38-170) against the reference's own
    challenge-sequence known answer (libs/fri/src/root.zig, "wire-compat", Goldilocks)."""
    kat = json.load(open(os.path.join(GOLDEN, "fri_proof.json")))["transcript_kat"]
    t = pyref.Transcript(kat["label"].encode())
    got = b"".join(t.challenge_field_checked(0xFFFFFFFF00000001, 8).to_bytes(8, "little")
                   for _ in range(kat["draws"]))
    assert got.hex() == kat["expect"], kat["source"]


def test_fri_proof_fixture_oracle_and_verifier():
    """The oracle's prove (commitment, fold and inverse transform in C++) reproduces the
    pure-Python proofs of fri_proof.json on all four fields; the restated verifier accepts
    them and rejects a tampered value, a tampered path, a tampered residual and another
    transcript label (the reference's own rejection tests, libs/fri/src/root.zig:834-902)."""
    d = json.load(open(os.path.join(GOLDEN, "fri_proof.json")))
    cfg = d["config"]
    args = (cfg["log_domain"], cfg["log_final"], cfg["log_residual_degree"], cfg["num_queries"])
    label = cfg["label"].encode()
    for c in d["cases"]:
        f = FIELD_IDS[c["field"]]
        p, nb = O.MODULI[f], O.element_bytes(f)
        evals = _mont_of(f, [int(v, 16) for v in c["evals"]])
        got = O.fri_prove(f, evals, *args, pyref.Transcript(label), workers=4)
        assert _proof_hex(got) == {k: c[k] for k in ("roots", "residual", "queries")}, c["field"]
        proof = _proof_bytes(c, cfg)
        assert pyref.fri_verify(p, nb, pyref.Transcript(label), proof, *args), c["field"]
        assert not pyref.fri_verify(p, nb, pyref.Transcript(b"another statement"), proof, *args)
        for where in ("value", "path", "residual"):
            bad = json.loads(json.dumps(c))
            if where == "value":
                v = bad["queries"][1]["values"][2]
                bad["queries"][1]["values"][2] = ("%02x" % (int(v[:2], 16) ^ 1)) + v[2:]
            elif where == "path":
                x = bad["queries"][0]["paths"][1][0]
                bad["queries"][0]["paths"][1][0] = ("%02x" % (int(x[:2], 16) ^ 0x80)) + x[2:]
            else:
                x = bad["residual"][0]
                bad["residual"][0] = ("%02x" % (int(x[:2], 16) ^ 1)) + x[2:]
            assert not pyref.fri_verify(p, nb, pyref.Transcript(label), _proof_bytes(bad, cfg), *args), where


@pytest.mark.parametrize("fname", ["goldilocks", "babybear"])
def test_small_field_coset_lde_vs_pure_python(fname):
    """The oracle's coset extension over the small fields (the checker of the device's
    small-field zntt_coset_lde_device) against pyref's independent composition."""
    f = FIELD_IDS[fname]
    p = O.MODULI[f]
    for log_in, log_blowup, shift in ((0, 1, 7), (3, 2, 7), (6, 1, 31), (8, 2, 1)):
        vals = pyref.random_field_values(p, 40 + log_in, 1 << log_in)
        got = _canon_ints(f, O.coset_lde(f, _mont_of(f, vals), log_in, log_blowup, _mont_of(f, [shift])[0]))
        assert got == pyref.coset_lde(vals, log_blowup, shift, p), (log_in, log_blowup, shift)


def test_row_commitment_fixture():
    """The oracle's row commitment (MerkleTree.init over rows, libs/merkle/src/merkle_tree.zig:
    70-103) against the pure-Python one in merkle_rows.json, all four fields, rows of one block
    to one full chunk."""
    d = json.load(open(os.path.join(GOLDEN, "merkle_rows.json")))
    for c in d["cases"]:
        f = FIELD_IDS[c["field"]]
        cols = [_mont_of(f, [int(v, 16) for v in col]) for col in c["values"]]
        nodes = O.merkle_commit_rows(f, cols, c["log_n"], workers=4)
        assert nodes[1].tobytes().hex() == c["root"], (c["field"], c["columns"])
        if "nodes" in c:
            assert [x.tobytes().hex() for x in nodes[1:]] == c["nodes"]
