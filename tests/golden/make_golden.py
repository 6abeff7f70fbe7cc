"""Regenerates the golden fixtures in this folder.

    python tests/golden/make_golden.py [--reference PATH]

Two kinds of fixture:

1. Vectors copied as data from the reference's own tests, read as text:
   * ntt_kat.json -- the known-answer DFT cases of libs/ntt/src/root.zig:438-449
     (Goldilocks and BabyBear, log_n 1-4, root / input / expected output).
   * chacha20_rfc8439.json -- the RFC 8439 keystream vectors that
     libs/rng/src/root.zig:182-228 checks the reference's ChaCha20 against.
2. Vectors computed here by pyref.py (pure Python, independent of the oracle
   and of the CUDA library) for the two scalar fields the transform serves:
   * fr_transforms.json -- seeded randomFieldElement inputs (ChaCha20, seed
     encoding u64 LE + zeros), the reference-derived primitive roots, and the
     forward / inverse transforms by definition (n <= 2^6) or by a radix-2 FFT
     checked against the definition (n = 2^12, the plain 2^12 BN254-Fr case).
   * coset_lde.json -- a small blowup-4 coset extension over BLS12-381-Fr with
     shift 5, the reference's quadratic non-residue.
   * fri_commit.json -- the reference's BLAKE3 known answer (libs/hash/src/root.zig,
     kat.blake3_hello_world, copied as data) and FRI layer commitments (hashPair
     leaves and the Merkle node array) of seeded layers over all four fields.
   * poly_mul.json -- polynomial products by the schoolbook sum over both
     fields: seeded factors of several lengths, trailing zero coefficients
     (normalized away), a zero factor, constants, and max_degree cases that
     fit exactly or raise DegreeTooLarge.
   * merkle_rows.json -- row commitments (MerkleTree.init over the rows of several columns,
     each row's toBytes values concatenated) for all four fields, rows of one block up to
     one full 1024-byte chunk.
   * fri_proof.json -- the reference's transcript known answer (four Goldilocks
     challenges from Transcript.init("wire-compat"), libs/fri/src/root.zig, copied as
     data and reproduced by pyref.Transcript) and whole FRI proofs of pyref.fri_prove
     over that transcript for low-degree evaluations in all four fields, each accepted
     by pyref.fri_verify.

Values are canonical (not Montgomery) hex strings.  Large vectors are stored as
a SHA-256 of their little-endian 32-byte encoding plus a few leading values.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import pyref  # noqa: E402


def vec_digest(values: list[int]) -> str:
    h = hashlib.sha256()
    for v in values:
        h.update(int(v).to_bytes(32, "little"))
    return h.hexdigest()


def parse_kats(ref: str) -> list[dict]:
    path = os.path.join(ref, "libs/ntt/src/root.zig")
    lines = open(path).read().splitlines()
    cases = []
    field = None
    for ln, text in enumerate(lines, start=1):
        if text.strip() == "// Goldilocks":
            field = "goldilocks"
        elif text.strip() == "// BabyBear":
            field = "babybear"
        m = re.search(r"\.log_n = (\d+), \.root = (0x[0-9a-f]+), \.input = &\.\{ ([^}]*) \}, "
                      r"\.expect = &\.\{ ([^}]*) \}", text)
        if m and field:
            cases.append({
                "field": field,
                "log_n": int(m.group(1)),
                "root": m.group(2),
                "input": [s.strip() for s in m.group(3).split(",")],
                "expect": [s.strip() for s in m.group(4).split(",")],
                "source": f"libs/ntt/src/root.zig:{ln}",
            })
    assert len(cases) == 8, len(cases)
    return cases


def parse_rfc(ref: str) -> dict:
    path = os.path.join(ref, "libs/rng/src/root.zig")
    text = open(path).read()
    hexes = re.findall(r'hexToBytes\(&want_\w+, "([0-9a-f]+)"\)', text)
    plain = re.search(r'const plaintext = "([^"]+)";', text).group(1)
    assert len(hexes) == 3
    return {
        "key": bytes(range(32)).hex(),
        "block_nonce": "000000090000004a00000000",
        "block_counter1": hexes[0],
        "cipher_nonce": "000000000000004a00000000",
        "keystream_counter1": hexes[1],
        "ciphertext": hexes[2],
        "plaintext": plain,
        "source": "libs/rng/src/root.zig:182-228 (RFC 8439 sections 2.3.2 and 2.4.2)",
    }


def fr_cases() -> list[dict]:
    out = []
    plan = [("bn254_fr", pyref.BN254_FR_P, [1, 2, 3, 4, 5, 6], 101),
            ("bls12_381_fr", pyref.BLS12_381_FR_P, [1, 2, 3, 4, 5, 6], 202)]
    for name, p, logs, seed0 in plan:
        for log_n in logs:
            n = 1 << log_n
            seed = seed0 + log_n
            x = pyref.random_field_values(p, seed, n)
            w = pyref.primitive_root(p, log_n)
            fwd = pyref.dft(x, w, p)
            assert pyref.fft(x, w, p) == fwd
            inv = pyref.inverse_transform(x, w, p)
            out.append({"field": name, "log_n": log_n, "seed": seed, "root": hex(w),
                        "input": [hex(v) for v in x], "forward": [hex(v) for v in fwd],
                        "inverse": [hex(v) for v in inv]})
    # The plain 2^12 BN254-Fr transform: forward by FFT, inverse round trip.
    p, log_n, seed = pyref.BN254_FR_P, 12, 12
    x = pyref.random_field_values(p, seed, 1 << log_n)
    w = pyref.primitive_root(p, log_n)
    fwd = pyref.fft(x, w, p)
    inv = pyref.inverse_transform(x, w, p)
    # Spot-check the FFT against the definition at a few indices.
    for k in (0, 1, 7, 2048, 4095):
        assert fwd[k] == sum(x[j] * pow(w, j * k, p) for j in range(len(x))) % p
    out.append({"field": "bn254_fr", "log_n": log_n, "seed": seed, "root": hex(w),
                "input_sha256": vec_digest(x), "input_head": [hex(v) for v in x[:8]],
                "forward_sha256": vec_digest(fwd), "forward_head": [hex(v) for v in fwd[:8]],
                "inverse_sha256": vec_digest(inv), "inverse_head": [hex(v) for v in inv[:8]]})
    return out


def lde_case() -> dict:
    p = pyref.BLS12_381_FR_P
    log_in, log_blowup, seed = 6, 2, 303
    evals = pyref.random_field_values(p, seed, 1 << log_in)
    shift = pyref.first_qnr(p)
    assert shift == 5
    out = pyref.coset_lde(evals, log_blowup, shift, p)
    return {"field": "bls12_381_fr", "log_in": log_in, "log_blowup": log_blowup, "seed": seed,
            "shift": shift, "evals": [hex(v) for v in evals], "output": [hex(v) for v in out]}


def poly_cases() -> list[dict]:
    out = []
    plan = [("bn254_fr", pyref.BN254_FR_P, 404), ("bls12_381_fr", pyref.BLS12_381_FR_P, 505)]
    shapes = [(1, 1), (1, 7), (5, 3), (16, 16), (33, 17), (64, 1), (100, 57)]
    for name, p, seed0 in plan:
        for q, (la, lb) in enumerate(shapes):
            a = pyref.random_field_values(p, seed0 + 2 * q, la)
            b = pyref.random_field_values(p, seed0 + 2 * q + 1, lb)
            c = pyref.poly_mul(a, b, p)
            d = len(c) - 1
            out.append({"field": name, "a": [hex(v) for v in a], "b": [hex(v) for v in b],
                        "max_degree": d + 3, "degree": d, "product": [hex(v) for v in c]})
        # Trailing zeros in the inputs are dropped; the product has exactly max_degree.
        a = pyref.random_field_values(p, seed0 + 50, 6) + [0, 0]
        b = pyref.random_field_values(p, seed0 + 51, 4) + [0]
        c = pyref.poly_mul(a, b, p)
        out.append({"field": name, "a": [hex(v) for v in a], "b": [hex(v) for v in b],
                    "max_degree": len(c) - 1, "degree": len(c) - 1, "product": [hex(v) for v in c]})
        # One degree short of fitting: DegreeTooLarge.
        out.append({"field": name, "a": [hex(v) for v in a], "b": [hex(v) for v in b],
                    "max_degree": len(c) - 2, "error": "DegreeTooLarge"})
        # A factor with more coefficients than the capacity: DegreeTooLarge (fromCoeffs).
        out.append({"field": name, "a": [hex(v) for v in a], "b": ["0x1"], "max_degree": len(a) - 2,
                    "error": "DegreeTooLarge"})
        # A zero factor (all coefficients zero, or none): the zero polynomial.
        out.append({"field": name, "a": ["0x0", "0x0"], "b": [hex(v) for v in b], "max_degree": 10,
                    "degree": -1, "product": []})
        out.append({"field": name, "a": [], "b": [hex(v) for v in b], "max_degree": 10, "degree": -1,
                    "product": []})
    return out


def parse_blake3_kat(ref: str) -> dict:
    path = os.path.join(ref, "libs/hash/src/root.zig")
    text = open(path).read()
    start = text.index("pub const blake3_hello_world")
    body = text[start:text.index("};", start)]
    lineno = text[:start].count("\n") + 1
    digest = bytes(int(b, 16) for b in re.findall(r"0x([0-9a-f]{2})", body))
    assert len(digest) == 32
    return {"message": "hello world", "blake3": digest.hex(), "source": f"libs/hash/src/root.zig:{lineno}"}


def fri_commit_cases(ref: str) -> dict:
    kat = parse_blake3_kat(ref)
    assert pyref.blake3(kat["message"].encode()).hex() == kat["blake3"]
    fields = [("bn254_fr", pyref.BN254_FR_P, 32), ("bls12_381_fr", pyref.BLS12_381_FR_P, 32),
              ("goldilocks", 0xFFFFFFFF00000001, 8), ("babybear", 0x78000001, 4)]
    cases = []
    for q, (name, p, nb) in enumerate(fields):
        for log_n in (1, 2, 5, 8):
            values = pyref.random_field_values(p, 1000 + 10 * q + log_n, 1 << log_n)
            nodes = pyref.fri_commit_layer(values, nb)
            case = {"field": name, "log_n": log_n, "num_bytes": nb, "values": [hex(v) for v in values],
                    "root": nodes[1].hex()}
            if log_n <= 5:  # the whole node array for the small layers, the root for the others
                case["nodes"] = [x.hex() for x in nodes[1:]]
            cases.append(case)
    return {"kat": kat, "empty": pyref.blake3(b"").hex(), "cases": cases}


def parse_transcript_kat(ref: str) -> dict:
    """The reference's challenge-sequence known answer (libs/fri/src/root.zig, test "fri: the
    transcript switch preserved the challenge sequence"): four Goldilocks challenges from
    Transcript.init("wire-compat"), toBytes concatenated."""
    path = os.path.join(ref, "libs/fri/src/root.zig")
    text = open(path).read()
    start = text.index('test "fri: the transcript switch preserved the challenge sequence"')
    m = re.search(r'if \(F == Goldilocks\)\s*"([0-9a-f]+)"', text[start:])
    label = re.search(r'Transcript\.init\("([^"]+)"\)', text[start:]).group(1)
    lineno = text[:start + m.start(1)].count("\n") + 1
    return {"label": label, "field": "goldilocks", "draws": 4, "expect": m.group(1),
            "source": f"libs/fri/src/root.zig:{lineno}"}


FRI_FIELDS = [("bn254_fr", pyref.BN254_FR_P, 32), ("bls12_381_fr", pyref.BLS12_381_FR_P, 32),
              ("goldilocks", 0xFFFFFFFF00000001, 8), ("babybear", 0x78000001, 4)]


def fri_proof_cases(ref: str) -> dict:
    """Whole FRI proofs of the pure-Python prove (pyref.fri_prove) over the reference's
    transcript, for the evaluations of a polynomial of degree < 2^log_initial_degree on the
    2^log_domain subgroup; each verifies under pyref.fri_verify."""
    kat = parse_transcript_kat(ref)
    t = pyref.Transcript(kat["label"].encode())
    got = b"".join(t.challenge_field_checked(0xFFFFFFFF00000001, 8).to_bytes(8, "little") for _ in range(4))
    assert got.hex() == kat["expect"], "transcript restatement differs from the reference's known answer"
    cfg = {"log_domain": 8, "log_initial_degree": 6, "log_final": 3, "log_residual_degree": 1, "num_queries": 3,
           "label": "zig-algebra-b200 fri golden"}
    cases = []
    for q, (name, p, nb) in enumerate(FRI_FIELDS):
        n = 1 << cfg["log_domain"]
        coeffs = pyref.random_field_values(p, 1100 + q, 1 << cfg["log_initial_degree"])
        evals = pyref.fft(coeffs + [0] * (n - len(coeffs)), pyref.primitive_root(p, cfg["log_domain"]), p)
        args = (cfg["log_domain"], cfg["log_final"], cfg["log_residual_degree"], cfg["num_queries"])
        proof = pyref.fri_prove(p, nb, pyref.Transcript(cfg["label"].encode()), evals, *args)
        assert pyref.fri_verify(p, nb, pyref.Transcript(cfg["label"].encode()), proof, *args)
        cases.append({"field": name, "evals": [hex(v) for v in evals],
                      "roots": [r.hex() for r in proof["roots"]], "residual": [c.hex() for c in proof["residual"]],
                      "queries": [{"pair_index": qq["pair_index"], "values": [v.hex() for v in qq["values"]],
                                   "paths": [[x.hex() for x in path] for path in qq["paths"]]}
                                  for qq in proof["queries"]]})
    return {"transcript_kat": kat, "config": cfg, "cases": cases}


def merkle_rows_cases() -> dict:
    """Row commitments (pyref.merkle_commit_rows: MerkleTree.init over rows of columns) for
    seeded columns of all four fields, with rows of one block, several blocks and exactly one
    chunk (1024 bytes)."""
    cases = []
    for q, (name, p, nb) in enumerate(FRI_FIELDS):
        for m, log_n in ((1, 3), (2, 4), (3, 2), (5, 5), (1024 // nb, 2)):
            cols = [pyref.random_field_values(p, 1500 + 37 * q + 7 * m + c, 1 << log_n) for c in range(m)]
            nodes = pyref.merkle_commit_rows(cols, nb)
            case = {"field": name, "columns": m, "log_n": log_n, "values": [[hex(v) for v in c] for c in cols],
                    "root": nodes[1].hex()}
            if log_n <= 4:
                case["nodes"] = [x.hex() for x in nodes[1:]]
            cases.append(case)
    return {"cases": cases}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("ZIG_ALGEBRA_SRC"),
                    help="the zig-algebra source tree the known answers are read from "
                         "(default: $ZIG_ALGEBRA_SRC)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference or set ZIG_ALGEBRA_SRC to the zig-algebra source tree")
    json.dump(parse_kats(args.reference), open(os.path.join(HERE, "ntt_kat.json"), "w"), indent=1)
    json.dump(parse_rfc(args.reference), open(os.path.join(HERE, "chacha20_rfc8439.json"), "w"), indent=1)
    json.dump(fr_cases(), open(os.path.join(HERE, "fr_transforms.json"), "w"), indent=1)
    json.dump(lde_case(), open(os.path.join(HERE, "coset_lde.json"), "w"), indent=1)
    json.dump(poly_cases(), open(os.path.join(HERE, "poly_mul.json"), "w"), indent=1)
    json.dump(fri_commit_cases(args.reference), open(os.path.join(HERE, "fri_commit.json"), "w"), indent=1)
    json.dump(fri_proof_cases(args.reference), open(os.path.join(HERE, "fri_proof.json"), "w"), indent=1)
    json.dump(merkle_rows_cases(), open(os.path.join(HERE, "merkle_rows.json"), "w"), indent=1)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
