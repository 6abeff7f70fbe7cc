"""C-ABI checks that need no GPU: the library loads, exports every declared
entry point, validates arguments in zig-ntt's error order before touching a
device (libs/ntt/src/root.zig:33-36, 43, 67-68, 150-152, 161), and computes
the host-side set-up values (roots of unity) exactly like the reference."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle as O


def test_library_exports_every_declared_symbol(zntt):
    declared = zntt.declared_symbols()
    assert len(declared) >= 19
    L = zntt.lib()
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing


def test_field_info(zntt):
    for F in zntt.FIELDS:
        mod = (ctypes.c_uint64 * 4)()
        adic = ctypes.c_uint32()
        assert zntt.lib().zntt_field_info(F.id, mod, ctypes.byref(adic)) == 0
        assert sum(int(v) << (64 * k) for k, v in enumerate(mod)) == F.modulus
        assert adic.value == F.two_adicity
    with pytest.raises(zntt.UnsupportedField):
        zntt._check(zntt.lib().zntt_field_info(7, mod, ctypes.byref(adic)))


@pytest.mark.parametrize("fname", ["bn254_fr", "bls12_381_fr"])
def test_primitive_root_matches_reference_derivation(zntt, oracle, fname):
    F = getattr(zntt, fname.upper())
    fid = {"bn254_fr": O.BN254_FR, "bls12_381_fr": O.BLS12_381_FR}[fname]
    for log_n in [0, 1, 2, 5, 12, 20, 24, F.two_adicity]:
        st, want = O.primitive_root(fid, log_n)
        assert st == 0
        got = zntt.primitiveRootOfUnity(F, log_n)
        np.testing.assert_array_equal(got, want)
    with pytest.raises(zntt.OrderTooLarge):
        zntt.primitiveRootOfUnity(F, F.two_adicity + 1)


def test_shape_errors_are_reported_before_any_device_work(zntt):
    F = zntt.BN254_FR
    root = zntt.primitiveRootOfUnity(F, 2)
    short = np.zeros((3, 4), dtype=np.uint64)
    with pytest.raises(zntt.LengthMismatch):
        zntt.ntt(F, short, 2, root)
    with pytest.raises(zntt.LengthMismatch):
        zntt.intt(F, short, 2, root)
    two = np.zeros((2, 4), dtype=np.uint64)
    with pytest.raises(zntt.LogTooLarge):
        zntt.ntt(F, two, 64, root)
    with pytest.raises(zntt.LogTooLarge):
        zntt.intt(F, two, 200, root)
    with pytest.raises(zntt.LogTooLarge):
        zntt.precomputeTwiddles(F, 64, root)
    with pytest.raises(zntt.InvalidLength):
        zntt.bitReverse(F, np.zeros((0, 4), dtype=np.uint64))
    with pytest.raises(zntt.InvalidLength):
        zntt.bitReverse(F, np.zeros((3, 4), dtype=np.uint64))
    data = np.zeros((8, 4), dtype=np.uint64)
    fake = [np.zeros((1 << s, 4), dtype=np.uint64) for s in range(3)]
    # table shorter than log_n
    with pytest.raises(zntt.InvalidTwiddles):
        zntt.nttWithTwiddles(F, data, 3, fake[:2])
    with pytest.raises(zntt.InvalidTwiddles):
        zntt.inttWithTwiddles(F, data, 3, fake[:2])
    # a stage of the wrong length
    with pytest.raises(zntt.InvalidTwiddles):
        zntt.nttWithTwiddles(F, data, 3, [fake[0], fake[1][:1], fake[2]])
    # order: LogTooLarge, then LengthMismatch, then InvalidTwiddles
    with pytest.raises(zntt.LogTooLarge):
        zntt.nttWithTwiddles(F, np.zeros((3, 4), dtype=np.uint64), 64, [])
    with pytest.raises(zntt.LengthMismatch):
        zntt.nttWithTwiddles(F, np.zeros((3, 4), dtype=np.uint64), 3, [])
    # on every error the data is untouched (validation precedes any mutation)
    d = np.arange(32, dtype=np.uint64).reshape(8, 4).copy()
    before = d.copy()
    with pytest.raises(zntt.InvalidTwiddles):
        zntt.nttWithTwiddles(F, d, 3, [fake[0], fake[1][:1], fake[2]])
    np.testing.assert_array_equal(d, before)


def test_unsupported_field_rejected(zntt):
    bogus = zntt.Field(9, "bogus", 7, 1)
    with pytest.raises(zntt.UnsupportedField):
        zntt.ntt(bogus, np.zeros((2, 4), dtype=np.uint64), 1, np.zeros(4, dtype=np.uint64))


def test_poly_mul_contract_before_any_device_work(zntt, oracle):
    """Polynomial.mul's results that need no transform (libs/poly/src/poly.zig:76-77, 198-200):
    a zero factor is the zero polynomial, and both DegreeTooLarge cases are raised before the
    library looks for a device."""
    for F, fid in ((zntt.BN254_FR, O.BN254_FR), (zntt.BLS12_381_FR, O.BLS12_381_FR)):
        b = O.random_elements(fid, 9, 4)
        for a in (np.zeros((3, 4), dtype=np.uint64), np.zeros((0, 4), dtype=np.uint64)):
            out, deg = zntt.poly_mul(F, a, b, 10)
            assert deg == -1 and not out.any() and out.shape == (11, 4)
        a = O.random_elements(fid, 10, 6)
        with pytest.raises(zntt.DegreeTooLarge):
            zntt.poly_mul(F, a, b, 7)  # product degree 8 > 7
        with pytest.raises(zntt.DegreeTooLarge):
            zntt.poly_mul(F, a, b[:1], 4)  # six coefficients do not fit max_degree 4
        # fromCoeffs checks the length before it normalizes: seven coefficients do not fit
        # max_degree 4 even when six of them are zero and the product (degree 2) would.
        padded = np.concatenate([b[:1], np.zeros((6, 4), dtype=np.uint64)])
        with pytest.raises(zntt.DegreeTooLarge):
            zntt.poly_mul(F, a[:3], padded, 4)
    with pytest.raises(zntt.UnsupportedField):
        zntt._check(zntt.lib().zntt_poly_mul(5, None, 0, None, 0, 0, None, None))
    with pytest.raises(zntt.InvalidArgument):
        zntt._check(zntt.lib().zntt_poly_mul(0, None, 2, None, 0, 4, None, None))


def test_fri_prover_loop_arguments_before_any_device_work(zntt):
    """The commit phase, the fused fold and commitment and the query openings check their sizes
    (Config.rounds' rules, libs/fri/src/root.zig:188-195), the field, alpha and their pointers
    before they look for a device."""
    F = zntt.BN254_FR
    never = lambda r, root: [0, 0, 0, 0]  # noqa: E731
    for log_domain, log_final in ((4, 4), (4, 5), (0, 0), (20, 13)):
        with pytest.raises(zntt.InvalidArgument):
            zntt.fri_commit_phase(F, log_domain, log_final, [1] * 30, [1] * 30, never)
    with pytest.raises(zntt.InvalidArgument):
        zntt.fri_commit_phase(F, 6, 2, [1, 1, 0, 1, 1], [1] * 4, never)  # a null layer
    with pytest.raises(zntt.UnsupportedField):
        zntt.fri_commit_phase(zntt.Field(9, "bogus", 7, 1), 6, 2, [1] * 5, [1] * 4, never)
    for log_domain, rounds in ((6, 0), (6, 7), (32, 4)):
        with pytest.raises(zntt.InvalidArgument):
            zntt.fri_query_extract(F, log_domain, rounds, [1] * 8, [16] * 8, [0])
    with pytest.raises(zntt.InvalidArgument):
        zntt.fri_query_extract(F, 6, 2, [1] * 3, [16] * 3, [64])  # a position outside the domain
    with pytest.raises(zntt.InvalidArgument):
        zntt.fri_query_extract(F, 6, 2, [1] * 3, [16] * 3, [])  # no queries
    with pytest.raises(zntt.InvalidArgument):
        zntt.fri_fold_commit(F, 1 << 20, 1, [0, 0, 0, 0], 1 << 24, 1 << 28)  # nothing left to commit
    with pytest.raises(zntt.InvalidArgument):
        zntt.fri_fold_commit(F, 1 << 20, 6, [2**64 - 1] * 4, 1 << 24, 1 << 28)  # alpha >= p
    with pytest.raises(zntt.UnsupportedField):
        zntt.fri_fold_commit(zntt.Field(9, "bogus", 7, 1), 1 << 20, 6, [0, 0, 0, 0], 1 << 24, 1 << 28)
    cols = (ctypes.c_void_p * 1)(1 << 20)
    for count in (0, 33, 1 << 27):  # no column, a row beyond one chunk, a byte size that wraps 32 bits
        with pytest.raises(zntt.InvalidArgument):
            zntt._check(zntt.lib().zntt_merkle_commit_rows(F.id, cols, count, 4, 1 << 28, None, None))
        with pytest.raises(zntt.InvalidArgument):
            zntt._check(zntt.lib().zntt_merkle_open_rows(F.id, cols, count, 4, 1 << 28,
                                                         (ctypes.c_uint64 * 1)(0), 1, b"x" * 64, b"x" * 64, None))


def test_small_field_poly_mul_contract_before_any_device_work(zntt):
    """Polynomial.mul's results that need no transform, for Goldilocks and BabyBear (one
    canonical u64 per coefficient): the zero polynomial, both DegreeTooLarge cases, and a
    non-canonical coefficient refused."""
    for F in (zntt.GOLDILOCKS, zntt.BABYBEAR):
        b = np.array([3, 1, 4], dtype=np.uint64)
        out, deg = zntt.poly_mul(F, np.zeros(3, dtype=np.uint64), b, 10)
        assert deg == -1 and not out.any() and out.shape == (11,)
        a = np.array([2, 7, 1, 8, 2, 8], dtype=np.uint64)
        with pytest.raises(zntt.DegreeTooLarge):
            zntt.poly_mul(F, a, b, 6)  # product degree 7 > 6
        with pytest.raises(zntt.DegreeTooLarge):
            zntt.poly_mul(F, a, b[:1], 4)  # six coefficients do not fit max_degree 4
        with pytest.raises(zntt.InvalidArgument):
            zntt.poly_mul(F, np.array([F.modulus], dtype=np.uint64), b, 10)


def test_column_entry_points_check_arguments_first(zntt):
    """The many-column entry points refuse null pointers, zero columns and unknown modes before
    they look at a table or a device."""
    L = zntt.lib()
    one = (ctypes.c_void_p * 1)(1 << 20)
    for args in ((None, one, one, 1, 0), (1, None, one, 1, 0), (1, one, one, 0, 0), (1, one, one, 1, 7)):
        with pytest.raises(zntt.InvalidArgument):
            zntt._check(L.zntt_ntt_device_columns(*args, None))
    shift = (ctypes.c_uint64 * 4)(7, 0, 0, 0)
    for args in ((None, 1, shift, one, one, 1), (1, 1, shift, None, one, 1), (1, 1, shift, one, one, 0)):
        with pytest.raises(zntt.InvalidArgument):
            zntt._check(L.zntt_coset_lde_columns(*args, None))


def test_small_fields_host_side(zntt, oracle):
    """Goldilocks and BabyBear: field info, primitive roots as zig-field derives them (the
    roots of the reference's KAT, libs/ntt/src/root.zig:437-447, and the oracle's at every
    order), and zig-ntt's error order before any device work."""
    import json
    import os
    kats = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ntt_kat.json")))
    for F, fid in ((zntt.GOLDILOCKS, O.GOLDILOCKS), (zntt.BABYBEAR, O.BABYBEAR)):
        mod = (ctypes.c_uint64 * 4)()
        adic = ctypes.c_uint32()
        assert zntt.lib().zntt_field_info(F.id, mod, ctypes.byref(adic)) == 0
        assert list(mod) == [F.modulus, 0, 0, 0] and adic.value == F.two_adicity
        for c in kats:
            if c["field"] == F.name:
                assert int(zntt.primitiveRootOfUnity(F, c["log_n"])[0]) == int(c["root"], 16)
        for log_n in range(F.two_adicity + 1):
            st, want = O.primitive_root(fid, log_n)
            assert st == 0
            got = zntt.primitiveRootOfUnity(F, log_n)
            assert int(got[0]) == O.to_ints(O.from_mont(fid, want.reshape(1, 4)))[0] and not got[1:].any()
        with pytest.raises(zntt.OrderTooLarge):
            zntt.primitiveRootOfUnity(F, F.two_adicity + 1)
        root = zntt.primitiveRootOfUnity(F, 2)
        with pytest.raises(zntt.LengthMismatch):
            zntt.ntt(F, np.zeros(3, dtype=np.uint64), 2, root)
        with pytest.raises(zntt.LogTooLarge):
            zntt.intt(F, np.zeros(2, dtype=np.uint64), 64, root)
        with pytest.raises(zntt.InvalidTwiddles):
            zntt.nttWithTwiddles(F, np.zeros(4, dtype=np.uint64), 2, [np.zeros(1, dtype=np.uint64)])
        with pytest.raises(zntt.InvalidLength):
            zntt.bitReverse(F, np.zeros(3, dtype=np.uint64))
        # The mirror refuses an array of the 256-bit layout for a small field, and vice versa,
        # so the library never reads past a buffer.
        with pytest.raises(zntt.InvalidArgument):
            zntt.ntt(F, np.zeros((4, 4), dtype=np.uint64), 2, root)
        with pytest.raises(zntt.InvalidTwiddles):
            zntt.nttWithTwiddles(zntt.BN254_FR, np.zeros((2, 4), dtype=np.uint64), 1, [np.zeros(1, dtype=np.uint64)])


def test_batch_spin_limit_and_pool_stats_need_no_device(zntt):
    """zntt_batch_set_spin_limit refuses a null batch before touching anything, and the pool
    counters read without a device."""
    L = zntt.lib()
    assert L.zntt_batch_set_spin_limit(None, 0) == 10  # ZNTT_ERR_INVALID_ARGUMENT
    assert "null batch" in L.zntt_last_error().decode()
    st = zntt.pool_stats()
    assert set(st) == {"acquires", "device_mallocs", "cached_bytes"}
    assert st["device_mallocs"] <= st["acquires"] * 2
    assert zntt.BATCH_SPIN_LIMIT == 1 << 22


def test_shipped_tuning_table_covers_every_size_and_shape(zntt):
    """The B200 table that bench.py loads has one entry per (field, log n, pass shape) for
    both 256-bit fields and log n 10..24, each with a stage count its shape's tile can hold,
    and it loads through zntt_tune_load (parsing needs no device)."""
    import json
    import os
    path = os.path.join(os.path.dirname(zntt.__file__), "tune", "b200.json")
    rows = json.load(open(path))
    log_tile = {0: 11, 1: 10, 2: 9, 3: 8, 4: 9}  # kShapes in csrc/kernels.cuh
    seen = {(r["field"], r["log_n"], r["shape"]) for r in rows}
    for f in (0, 1):
        for L in range(10, 25):
            for sh, lt in log_tile.items():
                assert (f, L, sh) in seen, (f, L, sh)
    for r in rows:
        assert r["gpu"] == "NVIDIA B200" and r["us"] > 0
        assert 2 <= r["kmax"] <= log_tile[r["shape"]], r
    assert zntt.lib().zntt_tune_load(path.encode()) == 0
    zntt.tune_clear()
