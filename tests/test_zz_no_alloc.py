"""The allocation-free in-place transform (zntt_ntt_device_inplace_noalloc).

Callers that may not allocate device memory while they transform -- a service
with a fixed up-front memory budget, a program whose memory belongs to another
allocator, a latency-critical path -- use this entry point; its scratch is an
8 MiB array inside the library.  The test calls it through the C ABI twice in a
row (so the second call starts from the scratch the first one left) and
checks each result bit-exactly against the existing entry point
zntt_ntt_device, and that the library's buffer pool saw no acquire and made no
cudaMalloc during the call (so a change that routed this entry point through
the pool would fail here); then checks that a transform larger than the array
is rejected without touching the data.  Collected last so that a failure here
leaves every other test already run.
"""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def z(zntt):
    zntt.init(0)
    return zntt


def _vec(z, F, seed, n):
    import torch
    x = torch.empty(n * 4, dtype=torch.int64, device="cuda")
    z.random_elements(F, seed, x.data_ptr(), n)
    return x


@pytest.mark.parametrize("log_n", [1, 11, 12, 16, 18])
def test_noalloc_matches_existing_entry_on_consecutive_calls(z, log_n):
    import torch
    for F in z.FIELDS:
        n = 1 << log_n
        with z.DeviceTwiddles(F, log_n, z.primitiveRootOfUnity(F, log_n)) as tw:
            for call, (seed, mode) in enumerate([(100 + log_n, z.FORWARD), (200 + log_n, z.INVERSE)]):
                x = _vec(z, F, seed, n)
                want = torch.empty_like(x)
                z.ntt_device(tw, x.data_ptr(), want.data_ptr(), mode)
                # The library runs on its own stream and torch on its: order the clone
                # after the input is made, and the in-place call after the clone.
                torch.cuda.synchronize()
                got = x.clone()
                torch.cuda.synchronize()
                before = z.pool_stats()
                z.ntt_device_inplace_noalloc(tw, got.data_ptr(), mode)
                torch.cuda.synchronize()
                after = z.pool_stats()
                assert after["acquires"] == before["acquires"], "the call took a pool buffer"
                assert after["device_mallocs"] == before["device_mallocs"], "the call allocated"
                assert torch.equal(got, want), f"{F} 2^{log_n} call {call}"


def test_noalloc_rejects_sizes_beyond_its_scratch(z):
    import torch
    F = z.BN254_FR
    with z.DeviceTwiddles(F, 19, z.primitiveRootOfUnity(F, 19)) as tw:
        x = _vec(z, F, 7, 1 << 19)
        torch.cuda.synchronize()
        before = x.clone()
        with pytest.raises(z.InvalidArgument, match="at most 2\\^18"):
            z.ntt_device_inplace_noalloc(tw, x.data_ptr(), z.FORWARD)
        torch.cuda.synchronize()
        assert torch.equal(x, before)
