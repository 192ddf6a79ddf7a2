"""lrt_prefix_sum_noalloc: the prefix sum for callers that cannot allocate
device memory (a plugin inside a host application that owns every device
allocation, or a frame-critical path where cudaMalloc would synchronise the
device). Its scratch is a fixed array compiled into the library, so these
checks compare it with the allocating lrt_prefix_sum and with a numpy scan on
the same inputs, on two calls in a row (the second call must not see the
first call's leftovers), on counts 0 and 1 and an input that is not 16-byte
aligned, and check that a count above its stated maximum is refused.

This file is collected last on purpose: a failure here leaves every other
test already run."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from lucabrtrender_b200 import _abi

pytestmark = pytest.mark.gpu


def _counts(n: int, seed: int) -> torch.Tensor:
    rng = np.random.default_rng(seed)
    c = rng.integers(0, 37, n, dtype=np.uint32)
    c[rng.random(n) < 0.125] = 0
    return torch.from_numpy(c.view(np.int32)).cuda()


def _noalloc(values: torch.Tensor):
    out = torch.full_like(values, -1)
    total = torch.full((1,), -1, dtype=torch.int32, device=values.device)
    code = _abi.load().lrt_prefix_sum_noalloc(values.data_ptr(), out.data_ptr(), total.data_ptr(), values.numel(),
                                              torch.cuda.current_stream().cuda_stream)
    assert code == _abi.OK, _abi.STATUS_NAMES.get(code, code)
    return out, total


def _allocating(rasterizer, values: torch.Tensor):
    out = torch.full_like(values, -1)
    total = torch.full((1,), -1, dtype=torch.int32, device=values.device)
    rasterizer.prefix_sum(values, out, total)
    return out, total


def _numpy_scan(values: torch.Tensor):
    """The exclusive prefix sum in 64-bit numpy, checked to stay below 2^32."""
    v = values.cpu().numpy().view(np.uint32).astype(np.uint64)
    inclusive = np.cumsum(v, dtype=np.uint64)
    total = int(inclusive[-1]) if v.size else 0
    assert total < 2**32
    exclusive = (inclusive - v).astype(np.uint32)
    return exclusive, total


def test_noalloc_prefix_sum_equals_the_allocating_one_twice_in_a_row(rasterizer):
    # A large call first, then a smaller one: the second must not read the first's status words.
    for n, seed in ((3_000_017, 1), (100_003, 2), (4096, 3)):
        values = _counts(n, seed)
        got, got_total = _noalloc(values)
        want, want_total = _allocating(rasterizer, values)
        assert torch.equal(got, want)
        assert torch.equal(got_total, want_total)
        # and against a scan that shares no code with either
        ref, ref_total = _numpy_scan(values)
        assert np.array_equal(got.cpu().numpy().view(np.uint32), ref)
        assert int(got_total.cpu().numpy().view(np.uint32)[0]) == ref_total


def test_noalloc_prefix_sum_edge_counts_and_an_unaligned_input():
    # count 0 and 1, and input/output one element past a 16-byte boundary
    # (the kernel's element-wise load and store path).
    for n in (0, 1, 5, 4097):
        values = _counts(max(n, 1), 10 + n)[:n]
        got, got_total = _noalloc(values)
        ref, ref_total = _numpy_scan(values)
        assert np.array_equal(got.cpu().numpy().view(np.uint32), ref)
        assert int(got_total.cpu().numpy().view(np.uint32)[0]) == ref_total
    backing = _counts(70_001, 4)
    values = backing[1:]
    assert values.data_ptr() % 16 != 0
    out = torch.full((70_001,), -1, dtype=torch.int32, device="cuda")[1:]
    total = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    code = _abi.load().lrt_prefix_sum_noalloc(values.data_ptr(), out.data_ptr(), total.data_ptr(), values.numel(),
                                              torch.cuda.current_stream().cuda_stream)
    assert code == _abi.OK
    ref, ref_total = _numpy_scan(values)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)
    assert int(total.cpu().numpy().view(np.uint32)[0]) == ref_total


def test_noalloc_prefix_sum_refuses_counts_above_its_maximum():
    values = torch.zeros(4, dtype=torch.int32, device="cuda")
    code = _abi.load().lrt_prefix_sum_noalloc(values.data_ptr(), values.data_ptr(), values.data_ptr(),
                                              _abi.PREFIX_SUM_NOALLOC_MAX + 1, None)
    assert code == _abi.INVALID_ARGUMENT
