"""lrt_prefix_sum_noalloc: the prefix sum for callers that cannot allocate
device memory (a plugin inside a host application that owns every device
allocation, or a frame-critical path where cudaMalloc would synchronise the
device). Its scratch is a fixed array compiled into the library, so these
checks compare it with the allocating lrt_prefix_sum on the same inputs, on
two calls in a row (the second call must not see the first call's leftovers),
and check that a count above its stated maximum is refused.

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


def test_noalloc_prefix_sum_equals_the_allocating_one_twice_in_a_row(rasterizer):
    # A large call first, then a smaller one: the second must not read the first's status words.
    for n, seed in ((3_000_017, 1), (100_003, 2), (4096, 3)):
        values = _counts(n, seed)
        got, got_total = _noalloc(values)
        want, want_total = _allocating(rasterizer, values)
        assert torch.equal(got, want)
        assert torch.equal(got_total, want_total)


def test_noalloc_prefix_sum_refuses_counts_above_its_maximum():
    values = torch.zeros(4, dtype=torch.int32, device="cuda")
    code = _abi.load().lrt_prefix_sum_noalloc(values.data_ptr(), values.data_ptr(), values.data_ptr(),
                                              _abi.PREFIX_SUM_NOALLOC_MAX + 1, None)
    assert code == _abi.INVALID_ARGUMENT
