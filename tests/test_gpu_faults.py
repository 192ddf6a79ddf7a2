"""The bounded device waits, made to run out without faulting the GPU.

Every wait in the library's kernels (the decoupled look-backs, the blend's
mbarrier waits) is bounded; when one gives up the kernel sets kErrTimeout,
returns, and the call reports LRT_TIMEOUT. Here the handle's test hook plants
the fault on the host side of a sort: the last digit pass starts its ticket
counter at 1, so partition 0 never publishes its counts and the partition
after it waits for nothing, up to a short poll limit. The call must return
TIMEOUT, and the same handle must go on to sort and render correctly."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L
from lucabrtrender_b200 import _abi

import helpers as H

pytestmark = pytest.mark.gpu


def _keys(count: int, seed: int):
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, 2**40, count, dtype=np.uint64)
    vals = np.arange(count, dtype=np.uint32)
    return keys, vals


def test_a_look_back_that_waits_for_nothing_times_out_and_the_handle_recovers():
    r = L.TileRasterizer.create(0)
    lib = _abi.load()
    try:
        keys, vals = _keys(100_003, 1)          # 33 partitions of 3072 keys, 5 passes of 8 bits
        kt = torch.from_numpy(keys.view(np.int64)).cuda()
        vt = torch.from_numpy(vals.view(np.int32)).cuda()
        assert lib.lrt_rast_debug_sort(r._handle, 1, 1024, 0) == _abi.OK
        with pytest.raises(_abi.LrtError) as info:
            r.radix_sort(kt, vt, 40)
        assert info.value.code == _abi.TIMEOUT
        torch.cuda.synchronize()                 # the context is still usable

        assert lib.lrt_rast_debug_sort(r._handle, 0, 0, 0) == _abi.OK
        keys, vals = _keys(100_003, 2)
        kt = torch.from_numpy(keys.view(np.int64)).cuda()
        vt = torch.from_numpy(vals.view(np.int32)).cuda()
        r.radix_sort(kt, vt, 40)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(kt.cpu().numpy().view(np.uint64), keys[order])
        assert np.array_equal(vt.cpu().numpy().view(np.uint32), vals[order])

        # and a frame on the same handle equals the oracle's bit for bit
        scene = H.reference_render_scenes()[0]
        targets = L.RenderTargets()
        stats = r.render(scene.camera, scene.gpu_instances(), scene.settings, targets)
        ref = scene.oracle_render()
        assert stats.pairs == ref["pairs"]
        assert np.array_equal(targets.colour.cpu().numpy(), ref["colour"])
    finally:
        r.close()


def test_the_fault_hook_with_the_normal_poll_limit_still_returns():
    """The same planted fault with the library's own limit (2^22 polls): the
    wait is long but bounded, and the call still comes back with TIMEOUT."""
    r = L.TileRasterizer.create(0)
    lib = _abi.load()
    try:
        keys, vals = _keys(20_000, 3)
        kt = torch.from_numpy(keys.view(np.int64)).cuda()
        assert lib.lrt_rast_debug_sort(r._handle, 1, 0, 0) == _abi.OK
        with pytest.raises(_abi.LrtError) as info:
            r.radix_sort(kt, None, 16)
        assert info.value.code == _abi.TIMEOUT
    finally:
        r.close()


@pytest.mark.parametrize("key_bits,with_values", [(40, True), (64, False), (24, True)])
def test_the_wide_look_back_words_sort_as_the_narrow_ones(key_bits, with_values):
    """Sorts of 2^30 keys or more count their look-back in 64-bit words; the
    hook asks for that form on a sort small enough to run here."""
    r = L.TileRasterizer.create(0)
    lib = _abi.load()
    try:
        rng = np.random.default_rng(key_bits)
        keys = rng.integers(0, 2**63, 500_009, dtype=np.uint64) & np.uint64((1 << key_bits) - 1 if key_bits < 64
                                                                            else 2**64 - 1)
        vals = np.arange(keys.size, dtype=np.uint32)
        assert lib.lrt_rast_debug_sort(r._handle, 0, 0, 1) == _abi.OK
        kt = torch.from_numpy(keys.view(np.int64)).cuda()
        vt = torch.from_numpy(vals.view(np.int32)).cuda() if with_values else None
        r.radix_sort(kt, vt, key_bits)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(kt.cpu().numpy().view(np.uint64), keys[order])
        if with_values:
            assert np.array_equal(vt.cpu().numpy().view(np.uint32), vals[order])
    finally:
        r.close()
