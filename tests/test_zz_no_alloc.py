"""mb2_radix_sort_pairs_static: the sort that allocates no device memory.

It must give exactly the result of the context sort (mb2_radix_sort_pairs) on
the same keys, and of a stable host sort (numpy argsort, kind "stable"), on
consecutive calls that share its static scratch, without changing the
device's free memory, and refuse sizes above its maximum before touching
anything. Called through the C ABI. This file is collected last so that it
also runs after every other GPU test in the same process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from mars_md_b200 import _lib

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _random_pairs(n, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    keys = torch.randint(-2**31, 2**31 - 1, (n,), dtype=torch.int32, device="cuda", generator=g)
    # A narrow key range too, so that many keys tie and stability matters.
    keys[: n // 2] &= 0xFF
    vals = torch.randperm(n, dtype=torch.int32, device="cuda", generator=g)
    return keys, vals


def test_static_sort_matches_context_sort_on_consecutive_calls(ctx_factory):
    lib = _lib.load()
    ctx = ctx_factory(16)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    # Set-up call (looks up the scratch address on this device).
    assert lib.mb2_radix_sort_pairs_static(ctx.h, None, None, 0, sp) == _lib.MB2_OK
    for n, seed in [(300_001, 11), (_lib.MB2_SORT_STATIC_MAX, 12), (2049, 13)]:
        keys, vals = _random_pairs(n, seed)
        k_host = keys.cpu().numpy().view(np.uint32)
        v_host = vals.cpu().numpy()
        order = np.argsort(k_host, kind="stable")
        k_ctx, v_ctx = keys.clone(), vals.clone()
        ctx.radix_sort_pairs(k_ctx, v_ctx, stream=stream)
        k_st, v_st = keys.clone(), vals.clone()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib.mb2_radix_sort_pairs_static(ctx.h, _ptr(k_st), _ptr(v_st), n, sp)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        assert rc == _lib.MB2_OK, lib.mb2_last_error(ctx.h)
        assert free_after == free_before
        # Integer sort: the results must be identical, payload order included.
        assert torch.equal(k_st, k_ctx)
        assert torch.equal(v_st, v_ctx)
        # Independent of either GPU sort: a stable sort of the same pairs on the host.
        assert np.array_equal(k_st.cpu().numpy().view(np.uint32), k_host[order])
        assert np.array_equal(v_st.cpu().numpy(), v_host[order])


def test_static_sort_rejects_sizes_above_maximum(ctx_factory):
    lib = _lib.load()
    ctx = ctx_factory(16)
    keys = torch.zeros(4, dtype=torch.int32, device="cuda")
    vals = torch.arange(4, dtype=torch.int32, device="cuda")
    # The size check runs on the host before any launch, so n may exceed the buffers.
    rc = lib.mb2_radix_sort_pairs_static(ctx.h, _ptr(keys), _ptr(vals),
                                         _lib.MB2_SORT_STATIC_MAX + 1, None)
    assert rc == _lib.MB2_ERR_CAPACITY
    assert b"MB2_SORT_STATIC_MAX" in lib.mb2_last_error(ctx.h)
    torch.cuda.synchronize()
    assert torch.equal(vals.cpu(), torch.arange(4, dtype=torch.int32))
