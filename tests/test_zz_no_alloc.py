"""The no-allocation Leopard reconstruction entry point.

rsgpu_leopard_reconstruct_noalloc serves callers that must not allocate
device memory while handling a request (memory reserved up front, or a fixed
quota where cudaMalloc can fail or synchronize the device).  It works out of
static device buffers, so these tests call it through the C ABI and compare
its bytes with the regular rsgpu_reconstruct entry point, twice in a row with
different erasure patterns (the static buffers keep the previous call's
contents, and the second call must not be affected by them).

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rs():
    import rsgpu

    return rsgpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    assert t.cuda.is_available()
    return t


def noalloc(rs, torch, codec, shards, present):
    """Call the entry point through the C ABI on device shard pointers."""
    n = len(shards)
    ptrs = (ctypes.c_void_p * n)(*[s.data_ptr() for s in shards])
    lens = (ctypes.c_size_t * n)(*[s.numel() for s in shards])
    pres = (ctypes.c_uint8 * n)(*[1 if p else 0 for p in present])
    stream = torch.cuda.current_stream().cuda_stream
    return rs.lib().rsgpu_leopard_reconstruct_noalloc(codec._h, ptrs, lens, pres, n, stream)


@pytest.mark.parametrize("family,k,m,size", [
    ("leopard_gf16", 2048, 1024, 1024),   # 4096 lanes: the global-work decode
    ("leopard_gf16", 64, 32, 4096),
    ("leopard_gf8", 32, 16, 4096),
])
def test_noalloc_matches_regular_entry_point_twice(rs, torch, family, k, m, size):
    codec = rs.ReedSolomon(k, m, rs.CodecOptions(codec_family=family))
    rng = np.random.default_rng(k * 31 + m)
    full = torch.zeros((k + m, size), dtype=torch.uint8, device="cuda")
    full[:k] = torch.from_numpy(rng.integers(0, 256, (k, size), dtype=np.uint8)).cuda()
    codec.encode([full[i] for i in range(k + m)])
    torch.cuda.synchronize()
    for call, n_lost in enumerate([m, max(1, m // 3)]):
        lost = set(rng.choice(k + m, size=n_lost, replace=False).tolist())
        present = [i not in lost for i in range(k + m)]
        # Regular entry point on one copy ...
        a = full.clone()
        for i in lost:
            a[i].fill_(0x5A)
        lst = [None if i in lost else a[i] for i in range(k + m)]
        codec.reconstruct(lst)
        # ... the no-allocation one on another.
        b = full.clone()
        for i in lost:
            b[i].fill_(0xA5)
        rc = noalloc(rs, torch, codec, [b[i] for i in range(k + m)], present)
        assert rc == 0, rs.ERROR_NAMES.get(rc, rc)
        torch.cuda.synchronize()
        for i in range(k + m):
            assert torch.equal(lst[i], b[i]), (family, call, i)
        assert torch.equal(b, full), (family, call)


def test_noalloc_rejects_codes_beyond_its_static_limit(rs, torch):
    # 14000 + 4000 needs 32768 transform lanes, more than the static buffers hold.
    k, m = 14000, 4000
    codec = rs.ReedSolomon(k, m, rs.CodecOptions(codec_family="leopard_gf16"))
    t = torch.zeros(64, dtype=torch.uint8, device="cuda")
    present = [i != 0 for i in range(k + m)]
    rc = noalloc(rs, torch, codec, [t] * (k + m), present)
    assert rs.ERROR_NAMES.get(rc) == "ScratchLimit"
    assert (t == 0).all()
