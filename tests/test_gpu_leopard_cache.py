"""The Leopard error-locator cache is bounded (least recently used patterns
out beyond its byte budget, as the reference bounds its decode-plan cache,
src/core/leopard_gf16/decode.rs:268-305), and batches prepared before their
patterns were evicted still rebuild the right bytes: every launch reads its
own copies of the locators."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

K, M, SIZE = 10000, 100, 64       # 2^14 transform lanes: 32 KiB of locators per pattern
BLOCK = 2 * 16384
BUDGET = max(32 << 20, 64 * BLOCK)


@pytest.fixture(scope="module")
def rs():
    import rsgpu

    return rsgpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    assert t.cuda.is_available()
    return t


def patterns(rng, n):
    out = np.ones((n, K + M), np.uint8)
    for s in range(n):
        e = int(rng.integers(1, M + 1))
        out[s, rng.choice(K + M, size=e, replace=False)] = 0
    return out


def test_locator_cache_stays_bounded_and_batches_keep_their_locators(rs, torch):
    rng = np.random.default_rng(77)
    codec = rs.ReedSolomon(K, M, rs.CodecOptions(codec_family="leopard_gf16"))
    n = 160
    # Non-codeword stripes; the expected rebuild of a few comes from the oracle.
    full = torch.randint(0, 256, (n, K + M, SIZE), dtype=torch.uint8, device="cuda")
    host_full = full.cpu().numpy()
    ptrs = rs.device_pointer_table(full.data_ptr(), np.arange(n * (K + M), dtype=np.uint64) * np.uint64(SIZE))
    first = patterns(rng, n)
    prepared = codec.prepare_batch("reconstruct", ptrs, SIZE, present=first)

    def expect(s, pres):
        ref = [host_full[s, i].copy() for i in range(K + M)]
        for i in range(K + M):
            if not pres[i]:
                ref[i][:] = 0
        assert O.leopard_reconstruct(16, K, M, ref, pres) == 0
        return ref

    checked = [0, n // 2, n - 1]
    want_first = {s: expect(s, first[s]) for s in checked}
    # Stream many more distinct patterns than the cache holds through the
    # per-call batch API, checking a few rebuilt stripes each round.
    rounds = (BUDGET // BLOCK) // n + 3
    for r in range(rounds):
        pats = patterns(rng, n)
        buf = full.clone()
        bptrs = rs.device_pointer_table(buf.data_ptr(), np.arange(n * (K + M), dtype=np.uint64) * np.uint64(SIZE))
        lost = torch.from_numpy(pats == 0).cuda()
        buf.masked_fill_(lost.unsqueeze(-1), 0xA5)
        codec.reconstruct_batch(buf, pats)
        st = codec.cache_stats()
        # A call may keep its own patterns beyond the budget, never more.
        assert st.retained_bytes <= BUDGET + n * BLOCK, (r, st.retained_bytes)
        if r in (0, rounds - 1):
            got = buf.cpu().numpy()
            ref = expect(7, pats[7])
            for i in range(K + M):
                assert np.array_equal(got[7, i], ref[i]), (r, i)
        del buf, lost
    st = codec.cache_stats()
    assert st.evictions > 0 and st.entries * BLOCK <= BUDGET + n * BLOCK
    assert st.inserts == st.misses and st.requests == st.hits + st.misses
    # The batch prepared at the start: its patterns have long left the cache.
    lost = torch.from_numpy(first == 0).cuda()
    full.masked_fill_(lost.unsqueeze(-1), 0xA5)
    prepared.launch()
    torch.cuda.synchronize()
    got = full.cpu().numpy()
    for s in checked:
        for i in range(K + M):
            assert np.array_equal(got[s, i], want_first[s][i]), (s, i)
