"""verify_with_buffer (src/core/verify.rs:157-200; Leopard: :35-57) on the GPU:
the caller's buffers receive the recomputed parity, byte-exact against the
oracle's encode, and the flag says whether it equals the stored parity --
classic GF(2^8) (one K1 pass that compares and stores), Leopard GF(2^8) /
GF(2^16) and the tower field (encode into the buffers, then compare)."""
import numpy as np
import pytest

import oracle as O

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


def classic_ref(k, m, data):
    rc, mat = O.build_matrix(k, m)
    ref = [d.copy() for d in data] + [np.zeros(data[0].size, np.uint8) for _ in range(m)]
    O.classic_encode(mat, ref)
    return ref


def leopard_ref(field, k, m, data):
    rc, par = O.leopard_encode(field, k, m, data)
    assert rc == 0
    return list(data) + par


def tower_ref(k, m, data):
    rc, mat = O.gf16t_build_matrix(k, m)
    ref = [d.copy() for d in data] + [np.zeros(data[0].size, np.uint8) for _ in range(m)]
    O.gf16t_encode(mat, ref)
    return ref


CASES = [("classic", 10, 4, 65536), ("classic", 16, 4, 4096 + 15), ("classic", 4, 2, 1), ("classic", 20, 10, 5000),
         ("classic", 8, 1, 777), ("lgf8", 32, 16, 4096), ("lgf8", 10, 4, 256 << 10), ("lgf16", 64, 32, 1024),
         ("lgf16", 10, 4, 4096), ("tower", 6, 3, 1000)]


def make_codec(rs, kind, k, m):
    if kind == "classic":
        return rs.ReedSolomon(k, m)
    if kind == "tower":
        return rs.ReedSolomon(k, m, field="gf16")
    return rs.ReedSolomon(k, m, rs.CodecOptions(codec_family="leopard_gf8" if kind == "lgf8" else "leopard_gf16"))


def reference(kind, k, m, data):
    if kind == "classic":
        return classic_ref(k, m, data)
    if kind == "tower":
        return tower_ref(k, m, data)
    return leopard_ref(8 if kind == "lgf8" else 16, k, m, data)


@pytest.mark.parametrize("where", ["device", "host"])
@pytest.mark.parametrize("kind,k,m,size", CASES)
def test_verify_with_buffer_matches_oracle(rs, torch, where, kind, k, m, size):
    rng = np.random.default_rng(k * 131 + m + size + len(kind) + len(where))
    data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
    ref = reference(kind, k, m, data)
    codec = make_codec(rs, kind, k, m)
    cases = [(list(ref), True)]
    bad = [s.copy() for s in ref]
    bad[k + m - 1][size // 2] ^= 0x81
    cases.append((bad, False))
    stale = [s.copy() for s in ref]
    stale[0][0] ^= 1  # data changed, parity not: the buffer holds the new parity
    cases.append((stale, False))
    for shards, expect in cases:
        want = reference(kind, k, m, shards[:k])[k:]
        if where == "device":
            sh = [torch.from_numpy(s.copy()).cuda() for s in shards]
            buf = [torch.full((size,), 0x77, dtype=torch.uint8, device="cuda") for _ in range(m)]
        else:
            sh = [s.copy() for s in shards]
            buf = [np.full(size, 0x77, np.uint8) for _ in range(m)]
        ok = codec.verify_with_buffer(sh, buf)
        assert ok == expect, (kind, k, m, size)
        got = [b.cpu().numpy() for b in buf] if where == "device" else buf
        for r in range(m):
            assert (got[r] == want[r]).all(), (kind, r)
        if kind == "classic":
            assert codec.verify(sh) == expect


def test_verify_with_buffer_misaligned_device_pointers(rs, torch):
    k, m, size = 10, 4, 4099
    rng = np.random.default_rng(3)
    data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
    ref = classic_ref(k, m, data)
    codec = rs.ReedSolomon(k, m)
    big = [torch.zeros(size + 7, dtype=torch.uint8, device="cuda") for _ in range(k + m)]
    views = [b[3:3 + size] for b in big]
    for v, d in zip(views, ref):
        v.copy_(torch.from_numpy(d))
    bbig = [torch.zeros(size + 5, dtype=torch.uint8, device="cuda") for _ in range(m)]
    bviews = [b[1:1 + size] for b in bbig]
    assert codec.verify_with_buffer(views, bviews)
    for r in range(m):
        assert (bviews[r].cpu().numpy() == ref[k + r]).all()


def test_verify_with_buffer_errors(rs, torch):
    codec = rs.ReedSolomon(4, 2)
    sh = [torch.zeros(64, dtype=torch.uint8, device="cuda") for _ in range(6)]
    buf = [torch.zeros(64, dtype=torch.uint8, device="cuda") for _ in range(2)]

    def err(shards, buffer):
        with pytest.raises(rs.RsError) as e:
            codec.verify_with_buffer(shards, buffer)
        return e.value.name

    assert err(sh[:5], buf) == "TooFewShards"
    assert err(sh + sh[:1], buf) == "TooManyShards"
    assert err(sh, buf[:1]) == "TooFewBufferShards"
    assert err(sh, buf + buf[:1]) == "TooManyBufferShards"
    assert err(sh, [buf[0], torch.zeros(32, dtype=torch.uint8, device="cuda")]) == "IncorrectShardSize"
    assert err(sh, [torch.zeros(0, dtype=torch.uint8, device="cuda")] * 2) == "EmptyShard"
    assert err(sh, [torch.zeros(32, dtype=torch.uint8, device="cuda")] * 2) == "IncorrectShardSize"
    leo = rs.ReedSolomon(4, 2, rs.CodecOptions(codec_family="leopard_gf8"))
    odd = [torch.zeros(96, dtype=torch.uint8, device="cuda") for _ in range(6)]
    obuf = [torch.zeros(96, dtype=torch.uint8, device="cuda") for _ in range(2)]
    with pytest.raises(rs.RsError) as e:
        leo.verify_with_buffer(odd, obuf)
    assert e.value.name == "IncorrectShardSize"
