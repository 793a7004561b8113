"""Incremental parity (encode_single, encode_single_sep, update,
ShardByShard), split / join and the encoding-format identity, against the
oracle and the reference's byte fixtures."""
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


def full_parity(codec, data):
    k, m = codec.data_shard_count(), codec.parity_shard_count()
    sh = [d.copy() for d in data] + [np.zeros(data[0].size, np.uint8) for _ in range(m)]
    if codec.field == "gf16":
        O.gf16t_encode(codec.encoding_matrix(), sh)
    else:
        O.classic_encode(codec.encoding_matrix(), sh)
    return sh[k:]


def codecs(rs):
    return [rs.ReedSolomon(10, 4), rs.ReedSolomon(4, 2), rs.ReedSolomon(20, 7),
            rs.ReedSolomon(5, 1, rs.CodecOptions(fast_one_parity=True)), rs.ReedSolomon(6, 3, field="gf16")]


@pytest.mark.parametrize("idx", range(5))
@pytest.mark.parametrize("device", [False, True])
def test_encode_single_in_order_gives_full_parity(rs, torch, idx, device):
    c = codecs(rs)[idx]
    k, m = c.data_shard_count(), c.parity_shard_count()
    rng = np.random.default_rng(idx)
    n = 10002
    data = [rng.integers(0, 256, n, dtype=np.uint8) for _ in range(k)]
    want = full_parity(c, data)
    shards = [d.copy() for d in data] + [np.full(n, 0x5A, np.uint8) for _ in range(m)]
    if device:
        shards = [torch.from_numpy(s).cuda() for s in shards]
    for i in range(k):
        c.encode_single(i, shards)
    got = [s.cpu().numpy() if device else s for s in shards[k:]]
    for r in range(m):
        assert np.array_equal(got[r], want[r]), r
    # encode_single_sep with separate parity buffers
    par = [np.full(n, 0xA5, np.uint8) for _ in range(m)]
    for i in range(k):
        c.encode_single_sep(i, data[i], par)
    assert all(np.array_equal(a, b) for a, b in zip(par, want))


@pytest.mark.parametrize("idx", range(5))
@pytest.mark.parametrize("device", [False, True])
def test_update_matches_reencode(rs, torch, idx, device):
    c = codecs(rs)[idx]
    k, m = c.data_shard_count(), c.parity_shard_count()
    rng = np.random.default_rng(100 + idx)
    n = 4096 + 6
    old = [rng.integers(0, 256, n, dtype=np.uint8) for _ in range(k)]
    par = full_parity(c, old)
    changed = sorted(rng.choice(k, size=max(1, k // 3), replace=False).tolist())
    new = [rng.integers(0, 256, n, dtype=np.uint8) if j in changed else None for j in range(k)]
    cur = [new[j] if new[j] is not None else old[j] for j in range(k)]
    want = full_parity(c, cur)
    if device:
        t_old = [torch.from_numpy(x).cuda() for x in old]
        t_new = [None if x is None else torch.from_numpy(x).cuda() for x in new]
        t_par = [torch.from_numpy(x.copy()).cuda() for x in par]
        c.update(t_old, t_new, t_par)
        got = [x.cpu().numpy() for x in t_par]
    else:
        got = [x.copy() for x in par]
        c.update(old, new, got)
    for r in range(m):
        assert np.array_equal(got[r], want[r]), r
    # no changes: parity untouched
    same = [x.copy() for x in par]
    c.update(old, [None] * k, same)
    assert all(np.array_equal(a, b) for a, b in zip(same, par))


def test_incremental_errors(rs, torch):
    c = rs.ReedSolomon(4, 2)
    sh = [np.zeros(64, np.uint8) for _ in range(6)]
    for i, want in [(4, "InvalidIndex")]:
        with pytest.raises(rs.RsError) as e:
            c.encode_single(i, sh)
        assert e.value.name == want
    with pytest.raises(rs.RsError) as e:
        c.encode_single(0, sh[:5])
    assert e.value.name == "TooFewShards"
    with pytest.raises(rs.RsError) as e:
        c.encode_single(0, sh + [sh[0]])
    assert e.value.name == "TooManyShards"
    with pytest.raises(rs.RsError) as e:
        c.encode_single(0, [np.zeros(0, np.uint8)] * 6)
    assert e.value.name == "EmptyShard"
    with pytest.raises(rs.RsError) as e:
        c.encode_single(0, sh[:5] + [np.zeros(63, np.uint8)])
    assert e.value.name == "IncorrectShardSize"
    with pytest.raises(rs.RsError) as e:
        c.encode_single_sep(0, np.zeros(64, np.uint8), sh[:3])
    assert e.value.name == "TooManyParityShards"
    with pytest.raises(rs.RsError) as e:
        c.update(sh[:3], [None] * 4, sh[4:])
    assert e.value.name == "TooFewDataShards"
    with pytest.raises(rs.RsError) as e:
        c.update(sh[:4], [None, np.zeros(10, np.uint8), None, None], sh[4:])
    assert e.value.name == "IncorrectShardSize"
    leo = rs.ReedSolomon(4, 2, rs.CodecOptions(codec_family="leopard_gf8"))
    with pytest.raises(rs.RsError) as e:
        leo.encode_single(0, sh)
    assert e.value.name == "UnsupportedCodecFamily"
    with pytest.raises(rs.RsError) as e:
        leo.update(sh[:4], [None] * 4, sh[4:])
    assert e.value.name == "UnsupportedCodecFamily"


def test_shard_by_shard(rs, torch):
    # src/core/shard_by_shard.rs doc example: 3 + 2, the third shard arrives late.
    c = rs.ReedSolomon(3, 2)
    sbs = rs.ShardByShard(c)
    shards = [np.array(x, np.uint8) for x in ([0, 1, 2, 3, 4], [5, 6, 7, 8, 9], [0] * 5, [0] * 5, [0] * 5)]
    sbs.encode(shards)
    sbs.encode(shards)
    with pytest.raises(rs.SBSError) as e:
        sbs.reset()
    assert e.value.kind == "LeftoverShards"
    shards[2][:] = [10, 11, 12, 13, 14]
    sbs.encode(shards)
    assert sbs.parity_ready() and c.verify(shards)
    with pytest.raises(rs.SBSError) as e:
        sbs.encode(shards)
    assert e.value.kind == "TooManyCalls"
    sbs.reset()
    assert sbs.cur_input_index() == 0
    par = [np.zeros(5, np.uint8) for _ in range(2)]
    data = shards[:3]
    for _ in range(3):
        sbs.encode_sep(data, par)
    assert all(np.array_equal(a, b) for a, b in zip(par, shards[3:]))


@pytest.mark.parametrize("fam,k,m", [("classic", 4, 2), ("classic", 10, 4), ("leopard_gf8", 4, 2),
                                     ("leopard_gf16", 10, 4)])
@pytest.mark.parametrize("length", [0, 1, 63, 1000, 4097])
def test_split_join(rs, torch, fam, k, m, length):
    c = rs.ReedSolomon(k, m, rs.CodecOptions(codec_family=fam))
    rng = np.random.default_rng(length)
    data = rng.integers(0, 256, length, dtype=np.uint8).tobytes()
    shards = c.split(data)
    assert len(shards) == k
    # src/core/codec.rs:486-507, src/core/leopard.rs:75-98
    per = -(-length // k)
    want = per if fam == "classic" else max(-(-per // 64) * 64, 64)
    assert all(s.size == want for s in shards)
    flat = b"".join(s.tobytes() for s in shards)
    assert flat[:length] == data and set(flat[length:]) <= {0}
    if want == 0:
        # join validates like the reference: empty shards are EmptyShard
        with pytest.raises(rs.RsError) as e:
            c.join(shards, length)
        assert e.value.name == "EmptyShard"
        return
    assert c.join(shards, length) == data
    assert c.join(shards, length + 10 ** 6) == flat


def test_format_ids_match_reference_fixtures(rs, torch, kats):
    g8 = rs.ReedSolomon.with_custom_matrix(1, 1, [[0x87]])
    assert g8.stable_id_bytes() == bytes(kats["format_id_gf8_custom_1x1"]["bytes"])
    tw = rs.ReedSolomon.with_custom_matrix(1, 1, [[[0x12, 0x34]]], field="gf16")
    assert tw.stable_id_bytes() == bytes(kats["format_id_tower_custom_1x1"]["bytes"])
    # Leopard: no matrix (rows = cols = 0), family tag 1 / 2
    leo = rs.ReedSolomon(4, 2, rs.CodecOptions(codec_family="leopard_gf16"))
    b = leo.stable_id_bytes()
    assert b[:8] == b"RSEFMT\0\0" and b[10] == 2 and len(b) == 59 + len("rustfs.gf8.poly-11d.u8.v1")
    # equal formats, equal ids; different matrices, different ids
    assert rs.ReedSolomon(10, 4).stable_id_bytes() == rs.ReedSolomon(10, 4).stable_id_bytes()
    assert rs.ReedSolomon(10, 4).stable_id_bytes() != rs.ReedSolomon(
        10, 4, rs.CodecOptions(matrix_mode="cauchy")).stable_id_bytes()
