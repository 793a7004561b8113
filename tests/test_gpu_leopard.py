"""Leopard GF(2^8) / GF(2^16) encode, reconstruct and verify on the GPU,
byte-exact against the CPU oracle through the C ABI."""
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


def codec(rs, field, k, m):
    fam = "leopard_gf8" if field == 8 else "leopard_gf16"
    c = rs.ReedSolomon(k, m, rs.CodecOptions(codec_family=fam))
    assert c.codec_family() == fam
    return c


def dev(torch, arrs):
    return [torch.from_numpy(a.copy()).cuda() for a in arrs]


def host(ts):
    return [t.cpu().numpy() for t in ts]


def test_lgf16_go_parity_kat_on_gpu(rs, torch, kats):
    v = kats["lgf16_3x2_parity_prefix"]
    data = [np.array([(i * 64 + j) & 0xFF for j in range(64)], np.uint8) for i in range(3)]
    c = codec(rs, 16, 3, 2)
    sh = dev(torch, data + [np.zeros(64, np.uint8)] * 2)
    c.encode(sh)
    out = host(sh)
    assert list(out[3][:16]) == v["go_parity0"]["values"]
    assert list(out[4][:16]) == v["go_parity1"]["values"]


ENC_SHAPES = [(8, 4, 2, 64), (8, 10, 4, 1024), (8, 32, 16, 4096), (8, 128, 64, 8192), (8, 3, 5, 192),
              (8, 120, 50, 640), (8, 1, 1, 64), (16, 3, 2, 64), (16, 10, 4, 1024), (16, 32, 16, 4096),
              (16, 64, 32, 4096), (16, 300, 100, 1280), (16, 5, 7, 128), (16, 1, 1, 64)]


@pytest.mark.parametrize("field,k,m,size", ENC_SHAPES)
def test_leopard_encode_matches_oracle(rs, torch, field, k, m, size):
    rng = np.random.default_rng(field * 1000 + k + m + size)
    data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
    rc, par = O.leopard_encode(field, k, m, data)
    assert rc == 0
    c = codec(rs, field, k, m)
    sh = dev(torch, data + [np.full(size, 0x77, np.uint8) for _ in range(m)])
    c.encode(sh)
    out = host(sh)
    for i in range(m):
        assert np.array_equal(out[k + i], par[i]), (field, k, m, i)
    assert c.verify(sh)
    bad = [t.clone() for t in sh]
    bad[k + m - 1][size - 1] ^= 1
    assert not c.verify(bad)


@pytest.mark.parametrize("k,m,size", [(10, 4, 262144), (4, 2, 131072), (1, 1, 131072), (7, 3, 131072 + 64)])
def test_lgf8_dense_encode_matches_oracle(rs, torch, k, m, size):
    # GF(2^8) codes with <= 4 parity shards encode and verify shards >= 128 KiB
    # through K1 with the dense encode map (the smaller shapes above run the
    # FFT kernels, so the two forms are each checked against the oracle).
    rng = np.random.default_rng(k * 100 + m)
    data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
    rc, par = O.leopard_encode(8, k, m, data)
    assert rc == 0
    c = codec(rs, 8, k, m)
    for _ in range(2):  # the second call reuses the cached device tables
        sh = dev(torch, data + [np.full(size, 0x33, np.uint8) for _ in range(m)])
        c.encode(sh)
        out = host(sh)
        for i in range(m):
            assert np.array_equal(out[k + i], par[i]), (k, m, i)
        assert c.verify(sh)
        bad = [t.clone() for t in sh]
        bad[k + m - 1][size // 2] ^= 0x10
        assert not c.verify(bad)


@pytest.mark.parametrize("field,k,m,size", ENC_SHAPES)
@pytest.mark.parametrize("codeword", [True, False])
def test_leopard_reconstruct_matches_oracle(rs, torch, field, k, m, size, codeword):
    rng = np.random.default_rng(field * 7 + k * 3 + m + size + int(codeword))
    data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
    if codeword:
        rc, par = O.leopard_encode(field, k, m, data)
        full = data + par
    else:
        full = data + [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(m)]
    c = codec(rs, field, k, m)
    for trial in range(4):
        e = m if trial == 0 else int(rng.integers(1, m + 1))
        lost = set(rng.choice(k + m, size=e, replace=False).tolist())
        pres = [0 if i in lost else 1 for i in range(k + m)]
        ref = [s.copy() for s in full]
        for i in lost:
            ref[i][:] = 0
        assert O.leopard_reconstruct(field, k, m, ref, pres) == 0
        lst = [None if i in lost else torch.from_numpy(full[i].copy()).cuda() for i in range(k + m)]
        c.reconstruct(lst)
        for i in range(k + m):
            assert np.array_equal(lst[i].cpu().numpy(), ref[i]), (field, k, m, i, sorted(lost))
        if codeword:
            for i in range(k + m):
                assert np.array_equal(ref[i], full[i])


@pytest.mark.parametrize("field", [8, 16])
def test_leopard_reconstruct_data_and_host_path(rs, field):
    k, m, size = 20, 10, 2048
    rng = np.random.default_rng(field)
    data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
    rc, par = O.leopard_encode(field, k, m, data)
    full = data + par
    c = codec(rs, field, k, m)
    shards = [d.copy() for d in data] + [np.zeros(size, np.uint8) for _ in range(m)]
    c.encode(shards)
    assert all(np.array_equal(a, b) for a, b in zip(shards, full))
    lost = [0, 5, 19, 21, 29]
    lst = [None if i in lost else full[i].copy() for i in range(k + m)]
    c.reconstruct_data(lst)
    for i in range(k + m):
        if i in lost and i >= k:
            assert lst[i] is None
        else:
            assert np.array_equal(lst[i], full[i])


def test_lgf16_config3_shape_bitexact(rs, torch):
    # GF(2^16) k=1024, m=512, 16 KiB shards; erase 512 shards chosen from a seed.
    k, m, size = 1024, 512, 16384
    rng = np.random.default_rng(0x00EC5EED)
    data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
    rc, par = O.leopard_encode(16, k, m, data)
    assert rc == 0
    c = codec(rs, 16, k, m)
    buf = torch.zeros((k + m, size), dtype=torch.uint8, device="cuda")
    buf[:k] = torch.from_numpy(np.stack(data)).cuda()
    sh = [buf[i] for i in range(k + m)]
    c.encode(sh)
    got = buf[k:].cpu().numpy()
    assert np.array_equal(got, np.stack(par))
    lost = set(rng.choice(k + m, size=m, replace=False).tolist())
    lst = [None if i in lost else buf[i] for i in range(k + m)]
    c.reconstruct(lst)
    for i in sorted(lost):
        want = data[i] if i < k else par[i - k]
        assert np.array_equal(lst[i].cpu().numpy(), want), i


def test_lgf16_wide_code_uses_global_work(rs, torch):
    # 2048+1024 -> 4096 transform lanes (the serving mix's widest code).
    k, m, size = 2048, 1024, 512
    rng = np.random.default_rng(5)
    data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
    rc, par = O.leopard_encode(16, k, m, data)
    c = codec(rs, 16, k, m)
    buf = torch.zeros((k + m, size), dtype=torch.uint8, device="cuda")
    buf[:k] = torch.from_numpy(np.stack(data)).cuda()
    c.encode([buf[i] for i in range(k + m)])
    assert np.array_equal(buf[k:].cpu().numpy(), np.stack(par))
    lost = set(rng.choice(k + m, size=m, replace=False).tolist())
    full = data + par
    lst = [None if i in lost else buf[i] for i in range(k + m)]
    c.reconstruct(lst)
    for i in sorted(lost):
        assert np.array_equal(lst[i].cpu().numpy(), full[i]), i


@pytest.mark.parametrize("k,m,size", [(1024, 512, 256), (2048, 1024, 128), (4000, 1000, 64)])
@pytest.mark.parametrize("codeword", [True, False])
def test_lgf16_wide_decode_matches_oracle(rs, torch, k, m, size, codeword):
    # 2048, 4096 and 8192 transform lanes: the decode's work rows exceed
    # shared memory and live in a global slab.  Arbitrary (non-codeword)
    # inputs pin the whole pipeline, not only the round trip.
    rng = np.random.default_rng(k + m + size + int(codeword))
    data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
    if codeword:
        rc, par = O.leopard_encode(16, k, m, data)
        assert rc == 0
        full = data + par
    else:
        full = data + [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(m)]
    c = codec(rs, 16, k, m)
    for e in (m, int(rng.integers(1, m))):
        lost = set(rng.choice(k + m, size=e, replace=False).tolist())
        pres = [0 if i in lost else 1 for i in range(k + m)]
        ref = [s.copy() for s in full]
        for i in lost:
            ref[i][:] = 0
        assert O.leopard_reconstruct(16, k, m, ref, pres) == 0
        buf = torch.from_numpy(np.stack(full)).cuda()
        lst = [None if i in lost else buf[i] for i in range(k + m)]
        c.reconstruct(lst)
        for i in sorted(lost):
            assert np.array_equal(lst[i].cpu().numpy(), ref[i]), (k, m, e, i)


@pytest.mark.parametrize("k,m,size", [(4, 2, 12 << 20), (32, 16, 1536 << 10), (128, 64, 384 << 10)])
def test_lgf8_dense_reconstruct_matches_oracle(rs, torch, k, m, size):
    # GF(2^8) reconstructs that move >= 64 MiB under a pattern (here one
    # ~72 MiB stripe) derive its dense map and run it through K1; the same
    # pattern on short shards then hits the cached map.  Arbitrary
    # (non-codeword) inputs pin the dense path to the reference's decode.
    rng = np.random.default_rng(k * 31 + m)
    full = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k + m)]
    c = codec(rs, 8, k, m)
    for e, goal in ((min(16, m), "all"), (max(1, m // 3), "all"), (min(16, m), "data")):
        lost = set(rng.choice(k + m, size=e, replace=False).tolist())
        pres = [0 if i in lost else 1 for i in range(k + m)]
        ref = [s.copy() for s in full]
        for i in lost:
            ref[i][:] = 0
        assert O.leopard_reconstruct(8, k, m, ref, pres) == 0
        buf = torch.from_numpy(np.stack(full)).cuda()
        lst = [None if i in lost else buf[i] for i in range(k + m)]
        (c.reconstruct if goal == "all" else c.reconstruct_data)(lst)
        for i in sorted(lost):
            if goal == "data" and i >= k:
                assert lst[i] is None
            else:
                assert np.array_equal(lst[i].cpu().numpy(), ref[i]), (k, m, e, goal, i)
        del buf, lst
        short = [s[:64].copy() for s in full]
        sref = [s[:64].copy() for s in ref]
        sbuf = torch.from_numpy(np.stack(short)).cuda()
        slst = [None if i in lost else sbuf[i] for i in range(k + m)]
        (c.reconstruct if goal == "all" else c.reconstruct_data)(slst)
        for i in sorted(lost):
            if not (goal == "data" and i >= k):
                assert np.array_equal(slst[i].cpu().numpy(), sref[i]), (k, m, e, goal, i, "short")


def test_lgf8_repeated_pattern_switches_to_dense(rs, torch):
    # 48 MiB per call under one pattern: the first call runs the FFT decode,
    # the second crosses the codec's 64 MiB tally and derives the dense map,
    # the third uses the cached map; every call must give the same bytes.
    k, m, size = 32, 16, 1 << 20
    rng = np.random.default_rng(4242)
    full = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k + m)]
    lost = set(rng.choice(k + m, size=7, replace=False).tolist())
    pres = [0 if i in lost else 1 for i in range(k + m)]
    ref = [s.copy() for s in full]
    for i in lost:
        ref[i][:] = 0
    assert O.leopard_reconstruct(8, k, m, ref, pres) == 0
    c = codec(rs, 8, k, m)
    for call in range(3):
        buf = torch.from_numpy(np.stack(full)).cuda()
        lst = [None if i in lost else buf[i] for i in range(k + m)]
        c.reconstruct(lst)
        for i in sorted(lost):
            assert np.array_equal(lst[i].cpu().numpy(), ref[i]), (call, i)


def test_lgf8_dense_and_fft_in_one_batch(rs, torch):
    # One host-memory batch: 24 stripes under one pattern (72 MiB: dense),
    # five stripes with patterns of their own (too few bytes: FFT decode, in
    # a second launch), one stripe with nothing to rebuild.
    k, m, size, n = 32, 16, 65536, 30
    rng = np.random.default_rng(77)
    c = codec(rs, 8, k, m)
    shared = set(rng.choice(k + m, size=9, replace=False).tolist())
    stripes, pats, refs = [], [], []
    for s in range(n):
        full = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k + m)]
        if s < 24:
            lost = shared
        elif s < 29:
            lost = set(rng.choice(k + m, size=int(rng.integers(1, m + 1)), replace=False).tolist())
        else:
            lost = set()
        pres = [0 if i in lost else 1 for i in range(k + m)]
        ref = [x.copy() for x in full]
        for i in lost:
            ref[i][:] = 0
        if lost:
            assert O.leopard_reconstruct(8, k, m, ref, pres) == 0
        work = [x.copy() for x in full]
        for i in lost:
            work[i][:] = 0x5A
        stripes.append(work)
        pats.append(pres)
        refs.append(ref)
    c.reconstruct_batch(stripes, pats)
    for s in range(n):
        for i in range(k + m):
            assert np.array_equal(stripes[s][i], refs[s][i]), (s, i)


def test_leopard_errors(rs, torch):
    c = codec(rs, 8, 4, 2)
    sh = [torch.zeros(100, dtype=torch.uint8, device="cuda") for _ in range(6)]
    with pytest.raises(rs.RsError) as e:
        c.encode(sh)
    assert e.value.name == "IncorrectShardSize"
    sh = [torch.zeros(64, dtype=torch.uint8, device="cuda") for _ in range(6)]
    with pytest.raises(rs.RsError) as e:
        c.reconstruct([None, None, None, sh[3], sh[4], sh[5]])
    assert e.value.name == "TooFewShardsPresent"
    with pytest.raises(rs.RsError) as e:
        codec(rs, 8, 200, 50)
    assert e.value.name == "TooManyShards"


@pytest.mark.parametrize("mode,total,parity,expect", [
    ("prefer_leopard", 48, 16, "leopard_gf8"), ("prefer_leopard", 300, 100, "leopard_gf16"),
    ("prefer_gf16", 14, 4, "leopard_gf16"), ("as_needed", 14, 4, "classic"), ("as_needed", 300, 100, "leopard_gf16"),
    ("disabled", 14, 4, "classic")])
def test_leopard_mode_resolution(rs, mode, total, parity, expect):
    # src/core/leopard.rs:191-223
    c = rs.ReedSolomon(total - parity, parity, rs.CodecOptions(leopard_mode=mode))
    assert c.codec_family() == expect


def test_tower_gf16_classic(rs, torch):
    for k, m, size in [(4, 2, 64), (10, 4, 4098), (20, 10, 1000)]:
        rc, mat = O.gf16t_build_matrix(k, m)
        c = rs.ReedSolomon(k, m, field="gf16")
        assert np.array_equal(c.encoding_matrix(), mat)
        rng = np.random.default_rng(k)
        data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
        ref = data + [np.zeros(size, np.uint8) for _ in range(m)]
        O.gf16t_encode(mat, ref)
        sh = dev(torch, data + [np.zeros(size, np.uint8) for _ in range(m)])
        c.encode(sh)
        assert all(np.array_equal(a, b) for a, b in zip(host(sh), ref))
        assert c.verify(sh)
        lost = set(rng.choice(k + m, size=m, replace=False).tolist())
        lst = [None if i in lost else sh[i] for i in range(k + m)]
        c.reconstruct(lst)
        assert all(np.array_equal(lst[i].cpu().numpy(), ref[i]) for i in range(k + m))


@pytest.mark.parametrize("goal", ["all", "data"])
def test_tower_gf16_reconstruct_non_codeword(rs, torch, goal):
    # Random shards that are not a codeword: the rebuilt shards must follow the
    # reference's survivor rule and row algebra, not merely round-trip.
    for k, m, size in [(4, 2, 64), (10, 4, 2 * 2049), (20, 10, 1000)]:
        rc, mat = O.gf16t_build_matrix(k, m)
        c = rs.ReedSolomon(k, m, field="gf16")
        rng = np.random.default_rng(k * 3 + m + len(goal))
        for _ in range(4):
            shards = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k + m)]
            e = int(rng.integers(1, m + 1))
            lost = set(rng.choice(k + m, size=e, replace=False).tolist())
            pres = [0 if i in lost else 1 for i in range(k + m)]
            ref = [s.copy() for s in shards]
            assert O.gf16t_reconstruct(mat, ref, pres, data_only=(goal == "data")) == 0
            lst = [None if i in lost else torch.from_numpy(shards[i].copy()).cuda() for i in range(k + m)]
            if goal == "all":
                c.reconstruct(lst)
            else:
                c.reconstruct_data(lst)
            for i in range(k + m):
                if i in lost and (goal == "all" or i < k):
                    assert np.array_equal(lst[i].cpu().numpy(), ref[i]), (k, m, goal, sorted(lost), i)
                elif i not in lost:
                    assert np.array_equal(lst[i].cpu().numpy(), shards[i])
                else:
                    assert lst[i] is None


@pytest.mark.parametrize("k,m,size", [(1500, 100, 192), (1000, 600, 320), (600, 1000, 64), (1024, 512, 4096)])
def test_lgf16_2048_lane_decode_shapes(rs, torch, k, m, size):
    # 2048 transform lanes with shard lengths down to one 64-byte block:
    # non-codeword inputs, truncated transforms (k + m well below n, few
    # parity lanes, more parity than data), goals all and data.
    rng = np.random.default_rng(k * 5 + m + size)
    full = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k + m)]
    c = codec(rs, 16, k, m)
    for e, goal in ((m, "all"), (int(rng.integers(1, m)), "all"), (int(rng.integers(1, m + 1)), "data")):
        lost = set(rng.choice(k + m, size=e, replace=False).tolist())
        pres = [0 if i in lost else 1 for i in range(k + m)]
        ref = [s.copy() for s in full]
        for i in lost:
            ref[i][:] = 0
        want = [1 if (goal == "all" or i < k) else 0 for i in range(k + m)]
        assert O.leopard_reconstruct(16, k, m, ref, pres, want) == 0
        buf = torch.from_numpy(np.stack(full)).cuda()
        lst = [None if i in lost else buf[i] for i in range(k + m)]
        (c.reconstruct if goal == "all" else c.reconstruct_data)(lst)
        for i in sorted(lost):
            if goal == "data" and i >= k:
                assert lst[i] is None
            else:
                assert np.array_equal(lst[i].cpu().numpy(), ref[i]), (k, m, e, goal, i)
