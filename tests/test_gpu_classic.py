"""Classic GF(2^8) encode / reconstruct / verify on the GPU, byte-exact against
the CPU oracle, through the C ABI (librsgpu.so)."""
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


def rand_shards(rng, n, size):
    return [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(n)]


def to_dev(torch, arrs):
    return [torch.from_numpy(a.copy()).cuda() for a in arrs]


def to_host(ts):
    return [t.cpu().numpy() for t in ts]


SHAPES = [(1, 1), (2, 2), (4, 2), (6, 3), (8, 4), (10, 4), (12, 4), (16, 4), (17, 3), (5, 7), (32, 8),
          (64, 32), (200, 56)]


@pytest.mark.parametrize("k,m", SHAPES)
@pytest.mark.parametrize("size", [1, 15, 16, 64, 1000, 4096 + 16, 65536])
def test_encode_matches_oracle_device(rs, torch, k, m, size):
    rng = np.random.default_rng(k * 7919 + m * 31 + size)
    data = rand_shards(rng, k, size)
    codec = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    assert (codec.encoding_matrix() == mat).all()
    ref = data + [np.zeros(size, np.uint8) for _ in range(m)]
    O.classic_encode(mat, ref)
    dev = to_dev(torch, data + [np.full(size, 0xEE, np.uint8) for _ in range(m)])
    codec.encode(dev)
    torch.cuda.synchronize()
    got = to_host(dev)
    for i in range(k + m):
        assert (got[i] == ref[i]).all(), (k, m, size, i)


@pytest.mark.parametrize("k,m", [(4, 2), (10, 4), (16, 4)])
def test_encode_host_path_and_sep(rs, k, m):
    rng = np.random.default_rng(k + m)
    size = 12345
    data = rand_shards(rng, k, size)
    codec = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    ref = data + [np.zeros(size, np.uint8) for _ in range(m)]
    O.classic_encode(mat, ref)
    shards = [d.copy() for d in data] + [np.zeros(size, np.uint8) for _ in range(m)]
    codec.encode(shards)
    assert all((a == b).all() for a, b in zip(shards, ref))
    par = [np.zeros(size, np.uint8) for _ in range(m)]
    codec.encode_sep([d.copy() for d in data], par)
    assert all((a == b).all() for a, b in zip(par, ref[k:]))


def test_misaligned_device_pointers(rs, torch):
    k, m, size = 10, 4, 4099
    rng = np.random.default_rng(3)
    data = rand_shards(rng, k, size)
    codec = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    ref = data + [np.zeros(size, np.uint8) for _ in range(m)]
    O.classic_encode(mat, ref)
    big = [torch.zeros(size + 7, dtype=torch.uint8, device="cuda") for _ in range(k + m)]
    views = [b[3: 3 + size] for b in big]
    for v, d in zip(views, data):
        v.copy_(torch.from_numpy(d))
    codec.encode(views)
    torch.cuda.synchronize()
    for i in range(k + m):
        assert (views[i].cpu().numpy() == ref[i]).all()


@pytest.mark.parametrize("mode", ["vandermonde", "cauchy", "jerasure_like"])
@pytest.mark.parametrize("k,m", [(4, 2), (10, 4), (16, 4), (20, 10)])
def test_matrix_modes(rs, torch, mode, k, m):
    rc, mat = O.build_matrix(k, m, mode)
    if rc != 0:
        with pytest.raises(rs.RsError):
            rs.ReedSolomon(k, m, rs.CodecOptions(matrix_mode=mode))
        return
    codec = rs.ReedSolomon(k, m, rs.CodecOptions(matrix_mode=mode))
    assert (codec.encoding_matrix() == mat).all()
    rng = np.random.default_rng(11)
    data = rand_shards(rng, k, 256)
    ref = data + [np.zeros(256, np.uint8) for _ in range(m)]
    O.classic_encode(mat, ref)
    dev = to_dev(torch, ref)
    for i in range(k, k + m):
        dev[i].zero_()
    codec.encode(dev)
    assert all((a == b).all() for a, b in zip(to_host(dev), ref))


def test_fast_one_parity(rs, torch):
    k = 9
    codec = rs.ReedSolomon(k, 1, rs.CodecOptions(fast_one_parity=True))
    rng = np.random.default_rng(5)
    data = rand_shards(rng, k, 777)
    dev = to_dev(torch, data + [np.zeros(777, np.uint8)])
    codec.encode(dev)
    x = np.zeros(777, np.uint8)
    for d in data:
        x ^= d
    assert (dev[k].cpu().numpy() == x).all()


def erase_patterns(rng, k, m, n):
    pats = []
    for _ in range(n):
        e = int(rng.integers(1, m + 1))
        lost = set(rng.choice(k + m, size=e, replace=False).tolist())
        pats.append([0 if i in lost else 1 for i in range(k + m)])
    return pats


@pytest.mark.parametrize("k,m", [(4, 2), (10, 4), (16, 4), (6, 3), (12, 4), (32, 8)])
@pytest.mark.parametrize("goal", ["all", "data", "required"])
def test_reconstruct_matches_oracle(rs, torch, k, m, goal):
    rng = np.random.default_rng(k * 100 + m + len(goal))
    size = 4096 + 48
    codec = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    for pres in erase_patterns(rng, k, m, 12):
        # Non-codeword input: reconstruct must still match the reference's algebra.
        shards = rand_shards(rng, k + m, size)
        req = [int(rng.integers(0, 2)) for _ in range(k + m)] if goal == "required" else None
        ref = [s.copy() for s in shards]
        assert O.classic_reconstruct(mat, ref, pres, goal, req) == 0
        dev = to_dev(torch, shards)
        lst = [dev[i] if pres[i] else None for i in range(k + m)]
        if goal == "all":
            codec.reconstruct(lst)
        elif goal == "data":
            codec.reconstruct_data(lst)
        else:
            codec.reconstruct_some(lst, req)
        torch.cuda.synchronize()
        for i in range(k + m):
            if pres[i]:
                assert (lst[i].cpu().numpy() == shards[i]).all()
            elif lst[i] is not None:
                assert (lst[i].cpu().numpy() == ref[i]).all(), (k, m, goal, pres, i)


def test_reconstruct_config1_pattern_host_and_device(rs, torch):
    # 10+4, erase {0, 3, 11, 13} (the single-stripe workload).
    k, m, size = 10, 4, 65536
    rng = np.random.default_rng(2024)
    codec = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    full = rand_shards(rng, k, size) + [np.zeros(size, np.uint8) for _ in range(m)]
    O.classic_encode(mat, full)
    lost = {0, 3, 11, 13}
    host = [None if i in lost else full[i].copy() for i in range(k + m)]
    codec.reconstruct(host)
    assert all((host[i] == full[i]).all() for i in range(k + m))
    dev = [None if i in lost else torch.from_numpy(full[i]).cuda() for i in range(k + m)]
    codec.reconstruct(dev)
    assert all((dev[i].cpu().numpy() == full[i]).all() for i in range(k + m))
    assert codec.verify(dev)
    st = codec.cache_stats()
    assert st.hits >= 1 and st.misses >= 1


@pytest.mark.parametrize("k,m", [(4, 2), (10, 4), (16, 4)])
def test_verify(rs, torch, k, m):
    rng = np.random.default_rng(77)
    size = 5000
    codec = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    full = rand_shards(rng, k, size) + [np.zeros(size, np.uint8) for _ in range(m)]
    O.classic_encode(mat, full)
    dev = to_dev(torch, full)
    assert codec.verify(dev)
    ws = rs.VerifyWorkspace(codec, size)
    assert codec.verify_with_workspace(dev, ws)
    for pos in [0, 16, size - 1, 4095, 4096]:
        for sh in [k, k + m - 1]:
            bad = [t.clone() for t in dev]
            bad[sh][pos] ^= 0x5A
            assert not codec.verify(bad), (pos, sh)
            assert not codec.verify_with_workspace(bad, ws)
    assert codec.verify([f.copy() for f in full])
    host_bad = [f.copy() for f in full]
    host_bad[k][3] ^= 0xFF
    assert not codec.verify(host_bad)


def test_batch_api_mixed_patterns(rs, torch):
    k, m, size, n = 10, 4, 8192, 64
    rng = np.random.default_rng(99)
    codec = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    stripes = []
    for s in range(n):
        full = rand_shards(rng, k, size) + [np.zeros(size, np.uint8) for _ in range(m)]
        stripes.append(full)
    dev = [to_dev(torch, st) for st in stripes]
    codec.encode_batch(dev)
    refs = []
    for st in stripes:
        r = [x.copy() for x in st]
        O.classic_encode(mat, r)
        refs.append(r)
    for d, r in zip(dev, refs):
        assert all((a.cpu().numpy() == b).all() for a, b in zip(d, r))
    assert all(codec.verify_batch(dev))
    pats = erase_patterns(rng, k, m, n)
    for d, p in zip(dev, pats):
        for i in range(k + m):
            if not p[i]:
                d[i].fill_(0xCC)
    codec.reconstruct_batch(dev, pats)
    for d, r in zip(dev, refs):
        assert all((a.cpu().numpy() == b).all() for a, b in zip(d, r))
    dev[5][k].view(-1)[77] ^= 1
    ok = codec.verify_batch(dev)
    assert ok[5] is False and sum(ok) == n - 1


def test_batch_host_path(rs):
    k, m, size, n = 10, 4, 4096, 20
    rng = np.random.default_rng(123)
    codec = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    stripes = [rand_shards(rng, k, size) + [np.zeros(size, np.uint8) for _ in range(m)] for _ in range(n)]
    refs = []
    for st in stripes:
        r = [x.copy() for x in st]
        O.classic_encode(mat, r)
        refs.append(r)
    codec.encode_batch(stripes)
    for st, r in zip(stripes, refs):
        assert all((a == b).all() for a, b in zip(st, r))
    pats = erase_patterns(rng, k, m, n)
    for st, p in zip(stripes, pats):
        for i in range(k + m):
            if not p[i]:
                st[i][:] = 0
    codec.reconstruct_batch(stripes, pats)
    for st, r in zip(stripes, refs):
        assert all((a == b).all() for a, b in zip(st, r))
    assert all(codec.verify_batch(stripes))


@pytest.mark.parametrize("where", ["host", "device"])
@pytest.mark.parametrize("size", [4096, 3000])
def test_batch_stripe_block(rs, torch, where, size):
    # One contiguous (stripes, k + m, length) block: pointers are computed in
    # one step, a host rebuild uploads only the first k present shards, and a
    # host verify reads back every chunk's flags once at the end.
    k, m, n = 10, 4, 40
    rng = np.random.default_rng(size + len(where))
    codec = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    ref = np.zeros((n, k + m, size), np.uint8)
    ref[:, :k] = rng.integers(0, 256, (n, k, size), dtype=np.uint8)
    for s in range(n):
        st = list(ref[s])
        O.classic_encode(mat, st)
    blk = ref.copy()
    blk[:, k:] = 0
    if where == "device":
        blk = torch.from_numpy(blk).cuda()
    codec.encode_batch(blk)
    got = blk if where == "host" else blk.cpu().numpy()
    assert (got == ref).all()
    pats = np.array(erase_patterns(rng, k, m, n), dtype=bool)
    if where == "host":
        blk[~pats] = 0xCC
    else:
        blk[torch.from_numpy(~pats).cuda()] = 0xCC
    codec.reconstruct_batch(blk, pats)
    got = blk if where == "host" else blk.cpu().numpy()
    assert (got == ref).all()
    assert codec.verify_batch(blk) == [True] * n
    bad = [3, 17, n - 1]
    for s in bad:
        blk[s, k + s % m, size // 3] ^= 0x21
    ok = codec.verify_batch(blk)
    assert [i for i, v in enumerate(ok) if not v] == bad
    with pytest.raises(rs.RsError) as e:
        codec.verify_batch(blk[:, : k + m - 1])
    assert e.value.name == "TooFewShards"
    with pytest.raises(rs.RsError) as e:
        codec.encode_batch([list(ref[0]) + [ref[0][0]]])
    assert e.value.name == "TooManyShards"


def test_error_precedence(rs, torch):
    codec = rs.ReedSolomon(4, 2)
    sh = [torch.zeros(64, dtype=torch.uint8, device="cuda") for _ in range(6)]
    with pytest.raises(rs.RsError) as e:
        codec.encode(sh[:5])
    assert e.value.name == "TooFewShards"
    with pytest.raises(rs.RsError) as e:
        codec.encode(sh + [sh[0]])
    assert e.value.name == "TooManyShards"
    empty = [torch.zeros(0, dtype=torch.uint8, device="cuda")] + sh[1:]
    with pytest.raises(rs.RsError) as e:
        codec.encode(empty)
    assert e.value.name == "EmptyShard"
    odd = sh[:5] + [torch.zeros(63, dtype=torch.uint8, device="cuda")]
    with pytest.raises(rs.RsError) as e:
        codec.encode(odd)
    assert e.value.name == "IncorrectShardSize"
    with pytest.raises(rs.RsError) as e:
        codec.reconstruct([None, None, None, sh[3], sh[4], sh[5]])
    assert e.value.name == "TooFewShardsPresent"
    with pytest.raises(rs.RsError) as e:
        codec.reconstruct_some([None] + sh[1:], [True, False, True])
    assert e.value.name == "InvalidShardFlags"
    with pytest.raises(rs.RsError) as e:
        codec.encode_sep(sh[:3], sh[4:])
    assert e.value.name == "TooFewDataShards"


def test_singular_custom_matrix_writes_nothing(rs, torch):
    # Two identical parity rows: losing two data shards leaves a singular system.
    k, m = 3, 2
    codec = rs.ReedSolomon.with_custom_matrix(k, m, [[1, 2, 3], [1, 2, 3]])
    sh = [torch.full((64,), i + 1, dtype=torch.uint8, device="cuda") for i in range(k + m)]
    out0 = torch.full((64,), 0xAB, dtype=torch.uint8, device="cuda")
    out1 = torch.full((64,), 0xAB, dtype=torch.uint8, device="cuda")
    lst = [out0, out1, sh[2], sh[3], sh[4]]
    mem, ptrs, lens, stream, keep = rs._buffer_info(lst)
    pres = rs._flags([0, 0, 1, 1, 1], 5)
    rc = rs.lib().rsgpu_reconstruct(codec._h, ptrs, lens, pres, 5, 0, rs._flags([], 1), 0, mem, stream)
    assert rc == 14  # InvalidCustomMatrix
    torch.cuda.synchronize()
    assert (out0.cpu().numpy() == 0xAB).all() and (out1.cpu().numpy() == 0xAB).all()
    rc2, mat = O.build_matrix(k, m, "custom", custom=np.array([[1, 2, 3], [1, 2, 3]], np.uint8))
    ref = [s.cpu().numpy() for s in sh]
    assert O.classic_reconstruct(mat, ref, [0, 0, 1, 1, 1]) == 14


def test_kernel_launch_counter_moves(rs, torch):
    before = rs.kernel_launch_count()
    codec = rs.ReedSolomon(4, 2)
    sh = [torch.zeros(4096, dtype=torch.uint8, device="cuda") for _ in range(6)]
    codec.encode(sh)
    assert rs.kernel_launch_count() > before


def test_prepared_batches_replay_in_a_cuda_graph(rs, torch):
    # Prepared batches only launch, so a step of them can be captured once
    # and replayed: each replay re-reads the shards as they are then.  The
    # replayed encode, rebuild of the erased shards and verify must give the
    # oracle's bytes and flags, for new data every time.
    k, m, size, n = 10, 4, 65536, 8
    rng = np.random.default_rng(123)
    codec = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    buf = torch.zeros((n, k + m, size), dtype=torch.uint8, device="cuda")
    offs = np.arange(n * (k + m), dtype=np.uint64) * np.uint64(size)
    ptrs = rs.device_pointer_table(buf.data_ptr(), offs)
    pats = np.ones((n, k + m), np.uint8)
    pats[:, [0, 3, 11, 13]] = 0
    enc = codec.prepare_batch("encode", ptrs, size)
    rec = codec.prepare_batch("reconstruct", ptrs, size, present=pats)
    ver = codec.prepare_batch("verify", ptrs, size)
    for b in (enc, rec, ver):  # first launches (kernel attributes, occupancy) before the capture
        b.launch()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        enc.launch()
        rec.launch()
        ver.launch()
    torch.cuda.synchronize()
    for rnd in range(3):
        data = rng.integers(0, 256, (n, k, size), dtype=np.uint8)
        buf[:, :k] = torch.from_numpy(data).cuda()
        buf[:, k:] = 0x5A  # stale parity; encode overwrites it
        g.replay()
        torch.cuda.synchronize()
        got = buf.cpu().numpy()
        for s in range(n):
            want = [data[s, j].copy() for j in range(k)] + [np.zeros(size, np.uint8) for _ in range(m)]
            O.classic_encode(mat, want)
            for j in range(k + m):
                assert np.array_equal(got[s, j], want[j]), (rnd, s, j)
        assert ver.verify_result().all(), rnd
    # A replay whose verify sees corrupted parity: the rebuild restores shard
    # 11 (erased in the pattern) but shard 12 is present and stays corrupted.
    g.replay()
    torch.cuda.synchronize()
    buf[2, 12, 100] ^= 1
    ver.launch()
    ok = ver.verify_result()
    assert not ok[2] and ok.sum() == n - 1
    del g
