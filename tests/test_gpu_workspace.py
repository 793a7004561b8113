"""Prepared reconstruction plans (rsgpu_prepare_reconstruct_ws /
rsgpu_reconstruct_with_ws, the reference's prepare_reconstruct_*workspace and
reconstruct_with_workspace, src/core/reconstruct.rs:539-726) on the GPU:
one plan applied to many stripes of its erasure pattern, non-codeword
inputs included, byte-exact against the oracle; and the reference's reuse
checks, which must write nothing."""
import ctypes

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


def pattern(rng, k, m):
    e = int(rng.integers(1, m + 1))
    lost = set(rng.choice(k + m, size=e, replace=False).tolist())
    return [0 if i in lost else 1 for i in range(k + m)]


def want(goal, i, k, req):
    return goal == "all" or (goal == "data" and i < k) or (goal == "required" and req[i])


@pytest.mark.parametrize("where", ["device", "host"])
@pytest.mark.parametrize("goal", ["all", "data", "required"])
@pytest.mark.parametrize("k,m,size", [(10, 4, 65536 + 48), (16, 4, 4096 + 15), (6, 3, 1000), (32, 8, 8192)])
def test_workspace_matches_oracle(rs, torch, where, goal, k, m, size):
    rng = np.random.default_rng(k * 1000 + m * 10 + size + len(goal) + len(where))
    codec = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    for _ in range(3):
        pres = pattern(rng, k, m)
        req = [int(rng.integers(0, 2)) for _ in range(k + m)] if goal == "required" else None
        ws = codec.prepare_reconstruct_workspace(pres, size, goal, req)
        assert ws.targets() == [i for i in range(k + m) if not pres[i] and want(goal, i, k, req)]
        for _stripe in range(3):
            # Non-codeword stripes: the plan must follow the reference's algebra.
            shards = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k + m)]
            ref = [s.copy() for s in shards]
            assert O.classic_reconstruct(mat, ref, pres, goal, req) == 0
            if where == "device":
                bufs = [torch.from_numpy(s.copy()).cuda() for s in shards]
                for i in range(k + m):
                    if not pres[i]:
                        bufs[i].fill_(0xA5)
            else:
                bufs = [s.copy() for s in shards]
                for i in range(k + m):
                    if not pres[i]:
                        bufs[i][:] = 0xA5
            codec.reconstruct_with_workspace(bufs, ws, present=pres)
            if where == "device":
                torch.cuda.synchronize()
                got = [b.cpu().numpy() for b in bufs]
            else:
                got = bufs
            for i in range(k + m):
                if pres[i]:
                    assert (got[i] == shards[i]).all()
                elif want(goal, i, k, req):
                    assert (got[i] == ref[i]).all(), (k, m, goal, pres, i)
                else:
                    assert (got[i] == 0xA5).all(), "a shard that is not a target was written"


def test_workspace_option_semantics_and_reuse(rs, torch):
    # None entries are missing; targets get new buffers, like Option<Vec<u8>>.
    k, m, size = 4, 3, 65
    codec = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    rng = np.random.default_rng(5)
    full = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8)
                                                                            for _ in range(m)]
    O.classic_encode(mat, full)
    pres = [1] * 7
    pres[0] = pres[1] = pres[4] = 0
    req = [0] * 7
    req[4] = 1
    ws = codec.prepare_reconstruct_some_workspace(pres, size, req)
    assert ws.targets() == [4]
    for _ in range(3):
        shards = [None if not pres[i] else torch.from_numpy(full[i].copy()).cuda() for i in range(7)]
        codec.reconstruct_with_workspace(shards, ws)
        assert shards[0] is None and shards[1] is None
        assert (shards[4].cpu().numpy() == full[4]).all()
    ws_data = codec.prepare_reconstruct_data_workspace(pres, size)
    shards = [None if not pres[i] else full[i].copy() for i in range(7)]
    codec.reconstruct_with_workspace(shards, ws_data)
    assert (shards[0] == full[0]).all() and (shards[1] == full[1]).all() and shards[4] is None


def _raw_with_ws(rs, codec, ws, bufs, pres):
    mem, ptrs, lens, stream, keep = rs._buffer_info(bufs)
    return rs.lib().rsgpu_reconstruct_with_ws(codec._h, ws._h, ptrs, lens, rs._flags(pres, len(pres)), len(bufs), mem,
                                              stream)


def test_workspace_reuse_checks_write_nothing(rs, torch):
    k, m, size = 10, 4, 4096
    codec = rs.ReedSolomon(k, m)
    pres = [1] * (k + m)
    pres[2] = pres[11] = 0
    ws = codec.prepare_reconstruct_workspace(pres, size)

    def bufs(length):
        return [torch.full((length,), 0x3C, dtype=torch.uint8, device="cuda") for _ in range(k + m)]

    # A different missing pattern: InvalidShardFlags.
    b = bufs(size)
    other = list(pres)
    other[3] = 0
    assert _raw_with_ws(rs, codec, ws, b, other) == 12
    # Same pattern, another length: IncorrectShardSize.
    b2 = bufs(size + 64)
    assert _raw_with_ws(rs, codec, ws, b2, pres) == 9
    # Present shards of different lengths: IncorrectShardSize; an empty one: EmptyShard.
    b3 = bufs(size)
    b3[0] = torch.full((size - 1,), 0x3C, dtype=torch.uint8, device="cuda")
    assert _raw_with_ws(rs, codec, ws, b3, pres) == 9
    b4 = bufs(size)
    b4[0] = torch.zeros(0, dtype=torch.uint8, device="cuda")
    assert _raw_with_ws(rs, codec, ws, b4, pres) == 11
    # Piece counts.
    assert _raw_with_ws(rs, codec, ws, bufs(size)[:-1], pres[:-1]) == 1
    assert _raw_with_ws(rs, codec, ws, bufs(size) + bufs(size)[:1], pres + [1]) == 2
    # A plan prepared by a codec of another shape or format.
    assert _raw_with_ws(rs, rs.ReedSolomon(9, 4), ws, bufs(size)[:13], pres[:13]) == 4  # TooManyDataShards
    assert _raw_with_ws(rs, rs.ReedSolomon(11, 3), ws, bufs(size), pres) == 3  # TooFewDataShards
    assert _raw_with_ws(rs, rs.ReedSolomon(10, 3), ws, bufs(size)[:13], pres[:13]) == 6  # TooManyParityShards
    cauchy = rs.ReedSolomon(k, m, rs.CodecOptions(matrix_mode="cauchy"))
    assert _raw_with_ws(rs, cauchy, ws, bufs(size), pres) == 14  # InvalidCustomMatrix
    torch.cuda.synchronize()
    for group in (b, b2, b3, b4):
        for t in group:
            assert (t.cpu().numpy() == 0x3C).all(), "a failed call wrote a shard"
    # An equivalent codec may reuse the plan.
    twin = rs.ReedSolomon(k, m)
    rc, mat = O.build_matrix(k, m)
    rng = np.random.default_rng(8)
    full = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8)
                                                                            for _ in range(m)]
    O.classic_encode(mat, full)
    dev = [torch.from_numpy(f.copy()).cuda() for f in full]
    dev[2].zero_()
    dev[11].zero_()
    twin.reconstruct_with_workspace(dev, ws, present=pres)
    assert all((d.cpu().numpy() == f).all() for d, f in zip(dev, full))


def test_workspace_prepare_errors(rs):
    codec = rs.ReedSolomon(4, 2)
    L = rs.lib()
    h = ctypes.c_void_p()

    def prep(c, pres, length, goal=0, req=None):
        req = req or []
        return L.rsgpu_prepare_reconstruct_ws(c._h, rs._flags(pres, max(1, len(pres))), len(pres), length, goal,
                                              rs._flags(req, max(1, len(req))), len(req), ctypes.byref(h))

    assert prep(codec, [1] * 5, 64) == 1
    assert prep(codec, [1] * 7, 64) == 2
    assert prep(codec, [0, 1, 1, 1, 1, 1], 0) == 11
    assert prep(codec, [0, 0, 0, 1, 1, 1], 64) == 10
    assert prep(codec, [0, 1, 1, 1, 1, 1], 64, 2, [1, 0, 1]) == 12  # required mask of 3 flags
    # Leopard families: the reference's workspaces are classic only.
    leo = rs.ReedSolomon(4, 2, rs.CodecOptions(codec_family="leopard_gf16"))
    assert prep(leo, [0, 1, 1, 1, 1, 1], 64) == 15
    # A singular survivor system of a custom matrix fails at prepare time.
    bad = rs.ReedSolomon.with_custom_matrix(3, 2, [[1, 2, 3], [1, 2, 3]])
    assert prep(bad, [0, 0, 1, 1, 1], 64) == 14


def test_workspace_all_present_is_a_no_op(rs, torch):
    codec = rs.ReedSolomon(4, 2)
    ws = codec.prepare_reconstruct_workspace([1] * 6, 128)
    assert ws.targets() == []
    sh = [torch.full((128,), i, dtype=torch.uint8, device="cuda") for i in range(6)]
    codec.reconstruct_with_workspace(sh, ws)
    assert all((t.cpu().numpy() == i).all() for i, t in enumerate(sh))


def test_workspace_tower_field(rs, torch):
    k, m, size = 6, 3, 2 * 700
    rc, mat = O.gf16t_build_matrix(k, m)
    codec = rs.ReedSolomon(k, m, field="gf16")
    rng = np.random.default_rng(21)
    pres = [1] * (k + m)
    pres[1] = pres[4] = pres[7] = 0
    ws = codec.prepare_reconstruct_workspace(pres, size)
    for _ in range(2):
        shards = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k + m)]
        ref = [s.copy() for s in shards]
        assert O.gf16t_reconstruct(mat, ref, pres) == 0
        dev = [torch.from_numpy(s.copy()).cuda() for s in shards]
        codec.reconstruct_with_workspace(dev, ws, present=pres)
        for i in range(k + m):
            assert (dev[i].cpu().numpy() == ref[i]).all(), i
