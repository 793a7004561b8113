"""Progressive recovery (decode_idx, src/galois_8/policy.rs:543-700) on the GPU:
inputs arrive in batches and every call's destinations are compared byte for
byte with the oracle after that call, on codewords and non-codewords, in
device and host memory; merge mode, and the reference's error cases, which
must leave the destinations unchanged."""
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


def encoded(k, m, size, rng):
    rc, mat = O.build_matrix(k, m)
    sh = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8)
                                                                          for _ in range(m)]
    O.classic_encode(mat, sh)
    return mat, sh


def to_dev(torch, lst):
    return [None if a is None else torch.from_numpy(a.copy()).cuda() for a in lst]


def to_host(lst):
    return [None if t is None else t.cpu().numpy() for t in lst]


def test_reference_progressive_case(rs, torch):
    # src/tests/mod.rs:3970-4005 on the GPU: two batches recover shards 1 and 4.
    rng = np.random.default_rng(11)
    mat, sh = encoded(5, 3, 256 * 1024, rng)
    codec = rs.ReedSolomon(5, 3)
    expect = [True, False, True, True, False, True, True, False]
    dst = [None] * 8
    dst[1] = torch.zeros(256 * 1024, dtype=torch.uint8, device="cuda")
    dst[4] = torch.zeros(256 * 1024, dtype=torch.uint8, device="cuda")
    first = [None] * 8
    first[0], first[2] = sh[0], sh[2]
    codec.decode_idx(dst, expect, to_dev(torch, first))
    second = [None] * 8
    second[3], second[5], second[6] = sh[3], sh[5], sh[6]
    codec.decode_idx(dst, expect, to_dev(torch, second))
    assert (dst[1].cpu().numpy() == sh[1]).all() and (dst[4].cpu().numpy() == sh[4]).all()


@pytest.mark.parametrize("where", ["device", "host"])
@pytest.mark.parametrize("k,m,size", [(5, 3, 4096), (10, 4, 65536 + 17), (16, 4, 8192), (64, 6, 65),
                                      (32, 8, 3000), (4, 2, 1)])
def test_progressive_batches_match_oracle(rs, torch, where, k, m, size):
    rng = np.random.default_rng(k * 97 + m + size + len(where))
    rc, mat = O.build_matrix(k, m)
    codec = rs.ReedSolomon(k, m)
    for trial in range(3):
        # Non-codeword shards: the product must follow the reference's rows.
        sh = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k + m)]
        selected = sorted(rng.choice(k + m, size=k, replace=False).tolist())
        expect = [i in selected for i in range(k + m)]
        n_out = int(rng.integers(1, min(k + m, 9) + 1))
        outs = sorted(rng.choice(k + m, size=n_out, replace=False).tolist())
        init = [rng.integers(0, 256, size, dtype=np.uint8) if i in outs else None for i in range(k + m)]
        ref = [None if a is None else a.copy() for a in init]
        dst = to_dev(torch, init) if where == "device" else [None if a is None else a.copy() for a in init]
        order = list(selected) + [i for i in range(k + m) if i not in selected]  # unselected inputs are ignored
        rng.shuffle(order)
        n_batches = int(rng.integers(1, 5))
        cuts = sorted(rng.choice(np.arange(1, len(order)), size=n_batches - 1, replace=False).tolist()) \
            if n_batches > 1 else []
        for batch in np.split(np.array(order), cuts):
            inp = [sh[i] if i in set(batch.tolist()) else None for i in range(k + m)]
            assert O.classic_decode_idx(mat, ref, expect, inp) == 0
            codec.decode_idx(dst, expect, to_dev(torch, inp) if where == "device" else inp)
            got = to_host(dst) if where == "device" else dst
            for i in outs:
                assert (got[i] == ref[i]).all(), (k, m, trial, i)


@pytest.mark.parametrize("where", ["device", "host"])
def test_merge_mode(rs, torch, where):
    # src/tests/mod.rs:4007-4047: two partial results merged by XOR.
    rng = np.random.default_rng(12)
    mat, sh = encoded(5, 3, 128 * 1024, rng)
    codec = rs.ReedSolomon(5, 3)
    expect = [True, False, True, True, False, True, True, False]
    conv = (lambda x: to_dev(torch, x)) if where == "device" else (lambda x: [None if a is None else a.copy()
                                                                                  for a in x])
    pa = conv([np.zeros(128 * 1024, np.uint8) if i in (1, 4) else None for i in range(8)])
    pb = conv([np.zeros(128 * 1024, np.uint8) if i in (1, 4) else None for i in range(8)])
    codec.decode_idx(pa, expect, conv([sh[i] if i in (0, 2) else None for i in range(8)]))
    codec.decode_idx(pb, expect, conv([sh[i] if i in (3, 5, 6) else None for i in range(8)]))
    codec.decode_idx(pa, None, pb)
    got = to_host(pa) if where == "device" else pa
    assert (got[1] == sh[1]).all() and (got[4] == sh[4]).all()
    # Lengths may differ between indices, and empty pairs are allowed.
    d = conv([np.full(n, 0x0F, np.uint8) if n is not None else None for n in [3, 0, 700, None, 5, None, None, None]])
    x = [np.full(n, 0xF0, np.uint8) if n is not None else None for n in [3, 0, 700, None, None, None, None, None]]
    codec.decode_idx(d, None, conv(x))
    got = to_host(d) if where == "device" else d
    assert (got[0] == 0xFF).all() and got[1].size == 0 and (got[2] == 0xFF).all() and (got[4] == 0x0F).all()


def test_errors_leave_destinations_unchanged(rs, torch):
    codec = rs.ReedSolomon(5, 3)

    def err(dst, expect, inp):
        with pytest.raises(rs.RsError) as e:
            codec.decode_idx(dst, expect, inp)
        return e.value.name

    z = lambda n: torch.full((n,), 0x5A, dtype=torch.uint8, device="cuda")  # noqa: E731
    expect = [True, False, True, True, False, True, True, False]
    assert err([None] * 8, [True, False], [None] * 8) == "InvalidShardFlags"
    assert err([None] * 7, [True] * 8, [None] * 8) == "TooFewShards"
    assert err([None] * 8, [True] * 8, [None] * 7) == "TooFewShards"
    assert err([None] * 9, [True] * 8, [None] * 8) == "TooManyShards"
    dst = [None] * 8
    dst[1] = z(16)
    inp = [None] * 8
    inp[0] = z(8)
    assert err(dst, expect, inp) == "IncorrectShardSize"
    inp = [None] * 8
    inp[1] = z(8)
    assert err([None] * 8, None, inp) == "TooFewShards"
    dst2 = [None] * 8
    dst2[1] = z(8)
    assert err(dst2, [True, False, True] + [False] * 5, [None] * 8) == "TooFewShardsPresent"
    # More than k expected inputs with work to do (src/core/reconstruct.rs:1176-1183).
    inp = [None] * 8
    inp[0] = z(8)
    assert err(dst2, [True] * 8, inp) == "TooFewShardsPresent"
    # Merge mode validates every pair before it writes any.
    md = [z(8), z(8), None, None, None, None, None, None]
    mi = [z(8), z(8), z(4), None, None, None, None, None]
    assert err(md, None, mi) == "TooFewShards"
    md[2] = z(8)
    assert err(md, None, mi) == "IncorrectShardSize"
    torch.cuda.synchronize()
    for t in [dst[1], dst2[1], md[0], md[1], md[2]]:
        assert (t.cpu().numpy() == 0x5A).all()
    for fam in ("leopard_gf8", "leopard_gf16"):
        leo = rs.ReedSolomon(32, 16, rs.CodecOptions(codec_family=fam))
        with pytest.raises(rs.RsError) as e:
            leo.decode_idx([None] * 48, None, [None] * 48)
        assert e.value.name == "UnsupportedCodecFamily"


def test_singular_custom_matrix(rs, torch):
    codec = rs.ReedSolomon.with_custom_matrix(3, 2, [[1, 2, 3], [1, 2, 3]])
    dst = [torch.full((64,), 0x11, dtype=torch.uint8, device="cuda")] + [None] * 4
    inp = [None, None, torch.ones(64, dtype=torch.uint8, device="cuda"), None, None]
    with pytest.raises(rs.RsError) as e:
        codec.decode_idx(dst, [False, False, True, True, True], inp)
    assert e.value.name == "InvalidCustomMatrix"
    torch.cuda.synchronize()
    assert (dst[0].cpu().numpy() == 0x11).all()
