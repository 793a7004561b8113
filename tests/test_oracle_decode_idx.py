"""The oracle's progressive recovery (decode_idx) against the reference's own
tests of it: src/tests/mod.rs:3970-4175 and tests/compact_decode_matrix.rs:270-300.
CPU only; these pin the restatement that the GPU tests compare against."""
import numpy as np

import oracle as O

ERR = {"TooFewShards": 1, "TooManyShards": 2, "IncorrectShardSize": 9, "TooFewShardsPresent": 10,
       "InvalidShardFlags": 12}


def encoded(k, m, size, seed):
    rng = np.random.default_rng(seed)
    rc, mat = O.build_matrix(k, m)
    assert rc == 0
    sh = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)] + [np.zeros(size, np.uint8)
                                                                          for _ in range(m)]
    O.classic_encode(mat, sh)
    return mat, sh


def reconstruct_some(mat, sh, lost, wanted):
    k = mat.shape[1]
    n = mat.shape[0]
    out = [s.copy() for s in sh]
    for i in lost:
        out[i][:] = 0
    pres = [0 if i in lost else 1 for i in range(n)]
    req = [1 if i in wanted else 0 for i in range(n)]
    assert O.classic_reconstruct(mat, out, pres, "required", req) == 0
    return out


def test_progressive_matches_reconstruct_some():
    # src/tests/mod.rs:3970-4005
    mat, sh = encoded(5, 3, 256 * 1024, 1)
    expected = reconstruct_some(mat, sh, {1, 4}, {1, 4})
    dst = [None] * 8
    dst[1] = np.zeros_like(sh[0])
    dst[4] = np.zeros_like(sh[0])
    expect = [True, False, True, True, False, True, True, False]
    first = [None] * 8
    first[0], first[2] = sh[0].copy(), sh[2].copy()
    assert O.classic_decode_idx(mat, dst, expect, first) == 0
    second = [None] * 8
    second[3], second[5], second[6] = sh[3].copy(), sh[5].copy(), sh[6].copy()
    assert O.classic_decode_idx(mat, dst, expect, second) == 0
    assert (dst[1] == expected[1]).all() and (dst[4] == expected[4]).all()


def test_merge_mode_accumulates_partial_results():
    # src/tests/mod.rs:4007-4047
    mat, sh = encoded(5, 3, 128 * 1024, 2)
    expect = [True, False, True, True, False, True, True, False]
    pa = [None] * 8
    pa[1], pa[4] = np.zeros_like(sh[0]), np.zeros_like(sh[0])
    ia = [None] * 8
    ia[0], ia[2] = sh[0].copy(), sh[2].copy()
    assert O.classic_decode_idx(mat, pa, expect, ia) == 0
    pb = [None] * 8
    pb[1], pb[4] = np.zeros_like(sh[0]), np.zeros_like(sh[0])
    ib = [None] * 8
    ib[3], ib[5], ib[6] = sh[3].copy(), sh[5].copy(), sh[6].copy()
    assert O.classic_decode_idx(mat, pb, expect, ib) == 0
    assert O.classic_decode_idx(mat, pa, None, pb) == 0
    expected = reconstruct_some(mat, sh, {1, 4}, {1, 4})
    assert (pa[1] == expected[1]).all() and (pa[4] == expected[4]).all()


def test_error_cases():
    rc, mat = O.build_matrix(5, 3)
    # invalid expect length (mod.rs:4049-4061)
    assert O.classic_decode_idx(mat, [None] * 8, [True, False], [None] * 8) == ERR["InvalidShardFlags"]
    # dst / input counts (mod.rs:4063-4092)
    assert O.classic_decode_idx(mat, [None] * 7, [True] * 8, [None] * 8) == ERR["TooFewShards"]
    assert O.classic_decode_idx(mat, [None] * 8, [True] * 8, [None] * 7) == ERR["TooFewShards"]
    assert O.classic_decode_idx(mat, [None] * 9, [True] * 8, [None] * 8) == ERR["TooManyShards"]
    # shard size mismatch (mod.rs:4130-4146): the length comes from input[0]
    dst = [None] * 8
    dst[1] = np.zeros(16, np.uint8)
    inp = [None] * 8
    inp[0] = np.ones(8, np.uint8)
    expect = [True, False, True, True, False, True, True, False]
    assert O.classic_decode_idx(mat, dst, expect, inp) == ERR["IncorrectShardSize"]
    assert (dst[1] == 0).all()
    # merge mode with a missing destination (mod.rs:4148-4160)
    inp = [None] * 8
    inp[1] = np.ones(8, np.uint8)
    assert O.classic_decode_idx(mat, [None] * 8, None, inp) == ERR["TooFewShards"]
    # too few expected inputs (mod.rs:4162-4175)
    dst = [None] * 8
    dst[1] = np.zeros(8, np.uint8)
    assert O.classic_decode_idx(mat, dst, [True, False, True] + [False] * 5, [None] * 8) == \
        ERR["TooFewShardsPresent"]
    # no destination buffer and no input at all: nothing gives a length
    assert O.classic_decode_idx(mat, [None] * 8, [True] * 8, [None] * 8) == ERR["TooFewShardsPresent"]


def test_more_than_k_expected_inputs():
    # get_data_decode_matrix (src/core/reconstruct.rs:1176-1183) takes exactly
    # k selected inputs: with more expected inputs, a call that has both
    # outputs and inputs fails, while one with nothing to do returns early.
    mat, sh = encoded(5, 3, 64, 3)
    dst = [None] * 8
    dst[1] = np.zeros(64, np.uint8)
    inp = [None] * 8
    inp[0] = sh[0].copy()
    assert O.classic_decode_idx(mat, dst, [True] * 8, inp) == ERR["TooFewShardsPresent"]
    assert O.classic_decode_idx(mat, dst, [True] * 8, [None] * 8) == 0
    assert (dst[1] == 0).all()


def test_progressive_batches_recover_identity_and_parity_rows():
    # tests/compact_decode_matrix.rs:270-300: 64+6, 65-byte shards, batches of
    # 11 survivors, targets that mix missing and present data and parity.
    k, m = 64, 6
    mat, sh = encoded(k, m, 65, 4)
    missing = [0, 21, 63, 64]
    survivors = [i for i in range(k + m) if i not in missing][:k]
    expect = [i in survivors for i in range(k + m)]
    targets = [0, 2, 21, 63, 64, 69]
    out = [np.zeros(65, np.uint8) if i in targets else None for i in range(k + m)]
    for b in range(0, len(survivors), 11):
        batch = survivors[b:b + 11]
        inp = [sh[i].copy() if i in batch else None for i in range(k + m)]
        assert O.classic_decode_idx(mat, out, expect, inp) == 0
    for i in range(k + m):
        if i in targets:
            assert (out[i] == sh[i]).all(), i
        else:
            assert out[i] is None
