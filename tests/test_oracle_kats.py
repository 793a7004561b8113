"""Pin the CPU oracle to the reference's own known-answer tests.

Every expected value comes from tests/golden/reference_kats.json, which
make_golden.py copies out of literal assertions in the reference test suite.
These run on CPU only.
"""
import numpy as np
import pytest

import oracle as O

M64 = (1 << 64) - 1


def smallrng_u8(seed, n):
    """rand 0.10 ``SmallRng`` (Xoshiro256++ seeded by SplitMix64) drawing
    ``random::<u8>()`` = the upper 32 bits of each output truncated to a byte.
    Used by tests/golden_vectors.rs:31-34 to build the seeded KAT input."""

    def rotl(x, k):
        return ((x << k) | (x >> (64 - k))) & M64

    st, s = seed, []
    for _ in range(4):
        st = (st + 0x9E3779B97F4A7C15) & M64
        z = st
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        s.append(z ^ (z >> 31))
    out = []
    for _ in range(n):
        r = (rotl((s[0] + s[3]) & M64, 23) + s[0]) & M64
        t = (s[1] << 17) & M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = rotl(s[3], 45)
        out.append((r >> 32) & 0xFF)
    return out


def split(data, k):
    """src/core/codec.rs:476-500: ceil(len/k) bytes per shard, zero padded."""
    per = -(-len(data) // k)
    shards = []
    for i in range(k):
        s = np.zeros(per, np.uint8)
        chunk = data[i * per: (i + 1) * per]
        s[: len(chunk)] = chunk
        shards.append(s)
    return shards


def fixed_4x2():
    return [np.arange(i * 16, i * 16 + 16, dtype=np.uint8) for i in range(4)] + [np.zeros(16, np.uint8)] * 2


def test_gf8_log_table_matches_backblaze(kats):
    lg, ex = O.gf8_tables()
    assert list(lg) == kats["gf8_backblaze_log_table"]["values"]
    # exp table wraps (build.rs:29-39)
    assert list(ex[:255]) == list(ex[255:510])


def test_gf8_mul_exp_kats(kats):
    for c in kats["gf8_mul"]:
        assert O.gf8_mul(c["a"], c["b"]) == c["expect"], c
    for c in kats["gf8_exp"]:
        assert O.gf8_exp(c["a"], c["n"]) == c["expect"], c


def test_gf8_slice_kats(kats):
    inp = np.array(kats["gf8_slice_ops"]["input"], np.uint8)
    out = np.zeros_like(inp)
    for op in kats["gf8_slice_ops"]["ops"]:
        if op["op"] == "mul_slice":
            out = O.gf8_mul_slice(op["c"], inp)
        else:
            out = O.gf8_mul_slice_xor(op["c"], inp, out)
        assert list(out) == op["expect"], op


def test_gf8_field_axioms_exhaustive():
    lg, ex = O.gf8_tables()
    for a in range(1, 256):
        assert O.gf8_mul(a, O.gf8_div(1, a)) == 1
    assert O.gf8_div(0, 7) == 0 and O.gf8_div(7, 0) == 0
    assert O.gf8_exp(0, 0) == 1 and O.gf8_exp(0, 5) == 0


def test_classic_4x2_encode_golden(kats):
    g = kats["classic_4x2_golden"]["golden_encode_4x2_incrementing_input"]
    rc, mat = O.build_matrix(4, 2)
    assert rc == 0
    shards = [s.copy() for s in fixed_4x2()]
    O.classic_encode(mat, shards)
    assert list(shards[4]) == g["parity4"]
    assert list(shards[5]) == g["parity5"]
    assert O.checksum_shards(shards) == g["checksum"]


def test_classic_4x2_reconstruct_golden(kats):
    rc, mat = O.build_matrix(4, 2)
    enc = [s.copy() for s in fixed_4x2()]
    O.classic_encode(mat, enc)
    # reconstruct_data with shards 1 and 4 missing: shard 4 stays empty.
    g = kats["classic_4x2_golden"]["golden_reconstruct_data_4x2_incrementing_input"]
    sh = [s.copy() for s in enc]
    sh[1][:] = 0
    sh[4][:] = 0
    pres = [1, 0, 1, 1, 0, 1]
    assert O.classic_reconstruct(mat, sh, pres, goal="data") == 0
    assert list(sh[1]) == list(range(16, 32))
    view = [bytes(s) for s in sh]
    view[4] = b""
    assert O.checksum_shards(view) == g["checksum"]
    # reconstruct (all) with shards 0 and 5 missing
    g = kats["classic_4x2_golden"]["golden_reconstruct_4x2_incrementing_input"]
    sh = [s.copy() for s in enc]
    sh[0][:] = 0
    sh[5][:] = 0
    assert O.classic_reconstruct(mat, sh, [0, 1, 1, 1, 1, 0]) == 0
    assert all((a == b).all() for a, b in zip(sh, enc))
    assert O.checksum_shards(sh) == g["checksum"]


def test_classic_4x2_verify_detects_corruption():
    rc, mat = O.build_matrix(4, 2)
    sh = [s.copy() for s in fixed_4x2()]
    O.classic_encode(mat, sh)
    assert O.classic_verify(mat, sh)
    sh[5][3] ^= 0xFF
    assert not O.classic_verify(mat, sh)


@pytest.mark.parametrize(
    "name,data",
    [
        ("golden_encode_4x2_seeded_random_input", smallrng_u8(0xA5A51024, 61)),
        ("golden_encode_4x2_all_zero_input", [0] * 61),
        ("golden_encode_4x2_repeated_pattern_input", ([0xDE, 0xAD, 0xBE, 0xEF] * 16)[:61]),
    ],
)
def test_classic_4x2_split_checksums(kats, name, data):
    rc, mat = O.build_matrix(4, 2)
    sh = split(np.array(data, np.uint8), 4)
    sh += [np.zeros(sh[0].size, np.uint8) for _ in range(2)]
    O.classic_encode(mat, sh)
    assert O.classic_verify(mat, sh)
    assert O.checksum_shards(sh) == kats["classic_4x2_golden"][name]["checksum"]


def test_classic_2x2_kat(kats):
    v = kats["classic_2x2"]
    rc, mat = O.build_matrix(2, 2)
    sh = [np.array(v["initial"][i * 3: i * 3 + 3], np.uint8) for i in range(4)]
    O.classic_encode(mat, sh)
    assert O.classic_verify(mat, sh)
    sh[0][:] = [101, 102, 103]
    assert O.classic_reconstruct(mat, sh, [0, 1, 1, 1]) == 0
    assert [int(x) for s in sh for x in s] == v["expect"]


@pytest.mark.parametrize("mode", ["vandermonde", "cauchy", "jerasure_like"])
@pytest.mark.parametrize("k,m", [(1, 1), (2, 2), (4, 2), (10, 4), (16, 4), (17, 3), (32, 8), (100, 28)])
def test_classic_matrix_modes_roundtrip(mode, k, m):
    rc, mat = O.build_matrix(k, m, mode)
    if rc != 0:
        pytest.skip(f"{mode} {k}+{m} rejected by the reference construction (rc={rc})")
    assert (mat[:k] == np.eye(k, dtype=np.uint8)).all()
    rng = np.random.default_rng(k * 1000 + m)
    sh = [rng.integers(0, 256, 48, dtype=np.uint8) for _ in range(k)] + [np.zeros(48, np.uint8)] * m
    sh = [s.copy() for s in sh]
    O.classic_encode(mat, sh)
    orig = [s.copy() for s in sh]
    lost = rng.choice(k + m, size=m, replace=False)
    pres = [0 if i in lost else 1 for i in range(k + m)]
    for i in lost:
        sh[i][:] = 0
    assert O.classic_reconstruct(mat, sh, pres) == 0
    assert all((a == b).all() for a, b in zip(sh, orig))


def test_classic_recovery_rows_match_two_stage():
    rng = np.random.default_rng(7)
    for k, m in [(10, 4), (16, 4), (4, 2), (6, 3)]:
        rc, mat = O.build_matrix(k, m)
        for trial in range(20):
            sh = [rng.integers(0, 256, 64, dtype=np.uint8) for _ in range(k + m)]  # non-codeword
            e = int(rng.integers(1, m + 1))
            lost = rng.choice(k + m, size=e, replace=False)
            pres = [0 if i in lost else 1 for i in range(k + m)]
            goal = ["all", "data", "required"][trial % 3]
            req = [int(rng.integers(0, 2)) for _ in range(k + m)] if goal == "required" else None
            two = [s.copy() for s in sh]
            assert O.classic_reconstruct(mat, two, pres, goal, req) == 0
            rc, surv, targ, rows = O.classic_recovery_rows(mat, pres, goal, req)
            assert rc == 0
            for t, idx in enumerate(targ):
                acc = np.zeros(64, np.uint8)
                for c, s in enumerate(surv):
                    acc = O.gf8_mul_slice_xor(int(rows[t, c]), sh[s], acc)
                assert (acc == two[idx]).all(), (k, m, goal, idx)


# ------------------------------------------------------------------ Leopard
def test_lgf16_fft_skew_prefix(kats):
    lg, ex, sk, wa = O.lgf16_tables()
    assert list(sk[:8]) == kats["lgf16_fft_skew_prefix"]["values"]


def test_lgf16_3x2_parity_matches_go(kats):
    v = kats["lgf16_3x2_parity_prefix"]
    data = [np.array([(i * 64 + j) & 0xFF for j in range(64)], np.uint8) for i in range(3)]
    rc, par = O.leopard_encode(16, 3, 2, data)
    assert rc == 0
    assert list(par[0][:16]) == v["go_parity0"]["values"]
    assert list(par[1][:16]) == v["go_parity1"]["values"]


def test_lgf16_3x2_coefficients(kats):
    rows = kats["lgf16_3x2_coefficients"]["rows"]
    for d in range(3):
        data = [np.zeros(64, np.uint8) for _ in range(3)]
        data[d][0] = 1
        rc, par = O.leopard_encode(16, 3, 2, data)
        for p in range(2):
            got = int(par[p][0]) | (int(par[p][1]) << 8)
            assert got == rows[p * 3 + d]


def test_lgf8_table_invariants(kats):
    lg, ex, sk, wa = O.lgf8_tables()
    assert lg[0] == kats["lgf8_table_invariants"]["log_lut0"]
    assert ex[0] == kats["lgf8_table_invariants"]["exp_lut0"]


def test_leopard_mul_is_linear_and_matches_log_exp():
    lg, ex, sk, wa = O.lgf8_tables()
    for lm in (0, 1, 77, 254, 255):
        for a in range(256):
            exp = 0 if a == 0 else ex[(int(lg[a]) + lm) % 255 if (int(lg[a]) + lm) != 255 else 255]
            assert O.lib().orc_lgf8_mul_log(a, lm) == exp


@pytest.mark.parametrize(
    "field,k,m,size",
    [(8, 4, 2, 64), (8, 10, 4, 128), (8, 32, 16, 64), (8, 128, 64, 64), (8, 3, 5, 64), (8, 120, 50, 64),
     (16, 3, 2, 64), (16, 10, 4, 128), (16, 32, 16, 64), (16, 300, 100, 64), (16, 1024, 512, 64),
     (16, 1, 1, 64), (16, 5, 7, 64)],
)
def test_leopard_roundtrip(field, k, m, size):
    rng = np.random.default_rng(field * 100000 + k * 100 + m)
    data = [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
    rc, par = O.leopard_encode(field, k, m, data)
    assert rc == 0
    full = data + par
    for trial in range(3):
        e = m if trial == 0 else int(rng.integers(1, m + 1))
        lost = rng.choice(k + m, size=e, replace=False)
        pres = [0 if i in lost else 1 for i in range(k + m)]
        sh = [s.copy() for s in full]
        for i in lost:
            sh[i][:] = 0xA5
        assert O.leopard_reconstruct(field, k, m, sh, pres) == 0
        for i in range(k + m):
            assert (sh[i] == full[i]).all(), (field, k, m, i)


def test_leopard_too_many_erasures():
    data = [np.zeros(64, np.uint8) for _ in range(4)]
    rc, par = O.leopard_encode(8, 4, 2, data)
    sh = data + par
    assert O.leopard_reconstruct(8, 4, 2, sh, [0, 0, 0, 1, 1, 1]) == 10  # TooFewShardsPresent


def test_gf16_tower_roundtrip():
    for k, m in [(4, 2), (10, 4), (20, 10)]:
        rc, mat = O.gf16t_build_matrix(k, m)
        assert rc == 0
        rng = np.random.default_rng(k)
        sh = [rng.integers(0, 256, 32, dtype=np.uint8) for _ in range(k)] + [np.zeros(32, np.uint8) for _ in range(m)]
        O.gf16t_encode(mat, sh)
        orig = [s.copy() for s in sh]
        lost = rng.choice(k + m, size=m, replace=False)
        pres = [0 if i in lost else 1 for i in range(k + m)]
        for i in lost:
            sh[i][:] = 0
        assert O.gf16t_reconstruct(mat, sh, pres) == 0
        assert all((a == b).all() for a, b in zip(sh, orig))


def test_leopard_combo_fit_rejected():
    # src/core/leopard.rs:225-237: ceil(k/m)*m must fit order - m.
    data = [np.zeros(64, np.uint8) for _ in range(200)]
    rc, _ = O.leopard_encode(8, 200, 50, data)
    assert rc == 2  # TooManyShards


def test_error_codes_are_the_reference_discriminants_plus_one(kats):
    # The C ABI returns the reference Error discriminant + 1 (src/errors.rs),
    # under the same names in the header and the Python mirror, with the
    # reference's own message text.
    import os
    import re

    import rsgpu

    ref = kats["error_enum"]
    header = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                               "rsgpu.h")).read()
    codes = {name: int(v) for name, v in re.findall(r"RSGPU_ERR_(\w+) = (\d+)", header)}
    assert len(ref["variants"]) == 16
    for i, variant in enumerate(ref["variants"]):
        snake = re.sub(r"(?<!^)(?=[A-Z])", "_", variant).upper()
        assert codes[snake] == i + 1, variant
        assert rsgpu.ERROR_NAMES[i + 1] == variant
        assert rsgpu.lib().rsgpu_error_string(i + 1).decode() == ref["messages"][variant], variant
    # device conditions sit outside the reference's range
    assert all(v >= 100 for k, v in codes.items() if k not in
               {re.sub(r"(?<!^)(?=[A-Z])", "_", x).upper() for x in ref["variants"]})


def test_default_options_are_the_references(kats):
    # rsgpu_options_default fills every field the way CodecOptions::default()
    # does (src/core/options.rs); enum values by the header's names.
    import os
    import re

    import rsgpu

    ref = kats["codec_options_default"]["fields"]
    header = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                               "rsgpu.h")).read()
    enum = {name: int(v) for name, v in re.findall(r"(RSGPU_\w+) = (\d+)", header)}
    prefix = {"codec_family": "RSGPU_FAMILY_", "leopard_mode": "RSGPU_LEOPARD_", "matrix_mode": "RSGPU_MATRIX_"}
    o = rsgpu._Options()
    rsgpu.lib().rsgpu_options_default(o)
    assert {f for f, _ in rsgpu._Options._fields_} == set(ref)
    for field, want in ref.items():
        got = getattr(o, field)
        if isinstance(want, str):
            want = enum[prefix[field] + re.sub(r"(?<!^)(?=[A-Z])", "_", want).upper()]
        assert got == want, (field, got, want)


def test_timed_cpu_row_kernel_matches_the_oracle_encode():
    # The benchmark's CPU baseline (GFNI rows at the host's widest vector, or
    # nibble tables) must compute the same parity as the scalar restatement,
    # including shard lengths with a ragged tail and recovery-row matrices.
    for k, m, size, n in [(10, 4, 4096 + 37, 3), (16, 4, 1000, 2), (4, 2, 70, 5), (20, 10, 999, 2)]:
        rc, mat = O.build_matrix(k, m)
        rng = np.random.default_rng(k + m + size)
        flat = []
        for _ in range(n):
            flat += [rng.integers(0, 256, size, dtype=np.uint8) for _ in range(k)]
            flat += [np.zeros(size, np.uint8) for _ in range(m)]
        for kernel in range(O.fast_best_kernel() + 1):
            O.fast_force_kernel(kernel)
            for s in range(n):
                for r in range(m):
                    flat[s * (k + m) + k + r][:] = 0xEE
            assert O.fast_encode_batch(mat, flat, n, size, 3) == 0
            for s in range(n):
                ref = [a.copy() for a in flat[s * (k + m): s * (k + m) + k]] + [np.zeros(size, np.uint8)
                                                                                for _ in range(m)]
                O.classic_encode(mat, ref)
                for i in range(k + m):
                    assert (ref[i] == flat[s * (k + m) + i]).all(), (k, m, s, i, O.fast_kernel_name())
        O.fast_force_kernel(-1)
