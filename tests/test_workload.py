"""The seeded mixed-geometry workload (rsgpu/workload.py) against the
distribution it stands for: 16384 operations over classic GF(2^8) {4+2, 6+3,
8+4, 12+4, 16+4} and Leopard GF(2^8) {32+16, 128+64}, shard sizes
log-uniform between 4 KiB and 4 MiB rounded to 64 bytes, erasure counts
uniform in 0..m at random positions, and encode / reconstruct / verify with
probabilities 0.5 / 0.4 / 0.1.  Host logic only: no GPU."""
import numpy as np
import pytest

from rsgpu import workload as W

SEED = 0x00EC5EED20260524


@pytest.fixture(scope="module")
def specs():
    return W.mixed_specs(16384, SEED + 4)


def test_same_seed_same_workload(specs):
    again = W.mixed_specs(512, SEED + 4)
    for a, b in zip(specs[:512], again):
        assert (a.geom, a.op, a.shard_len) == (b.geom, b.op, b.shard_len)
        assert (a.present is None) == (b.present is None)
        if a.present is not None:
            assert np.array_equal(a.present, b.present)
    other = W.mixed_specs(512, SEED + 5)
    assert [s.shard_len for s in other] != [s.shard_len for s in specs[:512]]


def test_geometries_are_uniform(specs):
    counts = {g: 0 for g in W.MIX_GEOMETRIES}
    for s in specs:
        counts[s.geom] += 1
    expect = len(specs) / len(W.MIX_GEOMETRIES)
    # 5 sigma of a binomial(16384, 1/7) count
    sigma = np.sqrt(len(specs) * (1 / 7) * (6 / 7))
    for g, c in counts.items():
        assert abs(c - expect) < 5 * sigma, (g, c)


def test_operation_mix(specs):
    n = len(specs)
    for op, p in zip(W.OPS, W.OP_PROBS):
        c = sum(s.op == op for s in specs)
        assert abs(c - n * p) < 5 * np.sqrt(n * p * (1 - p)), (op, c)


def test_shard_sizes_log_uniform_and_aligned(specs):
    lens = np.array([s.shard_len for s in specs], np.float64)
    assert (lens % 64 == 0).all()
    assert lens.min() >= 4096 - 32 and lens.max() <= (4 << 20) + 32
    # log-uniform: log2(len) is uniform on [12, 22], mean 17, sd 10 / sqrt(12)
    lg = np.log2(lens)
    assert abs(lg.mean() - 17.0) < 0.05
    assert abs(lg.std() - 10 / np.sqrt(12)) < 0.05
    # every decade of the range is populated in proportion
    hist, _ = np.histogram(lg, bins=10, range=(12, 22))
    assert hist.min() > 0.8 * len(specs) / 10


def test_erasures_uniform_in_0_to_m(specs):
    by_geom = {}
    for s in specs:
        if s.op != "reconstruct":
            assert s.present is None
            continue
        fam, k, m = s.geom
        assert s.present.shape == (k + m,) and s.present.dtype == np.uint8
        e = int((s.present == 0).sum())
        assert 0 <= e <= m
        by_geom.setdefault(s.geom, []).append(e)
    for (fam, k, m), es in by_geom.items():
        es = np.array(es)
        # uniform on 0..m: mean m/2, and both ends occur
        assert abs(es.mean() - m / 2) < 5 * np.sqrt(((m + 1) ** 2 - 1) / 12 / len(es)), (k, m)
        assert es.min() == 0 and es.max() == m


def test_erasure_positions_cover_data_and_parity(specs):
    lost_data = lost_parity = 0
    for s in specs:
        if s.present is None:
            continue
        k = s.geom[1]
        lost = np.flatnonzero(s.present == 0)
        lost_data += int((lost < k).sum())
        lost_parity += int((lost >= k).sum())
    assert lost_data > 0 and lost_parity > 0


def test_algorithmic_bytes_follow_the_roofline_accounting():
    k, m, S = 10, 4, 65536
    enc = W.MixOpSpec(("classic", k, m), "encode", S)
    ver = W.MixOpSpec(("classic", k, m), "verify", S)
    assert enc.algorithmic_bytes() == ver.algorithmic_bytes() == (k + m) * S
    pres = np.ones(k + m, np.uint8)
    pres[[0, 3, 11, 13]] = 0
    rec = W.MixOpSpec(("classic", k, m), "reconstruct", S, pres)
    assert rec.algorithmic_bytes() == (k + 4) * S  # reads k survivors, writes e
    lk, lm = 32, 16
    lp = np.ones(lk + lm, np.uint8)
    lp[:5] = 0
    lrec = W.MixOpSpec(("leopard_gf8", lk, lm), "reconstruct", S, lp)
    assert lrec.algorithmic_bytes() == (lk + lm) * S  # reads every present, writes e
    none = W.MixOpSpec(("classic", k, m), "reconstruct", S, np.ones(k + m, np.uint8))
    assert none.algorithmic_bytes() == 0


def test_waves_fit_the_arena_and_keep_order(specs):
    arena = 8 << 30
    groups = W.waves(specs, arena)
    assert [i for g in groups for i in g] == list(range(len(specs)))
    for g in groups:
        used = sum((specs[i].stripe_bytes + 255) // 256 * 256 for i in g)
        assert used <= arena or len(g) == 1
