"""Mixed batches (one persistent kernel over many codecs, lengths and
operations) against the CPU oracle, byte for byte, under every plan."""
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


@pytest.fixture(scope="module")
def codecs(rs):
    out = {}
    for fam, k, m in [("classic", 4, 2), ("classic", 10, 4), ("classic", 16, 4), ("leopard_gf8", 32, 16),
                      ("leopard_gf8", 128, 64), ("leopard_gf16", 64, 32), ("leopard_gf16", 10, 4)]:
        out[(fam, k, m)] = rs.ReedSolomon(k, m, rs.CodecOptions(codec_family=fam))
    return out


def field_of(fam):
    return 8 if fam == "leopard_gf8" else 16


def make_case(torch, codecs, seed, n_ops, lo, hi, geoms=None, align=64, odd=False):
    """Random ops over the codecs; returns (ops for MixedBatch, host copies, specs)."""
    from rsgpu import workload as W

    rng = np.random.default_rng(seed)
    geoms = geoms or list(codecs)
    specs, host, dev = [], [], []
    for i in range(n_ops):
        fam, k, m = geoms[int(rng.integers(len(geoms)))]
        op = ["encode", "reconstruct", "verify"][int(rng.choice(3, p=[0.45, 0.4, 0.15]))]
        length = W.log_uniform_len(rng, lo, hi, align)
        if odd and fam == "classic":
            length += int(rng.integers(1, 64))
        total = k + m
        data = rng.integers(0, 256, (total, length), dtype=np.uint8)
        present = None
        goal = "all"
        if op == "verify" and rng.integers(2) == 0:
            # a codeword: parity from the oracle
            data = oracle_encode((fam, k, m), codecs[(fam, k, m)], data)
        if op == "reconstruct":
            e = int(rng.integers(0, m + 1))
            lost = rng.choice(total, size=e, replace=False) if e else []
            present = np.ones(total, np.uint8)
            present[list(lost)] = 0
            goal = "data" if rng.integers(4) == 0 else "all"
        specs.append(dict(geom=(fam, k, m), op=op, present=present, goal=goal, len=length))
        host.append(data)
    # one device arena, each stripe 256-byte aligned
    offs, cur = [], 0
    for d in host:
        offs.append(cur)
        cur += (d.size + 255) // 256 * 256
    arena = torch.zeros(cur + 256, dtype=torch.uint8, device="cuda")
    for o, d in zip(offs, host):
        arena[o:o + d.size] = torch.from_numpy(d.reshape(-1)).cuda()
    ops = []
    for sp, o in zip(specs, offs):
        fam, k, m = sp["geom"]
        base = arena.data_ptr() + o
        ptrs = [base + j * sp["len"] for j in range(k + m)]
        ops.append(dict(codec=codecs[sp["geom"]], op=sp["op"], shards=ptrs, shard_len=sp["len"],
                        present=sp["present"], goal=sp["goal"]))
    return ops, host, specs, arena, offs


def oracle_encode(geom, codec, data):
    fam, k, m = geom
    out = data.copy()
    if fam == "classic":
        sh = [out[i] for i in range(k + m)]
        O.classic_encode(codec.encoding_matrix(), sh)
    else:
        rc, par = O.leopard_encode(field_of(fam), k, m, [out[i] for i in range(k)])
        assert rc == 0
        for r in range(m):
            out[k + r] = par[r]
    return out


def oracle_expect(specs, host, codecs):
    """Expected arena contents and verify flags per op."""
    exp, flags = [], []
    for sp, d in zip(specs, host):
        fam, k, m = sp["geom"]
        c = codecs[sp["geom"]]
        if sp["op"] == "encode":
            exp.append(oracle_encode(sp["geom"], c, d))
            flags.append(True)
        elif sp["op"] == "verify":
            want = oracle_encode(sp["geom"], c, d)
            exp.append(d.copy())
            flags.append(bool(np.array_equal(want, d)))
        else:
            out = d.copy()
            sh = [out[i] for i in range(k + m)]
            if fam == "classic":
                rc = O.classic_reconstruct(c.encoding_matrix(), sh, sp["present"], goal=sp["goal"])
            else:
                want = [1] * (k + m) if sp["goal"] == "all" else [1] * k + [0] * m
                rc = O.leopard_reconstruct(field_of(fam), k, m, sh, sp["present"], want)
            assert rc == 0
            exp.append(out)
            flags.append(True)
    return exp, flags


def check(torch, arena, offs, exp, specs, tag):
    got = arena.cpu().numpy()
    for i, (o, e) in enumerate(zip(offs, exp)):
        g = got[o:o + e.size].reshape(e.shape)
        if not np.array_equal(g, e):
            bad = np.argwhere(g != e)
            raise AssertionError(f"{tag}: op {i} {specs[i]['geom']} {specs[i]['op']} len {specs[i]['len']} "
                                 f"first mismatch (shard, col) {tuple(bad[0])} of {len(bad)}")


@pytest.mark.parametrize("seed", [1, 2])
@pytest.mark.parametrize("graph", [True, False])
def test_mix_default_plans_match_oracle(rs, torch, codecs, seed, graph):
    ops, host, specs, arena, offs = make_case(torch, codecs, seed, 40, 64, 40000)
    exp, flags = oracle_expect(specs, host, codecs)
    mb = rs.MixedBatch(ops, graph=graph)
    mb.launch()
    torch.cuda.synchronize()
    check(torch, arena, offs, exp, specs, f"seed {seed}")
    assert list(mb.results()) == flags
    info = mb.info()
    assert info.kernels_per_launch == 1 and info.n_ops == len(ops)
    # A second launch reads its own outputs as inputs only where the op says
    # so (encode/reconstruct outputs are functions of untouched inputs), so
    # the bytes do not change.
    mb.launch()
    torch.cuda.synchronize()
    check(torch, arena, offs, exp, specs, "relaunch")
    assert list(mb.results()) == flags


def plan_variants(specs):
    """Every valid plan family, applied to all ops it fits."""
    out = {}
    for name in ["apply8k", "apply4k", "fft1", "fft2", "fft3", "dense8k"]:
        plans = []
        for sp in specs:
            fam = sp["geom"][0]
            if fam == "classic":
                plans.append((0, 1 if name == "apply4k" else 0))
            elif name.startswith("fft") or fam == "leopard_gf16":
                t = int(name[3:]) if name.startswith("fft") else 1
                plans.append((1, t))
            elif name in ("apply8k", "dense8k"):
                plans.append((0, 0))
            else:
                plans.append((0, 1))
        out[name] = plans
    return out


@pytest.mark.parametrize("variant", ["apply8k", "apply4k", "fft1", "fft2", "fft3"])
def test_mix_every_plan_writes_the_same_bytes(rs, torch, codecs, variant):
    ops, host, specs, arena, offs = make_case(torch, codecs, 11, 36, 64, 20000)
    exp, flags = oracle_expect(specs, host, codecs)
    plans = plan_variants(specs)[variant]
    mb = rs.MixedBatch(ops, plans=plans, order="submit" if variant == "fft2" else "cost")
    assert mb.plans() == [tuple(p) for p in plans]
    mb.launch()
    torch.cuda.synchronize()
    check(torch, arena, offs, exp, specs, variant)
    assert list(mb.results()) == flags


@pytest.mark.parametrize("size,want_tile", [(4096, 1), (262144, 3)])
def test_small_batch_runs_transforms_at_the_finest_tile(rs, torch, codecs, size, want_tile):
    # The fixed rule gives a 128+64 encode 8 blocks per work item.  A batch
    # with fewer items than the kernel's resident CTAs (3 x 148; one 4 KiB
    # stripe: 8 items) runs at the finest tile instead, so more items run side
    # by side; one that fills the GPU (256 KiB: 512 items) keeps the planned
    # tile.
    # The bytes are the oracle's either way.
    g = ("leopard_gf8", 128, 64)
    c = codecs[g]
    k, m = 128, 64
    data = np.random.default_rng(size).integers(0, 256, (k + m, size), dtype=np.uint8)
    t = torch.from_numpy(data).cuda()
    op = dict(codec=c, op="encode", shards=[t[j] for j in range(k + m)], shard_len=size)
    mb = rs.MixedBatch([op], planner="fixed", graph=False)
    assert mb.plans() == [(rs.ALGO_FFT, want_tile)]
    mb.launch()
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), oracle_encode(g, c, data))


@pytest.mark.parametrize("plan", [None, 1, 2, 3])
def test_mix_wide_gf16_code_with_global_work_rows(rs, torch, plan):
    # GF(2^16) 600+300: 1024 encode rows and 2048 decode lanes, more than a
    # k_mix CTA's shared memory holds, so the work rows live in the batch's
    # global scratch.  Encode, rebuild (goals all and data), and verify of a
    # codeword and of a corrupted stripe in one batch, at the planner's tile
    # (None) and at every forced tile, against the oracle on inputs that are
    # not codewords.
    geom = ("leopard_gf16", 600, 300)
    k, m = geom[1], geom[2]
    total = k + m
    cods = {geom: rs.ReedSolomon(k, m, rs.CodecOptions(codec_family="leopard_gf16"))}
    rng = np.random.default_rng(600 + (plan or 0))
    specs, host = [], []
    for op, length, goal in [("encode", 2048, "all"), ("reconstruct", 1024, "all"), ("reconstruct", 3072, "data"),
                             ("verify", 1024, "all"), ("verify", 2048, "all")]:
        data = rng.integers(0, 256, (total, length), dtype=np.uint8)
        present = None
        if op == "verify":
            data = oracle_encode(geom, cods[geom], data)
            if length == 2048:
                data[k + 7, 100] ^= 0x40
        if op == "reconstruct":
            present = np.ones(total, np.uint8)
            present[rng.choice(total, size=m, replace=False)] = 0
        specs.append(dict(geom=geom, op=op, present=present, goal=goal, len=length))
        host.append(data)
    offs, cur = [], 0
    for d in host:
        offs.append(cur)
        cur += (d.size + 255) // 256 * 256
    arena = torch.zeros(cur + 256, dtype=torch.uint8, device="cuda")
    for o, d in zip(offs, host):
        arena[o:o + d.size] = torch.from_numpy(d.reshape(-1)).cuda()
    ops = [dict(codec=cods[geom], op=sp["op"], shard_len=sp["len"], present=sp["present"], goal=sp["goal"],
                shards=[arena.data_ptr() + o + j * sp["len"] for j in range(total)]) for sp, o in zip(specs, offs)]
    exp, flags = oracle_expect(specs, host, cods)
    assert flags == [True, True, True, True, False]
    plans = None if plan is None else [(rs.ALGO_FFT, plan)] * len(ops)
    mb = rs.MixedBatch(ops, plans=plans, graph=False)
    if plan is None:  # a small batch: the finest tile
        assert mb.plans() == [(rs.ALGO_FFT, 1)] * len(ops)
    mb.launch()
    torch.cuda.synchronize()
    check(torch, arena, offs, exp, specs, f"tile {plan}")
    assert list(mb.results()) == flags


def test_mix_dense_leopard_maps_are_exact_on_non_codewords(rs, torch, codecs):
    # Leopard GF(2^8) operations run as dense matrices over the Leopard field:
    # the reconstruction map uses every present shard, like the FFT decode, so
    # the bytes agree even when the inputs are not a codeword.
    geoms = [("leopard_gf8", 32, 16), ("leopard_gf8", 128, 64)]
    ops, host, specs, arena, offs = make_case(torch, codecs, 5, 24, 64, 16384, geoms=geoms)
    exp, flags = oracle_expect(specs, host, codecs)
    plans = [(0, i % 2) for i in range(len(ops))]
    mb = rs.MixedBatch(ops, plans=plans)
    mb.launch()
    torch.cuda.synchronize()
    check(torch, arena, offs, exp, specs, "dense")
    assert list(mb.results()) == flags


def test_mix_odd_lengths_and_misaligned_pointers(rs, torch, codecs):
    # Classic shards whose length is not a multiple of 16 take the byte tail
    # path; a stripe whose pointers are misaligned runs entirely on it.
    geoms = [("classic", 4, 2), ("classic", 10, 4)]
    ops, host, specs, arena, offs = make_case(torch, codecs, 9, 20, 64, 9000, geoms=geoms, odd=True)
    # shift the last stripe by one byte
    last = len(ops) - 1
    fam, k, m = specs[last]["geom"]
    n = specs[last]["len"]
    d = host[last]
    o = offs[last] + 1
    arena[o:o + d.size] = torch.from_numpy(d.reshape(-1)).cuda()
    offs[last] = o
    ops[last]["shards"] = [arena.data_ptr() + o + j * n for j in range(k + m)]
    exp, flags = oracle_expect(specs, host, codecs)
    mb = rs.MixedBatch(ops)
    mb.launch()
    torch.cuda.synchronize()
    check(torch, arena, offs, exp, specs, "odd")
    assert list(mb.results()) == flags


def test_mix_errors(rs, torch, codecs):
    t = torch.zeros(64 * 200, dtype=torch.uint8, device="cuda")
    base = t.data_ptr()
    c = codecs[("leopard_gf8", 32, 16)]
    ptrs = [base + 64 * i for i in range(48)]
    with pytest.raises(rs.RsError) as e:
        rs.MixedBatch([dict(codec=c, op="encode", shards=ptrs, shard_len=100)])
    assert e.value.name == "IncorrectShardSize"
    with pytest.raises(rs.RsError) as e:
        pres = np.zeros(48, np.uint8)
        rs.MixedBatch([dict(codec=c, op="reconstruct", shards=ptrs, shard_len=64, present=pres)])
    assert e.value.name == "TooFewShardsPresent"
    with pytest.raises(rs.RsError) as e:
        rs.MixedBatch([dict(codec=c, op="encode", shards=ptrs, shard_len=64)], plans=[(1, 7)])
    assert e.value.name == "InvalidArgument"
    cl = codecs[("classic", 4, 2)]
    with pytest.raises(rs.RsError) as e:
        rs.MixedBatch([dict(codec=cl, op="encode", shards=ptrs[:6], shard_len=64)], plans=[(1, 0)])
    assert e.value.name == "InvalidArgument"
    g16 = codecs[("leopard_gf16", 10, 4)]
    with pytest.raises(rs.RsError) as e:
        rs.MixedBatch([dict(codec=g16, op="encode", shards=ptrs[:14], shard_len=64)], plans=[(0, 0)])
    assert e.value.name == "InvalidArgument"
    tower = rs.ReedSolomon(4, 2, field="gf16")
    with pytest.raises(rs.RsError) as e:
        rs.MixedBatch([dict(codec=tower, op="encode", shards=ptrs[:6], shard_len=64)])
    assert e.value.name == "UnsupportedCodecFamily"
    with pytest.raises(rs.RsError) as e:
        rs.MixedBatch([dict(codec=cl, op="encode", shards=ptrs[:6], shard_len=0)])
    assert e.value.name == "EmptyShard"
    # an empty batch is valid and launches nothing
    mb = rs.MixedBatch([])
    mb.launch()
    assert mb.info().kernels_per_launch == 0


def test_prepared_batch_survives_decode_cache_eviction(rs, torch):
    # A prepared batch keeps private copies of its decode tables: evicting
    # them from the codec's cache afterwards must not change its output.
    k, m, n = 10, 4, 4096
    c = rs.ReedSolomon(k, m, rs.CodecOptions(inversion_cache_capacity=4))
    rng = np.random.default_rng(3)
    data = rng.integers(0, 256, (k + m, n), dtype=np.uint8)
    full = oracle_encode(("classic", k, m), c, data)
    buf = torch.from_numpy(full.copy()).cuda()
    pres = np.ones(k + m, np.uint8)
    pres[[0, 3, 11, 13]] = 0
    ptrs = rs.device_pointer_table(buf.data_ptr(), [i * n for i in range(k + m)])
    pb = c.prepare_batch("reconstruct", ptrs, n, present=pres[None, :])
    # churn the cache with other patterns
    scratch = torch.from_numpy(full.copy()).cuda()
    for trial in range(12):
        lost = set(rng.choice(k + m, size=3, replace=False).tolist())
        lst = [None if i in lost else scratch[i] for i in range(k + m)]
        c.reconstruct(lst)
    assert c.cache_stats().evictions > 0
    for i in [0, 3, 11, 13]:
        buf[i].fill_(0)
    pb.launch()
    torch.cuda.synchronize()
    assert np.array_equal(buf.cpu().numpy(), full)
