"""The request server: every result is byte-identical whether the request
ran alone or in a continuous-batching mix with others, equal to the CPU
oracle, and admission never exceeds the device-memory budget."""
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


GEOMS = [("classic", 4, 2), ("classic", 10, 4), ("leopard_gf8", 32, 16), ("leopard_gf16", 64, 32),
         ("leopard_gf8", 10, 4)]


@pytest.fixture(scope="module")
def codecs(rs):
    return {g: rs.ReedSolomon(g[1], g[2], rs.CodecOptions(codec_family=g[0])) for g in GEOMS}


def make_requests(codecs, seed, n):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        g = GEOMS[int(rng.integers(len(GEOMS)))]
        fam, k, m = g
        op = ["encode", "reconstruct", "verify"][int(rng.choice(3, p=[0.45, 0.4, 0.15]))]
        length = int(rng.integers(1, 200)) * 64
        data = rng.integers(0, 256, (k + m, length), dtype=np.uint8)
        present, goal = None, "all"
        if op == "reconstruct":
            e = int(rng.integers(1, m + 1))
            present = np.ones(k + m, np.uint8)
            present[rng.choice(k + m, size=e, replace=False)] = 0
            goal = "data" if rng.integers(3) == 0 else "all"
        if op == "verify" and rng.integers(2):
            data = oracle_apply(g, codecs[g], "encode", data, None, "all")[0]
        reqs.append(dict(geom=g, op=op, data=data, present=present, goal=goal, len=length))
    return reqs


def oracle_apply(g, codec, op, data, present, goal):
    fam, k, m = g
    out = data.copy()
    sh = [out[i] for i in range(k + m)]
    field = 8 if fam == "leopard_gf8" else 16
    if op in ("encode", "verify"):
        if fam == "classic":
            O.classic_encode(codec.encoding_matrix(), sh)
        else:
            rc, par = O.leopard_encode(field, k, m, sh[:k])
            for r in range(m):
                out[k + r] = par[r]
        if op == "verify":
            return data.copy(), bool(np.array_equal(out, data))
        return out, True
    if fam == "classic":
        assert O.classic_reconstruct(codec.encoding_matrix(), sh, present, goal=goal) == 0
    else:
        want = [1] * (k + m) if goal == "all" else [1] * k + [0] * m
        assert O.leopard_reconstruct(field, k, m, sh, present, want) == 0
    return out, True


def run(rs, server, codecs, reqs, one_at_a_time, device=None):
    """Submit every request (host buffers, or device tensors when `device`),
    return (outputs, verify results, completions)."""
    bufs, oks, comps = [], {}, []
    for i, r in enumerate(reqs):
        b = r["data"].copy()
        if device is not None:
            t = device.from_numpy(b).cuda()
            bufs.append(t)
            shards = [t[j] for j in range(t.shape[0])]
        else:
            bufs.append(b)
            shards = [b[j] for j in range(b.shape[0])]
        server.submit(codecs[r["geom"]], r["op"], shards, r["len"], present=r["present"], goal=r["goal"], tag=i + 1)
        if one_at_a_time:
            comps += server.wait(1)
    if not one_at_a_time:
        comps += server.wait(len(reqs))
    for c in comps:
        assert c["status"] == 0, c
        oks[c["tag"] - 1] = c["ok"]
    outs = [b.cpu().numpy() if device is not None else b for b in bufs]
    return outs, [oks[i] for i in range(len(reqs))], comps


def test_results_identical_alone_and_in_the_mix(rs, torch, codecs):
    reqs = make_requests(codecs, 3, 80)
    srv = rs.Server(streams=3, max_batch=16)
    alone, ok_alone, _ = run(rs, srv, codecs, reqs, one_at_a_time=True)
    mixed, ok_mixed, comps = run(rs, srv, codecs, reqs, one_at_a_time=False)
    st = srv.stats()
    srv.close()
    assert st["launches"] >= 80 + 5  # 80 alone, then several mixed launches
    for i, r in enumerate(reqs):
        want, want_ok = oracle_apply(r["geom"], codecs[r["geom"]], r["op"], r["data"], r["present"], r["goal"])
        assert np.array_equal(alone[i], want), (i, r["geom"], r["op"])
        assert np.array_equal(mixed[i], alone[i]), (i, r["geom"], r["op"])
        assert ok_alone[i] == ok_mixed[i] == want_ok, i


def test_device_resident_requests_and_concurrent_launches(rs, torch, codecs):
    reqs = make_requests(codecs, 9, 120)
    srv = rs.Server(streams=3, max_batch=8)
    outs, oks, comps = run(rs, srv, codecs, reqs, one_at_a_time=False, device=torch)
    st = srv.stats()
    srv.close()
    for i, r in enumerate(reqs):
        want, want_ok = oracle_apply(r["geom"], codecs[r["geom"]], r["op"], r["data"], r["present"], r["goal"])
        assert np.array_equal(outs[i], want), i
        assert oks[i] == want_ok
    assert st["launches"] >= 15 and st["max_concurrent_launches"] >= 2, st


def test_admission_respects_the_memory_budget(rs, torch, codecs):
    reqs = make_requests(codecs, 4, 60)
    largest = max((r["geom"][1] + r["geom"][2]) * r["len"] for r in reqs)
    budget = 2 * largest
    srv = rs.Server(device_budget=budget, streams=2)
    outs, oks, comps = run(rs, srv, codecs, reqs, one_at_a_time=False)
    st = srv.stats()
    srv.close()
    assert st["max_reserved_bytes"] <= budget and st["completed"] == 60
    # requests waited for memory: some were admitted well after submission
    assert max(c["admit_s"] - c["submit_s"] for c in comps) >= 0.0
    for i, r in enumerate(reqs):
        want, _ = oracle_apply(r["geom"], codecs[r["geom"]], r["op"], r["data"], r["present"], r["goal"])
        assert np.array_equal(outs[i], want), i


def test_server_errors(rs, torch, codecs):
    srv = rs.Server(device_budget=1 << 20)
    c = codecs[("leopard_gf8", 32, 16)]
    big = np.zeros((48, 64 << 10), np.uint8)
    with pytest.raises(rs.RsError) as e:
        srv.submit(c, "encode", [big[i] for i in range(48)], 64 << 10)
    assert e.value.name == "OutOfMemory"
    small = np.zeros((48, 100), np.uint8)
    with pytest.raises(rs.RsError) as e:
        srv.submit(c, "encode", [small[i] for i in range(48)], 100)
    assert e.value.name == "IncorrectShardSize"
    pres = np.zeros(48, np.uint8)
    ok = np.zeros((48, 64), np.uint8)
    with pytest.raises(rs.RsError) as e:
        srv.submit(c, "reconstruct", [ok[i] for i in range(48)], 64, present=pres)
    assert e.value.name == "TooFewShardsPresent"
    srv.close()


def test_repeated_leopard_pattern_fft_then_dense_map(rs, torch, codecs):
    # A Leopard GF(2^8) rebuild the plan table sends to the dense map: the
    # server's batches run the FFT decode until the pattern is due under the
    # per-call rule, then derive its map and use it.  Every result must equal
    # the oracle, whichever path ran, alone or beside other batches.
    from rsgpu import tune_mix

    g = ("leopard_gf8", 32, 16)
    c = codecs[g]
    k, m = 32, 16
    rng = np.random.default_rng(31)
    pres = np.ones(k + m, np.uint8)
    pres[rng.choice(k + m, size=4, replace=False)] = 0
    rs.Tuner.clear()
    rs.Tuner.load(tune_mix.DEFAULT_TABLE)
    try:
        size = None
        for cand in (1 << 20, 2 << 20, 4 << 20):
            op = dict(codec=c, op="reconstruct", shards=[0] * (k + m), shard_len=cand, present=pres, goal="all")
            p = rs.Tuner.lookup(op)
            if p is not None and p[0] == 0:
                size = cand
                break
        if size is None:
            pytest.skip("the plan table keeps 32+16 rebuilds on the FFT decode")
        data = rng.integers(0, 256, (k + m, size), dtype=np.uint8)
        want, _ = oracle_apply(g, c, "reconstruct", data, pres, "all")
        srv = rs.Server(streams=2, max_batch=4, planner="model")
        for call in range(5):  # one at a time
            t = torch.from_numpy(data).cuda()
            t[torch.from_numpy(pres == 0).cuda()] = 0
            srv.submit(c, "reconstruct", [t[j] for j in range(k + m)], size, present=pres, tag=call + 1)
            comp = srv.wait(1)
            assert comp[0]["status"] == 0
            assert np.array_equal(t.cpu().numpy(), want), call
            torch.cuda.synchronize()
        srv.close()
        # Several new patterns at once, one request per batch, built while
        # earlier batches run.
        pats = []
        for _ in range(3):
            p2 = np.ones(k + m, np.uint8)
            p2[rng.choice(k + m, size=3, replace=False)] = 0
            pats.append(p2)
        wants = [oracle_apply(g, c, "reconstruct", data, p2, "all")[0] for p2 in pats]
        srv = rs.Server(streams=3, max_batch=1, planner="model")
        for rnd in range(3):
            bufs = []
            for i, p2 in enumerate(pats):
                t = torch.from_numpy(data).cuda()
                t[torch.from_numpy(p2 == 0).cuda()] = 0
                bufs.append(t)
                srv.submit(c, "reconstruct", [t[j] for j in range(k + m)], size, present=p2, tag=10 * rnd + i + 1)
            comps = srv.wait(len(pats))
            assert all(x["status"] == 0 for x in comps)
            torch.cuda.synchronize()
            for i, t in enumerate(bufs):
                assert np.array_equal(t.cpu().numpy(), wants[i]), (rnd, i)
        srv.close()
    finally:
        rs.Tuner.clear()


def test_wide_leopard_decodes_run_by_the_codec_kernel(rs, torch):
    # Leopard GF(2^16) reconstructions whose work rows do not fit k_mix's
    # shared memory (here 1024 and 2048 lanes) leave the server's mixed batch
    # for their codec's own decode kernel on the batch's stream.  Their bytes
    # must equal the oracle's, alone and in batches that mix them with
    # encodes, classic rebuilds and each other (goals all and data).
    geoms = [("leopard_gf16", 300, 100), ("leopard_gf16", 1024, 512), ("classic", 10, 4)]
    cods = {g: rs.ReedSolomon(g[1], g[2], rs.CodecOptions(codec_family=g[0])) for g in geoms}
    rng = np.random.default_rng(77)
    reqs = []
    for i in range(30):
        g = geoms[i % 3]
        fam, k, m = g
        op = "reconstruct" if i % 5 else "encode"
        length = int(rng.integers(1, 4)) * 64
        data = rng.integers(0, 256, (k + m, length), dtype=np.uint8)
        present, goal = None, "all"
        if op == "reconstruct":
            e = int(rng.integers(1, m + 1))
            present = np.ones(k + m, np.uint8)
            present[rng.choice(k + m, size=e, replace=False)] = 0
            goal = "data" if i % 4 == 0 else "all"
        reqs.append(dict(geom=g, op=op, data=data, present=present, goal=goal, len=length))
    srv = rs.Server(streams=3, max_batch=8)
    alone, _, _ = run(rs, srv, cods, reqs, one_at_a_time=True, device=torch)
    mixed, _, _ = run(rs, srv, cods, reqs, one_at_a_time=False, device=torch)
    srv.close()
    for i, r in enumerate(reqs):
        want, _ = oracle_apply(r["geom"], cods[r["geom"]], r["op"], r["data"], r["present"], r["goal"])
        assert np.array_equal(alone[i], want), (i, r["geom"], r["op"], r["goal"])
        assert np.array_equal(mixed[i], want), (i, r["geom"], r["op"], r["goal"])


def test_large_leopard_gf8_rebuilds_through_maps_derived_on_the_stream(rs, torch):
    # Leopard GF(2^8) rebuilds of 32 MiB stripes and more whose dense map is
    # not cached run, in the server's batches, through a map derived on the
    # batch's stream (FFT decode of unit vectors, then device packing).  Every
    # fresh pattern must give the oracle's bytes, goals all and data, in
    # batches alone and together with other requests.
    geoms = [("leopard_gf8", 32, 16), ("leopard_gf8", 128, 64), ("classic", 10, 4)]
    cods = {g: rs.ReedSolomon(g[1], g[2], rs.CodecOptions(codec_family=g[0])) for g in geoms}
    rng = np.random.default_rng(91)
    reqs = []
    for i in range(9):
        g = geoms[i % 3]
        fam, k, m = g
        length = (1 << 20) if g[1] == 32 else (256 << 10) if g[1] == 128 else (64 << 10)
        data = rng.integers(0, 256, (k + m, length), dtype=np.uint8)
        e = int(rng.integers(1, m + 1))
        present = np.ones(k + m, np.uint8)
        present[rng.choice(k + m, size=e, replace=False)] = 0
        goal = "data" if i % 4 == 1 else "all"
        reqs.append(dict(geom=g, op="reconstruct", data=data, present=present, goal=goal, len=length))
    srv = rs.Server(streams=2, max_batch=4)
    alone, _, _ = run(rs, srv, cods, reqs, one_at_a_time=True, device=torch)
    mixed, _, _ = run(rs, srv, cods, reqs, one_at_a_time=False, device=torch)
    srv.close()
    for i, r in enumerate(reqs):
        want, _ = oracle_apply(r["geom"], cods[r["geom"]], r["op"], r["data"], r["present"], r["goal"])
        assert np.array_equal(alone[i], want), (i, r["geom"], r["goal"])
        assert np.array_equal(mixed[i], want), (i, r["geom"], r["goal"])
