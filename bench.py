"""Benchmark: batched classic encode + rebuild + verify on one B200 per rank.

Workload (the reference's config quoted for the headline metric): classic
galois_8 10+4 and 16+4, 1 MiB shards, 4096 stripes each, uniform-random u8
data from a seed; every stripe gets a seeded erasure pattern of 1..m shards
among k+m (data and parity mixed).  One step = encode, reconstruct and
verify_with_workspace over all stripes of both geometries.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Metric: GB/s of algorithmic bytes (encode (k+m)S, reconstruct (k+e)S, verify
(k+m)S), the same accounting as the roofline.  Inputs (137 GiB) are far
larger than L2, so no flush is needed between steps.  Under torchrun each rank
runs the same per-GPU workload (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rustfs-erasure-codec_b200"))

SEED = 0x00EC5EED20260524  # the reference benches' BASE_SEED (benches/common/mod.rs:10)
GEOMS = [(10, 4), (16, 4)]
SHARD = 1 << 20
STRIPES = 4096
MIX_OPS = 16384  # stripes of the mixed-geometry workload
# Both arms (this build and the reference's CPU path) report this metric.
METRIC = "batched classic encode+rebuild+verify GB/s (algorithmic bytes)"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
PROFILE_FILE = os.path.join(ROOT, "profiles", "k_apply_tma_encode_10x4.txt")


def erasure_patterns(k, m, n, seed):
    """Seeded per-stripe erasure sets of 1..m shards among k+m."""
    rng = np.random.default_rng(seed)
    pats = np.ones((n, k + m), np.uint8)
    counts = rng.integers(1, m + 1, size=n)
    for s in range(n):
        lost = rng.choice(k + m, size=int(counts[s]), replace=False)
        pats[s, lost] = 0
    return pats


def step_bytes(k, m, pats, size):
    n = pats.shape[0]
    e = (k + m) - pats.sum(axis=1)
    return int(n * (k + m) * size), int(((k + e) * size).sum()), int(n * (k + m) * size)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        import tempfile

        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def pin_to_gpu_numa(torch, device):
    """Restrict this process to the CPUs NVML reports as local to the GPU, so
    pinned host buffers are allocated on the GPU's NUMA node (a buffer on the
    far socket crosses the inter-socket link and halves the host<->device
    rate).  Returns (original CPU set, local CPU count); (None, None) when
    NVML cannot tell.  Only this process's scheduling changes."""
    try:
        import pynvml

        p = torch.cuda.get_device_properties(device)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            words = pynvml.nvmlDeviceGetCpuAffinity(h, (os.cpu_count() + 63) // 64)
        finally:
            pynvml.nvmlShutdown()
        cpus = {w * 64 + b for w, word in enumerate(words) for b in range(64) if (int(word) >> b) & 1}
        orig = os.sched_getaffinity(0)
        cpus &= orig
        if not cpus:
            return None, None
        os.sched_setaffinity(0, cpus)
        return orig, len(cpus)
    except Exception:
        return None, None


def measured_hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic_ratio():
    """DRAM bytes per algorithmic byte of the encode kernel, from the committed
    ncu summary (None when absent)."""
    try:
        for line in open(PROFILE_FILE):
            if line.startswith("dram_bytes_per_algorithmic_byte:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


# --------------------------------------------------------------------- CPU side
def cpu_widths():
    """GFNI kernels the host can run, widest first (the reference's order),
    or the nibble kernel alone."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    best = O.fast_best_kernel()
    return [2, 1] if best == 2 else [best]


def cpu_best(threads, keep=False):
    """cpu_sample with each GFNI width the host has; the faster is reported
    (the reference picks the widest, src/galois_8/backend.rs:396-413, which
    is not always the faster on every host, so the baseline takes the better
    of the two rather than risk under-reporting it)."""
    best = None
    for kernel in cpu_widths():
        r = cpu_sample(threads, keep=keep, kernel=kernel)
        if best is None or r[0] > best[0]:
            best = r
    return best


def cpu_sample(threads, keep=False, kernel=-1):
    """Time the oracle's threaded restatement of the reference's fastest x86
    classic path (GFNI row dot products at the host's widest vector width,
    src/galois_8/x86/gfni_rows.rs, chosen as src/galois_8/backend.rs:396-413
    chooses) on a bounded sample: 64 stripes per geometry, encode + rebuild
    (the same row kernel applied to recovery rows) + verify.  Recovery rows
    are derived once per distinct erasure pattern before the timed region,
    as the reference's inversion cache keeps them (src/core/inversion_cache.rs),
    and every output buffer is allocated before it; the timed region holds the
    row-kernel calls and verify's comparison only.
    Returns (GB/s of algorithmic bytes, kernel name, stripes per geometry,
    GiB/s in the reference's data-bytes convention, sample) where sample,
    with keep=True, holds per geometry the inputs and every output (for the
    GPU's byte-for-byte check on the same stripes)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    O.fast_force_kernel(kernel)
    n = 64
    total_bytes = data_bytes = 0
    t_total = 0.0
    sample = []
    for gi, (k, m) in enumerate(GEOMS):
        rng = np.random.default_rng(SEED + gi)
        rc, mat = O.build_matrix(k, m)
        block = rng.integers(0, 256, 64 * SHARD, dtype=np.uint8)
        # Every buffer is written once before the timed region, so no page is
        # first touched (and faulted in) while the row kernel is timed.
        stripes = np.empty((n, k + m, SHARD), np.uint8)
        stripes[:, k:].fill(0)
        for s in range(n):
            for i in range(k):
                j = s * k + i
                stripes[s, i] = np.roll(block[(j % 64) * SHARD:(j % 64 + 1) * SHARD], j // 64)
        flat = [stripes[s, i] for s in range(n) for i in range(k + m)]
        pats = erasure_patterns(k, m, n, SEED + 100 + gi)
        eb, rb, vb = step_bytes(k, m, pats, SHARD)
        # Untimed: recovery rows per distinct pattern, rebuild outputs, verify scratch.
        rows_of = {}
        rebuild = []
        for s in range(n):
            key = pats[s].tobytes()
            if key not in rows_of:
                rc, surv, targ, rows = O.classic_recovery_rows(mat, pats[s])
                sub = np.zeros((k + len(targ), k), np.uint8)
                sub[:k] = np.eye(k, dtype=np.uint8)
                sub[k:] = rows
                rows_of[key] = (surv, targ, sub)
            surv, targ, sub = rows_of[key]
            outs = np.empty((len(targ), SHARD), np.uint8)
            outs.fill(0)
            rebuild.append((sub, [flat[s * (k + m) + i] for i in surv] + [outs[j] for j in range(len(targ))],
                            targ, outs))
        scratch_par = np.empty((n, m, SHARD), np.uint8)
        scratch_par.fill(0)
        scratch = []
        for s in range(n):
            scratch += [flat[s * (k + m) + i] for i in range(k)] + [scratch_par[s, r] for r in range(m)]
        t0 = time.perf_counter()
        O.fast_encode_batch(mat, flat, n, SHARD, threads)
        t_enc = time.perf_counter() - t0
        t0 = time.perf_counter()
        for sub, ptrs, targ, outs in rebuild:
            O.fast_encode_batch(sub, ptrs, 1, SHARD, threads)
        t_rec = time.perf_counter() - t0
        t0 = time.perf_counter()
        O.fast_encode_batch(mat, scratch, n, SHARD, threads)
        ok = all(np.array_equal(scratch_par[s, r], stripes[s, k + r]) for s in range(n) for r in range(m))
        t_ver = time.perf_counter() - t0
        assert ok
        total_bytes += eb + rb + vb
        data_bytes += 3 * n * k * SHARD
        t_total += t_enc + t_rec + t_ver
        if keep:
            sample.append(dict(k=k, m=m, stripes=stripes, pats=pats,
                               rebuilt=[(targ, outs) for sub, ptrs, targ, outs in rebuild]))
    return total_bytes / t_total / 1e9, O.fast_kernel_name(), n, data_bytes / t_total / 2**30, sample


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def sample_check(torch, rsgpu, sample):
    """Run the GPU's batched encode, rebuild and verify (the timed prepared
    batches' path, device memory) on the CPU baseline's own sample stripes
    and compare every output byte with the CPU's: parity, every rebuilt shard
    (the erased shards are poisoned first), and the verify flags (all true,
    then false exactly for the stripes whose parity had a byte flipped)."""
    mism = flag_err = stripes_n = 0
    for g in sample:
        k, m, cpu = g["k"], g["m"], g["stripes"]
        n = cpu.shape[0]
        codec = rsgpu.ReedSolomon(k, m)
        buf = torch.from_numpy(cpu).cuda()
        buf[:, k:] = 0xA5
        ptrs = rsgpu.device_pointer_table(buf.data_ptr(), np.arange(n * (k + m), dtype=np.uint64) * np.uint64(SHARD))
        codec.prepare_batch("encode", ptrs, SHARD).launch()
        torch.cuda.synchronize()
        mism += int((buf[:, k:].cpu().numpy() != cpu[:, k:]).sum())
        lost = torch.from_numpy(g["pats"] == 0).cuda()
        buf.masked_fill_(lost.unsqueeze(-1), 0xA5)
        codec.prepare_batch("reconstruct", ptrs, SHARD, present=g["pats"]).launch()
        torch.cuda.synchronize()
        got = buf.cpu().numpy()
        for s, (targ, outs) in enumerate(g["rebuilt"]):
            for j, t in enumerate(targ):
                mism += int((got[s, t] != outs[j]).sum())  # rebuilt shards against the CPU's rebuild
            keep = [i for i in range(k + m) if i not in set(targ)]
            mism += int((got[s, keep] != cpu[s, keep]).sum())  # nothing else may change
        ver = codec.prepare_batch("verify", ptrs, SHARD)
        ver.launch()
        flag_err += int((~ver.verify_result()).sum())
        bad = np.arange(0, n, 3)
        for s in bad:
            buf[s, k + s % m, (s * 7919) % SHARD] ^= 0x10
        ver.launch()
        ok = ver.verify_result()
        want = np.ones(n, bool)
        want[bad] = False
        flag_err += int((ok != want).sum())
        stripes_n += n
        del buf
    torch.cuda.synchronize()
    return {"against": "the CPU baseline's outputs (reference CPU path, oracle restatement) on its own sample",
            "stripes": stripes_n, "mismatched_bytes": mism, "verify_flag_errors": flag_err}


def stripe_digests(torch, buf, key):
    """64-bit keyed linear digest of every stripe of a (stripes, shards,
    length) device buffer: sum over its 8-byte words of word * key word, mod
    2^64, with odd random key words (so any single changed word changes the
    digest; unequal stripes collide with probability about 2^-64)."""
    n = buf.shape[0]
    out = torch.empty(n, dtype=torch.int64, device=buf.device)
    step = max(1, (2 << 30) // (buf[0].numel()))
    for a in range(0, n, step):
        b = min(n, a + step)
        out[a:b] = (buf[a:b].reshape(b - a, -1).view(torch.int64) * key).sum(dim=1)
    return out


def digest_key(torch, words, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    key = torch.randint(-2**62, 2**62, (words,), dtype=torch.int64, device="cuda", generator=g)
    return key | 1


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path (restated: no Rust toolchain
    on this image) on the host cores, on a bounded sample of the workload."""
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    vals, dvals = [], []
    # The faster GFNI width on this host (untimed), then the timed steps with it.
    kernel = max(cpu_widths(), key=lambda w: cpu_sample(threads, kernel=w)[0])
    for _ in range(args.warmup):
        cpu_sample(threads, kernel=kernel)
    for _ in range(args.steps):
        v, kern, n, dv, _ = cpu_sample(threads, kernel=kernel)
        vals.append(v)
        dvals.append(dv)
    value = float(np.median(vals))
    line = {
        "impl": "reference", "metric": METRIC,
        "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "data_gibs": round(float(np.median(dvals)), 3),
        "config": {"workload": "classic galois_8 10+4 and 16+4, 1 MiB shards, seeded erasures 1..m",
                   "stripes_per_geometry_per_step": n, "flush": "inputs larger than L2"},
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": f"{n} stripes per geometry per step, {kern} rows kernel (oracle restatement; "
                                   "the faster GFNI width on this host)", "cpu_model": cpu_model()},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------- profiling cases
def _case_encode_10x4_64k():
    """512 stripes x 10+4 x 64 KiB (470 MB per launch, above L2): three encode launches."""
    import torch

    import rsgpu

    k, m, size, n = 10, 4, 65536, 512
    codec = rsgpu.ReedSolomon(k, m)
    buf = torch.randint(0, 256, (n, k + m, size), dtype=torch.uint8, device="cuda")
    offs = np.arange(n * (k + m), dtype=np.uint64) * np.uint64(size)
    enc = codec.prepare_batch("encode", rsgpu.device_pointer_table(buf.data_ptr(), offs), size)
    for _ in range(3):
        enc.launch()
    torch.cuda.synchronize()
    print("case encode-10x4-64k done")
    return 0


def _case_leopard(field, k, m, size, n, op):
    import torch

    import rsgpu

    fam = "leopard_gf8" if field == 8 else "leopard_gf16"
    codec = rsgpu.ReedSolomon(k, m, rsgpu.CodecOptions(codec_family=fam))
    buf = torch.randint(0, 256, (n, k + m, size), dtype=torch.uint8, device="cuda")
    offs = np.arange(n * (k + m), dtype=np.uint64) * np.uint64(size)
    ptrs = rsgpu.device_pointer_table(buf.data_ptr(), offs)
    if op == "encode":
        b = codec.prepare_batch("encode", ptrs, size)
    else:
        rng = np.random.default_rng(SEED)
        pats = np.ones((n, k + m), np.uint8)
        for s in range(n):
            pats[s, rng.choice(k + m, size=m, replace=False)] = 0
        b = codec.prepare_batch("reconstruct", ptrs, size, present=pats)
    for _ in range(3):
        b.launch()
    torch.cuda.synchronize()
    print(f"case leopard gf{field} {k}+{m} {op} done")
    return 0


def _case_mix():
    """The first ~2 GB wave of the mixed workload (model-planned, no graph):
    three launches of the persistent mixed kernel."""
    import torch

    import rsgpu
    from rsgpu import tune_mix
    from rsgpu import workload as W

    specs = W.mixed_specs(2048, SEED + 4)
    g = W.waves(specs, 2 << 30)[0]
    off, size = W.layout(specs, g)
    arena = torch.randint(0, 256, (size + 4096,), dtype=torch.uint8, device="cuda")
    base = arena.data_ptr()
    codecs = tune_mix.make_codecs(W.MIX_GEOMETRIES)
    rsgpu.Tuner.clear()
    rsgpu.Tuner.load(tune_mix.DEFAULT_TABLE)
    rsgpu.Tuner.train_from_tuner(epochs=3000, lr=3e-3, seed=1)
    ops = [tune_mix.spec_op(specs[i], codecs, [base + off[i] + j * specs[i].shard_len for j in range(specs[i].total)])
           for i in g]
    b = rsgpu.MixedBatch(ops, planner="model", graph=False)
    for _ in range(3):
        b.launch()
    torch.cuda.synchronize()
    print(f"case mix done: {len(ops)} ops, {size / 2**30:.2f} GiB, "
          f"{b.info().algorithmic_bytes / 1e9:.2f} GB algorithmic per launch")
    return 0


PROFILE_CASES = {
    "mix-2g": _case_mix,
    "encode-10x4-64k": _case_encode_10x4_64k,
    "lgf16-decode-1024x512": lambda: _case_leopard(16, 1024, 512, 16384, 16, "decode"),
    "lgf16-encode-1024x512": lambda: _case_leopard(16, 1024, 512, 16384, 16, "encode"),
    "lgf8-encode-32x16": lambda: _case_leopard(8, 32, 16, 1 << 20, 16, "encode"),
    "lgf8-decode-32x16": lambda: _case_leopard(8, 32, 16, 1 << 20, 16, "decode"),
    "lgf8-encode-128x64": lambda: _case_leopard(8, 128, 64, 1 << 19, 16, "encode"),
    "lgf8-decode-128x64": lambda: _case_leopard(8, 128, 64, 1 << 19, 16, "decode"),
}


# --------------------------------------------------------------------- GPU side
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--stripes", type=int, default=STRIPES)
    ap.add_argument("--e2e-stripes", type=int, default=256)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mix", action="store_true", help="skip the mixed-geometry workload")
    ap.add_argument("--mix-ops", type=int, default=MIX_OPS)
    ap.add_argument("--retune", action="store_true", help="re-run the autotuner instead of loading its table")
    ap.add_argument("--no-serve", action="store_true", help="skip the request-server workload")
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-loads", type=float, nargs="+", default=[50.0, 200.0, 800.0],
                    help="offered loads (GB/s of algorithmic bytes) of the Poisson request stream")
    ap.add_argument("--case", default=None, choices=sorted(PROFILE_CASES),
                    help="run one small profiling case (three launches of one kernel) and exit")
    args = ap.parse_args()
    if args.case:
        return PROFILE_CASES[args.case]()

    if args.impl == "reference":  # the reference arm loads nothing of this package
        return run_reference(args, int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")))

    import torch

    import rsgpu
    from rsgpu import ranks as R

    rk = R.from_env()
    rank, world = rk.rank, rk.world

    torch.cuda.set_device(rk.local)
    group = R.Group(rk, "nccl", timeout_s=120.0, device="cuda")
    cpus_all, cpus_local = pin_to_gpu_numa(torch, rk.local)

    def barrier():
        group.barrier()
        torch.cuda.synchronize()

    stream = torch.cuda.current_stream()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(SEED + rank)
    work = []  # per geometry: dict
    for gi, (k, m) in enumerate(GEOMS):
        n = args.stripes
        buf = torch.empty((n, k + m, SHARD), dtype=torch.uint8, device="cuda")
        buf[:, :k].random_(0, 256, generator=gen)
        codec = rsgpu.ReedSolomon(k, m)
        offs = np.arange(n * (k + m), dtype=np.uint64) * np.uint64(SHARD)
        ptrs = rsgpu.device_pointer_table(buf.data_ptr(), offs)
        pats = erasure_patterns(k, m, n, SEED + 100 + gi + 1000 * rank)
        enc = codec.prepare_batch("encode", ptrs, SHARD)
        enc.launch()
        torch.cuda.synchronize()
        # Every stripe's digest after encode; erase, then prepare (plans +
        # device decode tables) and rebuild once: the digests must come back.
        key = digest_key(torch, (k + m) * SHARD // 8, SEED + 300 + gi)
        digest = stripe_digests(torch, buf, key)
        lost = torch.from_numpy(pats == 0).cuda()
        buf.masked_fill_(lost.unsqueeze(-1), 0)
        rec = codec.prepare_batch("reconstruct", ptrs, SHARD, present=pats)
        ver = codec.prepare_batch("verify", ptrs, SHARD)
        rec.launch()
        ver.launch()
        torch.cuda.synchronize()
        bad_rebuild = int((stripe_digests(torch, buf, key) != digest).sum())
        bad_verify = int((~ver.verify_result()).sum())
        eb, rb, vb = step_bytes(k, m, pats, SHARD)
        work.append(dict(k=k, m=m, n=n, buf=buf, codec=codec, enc=enc, rec=rec, ver=ver, pats=pats, ptrs=ptrs,
                         bytes=(eb, rb, vb), key=key, digest=digest, bad=bad_rebuild + bad_verify))
    total_bytes = sum(sum(w["bytes"]) for w in work)

    def step():
        for w in work:
            w["enc"].launch()
            w["rec"].launch()
            w["ver"].launch()

    for _ in range(args.warmup):
        step()
    barrier()
    launches0 = rsgpu.kernel_launch_count()
    kern_per_step = sum(w[x].kernel_count() for w in work for x in ("enc", "rec", "ver"))
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(rk.local) as clk:
        barrier()
        st.record(stream)
        for _ in range(args.steps):
            step()
        en.record(stream)
        barrier()
    ms = st.elapsed_time(en) / args.steps
    # After the timed steps (each re-encodes, rebuilds and verifies every
    # stripe) every stripe must still hold the codeword it held after encode.
    stripes_checked = stripes_bad = 0
    for w in work:
        stripes_checked += w["n"]
        stripes_bad += w["bad"] + int((~w["ver"].verify_result()).sum())
        stripes_bad += int((stripe_digests(torch, w["buf"], w["key"]) != w["digest"]).sum())
    gpu_launches = kern_per_step * args.steps
    assert rsgpu.kernel_launch_count() - launches0 == gpu_launches
    ms_max = group.max(ms)
    value = total_bytes * world / (ms_max / 1e3) / 1e9
    # The reference's own convention (data shards x shard bytes per operation,
    # GiB/s; benches/throughput_matrix.rs:167-172): three operations per stripe.
    data_bytes = sum(3 * w["n"] * w["k"] * SHARD for w in work)
    data_gibs = data_bytes * world / (ms_max / 1e3) / 2**30

    # Dominant kernel (10+4 encode) timed alone with events on its stream.
    w0 = work[0]
    enc_ms = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        w0["enc"].launch()
        e1.record(stream)
        torch.cuda.synchronize()
        enc_ms.append(e0.elapsed_time(e1))
    enc_t = float(np.mean(enc_ms)) / 1e3
    enc_bytes = w0["bytes"][0]
    peak, peak_kind = measured_hbm_peak()
    achieved = enc_bytes / enc_t / 1e9
    ratio = profiled_traffic_ratio()

    # Per-stripe kernel comparison (the reference's one-stripe-per-call shape)
    # on the first 512 stripes of each geometry: one launch per stripe and op.
    per = []
    n_ps = min(512, args.stripes)
    for w in work:
        k, m = w["k"], w["m"]
        sb = []
        for s in range(n_ps):
            p = w["ptrs"][s * (k + m):(s + 1) * (k + m)]
            sb.append((w["codec"].prepare_batch("encode", p, SHARD),
                       w["codec"].prepare_batch("reconstruct", p, SHARD, present=w["pats"][s:s + 1]),
                       w["codec"].prepare_batch("verify", p, SHARD)))
        per.append(sb)
    ps_bytes = 0
    for w in work:
        eb, rb, vb = step_bytes(w["k"], w["m"], w["pats"][:n_ps], SHARD)
        ps_bytes += eb + rb + vb

    def per_stripe_step():
        for sb in per:
            for e, r, v in sb:
                e.launch()
                r.launch()
                v.launch()

    per_stripe_step()
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    per_stripe_step()
    p1.record(stream)
    torch.cuda.synchronize()
    ps_value = ps_bytes / (p0.elapsed_time(p1) / 1e3) / 1e9
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sub_batches = []
    for w in work:
        k, m = w["k"], w["m"]
        p = w["ptrs"][: n_ps * (k + m)]
        sub_batches.append((w["codec"].prepare_batch("encode", p, SHARD),
                            w["codec"].prepare_batch("reconstruct", p, SHARD, present=w["pats"][:n_ps]),
                            w["codec"].prepare_batch("verify", p, SHARD)))
    for e, r, v in sub_batches:
        e.launch(), r.launch(), v.launch()
    torch.cuda.synchronize()
    b0.record(stream)
    for e, r, v in sub_batches:
        e.launch(), r.launch(), v.launch()
    b1.record(stream)
    torch.cuda.synchronize()
    batched_same = ps_bytes / (b0.elapsed_time(b1) / 1e3) / 1e9
    del per, sub_batches

    # End to end through the public API with pinned host buffers.
    e2e = e2e_measure(torch, rsgpu, args, group)
    e2e["host_cpus_local_to_gpu"] = cpus_local

    for item in work:
        item.clear()  # drops the config-2 shard buffers (137 GiB)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    # Config 1 (the reference's CPU-runnable case) and config 3 (Leopard
    # GF(2^16) 1024+512): per-operation times, bytes checked.
    config1 = config1_workload(torch, rsgpu, stream, gen)
    leopard16 = leopard16_workload(torch, rsgpu, stream, gen)
    torch.cuda.empty_cache()

    # Mixed geometries in one persistent kernel (batched, model-scheduled)
    # against the per-stripe kernel loop.
    mixed = None
    if not args.no_mix:
        mixed = mixed_workload(args, torch, rsgpu, rank, stream, gen)
    serving = None
    if not args.no_serve:
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        serving = serving_workload(args, torch, rsgpu, rank, gen)

    if cpus_all is not None:
        os.sched_setaffinity(0, cpus_all)  # the CPU baseline gets every host core
    cpu = None
    sample = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        v, kern, n, dv, cpu_stripes = cpu_best(threads, keep=True)
        cpu = {"value": round(v, 3), "unit": "GB/s", "data_gibs": round(dv, 3), "cores": threads, "kind": "port",
               "sample": f"{n} stripes per geometry: encode+rebuild+verify with the oracle's {kern} rows kernel "
                         "(the faster GFNI width on this host; recovery rows derived per distinct pattern before "
                         "timing)", "cpu_model": cpu_model()}
        sample = sample_check(torch, rsgpu, cpu_stripes)
        del cpu_stripes
    check = {"digest": "64-bit keyed linear digest per stripe",
             "stripes": stripes_checked, "mismatched_stripes": stripes_bad, "sample": sample}
    mismatches = stripes_bad + (0 if sample is None else sample["mismatched_bytes"] + sample["verify_flag_errors"])
    for part in (config1, leopard16):
        mismatches += part["mismatched_bytes"]
    if mixed is not None:
        mismatches += mixed["check"]["mismatched_bytes"] + mixed["check"]["verify_flag_errors"]
    if serving is not None:
        mismatches += serving["mismatched_stripes"]

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": round(value, 1), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max, 3), "higher_is_better": True,
            "data_gibs": round(data_gibs, 1),
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": "classic galois_8 10+4 and 16+4, 1 MiB shards, seeded erasures 1..m",
                       "stripes_per_geometry": args.stripes, "ops_per_step": "encode, reconstruct, verify",
                       "bytes_per_step_per_gpu": total_bytes, "flush": "inputs (137 GiB/GPU) larger than L2",
                       "parallelism": f"stripes x{world} (weak, no collective)"},
            "roofline": {"bound": "hbm", "kernel": "k_apply_tma (10+4 encode, 4096 x 1 MiB)",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "frac_of_nominal_8tbs": round(achieved / 8000.0, 4),
                         "traffic": None if ratio is None else int(enc_bytes * ratio),
                         "algorithmic_bytes": enc_bytes},
            "per_stripe": {"value": round(ps_value, 1), "unit": "GB/s", "stripes_per_geometry": n_ps,
                           "batched_same_stripes": round(batched_same, 1),
                           "batched_speedup": round(batched_same / ps_value, 3)},
            "clocks": clk.summary(),
            "check": check,
            "mismatches_total": mismatches,
            "config1": config1,
            "leopard_gf16": leopard16,
            "mixed": mixed,
            "serving": serving,
            "e2e": e2e,
            "gpu_launches": gpu_launches,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    group.close()
    if rank == 0 and mismatches:
        print(f"bench: {mismatches} mismatches against the expected bytes", file=sys.stderr)
        return 1
    return 0


def _median_ms(torch, stream, fn, reps):
    """Median CUDA-event time of fn() on `stream` over reps launches."""
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts)), float(np.percentile(ts, 99))


def config1_workload(torch, rsgpu, stream, gen):
    """Classic 10+4, 64 KiB shards, 256 stripes: encode, erase {0,3,11,13},
    reconstruct, verify; every byte checked against the original stripes.
    Times are per operation over all 256 stripes (inputs 235 MB > L2)."""
    k, m, size, n = 10, 4, 65536, 256
    codec = rsgpu.ReedSolomon(k, m)
    buf = torch.empty((n, k + m, size), dtype=torch.uint8, device="cuda")
    buf[:, :k].random_(0, 256, generator=gen)
    offs = np.arange(n * (k + m), dtype=np.uint64) * np.uint64(size)
    ptrs = rsgpu.device_pointer_table(buf.data_ptr(), offs)
    enc = codec.prepare_batch("encode", ptrs, size)
    enc.launch()
    torch.cuda.synchronize()
    orig = buf.clone()
    pats = np.ones((n, k + m), np.uint8)
    pats[:, [0, 3, 11, 13]] = 0
    buf[:, [0, 3, 11, 13]] = 0
    rec = codec.prepare_batch("reconstruct", ptrs, size, present=pats)
    ver = codec.prepare_batch("verify", ptrs, size)
    rec.launch()
    ver.launch()
    torch.cuda.synchronize()
    mism = int((buf != orig).sum()) + int((~ver.verify_result()).sum())
    out = {"workload": "classic 10+4, 64 KiB shards, 256 stripes, erase {0,3,11,13}", "bit_exact": mism == 0,
           "mismatched_bytes": mism}
    nbytes = n * (k + m) * size  # encode, reconstruct ((k + 4) S) and verify move the same bytes
    for name, b in (("encode", enc), ("reconstruct", rec), ("verify", ver)):
        med, p99 = _median_ms(torch, stream, b.launch, 20)
        out[name] = {"us": round(med * 1e3, 1), "p99_us": round(p99 * 1e3, 1),
                     "gbs": round(nbytes / (med / 1e3) / 1e9, 1),
                     "data_gibs": round(n * k * size / (med / 1e3) / 2**30, 1)}
    # One step (encode, rebuild, verify) as one CUDA graph of the three
    # prepared launches, so no host launch latency sits between them (the
    # per-operation times above include it: each launch starts on an idle
    # stream).
    try:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            enc.launch()
            rec.launch()
            ver.launch()
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        med, p99 = _median_ms(torch, stream, g.replay, 20)
        out["step_graph"] = {"ops": "encode + reconstruct + verify, one CUDA graph",
                             "us": round(med * 1e3, 1), "p99_us": round(p99 * 1e3, 1),
                             "gbs": round(3 * nbytes / (med / 1e3) / 1e9, 1),
                             "data_gibs": round(3 * n * k * size / (med / 1e3) / 2**30, 1)}
        del g
    except Exception as e:  # reported, not fatal: the per-operation figures stand
        out["step_graph"] = {"error": str(e)[:200]}
    # The timed launches rewrote parity and the erased shards: still the same bytes.
    out["mismatched_bytes"] += int((buf != orig).sum()) + int((~ver.verify_result()).sum())
    out["bit_exact"] = out["mismatched_bytes"] == 0
    del buf, orig
    return out


def leopard16_workload(torch, rsgpu, stream, gen):
    """Leopard GF(2^16) k=1024, m=512, 16 KiB shards, 64 stripes (1.6 GB):
    encode, erase 512 seeded shards per stripe, reconstruct; the rebuilt
    stripes must equal the originals byte for byte.  Multiply-XOR counts per
    element column: encode 2 * 256 * 9 (two IFFT chunks of 512) + 256 * 9
    (the FFT), decode 2 * 1024 * 11 (IFFT and FFT of n = 2048)."""
    k, m, size, n = 1024, 512, 16384, 64
    codec = rsgpu.ReedSolomon(k, m, rsgpu.CodecOptions(codec_family="leopard_gf16"))
    buf = torch.empty((n, k + m, size), dtype=torch.uint8, device="cuda")
    buf[:, :k].random_(0, 256, generator=gen)
    offs = np.arange(n * (k + m), dtype=np.uint64) * np.uint64(size)
    ptrs = rsgpu.device_pointer_table(buf.data_ptr(), offs)
    enc = codec.prepare_batch("encode", ptrs, size)
    enc.launch()
    torch.cuda.synchronize()
    orig = buf.clone()
    rng = np.random.default_rng(SEED + 3)
    pats = np.ones((n, k + m), np.uint8)
    for s in range(n):
        pats[s, rng.choice(k + m, size=m, replace=False)] = 0
    lost = torch.from_numpy(pats == 0).cuda()
    buf.masked_fill_(lost.unsqueeze(-1), 0)
    rec = codec.prepare_batch("reconstruct", ptrs, size, present=pats)
    rec.launch()
    torch.cuda.synchronize()
    mism = int((buf != orig).sum())
    cols = size // 2
    mx = {"encode": (2 * 256 * 9 + 256 * 9) * cols * n, "reconstruct": 2 * 1024 * 11 * cols * n}
    # Shuffle bound of a GF(2^16) multiply-XOR: 6 table shuffles per 32-bit
    # word (two elements; 5+5+5 bits by shuffle, bit 15 by a mask), one
    # warp-wide shuffle per SM clock.
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    bound = props.multi_processor_count * 1.965e9 * 32 / 6 * 2
    nbytes = n * (k + m) * size  # encode reads k, writes m; reconstruct reads k + m - e, writes e
    out = {"workload": "Leopard GF16 1024+512, 16 KiB shards, 64 stripes, 512 seeded erasures each",
           "bit_exact": mism == 0, "mismatched_bytes": mism}
    for name, b in (("encode", enc), ("reconstruct", rec)):
        med, p99 = _median_ms(torch, stream, b.launch, 10)
        out[name] = {"ms": round(med, 3), "p99_ms": round(p99, 3),
                     "gbs": round(nbytes / (med / 1e3) / 1e9, 1),
                     "data_gibs": round(n * k * size / (med / 1e3) / 2**30, 1),
                     "mul_xor_per_s": float(f"{mx[name] / (med / 1e3):.4g}"),
                     "frac_of_shuffle_bound": round(mx[name] / (med / 1e3) / bound, 3)}
    out["shuffle_bound_mul_xor_per_s"] = float(f"{bound:.4g}")
    out["mismatched_bytes"] += int((buf != orig).sum())
    out["bit_exact"] = out["mismatched_bytes"] == 0
    del buf, orig
    return out


def mixed_workload(args, torch, rsgpu, rank, stream, gen):
    """16384 stripes: geometries uniform over classic GF(2^8) {4+2, 6+3, 8+4,
    12+4, 16+4} and Leopard GF(2^8) {32+16, 128+64}; shard sizes log-uniform
    4 KiB..4 MiB (64-byte multiples); erasures uniform 0..m; encode /
    reconstruct / verify with probabilities 0.5 / 0.4 / 0.1 (rsgpu.workload).
    The stripes do not fit HBM at once (~0.4 TB), so they run in waves that
    share one arena (a wave's inputs are whatever the previous wave left
    there); every mode runs the same waves in the same order.

    Modes, all on device-resident shards, timed with CUDA events:
      batched_model: one persistent-kernel mixed batch per wave (CUDA graph),
                     plans from the measured table + cost model;
      batched_fixed: the same with the fixed plan rule;
      per_stripe:    one prepared launch per stripe and operation (the codec's
                     own kernels, the plain per-stripe loop);
      per_stripe_api: one rsgpu_encode / _reconstruct / _verify call per stripe.
    """
    import ctypes

    from rsgpu import tune_mix
    from rsgpu import workload as W

    specs = W.mixed_specs(args.mix_ops, SEED + 4 + 1000 * rank)
    free, _ = torch.cuda.mem_get_info()
    arena_bytes = int(min(free * 0.5, 80e9))
    groups = W.waves(specs, arena_bytes)
    size = max(W.layout(specs, g)[1] for g in groups)
    arena = torch.empty(size + 4096, dtype=torch.uint8, device="cuda")
    arena.random_(0, 256, generator=gen)
    base = arena.data_ptr()
    codecs = tune_mix.make_codecs(W.MIX_GEOMETRIES)
    T = rsgpu.Tuner
    T.clear()
    t0 = time.perf_counter()
    if os.path.exists(tune_mix.DEFAULT_TABLE) and not args.retune:
        T.load(tune_mix.DEFAULT_TABLE)
        table_src = "loaded " + os.path.relpath(tune_mix.DEFAULT_TABLE, ROOT)
    else:
        sample = tune_mix.class_sample(W.mixed_specs(20000, 0x5EED), codecs, 160)
        T.tune(sample, target_bytes=96 << 20, repeats=2)
        table_src = "tuned in-process"
    tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    loss = T.train_from_tuner(epochs=3000, lr=3e-3, seed=1)
    train_s = time.perf_counter() - t0

    waves, abytes = [], 0
    t0 = time.perf_counter()
    for g in groups:
        off, _ = W.layout(specs, g)
        ops = []
        for i in g:
            s = specs[i]
            ops.append(tune_mix.spec_op(s, codecs, [base + off[i] + j * s.shard_len for j in range(s.total)]))
        bm = rsgpu.MixedBatch(ops, planner="model", graph=True)
        bf = rsgpu.MixedBatch(ops, planner="fixed", graph=True)
        abytes += bm.info().algorithmic_bytes
        per = []
        for o in ops:
            if o["op"] == "reconstruct" and np.asarray(o["present"]).all():
                continue
            ptrs = np.array(o["shards"], np.uint64)
            pres = None if o["op"] != "reconstruct" else np.asarray(o["present"], np.uint8)[None, :]
            per.append(o["codec"].prepare_batch(o["op"], ptrs, o["shard_len"], present=pres))
        waves.append(dict(ops=ops, model=bm, fixed=bf, per=per))
    prep_s = time.perf_counter() - t0
    plans = {}
    for w in waves:
        for p in w["model"].plans():
            plans[p] = plans.get(p, 0) + 1

    def run(mode):
        lat = []
        for w in waves:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if mode == "per":
                for pb in w["per"]:
                    pb.launch()
            else:
                w[mode].launch()
            e1.record(stream)
            lat.append((e0, e1))
        return lat

    out = {"workload": f"{args.mix_ops} stripes, 7 geometries (classic GF8 4+2/6+3/8+4/12+4/16+4, Leopard GF8 "
                       "32+16/128+64), shards 4 KiB-4 MiB log-uniform, erasures 0..m, enc/rec/ver 0.5/0.4/0.1",
           "waves": len(waves), "algorithmic_bytes": int(abytes), "unit": "GB/s",
           "planner": {"table": table_src, "classes": T.table_size(), "samples": len(T.samples()),
                       "model_loss": round(loss, 4), "tune_s": round(tune_s, 1), "train_s": round(train_s, 2),
                       "prepare_s": round(prep_s, 1),
                       "plans": {f"{'apply' if a == 0 else 'fft'}{t}": c for (a, t), c in sorted(plans.items())}}}
    steps = max(1, min(args.steps, 5))
    for mode, key in [("model", "batched_model"), ("fixed", "batched_fixed"), ("per", "per_stripe")]:
        run(mode)
        torch.cuda.synchronize()
        times, wave_ms = [], []
        for _ in range(steps):
            lat = run(mode)
            torch.cuda.synchronize()
            times.append(lat[0][0].elapsed_time(lat[-1][1]))
            wave_ms += [a.elapsed_time(b) for a, b in lat]
        ms = float(np.median(times))
        out[key] = {"value": round(abytes / (ms / 1e3) / 1e9, 1), "ms_per_pass": round(ms, 2),
                    "wave_ms_p50": round(float(np.percentile(wave_ms, 50)), 2),
                    "wave_ms_p99": round(float(np.percentile(wave_ms, 99)), 2)}
    # One pass of the per-stripe public API (host-side call per stripe).
    L = rsgpu.lib()
    st = stream.cuda_stream
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for w in waves:
        for o in w["ops"]:
            n = len(o["shards"])
            ptrs = (ctypes.c_void_p * n)(*o["shards"])
            lens = (ctypes.c_size_t * n)(*([o["shard_len"]] * n))
            c = o["codec"]._h
            if o["op"] == "encode":
                rc = L.rsgpu_encode(c, ptrs, lens, n, 1, st)
            elif o["op"] == "verify":
                ok = ctypes.c_int32()
                rc = L.rsgpu_verify(c, ptrs, lens, n, ctypes.byref(ok), 1, st)
            else:
                pres = (ctypes.c_uint8 * n)(*np.asarray(o["present"]).tolist())
                rc = L.rsgpu_reconstruct(c, ptrs, lens, pres, n, 0, None, 0, 1, st)
            assert rc == 0, rc
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    out["per_stripe_api"] = {"value": round(abytes / dt / 1e9, 1), "s_per_pass": round(dt, 2)}
    out["speedup_vs_per_stripe"] = round(out["batched_model"]["value"] / out["per_stripe"]["value"], 3)
    out["speedup_vs_per_stripe_api"] = round(out["batched_model"]["value"] / out["per_stripe_api"]["value"], 3)
    out["fixed_vs_per_stripe_api"] = round(out["batched_fixed"]["value"] / out["per_stripe_api"]["value"], 3)
    del waves
    out["check"] = mixed_mode_check(torch, rsgpu, specs, groups[0], arena, codecs)
    del arena
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out


def count_diff(a, b, chunk=1 << 30):
    """Number of differing bytes of two equally long uint8 device tensors."""
    a, b = a.reshape(-1), b.reshape(-1)
    return sum(int((a[i:i + chunk] != b[i:i + chunk]).sum()) for i in range(0, a.numel(), chunk))


def mixed_mode_check(torch, rsgpu, specs, group, arena, codecs, limit=8 << 30):
    """Every mode must write the same bytes: the first operations of the first
    wave (up to `limit` bytes of stripes) run from one saved arena state as a
    model-planned and a fixed-plan mixed batch and as the per-stripe launch
    loop; the arena after each is compared byte for byte with the model
    batch's, and the verify results with its flags."""
    from rsgpu import tune_mix
    from rsgpu import workload as W

    idx, used = [], 0
    for i in group:
        need = (specs[i].stripe_bytes + 255) // 256 * 256
        if idx and used + need > limit:
            break
        idx.append(i)
        used += need
    off, size = W.layout(specs, idx)
    base = arena.data_ptr()
    ops = [tune_mix.spec_op(specs[i], codecs, [base + off[i] + j * specs[i].shard_len for j in range(specs[i].total)])
           for i in idx]
    region = arena[:size]
    saved = region.clone()

    model = rsgpu.MixedBatch(ops, planner="model", graph=True)
    model.launch()
    want_flags = model.results().astype(bool)
    want = region.clone()
    mism, flag_err = 0, 0
    fixed = rsgpu.MixedBatch(ops, planner="fixed", graph=True)
    region.copy_(saved)
    fixed.launch()
    torch.cuda.synchronize()
    mism += count_diff(region, want)
    flag_err += int((fixed.results().astype(bool) != want_flags).sum())
    region.copy_(saved)
    per, kinds = [], []
    for o in ops:
        if o["op"] == "reconstruct" and np.asarray(o["present"]).all():
            per.append(None)
            kinds.append("none")
            continue
        pres = None if o["op"] != "reconstruct" else np.asarray(o["present"], np.uint8)[None, :]
        per.append(o["codec"].prepare_batch(o["op"], np.array(o["shards"], np.uint64), o["shard_len"], present=pres))
        kinds.append(o["op"])
    for b in per:
        if b is not None:
            b.launch()
    torch.cuda.synchronize()
    mism += count_diff(region, want)
    per_flags = np.array([bool(b.verify_result()[0]) if k == "verify" else True for b, k in zip(per, kinds)])
    flag_err += int((per_flags != want_flags).sum())
    del saved, want, model, fixed, per
    torch.cuda.synchronize()
    return {"against": "model batch vs fixed-plan batch vs per-stripe launches, from one saved arena state",
            "ops": len(ops), "stripe_bytes": int(size), "mismatched_bytes": mism, "verify_flag_errors": flag_err}


def serving_workload(args, torch, rsgpu, rank, gen):
    """Requests of the mixed workload plus Leopard GF(2^16) 2048+1024 at
    8 KiB shards (one request in eight), arriving as a seeded Poisson stream
    at a sweep of offered loads, served by the request server (continuous
    batching, model planner with the measured table, admission by a device
    memory budget) on device-resident shards.  Reports per-request latency
    p50 / p99 (submit -> completion) and GB/s of algorithmic bytes; the arena
    checksum after every load level must be identical (no byte differs
    whatever the batching)."""
    from rsgpu import tune_mix
    from rsgpu import workload as W

    rng = np.random.default_rng(SEED + 5 + 1000 * rank)
    specs = W.mixed_specs(args.serve_requests, SEED + 6 + 1000 * rank)
    wide = ("leopard_gf16", 2048, 1024)
    for i, s in enumerate(specs):
        if rng.integers(8) == 0:
            op = W.OPS[int(rng.choice(3, p=np.asarray(W.OP_PROBS, float)))]
            present = None
            if op == "reconstruct":
                e = int(rng.integers(0, 1025))
                present = np.ones(3072, np.uint8)
                present[rng.choice(3072, size=e, replace=False)] = 0
            specs[i] = W.MixOpSpec(wide, op, 8192, present)
    codecs = tune_mix.make_codecs(W.MIX_GEOMETRIES + [wide])
    idx = list(range(len(specs)))
    off, size = W.layout(specs, idx)
    arena = torch.empty(size + 4096, dtype=torch.uint8, device="cuda")
    arena.random_(0, 256, generator=gen)
    base = arena.data_ptr()
    ptrs = [[base + off[i] + j * s.shard_len for j in range(s.total)] for i, s in enumerate(specs)]
    abytes = np.array([s.algorithmic_bytes() for s in specs], np.float64)
    mean_bytes = float(abytes.mean())
    out = {"workload": f"{len(specs)} requests: mixed workload + Leopard GF16 2048+1024 at 8 KiB (1 in 8), "
                       "Poisson arrivals, device-resident shards",
           "unit": "GB/s", "levels": []}
    # Each request alone first (one C-ABI call per request, device memory):
    # the stripes' digests and verify flags every load level must reproduce.
    # Requests own disjoint stripes and every operation is idempotent on its
    # stripe, so the arena holds the same bytes after every full pass.
    key = digest_key(torch, max(s.stripe_bytes for s in specs) // 8, SEED + 400 + rank)
    lone_flags = lone_pass(torch, rsgpu, specs, codecs, ptrs)

    def digests():
        torch.cuda.synchronize()
        return [int((arena[off[i]:off[i] + s.stripe_bytes].view(torch.int64) * key[:s.stripe_bytes // 8]).sum())
                for i, s in enumerate(specs)]

    lone = digests()
    mismatched = 0
    budget = 16 << 30
    # Untimed warm-up: the first 256 requests at once, so first-use costs
    # (kernel loading, Leopard plans, pool growth) stay out of the latencies.
    # Every request rewrites only its own stripe from the same inputs, so
    # running them again leaves the arena unchanged.
    srv = rsgpu.Server(device_budget=budget, streams=3, max_batch=64, planner="model")
    warm = min(256, len(specs))
    for i in range(warm):
        s = specs[i]
        srv.submit(codecs[s.geom], s.op, ptrs[i], s.shard_len, present=s.present, tag=i + 1)
    srv.wait(warm)
    srv.close()
    for load in args.serve_loads:
        lam = load * 1e9 / mean_bytes
        arrivals = np.cumsum(rng.exponential(1.0 / lam, size=len(specs)))
        srv = rsgpu.Server(device_budget=budget, streams=3, max_batch=64, planner="model")
        comps = []
        t0 = time.perf_counter()
        for i, s in enumerate(specs):
            while time.perf_counter() - t0 < arrivals[i]:
                pass
            srv.submit(codecs[s.geom], s.op, ptrs[i], s.shard_len, present=s.present, tag=i + 1)
            if i % 64 == 0:
                comps += srv.poll(timeout_ms=0)
        comps += srv.wait(len(specs) - len(comps))
        st = srv.stats()
        srv.close()
        assert all(c["status"] == 0 for c in comps)
        lat = np.array([c["done_s"] - c["submit_s"] for c in comps]) * 1e3
        span = max(c["done_s"] for c in comps) - min(c["submit_s"] for c in comps)
        level = digests()
        flags = {c["tag"] - 1: bool(c["ok"]) for c in comps}
        bad = sum(1 for i in range(len(specs)) if level[i] != lone[i] or flags[i] != lone_flags[i])
        mismatched += bad
        out["levels"].append({"offered_gbs": load, "achieved_gbs": round(float(abytes.sum()) / span / 1e9, 1),
                              "p50_ms": round(float(np.percentile(lat, 50)), 3),
                              "p99_ms": round(float(np.percentile(lat, 99)), 3),
                              "launches": int(st["launches"]),
                              "host_prepare_frac": round(st["prepare_seconds"] / span, 3),
                              "max_prepare_ms": round(st["max_prepare_seconds"] * 1e3, 2),
                              "max_worker_gap_ms": round(st["max_loop_gap_seconds"] * 1e3, 2),
                              "max_concurrent_launches": int(st["max_concurrent_launches"]),
                              "max_reserved_gib": round(st["max_reserved_bytes"] / 2**30, 2),
                              "mismatched_stripes": bad})
    out["budget_gib"] = budget / 2**30
    out["check"] = "every request's stripe digest (64-bit keyed) and verify flag equal to its lone run"
    out["mismatched_stripes"] = mismatched
    out["identical_across_loads"] = mismatched == 0
    del arena
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out


def lone_pass(torch, rsgpu, specs, codecs, ptrs):
    """Every request alone, in order, through the per-call C ABI on device
    memory; returns the verify flag of each request (True for the others)."""
    import ctypes

    L = rsgpu.lib()
    st = torch.cuda.current_stream().cuda_stream
    flags = []
    for i, s in enumerate(specs):
        n = s.total
        p = (ctypes.c_void_p * n)(*ptrs[i])
        lens = (ctypes.c_size_t * n)(*([s.shard_len] * n))
        c = codecs[s.geom]._h
        ok = ctypes.c_int32(1)
        if s.op == "encode":
            rc = L.rsgpu_encode(c, p, lens, n, 1, st)
        elif s.op == "verify":
            rc = L.rsgpu_verify(c, p, lens, n, ctypes.byref(ok), 1, st)
        else:
            pres = (ctypes.c_uint8 * n)(*np.asarray(s.present).tolist())
            rc = L.rsgpu_reconstruct(c, p, lens, pres, n, 0, None, 0, 1, st)
        assert rc == 0, rc
        flags.append(bool(ok.value))
    torch.cuda.synchronize()
    return flags


def e2e_measure(torch, rsgpu, args, group):
    """Same operations through ReedSolomon.*_batch with pinned host shards: each
    step copies inputs host->device and results (parity, rebuilt shards, verify
    flags) device->host inside the timed region.  Every rank runs the same
    per-GPU work; the figure is all ranks' bytes over the slowest rank's
    time."""
    n = args.e2e_stripes
    stripes = []
    h2d = d2h = 0
    total = 0
    for gi, (k, m) in enumerate(GEOMS):
        codec = rsgpu.ReedSolomon(k, m)
        host = torch.empty((n, k + m, SHARD), dtype=torch.uint8, pin_memory=True)
        block = np.random.default_rng(SEED + 7 + gi).integers(0, 256, 64 << 20, dtype=np.uint8)
        arr = host.numpy()
        flat = arr[:, :k].reshape(-1)
        for off in range(0, flat.size, block.size):
            flat[off:off + block.size] = block[: flat.size - off]
        lists = arr  # (stripes, k+m, S) host array
        pats = erasure_patterns(k, m, n, SEED + 200 + gi)
        eb, rb, vb = step_bytes(k, m, pats, SHARD)
        total += eb + rb + vb
        e = (k + m) - pats.sum(axis=1)
        # encode uploads the data shards, rebuild the first k present shards
        # (the survivors a classic decode reads), verify every shard.
        h2d += n * k * SHARD + n * k * SHARD + n * (k + m) * SHARD
        d2h += n * m * SHARD + int((e * SHARD).sum()) + n
        stripes.append((codec, lists, pats, host))

    def step():
        for codec, lists, pats, host in stripes:
            codec.encode_batch(lists)
            codec.reconstruct_batch(lists, pats)
            ok = codec.verify_batch(lists)
            assert all(ok)

    step()
    # Each step timed on its own; the median step is reported, since the host
    # link is shared with whatever else runs on the machine and single steps
    # can stall on it.
    steps = max(3, min(args.steps, 5))
    torch.cuda.synchronize()
    group.barrier()
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        step()
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    dt = group.max(float(np.median(times)))
    for codec, lists, pats, host in stripes:
        del host
    link = host_link_gbs(torch)
    # The link's own bound for this step: each direction alone, and both
    # together at the rate the link sustains with copies in flight both ways.
    bound = max(h2d / (link["h2d_gbs"] * 1e9), d2h / (link["d2h_gbs"] * 1e9),
                (h2d + d2h) / (link["both_gbs"] * 1e9))
    total *= group.ranks.world
    h2d *= group.ranks.world
    d2h *= group.ranks.world
    return {"value": round(total / dt / 1e9, 2), "unit": "GB/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "stripes_per_geometry": n, "api": "ReedSolomon.*_batch, host memory",
            "s_per_step": round(dt, 4), "s_per_step_all": [round(t, 4) for t in times], "link": link,
            "link_bound_s_per_step": round(bound, 4),
            "link_frac": round(bound / dt, 3)}


def host_link_gbs(torch, nbytes=2 << 30, reps=5):
    """Pinned host <-> device copy bandwidth of this GPU (a 2 GiB copy each
    way alone, and one each way at once; best of reps, CUDA events): the
    ceiling of the host-memory path."""
    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    out = {}
    for name, fn in (("h2d_gbs", lambda: d.copy_(h, non_blocking=True)),
                     ("d2h_gbs", lambda: h.copy_(d, non_blocking=True))):
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 1e3
            best = t if best is None else min(best, t)
        out[name] = round(nbytes / best / 1e9, 1)
    # Both directions at once on two streams (a second pair of buffers):
    # bytes moved both ways over the time until both copies finished.
    h2 = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d2 = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s_up, s_down = torch.cuda.Stream(), torch.cuda.Stream()
    best = None
    for _ in range(reps):
        cur = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(cur)
        s_up.wait_stream(cur)
        s_down.wait_stream(cur)
        with torch.cuda.stream(s_up):
            d.copy_(h, non_blocking=True)
        with torch.cuda.stream(s_down):
            h2.copy_(d2, non_blocking=True)
        cur.wait_stream(s_up)
        cur.wait_stream(s_down)
        e1.record(cur)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        best = t if best is None else min(best, t)
    out["both_gbs"] = round(2 * nbytes / best / 1e9, 1)
    del h, d, h2, d2
    return out


if __name__ == "__main__":
    sys.exit(main())
