"""Autotune the mixed-batch planner for the mixed storage workload and save
the measured plan table.

    python -m rsgpu.tune_mix [--out PATH] [--classes N] [--target-mib M]

Draws a seeded sample of the mixed workload (rsgpu.workload), keeps one
operation per planner class (family, k, m, operation, goal, erasure bucket,
length bucket), measures every valid plan of each class on the GPU
(rsgpu_tune) and writes the table and the raw samples to PATH (default:
tuning/plans_b200.txt next to this package).  The cost model is trained from
those samples at load time (Tuner.train_from_tuner), so classes the sweep did
not cover get a predicted plan instead of a sweep.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TABLE = os.path.join(os.path.dirname(HERE), "tuning", "plans_b200.txt")


def class_sample(specs, codecs, limit, seed=1):
    """One op per planner class among specs (at most `limit`, spread over the
    classes in a seeded order)."""
    import rsgpu

    seen = {}
    for s in specs:
        op = spec_op(s, codecs)
        key = tuple(np.round(rsgpu.Tuner.features(op), 4)) + (op.get("goal", "all"),)
        seen.setdefault(key, op)
    keys = list(seen)
    rng = np.random.default_rng(seed)
    rng.shuffle(keys)
    return [seen[k] for k in keys[:limit]]


def spec_op(s, codecs, shards=None):
    fam, k, m = s.geom
    return dict(codec=codecs[s.geom], op=s.op, shards=shards if shards is not None else [1] * (k + m),
                shard_len=s.shard_len, present=s.present, goal=s.goal)


def make_codecs(geoms):
    import rsgpu

    return {g: rsgpu.ReedSolomon(g[1], g[2], rsgpu.CodecOptions(codec_family=g[0])) for g in geoms}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--classes", type=int, default=400)
    ap.add_argument("--target-mib", type=int, default=128)
    ap.add_argument("--seed", type=int, default=0x5EED)
    args = ap.parse_args(argv)
    import torch

    import rsgpu
    from rsgpu import workload as W

    torch.cuda.init()
    codecs = make_codecs(W.MIX_GEOMETRIES)
    specs = W.mixed_specs(20000, args.seed)
    ops = class_sample(specs, codecs, args.classes)
    rsgpu.Tuner.clear()
    n = rsgpu.Tuner.tune(ops, target_bytes=args.target_mib << 20, repeats=3)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    rsgpu.Tuner.save(args.out)
    print(f"tuned {n} classes, {len(rsgpu.Tuner.samples())} samples -> {args.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
