"""Seeded mixed-geometry workloads for mixed batches, the autotuner and the
serving loop.

The mix follows the storage-node traffic the batched path is built for:
geometries drawn uniformly from classic GF(2^8) {4+2, 6+3, 8+4, 12+4, 16+4}
and Leopard GF(2^8) {32+16, 128+64}; shard sizes log-uniform between a lower
and an upper bound, rounded to 64 bytes; an erasure count uniform in 0..m at
uniformly random positions; and operations encode / reconstruct / verify with
probabilities 0.5 / 0.4 / 0.1.  Everything is drawn from one numpy
``default_rng(seed)`` stream, so a seed names a workload.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

CLASSIC_GEOMETRIES = [("classic", 4, 2), ("classic", 6, 3), ("classic", 8, 4), ("classic", 12, 4),
                      ("classic", 16, 4)]
LEOPARD8_GEOMETRIES = [("leopard_gf8", 32, 16), ("leopard_gf8", 128, 64)]
MIX_GEOMETRIES = CLASSIC_GEOMETRIES + LEOPARD8_GEOMETRIES
OPS = ("encode", "reconstruct", "verify")
OP_PROBS = (0.5, 0.4, 0.1)


@dataclass
class MixOpSpec:
    """One operation of a mixed workload (no buffers yet)."""
    geom: Tuple[str, int, int]
    op: str
    shard_len: int
    present: Optional[np.ndarray] = None  # reconstruct: k + m flags
    goal: str = "all"

    @property
    def total(self) -> int:
        return self.geom[1] + self.geom[2]

    @property
    def stripe_bytes(self) -> int:
        return self.total * self.shard_len

    def algorithmic_bytes(self) -> int:
        """Bytes one run of this op reads plus writes (the roofline numerator):
        encode / verify (k+m)*S; classic reconstruct (k+e)*S; Leopard
        reconstruct (present+e)*S."""
        fam, k, m = self.geom
        if self.op != "reconstruct":
            return self.total * self.shard_len
        e = int(self.total - int(self.present.sum()))
        if e == 0:
            return 0
        if fam == "classic":
            return (k + e) * self.shard_len
        return (self.total - e + e) * self.shard_len


def log_uniform_len(rng, lo: int, hi: int, align: int = 64) -> int:
    v = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
    return max(align, int(round(v / align)) * align)


def mixed_specs(n: int, seed: int, lo: int = 4096, hi: int = 4 << 20,
                geometries: Sequence[Tuple[str, int, int]] = MIX_GEOMETRIES,
                probs: Sequence[float] = OP_PROBS) -> List[MixOpSpec]:
    """n operations of the mixed workload, drawn from ``default_rng(seed)``."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        geom = geometries[int(rng.integers(len(geometries)))]
        op = OPS[int(rng.choice(len(OPS), p=np.asarray(probs, float)))]
        length = log_uniform_len(rng, lo, hi)
        fam, k, m = geom
        present = None
        if op == "reconstruct":
            e = int(rng.integers(0, m + 1))
            lost = rng.choice(k + m, size=e, replace=False) if e else np.zeros(0, np.int64)
            present = np.ones(k + m, np.uint8)
            present[lost] = 0
        out.append(MixOpSpec(geom, op, length, present))
    return out


def waves(specs: Sequence[MixOpSpec], arena_bytes: int) -> List[List[int]]:
    """Split ops (in order) into consecutive groups whose stripes fit an arena
    of arena_bytes (each stripe 256-byte aligned)."""
    groups, cur, used = [], [], 0
    for i, s in enumerate(specs):
        need = (s.stripe_bytes + 255) // 256 * 256
        if cur and used + need > arena_bytes:
            groups.append(cur)
            cur, used = [], 0
        cur.append(i)
        used += need
    if cur:
        groups.append(cur)
    return groups


def layout(specs: Sequence[MixOpSpec], idx: Sequence[int]) -> Tuple[Dict[int, int], int]:
    """Byte offset of each op's stripe (shard-major, k + m shards of shard_len
    bytes back to back) inside an arena, and the arena size."""
    off, cur = {}, 0
    for i in idx:
        off[i] = cur
        cur += (specs[i].stripe_bytes + 255) // 256 * 256
    return off, cur
