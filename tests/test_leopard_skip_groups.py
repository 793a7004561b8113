"""Host-side checks of what the Leopard register stages rely on to skip the
per-butterfly test (csrc/leo_fft.cuh, group_may_skip):

- in both fields' skew tables the entries whose log is the modulus (the
  reference skips those multiplies, src/core/leopard_gf16/ops.rs:375-465) are
  exactly the entries 2^i - 1 (the oracle's tables restate the reference's
  construction, src/core/leopard_gf16/tables.rs and leopard_gf8/tables.rs);
- the predicate, restated here, is true for every group of lanes whose
  butterfly constants (entries skb + R + dm * t, 0 < t < G) include such an
  entry, over the skew bases and group shapes the transforms use.
"""
import ctypes

import numpy as np

import oracle as O


def skew_tables():
    L = O.lib()
    p16 = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))
    p8 = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    log = np.zeros(65536, np.uint16)
    exp = np.zeros(131072, np.uint16)
    sk16 = np.zeros(65535, np.uint16)
    walsh = np.zeros(65536, np.uint16)
    L.orc_lgf16_tables(p16(log), p16(exp), p16(sk16), p16(walsh))
    log8 = np.zeros(256, np.uint8)
    exp8 = np.zeros(512, np.uint8)
    sk8 = np.zeros(255, np.uint8)
    walsh8 = np.zeros(256, np.uint8)
    L.orc_lgf8_tables(p8(log8), p8(exp8), p8(sk8), p8(walsh8))
    return {16: (sk16, 65535), 8: (sk8, 255)}


def group_may_skip(skb, R, dm, G):
    """Restatement of the device predicate (dm a power of two)."""
    base = (skb + 1 + R) & 0xFFFFFFFF
    if base & (dm - 1):
        return False
    q = base // dm + 1
    p2 = 1 if q <= 1 else 1 << (q - 1).bit_length()
    return p2 <= q + G - 2


def test_modulus_logs_sit_at_two_to_the_i_minus_one():
    for bits, (sk, mod) in skew_tables().items():
        idx = np.arange(sk.size)
        at_mod = sk == mod
        pow2_minus_one = ((idx + 1) & idx) == 0
        assert np.array_equal(at_mod, pow2_minus_one), bits


def test_group_predicate_covers_every_skipped_constant():
    tables = skew_tables()
    rng = np.random.default_rng(0x5EED)
    for bits, (sk, mod) in tables.items():
        n_max = sk.size + 1
        checked = 0
        for lg in (1, 2, 3, 4):
            G = 1 << lg
            for lgdm in range(0, 15 if bits == 16 else 7):
                dm = 1 << lgdm
                for _ in range(400):
                    # skew bases of the transforms: -1 (decode, FFT encode)
                    # and m * (g + 1) - 1 (encode IFFT chunks)
                    m = 1 << int(rng.integers(lg, 16 if bits == 16 else 8))
                    skb = -1 if rng.integers(2) else m * int(rng.integers(1, 4)) - 1
                    span = G * dm
                    R = int(rng.integers(0, max(1, n_max // span))) * span
                    idx = [skb + R + dm * t for t in range(1, G)]
                    if max(idx) >= sk.size or min(idx) < 0:
                        continue
                    hits = any(sk[i] == mod for i in idx)
                    if hits:
                        assert group_may_skip(skb, R, dm, G), (bits, skb, R, dm, G)
                    checked += 1
        assert checked > 1000, (bits, checked)


def test_group_predicate_is_exact_at_the_transform_origin():
    # Groups at lane 0 of a transform from skew base -1 always meet entry
    # dm - 1, a power of two minus one.
    for lg in (1, 2, 3, 4):
        for lgdm in range(12):
            assert group_may_skip(-1, 0, 1 << lgdm, 1 << lg)
