"""The Leopard decode's formal derivative as the device computes it
(csrc/leo_fft.cuh, smem_derivative), restated on the host: 16-lane groups
taken in ascending rounds of W groups, each round reading every value it
needs before writing; bits 0-3 from the group's own lanes by an ascending
in-place pass, higher zero bits by the group 2^t lanes above.  It must equal
the direct formula (lane l gains the XOR of the old lanes l | 2^t over the
zero bits t of l, src/core/leopard_gf16/decode.rs:1100-1116) and the
reference's own in-place loop over i = 1 .. n - 1 (width = lowest set bit of
i: lanes [i - width, i) ^= lanes [i, i + width)).
"""
import numpy as np
import pytest


def derivative_direct(v):
    n = len(v)
    out = v.copy()
    for l in range(n):
        t = 1
        while (l | t) < n:
            if not (l & t):
                out[l] ^= v[l | t]
            t <<= 1
    return out


def derivative_reference_loop(v):
    w = v.copy()
    n = len(w)
    for i in range(1, n):
        width = ((i ^ (i - 1)) + 1) >> 1
        w[i - width:i] ^= w[i:i + width]
    return w


def derivative_grouped(v, warps):
    S = v.copy()
    n = len(S)
    lgn = n.bit_length() - 1
    groups = n // 16
    for r0 in range(0, groups, warps):
        staged = []
        for g in range(r0, min(groups, r0 + warps)):
            R = g * 16
            x = S[R:R + 16].copy()
            for j in range(16):  # ascending, in place: sources above j are still old
                t = 1
                while t < 16:
                    if not (j & t):
                        x[j] ^= x[j | t]
                    t <<= 1
            for t in range(4, lgn):
                if R & (1 << t):
                    continue
                x ^= S[R + (1 << t):R + (1 << t) + 16]
            staged.append((R, x))
        for R, x in staged:  # written only after the round's reads
            S[R:R + 16] = x
    return S


@pytest.mark.parametrize("n", [32, 64, 256, 1024, 2048, 4096])
@pytest.mark.parametrize("warps", [1, 3, 8, 32])
def test_grouped_derivative_matches_the_formula_and_the_reference_loop(n, warps):
    rng = np.random.default_rng(n * 131 + warps)
    v = rng.integers(0, 1 << 16, n, dtype=np.uint32)
    want = derivative_direct(v)
    assert np.array_equal(derivative_reference_loop(v), want)
    assert np.array_equal(derivative_grouped(v, warps), want)
