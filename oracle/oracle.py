"""ctypes front end for the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY.  The oracle restates the rustfs-erasure-codec 9.1.0
algorithms on the CPU so the CUDA path can be checked byte for byte.  Only the
test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lock = threading.Lock()
_lib = None

u8p = ctypes.POINTER(ctypes.c_uint8)
u16p = ctypes.POINTER(ctypes.c_uint16)
szp = ctypes.POINTER(ctypes.c_size_t)
size_t = ctypes.c_size_t


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                build()
            L = ctypes.CDLL(LIB_PATH)
            sig = {
                "orc_gf8_tables": (None, [u8p, u8p]),
                "orc_gf8_mul": (ctypes.c_uint8, [ctypes.c_uint8, ctypes.c_uint8]),
                "orc_gf8_div": (ctypes.c_uint8, [ctypes.c_uint8, ctypes.c_uint8]),
                "orc_gf8_exp": (ctypes.c_uint8, [ctypes.c_uint8, size_t]),
                "orc_gf8_mul_slice": (None, [ctypes.c_uint8, u8p, u8p, size_t]),
                "orc_gf8_mul_slice_xor": (None, [ctypes.c_uint8, u8p, u8p, size_t]),
                "orc_build_matrix": (ctypes.c_int, [size_t, size_t, ctypes.c_int, ctypes.c_int, u8p, u8p]),
                "orc_gf8_invert": (ctypes.c_int, [size_t, u8p, u8p]),
                "orc_classic_encode": (None, [size_t, size_t, u8p, ctypes.POINTER(u8p), ctypes.POINTER(u8p), size_t]),
                "orc_classic_reconstruct": (ctypes.c_int, [size_t, size_t, u8p, ctypes.POINTER(u8p), u8p, size_t,
                                                           ctypes.c_int, u8p, size_t]),
                "orc_classic_recovery_rows": (ctypes.c_int, [size_t, size_t, u8p, u8p, ctypes.c_int, u8p, size_t,
                                                             szp, szp, szp, u8p]),
                "orc_classic_verify": (ctypes.c_int, [size_t, size_t, u8p, ctypes.POINTER(u8p), size_t]),
                "orc_classic_decode_idx": (ctypes.c_int, [size_t, size_t, u8p, ctypes.POINTER(u8p), szp, size_t, u8p,
                                                          size_t, ctypes.POINTER(u8p), szp, size_t]),
                "orc_lgf8_tables": (None, [u8p, u8p, u8p, u8p]),
                "orc_lgf8_mul_log": (ctypes.c_uint8, [ctypes.c_uint8, ctypes.c_uint8]),
                "orc_lgf8_encode": (ctypes.c_int, [size_t, size_t, ctypes.POINTER(u8p), ctypes.POINTER(u8p), size_t]),
                "orc_lgf8_reconstruct": (ctypes.c_int, [size_t, size_t, ctypes.POINTER(u8p), u8p, u8p, size_t]),
                "orc_lgf8_error_locators": (None, [size_t, size_t, u8p, u8p]),
                "orc_lgf16_tables": (None, [u16p, u16p, u16p, u16p]),
                "orc_lgf16_mul_log": (ctypes.c_uint16, [ctypes.c_uint16, ctypes.c_uint16]),
                "orc_lgf16_encode": (ctypes.c_int, [size_t, size_t, ctypes.POINTER(u8p), ctypes.POINTER(u8p), size_t]),
                "orc_lgf16_reconstruct": (ctypes.c_int, [size_t, size_t, ctypes.POINTER(u8p), u8p, u8p, size_t]),
                "orc_lgf16_error_locators": (None, [size_t, size_t, u8p, u16p]),
                "orc_gf16t_mul": (None, [u8p, u8p, u8p]),
                "orc_gf16t_build_matrix": (ctypes.c_int, [size_t, size_t, u8p]),
                "orc_gf16t_encode": (None, [size_t, size_t, u8p, ctypes.POINTER(u8p), ctypes.POINTER(u8p), size_t]),
                "orc_gf16t_reconstruct": (ctypes.c_int, [size_t, size_t, u8p, ctypes.POINTER(u8p), u8p, size_t,
                                                         ctypes.c_int]),
                "orc_fast_encode_batch": (ctypes.c_int, [size_t, size_t, u8p, ctypes.POINTER(u8p), size_t, size_t,
                                                         ctypes.c_int]),
                "orc_fast_kernel_name": (ctypes.c_char_p, []),
                "orc_fast_force_kernel": (None, [ctypes.c_int]),
                "orc_fast_best_kernel": (ctypes.c_int, []),
            }
            for name, (res, args) in sig.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
        return _lib


def _p8(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(u8p)


def _ptrs(arrs):
    arr = (u8p * len(arrs))()
    for i, a in enumerate(arrs):
        arr[i] = _p8(a)
    return arr


# ---------------------------------------------------------------- GF(2^8)
def gf8_tables():
    lg = np.zeros(256, np.uint8)
    ex = np.zeros(510, np.uint8)
    lib().orc_gf8_tables(_p8(lg), _p8(ex))
    return lg, ex


def gf8_mul(a, b):
    return lib().orc_gf8_mul(a, b)


def gf8_div(a, b):
    return lib().orc_gf8_div(a, b)


def gf8_exp(a, n):
    return lib().orc_gf8_exp(a, n)


def gf8_mul_slice(c, inp):
    inp = np.ascontiguousarray(inp, np.uint8)
    out = np.zeros_like(inp)
    lib().orc_gf8_mul_slice(c, _p8(inp), _p8(out), inp.size)
    return out


def gf8_mul_slice_xor(c, inp, out):
    inp = np.ascontiguousarray(inp, np.uint8)
    out = np.array(out, np.uint8)
    lib().orc_gf8_mul_slice_xor(c, _p8(inp), _p8(out), inp.size)
    return out


MATRIX_MODES = {"vandermonde": 0, "cauchy": 1, "jerasure_like": 2, "custom": 3}


def build_matrix(k, m, mode="vandermonde", fast_one_parity=False, custom=None):
    out = np.zeros((k + m) * k, np.uint8)
    cust = np.ascontiguousarray(custom if custom is not None else np.zeros(max(1, m * k)), np.uint8).ravel()
    rc = lib().orc_build_matrix(k, m, MATRIX_MODES[mode], int(fast_one_parity), _p8(cust), _p8(out))
    return rc, out.reshape(k + m, k)


def invert(mat):
    mat = np.ascontiguousarray(mat, np.uint8)
    n = mat.shape[0]
    out = np.zeros_like(mat)
    rc = lib().orc_gf8_invert(n, _p8(mat), _p8(out))
    return rc, out


# ---------------------------------------------------------------- classic codec
def classic_encode(matrix, shards):
    """shards: list of k+m uint8 arrays (parity overwritten in place)."""
    matrix = np.ascontiguousarray(matrix, np.uint8)
    k = matrix.shape[1]
    m = matrix.shape[0] - k
    length = shards[0].size
    lib().orc_classic_encode(k, m, _p8(matrix), _ptrs(shards[:k]), _ptrs(shards[k:]), length)


GOALS = {"all": 0, "data": 1, "required": 2}


def classic_reconstruct(matrix, shards, present, goal="all", required=None):
    matrix = np.ascontiguousarray(matrix, np.uint8)
    k = matrix.shape[1]
    m = matrix.shape[0] - k
    pres = np.ascontiguousarray(np.array(present, np.uint8))
    req = np.ascontiguousarray(np.array(required if required is not None else [0], np.uint8))
    nreq = len(required) if required is not None else 0
    return lib().orc_classic_reconstruct(k, m, _p8(matrix), _ptrs(shards), _p8(pres), shards[0].size,
                                         GOALS[goal], _p8(req), nreq)


def classic_recovery_rows(matrix, present, goal="all", required=None):
    matrix = np.ascontiguousarray(matrix, np.uint8)
    k = matrix.shape[1]
    m = matrix.shape[0] - k
    pres = np.ascontiguousarray(np.array(present, np.uint8))
    req = np.ascontiguousarray(np.array(required if required is not None else [0], np.uint8))
    nreq = len(required) if required is not None else 0
    surv = (size_t * k)()
    targ = (size_t * (k + m))()
    nt = size_t(0)
    rows = np.zeros((k + m) * k, np.uint8)
    rc = lib().orc_classic_recovery_rows(k, m, _p8(matrix), _p8(pres), GOALS[goal], _p8(req), nreq,
                                         surv, targ, ctypes.byref(nt), _p8(rows))
    n = nt.value
    return rc, list(surv), list(targ)[:n], rows[: n * k].reshape(n, k)


def classic_verify(matrix, shards):
    matrix = np.ascontiguousarray(matrix, np.uint8)
    k = matrix.shape[1]
    m = matrix.shape[0] - k
    return bool(lib().orc_classic_verify(k, m, _p8(matrix), _ptrs(shards), shards[0].size))


def _opt_ptrs(arrs):
    """Pointer and length arrays for a list whose None entries stand for Option::None."""
    ptrs = (u8p * max(1, len(arrs)))()
    lens = (size_t * max(1, len(arrs)))()
    for i, a in enumerate(arrs):
        if a is not None:
            ptrs[i] = _p8(a)
            lens[i] = a.size
    return ptrs, lens


def classic_decode_idx(matrix, dst, expect, inputs):
    """src/galois_8/policy.rs:543-700: accumulate into the non-None entries of
    dst (uint8 arrays, changed in place); expect=None selects merge mode."""
    matrix = np.ascontiguousarray(matrix, np.uint8)
    k = matrix.shape[1]
    m = matrix.shape[0] - k
    dp, dl = _opt_ptrs(dst)
    ip, il = _opt_ptrs(inputs)
    if expect is None:
        ex, nex = None, 0
    else:
        ex = np.ascontiguousarray(np.array(expect, np.uint8).reshape(-1))
        ex, nex = (_p8(ex) if ex.size else _p8(np.zeros(1, np.uint8))), ex.size
    return lib().orc_classic_decode_idx(k, m, _p8(matrix), dp, dl, len(dst), ex, nex, ip, il, len(inputs))


# ---------------------------------------------------------------- Leopard
def lgf8_tables():
    lg, ex, sk, wa = (np.zeros(256, np.uint8), np.zeros(256, np.uint8), np.zeros(255, np.uint8),
                      np.zeros(256, np.uint8))
    lib().orc_lgf8_tables(_p8(lg), _p8(ex), _p8(sk), _p8(wa))
    return lg, ex, sk, wa


def lgf16_tables():
    lg = np.zeros(65536, np.uint16)
    ex = np.zeros(131072, np.uint16)
    sk = np.zeros(65535, np.uint16)
    wa = np.zeros(65536, np.uint16)
    lib().orc_lgf16_tables(lg.ctypes.data_as(u16p), ex.ctypes.data_as(u16p), sk.ctypes.data_as(u16p),
                           wa.ctypes.data_as(u16p))
    return lg, ex, sk, wa


def leopard_encode(field, k, m, data):
    length = data[0].size
    parity = [np.zeros(length, np.uint8) for _ in range(m)]
    fn = lib().orc_lgf8_encode if field == 8 else lib().orc_lgf16_encode
    rc = fn(k, m, _ptrs(data), _ptrs(parity), length)
    return rc, parity


def leopard_reconstruct(field, k, m, shards, present, want=None):
    pres = np.ascontiguousarray(np.array(present, np.uint8))
    w = np.ascontiguousarray(np.array(want if want is not None else [1] * (k + m), np.uint8))
    fn = lib().orc_lgf8_reconstruct if field == 8 else lib().orc_lgf16_reconstruct
    return fn(k, m, _ptrs(shards), _p8(pres), _p8(w), shards[0].size)


def leopard_error_locators(field, k, m, present):
    pres = np.ascontiguousarray(np.array(present, np.uint8))
    if field == 8:
        out = np.zeros(256, np.uint8)
        lib().orc_lgf8_error_locators(k, m, _p8(pres), _p8(out))
    else:
        out = np.zeros(65536, np.uint16)
        lib().orc_lgf16_error_locators(k, m, _p8(pres), out.ctypes.data_as(u16p))
    return out


# ---------------------------------------------------------------- tower GF(2^16)
def gf16t_build_matrix(k, m):
    out = np.zeros((k + m) * k * 2, np.uint8)
    rc = lib().orc_gf16t_build_matrix(k, m, _p8(out))
    return rc, out.reshape(k + m, k, 2)


def gf16t_encode(matrix, shards):
    matrix = np.ascontiguousarray(matrix, np.uint8)
    k = matrix.shape[1]
    m = matrix.shape[0] - k
    lib().orc_gf16t_encode(k, m, _p8(matrix), _ptrs(shards[:k]), _ptrs(shards[k:]), shards[0].size // 2)


def gf16t_reconstruct(matrix, shards, present, data_only=False):
    matrix = np.ascontiguousarray(matrix, np.uint8)
    k = matrix.shape[1]
    m = matrix.shape[0] - k
    pres = np.ascontiguousarray(np.array(present, np.uint8))
    return lib().orc_gf16t_reconstruct(k, m, _p8(matrix), _ptrs(shards), _p8(pres), shards[0].size // 2,
                                       int(data_only))


# ---------------------------------------------------------------- CPU baseline
def fast_encode_batch(matrix, shard_arrays, n_stripes, length, threads):
    """shard_arrays: flat list of n_stripes*(k+m) uint8 arrays."""
    matrix = np.ascontiguousarray(matrix, np.uint8)
    k = matrix.shape[1]
    m = matrix.shape[0] - k
    return lib().orc_fast_encode_batch(k, m, _p8(matrix), _ptrs(shard_arrays), n_stripes, length, threads)


def fast_kernel_name():
    return lib().orc_fast_kernel_name().decode()


def fast_force_kernel(kernel: int) -> None:
    """-1: the host's widest GFNI (the reference's choice); 2 / 1: GFNI at 64 /
    32 bytes; 0: nibble tables."""
    lib().orc_fast_force_kernel(kernel)


def fast_best_kernel() -> int:
    return int(lib().orc_fast_best_kernel())


# ---------------------------------------------------------------- checksums
def fnv1a(data: bytes) -> int:
    """FNV-1a 64 as used by the reference's golden tests (tests/golden_vectors.rs:5-9)."""
    acc = 0xCBF29CE484222325
    for b in bytes(data):
        acc = ((acc ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return acc


def checksum_shards(shards) -> int:
    """tests/golden_vectors.rs:11-18."""
    acc = 0xCBF29CE484222325
    for s in shards:
        acc ^= fnv1a(bytes(s))
        acc = (acc * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return acc
