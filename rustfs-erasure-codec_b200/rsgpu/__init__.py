"""Python mirror of the rustfs-erasure-codec ``ReedSolomon`` API over librsgpu.so.

This module is a thin ctypes layer over the C ABI declared in
``include/rsgpu.h``; every byte is computed by the sm_100a kernels inside
librsgpu.so.  There is no CPU fallback: importing this module without the
built library raises ``ImportError``.

Shards may be NumPy ``uint8`` arrays (host memory, staged through the GPU by
the library) or ``torch.uint8`` CUDA tensors (device memory; work is queued on
the current torch stream).  Method names and error behaviour follow the
reference (src/core/codec.rs, encode.rs, reconstruct.rs, verify.rs): errors
are raised as :class:`RsError` carrying the reference ``Error`` name.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "librsgpu.so")

ERROR_NAMES = {
    1: "TooFewShards", 2: "TooManyShards", 3: "TooFewDataShards", 4: "TooManyDataShards",
    5: "TooFewParityShards", 6: "TooManyParityShards", 7: "TooFewBufferShards", 8: "TooManyBufferShards",
    9: "IncorrectShardSize", 10: "TooFewShardsPresent", 11: "EmptyShard", 12: "InvalidShardFlags",
    13: "InvalidIndex", 14: "InvalidCustomMatrix", 15: "UnsupportedCodecFamily",
    16: "UnsupportedLeopardPrototype", 100: "Cuda", 101: "OutOfMemory", 102: "InvalidArgument",
    103: "DeviceTimeout", 104: "NoDevice", 105: "ScratchLimit", 106: "StreamIo",
}

MEM_HOST, MEM_DEVICE = 0, 1
FAMILY = {"classic": 0, "leopard_gf8": 1, "leopard_gf16": 2}
LEOPARD_MODE = {"disabled": 0, "as_needed": 1, "prefer_gf16": 2, "prefer_leopard": 3}
MATRIX_MODE = {"vandermonde": 0, "cauchy": 1, "jerasure_like": 2, "custom": 3}
GOAL = {"all": 0, "data": 1, "required": 2}


class RsError(Exception):
    """A reference ``Error`` (or a device condition) returned by the library."""

    def __init__(self, code: int):
        self.code = int(code)
        self.name = ERROR_NAMES.get(self.code, f"Error{code}")
        super().__init__(f"{self.name}: {_lib().rsgpu_error_string(self.code).decode()}")


class _Options(ctypes.Structure):
    _fields_ = [
        ("fast_one_parity", ctypes.c_int32),
        ("inversion_cache", ctypes.c_int32),
        ("inversion_cache_capacity", ctypes.c_size_t),
        ("inversion_cache_max_bytes", ctypes.c_size_t),
        ("codec_family", ctypes.c_int32),
        ("leopard_mode", ctypes.c_int32),
        ("matrix_mode", ctypes.c_int32),
        ("max_parallel_jobs", ctypes.c_size_t),
    ]


class MixOp(ctypes.Structure):
    """rsgpu_mix_op: one operation of a mixed batch."""
    _fields_ = [
        ("codec", ctypes.c_void_p),
        ("op", ctypes.c_int32),
        ("goal", ctypes.c_int32),
        ("shards", ctypes.c_void_p),
        ("present", ctypes.c_void_p),
        ("shard_len", ctypes.c_size_t),
    ]


class Plan(ctypes.Structure):
    """rsgpu_plan: algorithm (ALGO_APPLY / ALGO_FFT) and tile."""
    _fields_ = [("algo", ctypes.c_int32), ("tile", ctypes.c_int32)]

    def tuple(self):
        return (int(self.algo), int(self.tile))


class MixOptions(ctypes.Structure):
    _fields_ = [("planner", ctypes.c_int32), ("order", ctypes.c_int32), ("graph", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32)]


class MixInfo(ctypes.Structure):
    _fields_ = [("n_ops", ctypes.c_size_t), ("n_jobs", ctypes.c_size_t), ("n_items", ctypes.c_size_t),
                ("n_classes", ctypes.c_size_t), ("algorithmic_bytes", ctypes.c_uint64),
                ("device_bytes", ctypes.c_size_t), ("grid", ctypes.c_uint32), ("smem_bytes", ctypes.c_uint32),
                ("kernels_per_launch", ctypes.c_uint32), ("pad", ctypes.c_uint32)]


class TuneOptions(ctypes.Structure):
    _fields_ = [("target_bytes", ctypes.c_size_t), ("repeats", ctypes.c_int32), ("pad", ctypes.c_int32)]


MODEL_FEATURES, MODEL_PLANS, MODEL_HIDDEN = 11, 6, 32


class TuneSample(ctypes.Structure):
    _fields_ = [("features", ctypes.c_float * MODEL_FEATURES), ("plan", Plan), ("gbps", ctypes.c_float)]


class TrainOptions(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_int32), ("lr", ctypes.c_float), ("seed", ctypes.c_uint64)]


class ServerOptions(ctypes.Structure):
    _fields_ = [("device_budget", ctypes.c_size_t), ("max_inflight", ctypes.c_uint32), ("max_batch", ctypes.c_uint32),
                ("streams", ctypes.c_uint32), ("planner", ctypes.c_int32)]


class Request(ctypes.Structure):
    _fields_ = [("codec", ctypes.c_void_p), ("op", ctypes.c_int32), ("goal", ctypes.c_int32),
                ("shards", ctypes.c_void_p), ("present", ctypes.c_void_p), ("shard_len", ctypes.c_size_t),
                ("mem", ctypes.c_int32), ("pad", ctypes.c_int32), ("tag", ctypes.c_uint64)]


class Completion(ctypes.Structure):
    _fields_ = [("tag", ctypes.c_uint64), ("status", ctypes.c_int32), ("ok", ctypes.c_int32),
                ("submit_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("pending", ctypes.c_size_t), ("inflight", ctypes.c_size_t), ("budget_bytes", ctypes.c_size_t),
                ("reserved_bytes", ctypes.c_size_t), ("max_reserved_bytes", ctypes.c_size_t),
                ("max_concurrent_launches", ctypes.c_uint32), ("pad", ctypes.c_uint32),
                ("prepare_seconds", ctypes.c_double), ("max_prepare_seconds", ctypes.c_double),
                ("max_loop_gap_seconds", ctypes.c_double)]


class StreamOptions(ctypes.Structure):
    _fields_ = [("block_size", ctypes.c_size_t)]


class StreamStatus(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("code", ctypes.c_int32), ("shard_index", ctypes.c_size_t)]


_READFN = ctypes.CFUNCTYPE(ctypes.c_int64, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t)
_WRITEFN = ctypes.CFUNCTYPE(ctypes.c_int64, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t)
STREAM_KINDS = {1: "codec", 2: "read", 3: "write"}


class StreamError(Exception):
    """src/core/stream.rs StreamError: the shard index and what failed
    (a codec error, or the reader's / writer's exception)."""

    def __init__(self, kind: str, shard_index: int, error):
        self.kind = kind
        self.shard_index = int(shard_index)
        self.error = error
        super().__init__(f"{kind} error at shard {shard_index}: {error}")


ALGO_APPLY, ALGO_FFT = 0, 1
# Order of the cost model's outputs (rsgpu_plan_index).
MODEL_PLAN_ORDER = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (1, 3)]
PLANNER = {"fixed": 0, "table": 1, "model": 2}
ORDER = {"submit": 0, "cost": 1}


class CacheStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("requests", "hits", "misses", "inserts", "evictions", "entries", "retained_bytes")]


_L = None

P = ctypes.c_void_p
SZ = ctypes.c_size_t
I32 = ctypes.c_int32
PP = ctypes.POINTER(ctypes.c_void_p)
SZP = ctypes.POINTER(ctypes.c_size_t)
U8P = ctypes.POINTER(ctypes.c_uint8)


def _free_handle(owner, fn_name: str) -> None:
    """Release owner._h through the named C-ABI free call.  Safe from __del__
    during interpreter shutdown, when module globals may already be gone
    (callers bind this function as a default argument for that reason)."""
    h = getattr(owner, "_h", None)
    if not h:
        return
    lib = _L
    fn = getattr(lib, fn_name, None) if lib is not None else None
    if fn is not None:
        fn(h)
    owner._h = None


def _lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"librsgpu.so not found at {LIB_PATH}; build it with `python rustfs-erasure-codec_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        sigs = {
            "rsgpu_options_default": (None, [ctypes.POINTER(_Options)]),
            "rsgpu_codec_new": (I32, [SZ, SZ, ctypes.POINTER(_Options), PP]),
            "rsgpu_codec_with_custom_matrix": (I32, [SZ, SZ, U8P, ctypes.POINTER(_Options), PP]),
            "rsgpu_codec_new_gf16": (I32, [SZ, SZ, PP]),
            "rsgpu_codec_gf16_with_custom_matrix": (I32, [SZ, SZ, U8P, PP]),
            "rsgpu_encode_single": (I32, [P, SZ, PP, SZP, SZ, I32, P]),
            "rsgpu_encode_single_sep": (I32, [P, SZ, P, SZ, PP, SZP, SZ, I32, P]),
            "rsgpu_update": (I32, [P, PP, SZP, SZ, PP, SZP, SZ, PP, SZP, SZ, I32, P]),
            "rsgpu_split_shard_len": (SZ, [P, SZ]),
            "rsgpu_split": (I32, [P, P, SZ, P, SZ]),
            "rsgpu_join": (I32, [P, PP, SZP, SZ, P, SZ, SZP]),
            "rsgpu_format_id": (I32, [P, P, SZ, SZP]),
            "rsgpu_codec_free": (None, [P]),
            "rsgpu_data_shard_count": (SZ, [P]),
            "rsgpu_parity_shard_count": (SZ, [P]),
            "rsgpu_total_shard_count": (SZ, [P]),
            "rsgpu_codec_family": (I32, [P]),
            "rsgpu_encoding_matrix": (I32, [P, U8P, SZ]),
            "rsgpu_encode": (I32, [P, PP, SZP, SZ, I32, P]),
            "rsgpu_encode_sep": (I32, [P, PP, SZP, SZ, PP, SZP, SZ, I32, P]),
            "rsgpu_reconstruct": (I32, [P, PP, SZP, U8P, SZ, I32, U8P, SZ, I32, P]),
            "rsgpu_verify": (I32, [P, PP, SZP, SZ, ctypes.POINTER(I32), I32, P]),
            "rsgpu_verify_ws_new": (I32, [P, SZ, PP]),
            "rsgpu_verify_ws_free": (None, [P]),
            "rsgpu_verify_with_workspace": (I32, [P, PP, SZP, SZ, P, ctypes.POINTER(I32), I32, P]),
            "rsgpu_verify_with_buffer": (I32, [P, PP, SZP, SZ, PP, SZP, SZ, ctypes.POINTER(I32), I32, P]),
            "rsgpu_decode_idx": (I32, [P, PP, SZP, SZ, U8P, SZ, PP, SZP, SZ, I32, P]),
            "rsgpu_prepare_reconstruct_ws": (I32, [P, U8P, SZ, SZ, I32, U8P, SZ, PP]),
            "rsgpu_reconstruct_ws_free": (None, [P]),
            "rsgpu_reconstruct_ws_targets": (SZ, [P, SZP, SZ]),
            "rsgpu_reconstruct_with_ws": (I32, [P, P, PP, SZP, U8P, SZ, I32, P]),
            "rsgpu_encode_batch": (I32, [P, SZ, PP, SZ, I32, P]),
            "rsgpu_reconstruct_batch": (I32, [P, SZ, PP, U8P, SZ, I32, I32, P]),
            "rsgpu_verify_batch": (I32, [P, SZ, PP, SZ, U8P, I32, P]),
            "rsgpu_get_cache_stats": (I32, [P, ctypes.POINTER(CacheStats)]),
            "rsgpu_batch_prepare": (I32, [P, I32, SZ, P, P, SZ, I32, PP]),
            "rsgpu_batch_launch": (I32, [P, P]),
            "rsgpu_batch_verify_result": (I32, [P, U8P, P]),
            "rsgpu_batch_kernel_count": (ctypes.c_uint32, [P]),
            "rsgpu_batch_free": (None, [P]),
            "rsgpu_leopard_reconstruct_noalloc": (I32, [P, PP, SZP, U8P, SZ, P]),
            "rsgpu_mix_options_default": (None, [ctypes.POINTER(MixOptions)]),
            "rsgpu_mix_prepare": (I32, [P, SZ, ctypes.POINTER(MixOptions), PP]),
            "rsgpu_mix_prepare_planned": (I32, [P, SZ, P, ctypes.POINTER(MixOptions), PP]),
            "rsgpu_mix_launch": (I32, [P, P]),
            "rsgpu_mix_results": (I32, [P, U8P, P]),
            "rsgpu_mix_get_info": (I32, [P, ctypes.POINTER(MixInfo)]),
            "rsgpu_mix_get_plans": (I32, [P, P, SZ]),
            "rsgpu_mix_free": (None, [P]),
            "rsgpu_plan_features": (I32, [P, P]),
            "rsgpu_plan_index": (I32, [Plan]),
            "rsgpu_tune": (I32, [P, SZ, ctypes.POINTER(TuneOptions), SZP]),
            "rsgpu_tuner_samples": (SZ, [P, SZ]),
            "rsgpu_tuner_table_size": (SZ, []),
            "rsgpu_tuner_lookup": (I32, [P, ctypes.POINTER(Plan)]),
            "rsgpu_tuner_save": (I32, [ctypes.c_char_p]),
            "rsgpu_tuner_load": (I32, [ctypes.c_char_p]),
            "rsgpu_tuner_clear": (None, []),
            "rsgpu_model_param_count": (SZ, []),
            "rsgpu_model_get_params": (I32, [P, SZ]),
            "rsgpu_model_set_params": (I32, [P, SZ]),
            "rsgpu_model_train": (I32, [P, P, P, SZ, ctypes.POINTER(TrainOptions), ctypes.POINTER(ctypes.c_float)]),
            "rsgpu_model_train_from_tuner": (I32, [ctypes.POINTER(TrainOptions), ctypes.POINTER(ctypes.c_float)]),
            "rsgpu_model_predict": (I32, [P, SZ, P]),
            "rsgpu_model_gradients": (I32, [P, P, P, P, SZ, ctypes.POINTER(ctypes.c_float), P]),
            "rsgpu_model_ready": (I32, []),
            "rsgpu_stream_options_default": (None, [ctypes.POINTER(StreamOptions)]),
            "rsgpu_encode_stream": (I32, [P, SZ, _READFN, P, SZ, _WRITEFN, P, ctypes.POINTER(StreamOptions),
                                          ctypes.POINTER(StreamStatus)]),
            "rsgpu_verify_stream": (I32, [P, SZ, _READFN, P, ctypes.POINTER(StreamOptions), ctypes.POINTER(I32),
                                          ctypes.POINTER(StreamStatus)]),
            "rsgpu_reconstruct_stream_from": (I32, [P, SZ, U8P, _READFN, P, U8P, _WRITEFN, P,
                                                    ctypes.POINTER(StreamOptions), ctypes.POINTER(StreamStatus)]),
            "rsgpu_server_options_default": (None, [ctypes.POINTER(ServerOptions)]),
            "rsgpu_server_new": (I32, [ctypes.POINTER(ServerOptions), PP]),
            "rsgpu_server_submit": (I32, [P, ctypes.POINTER(Request)]),
            "rsgpu_server_poll": (SZ, [P, P, SZ, I32]),
            "rsgpu_server_get_stats": (I32, [P, ctypes.POINTER(ServerStats)]),
            "rsgpu_server_free": (None, [P]),
            "rsgpu_kernel_launch_count": (ctypes.c_uint64, []),
            "rsgpu_error_string": (ctypes.c_char_p, [I32]),
            "rsgpu_version": (ctypes.c_char_p, []),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _L = L
    return _L


def lib():
    """The loaded librsgpu.so (raises ImportError when it is not built)."""
    return _lib()


def kernel_launch_count() -> int:
    return int(_lib().rsgpu_kernel_launch_count())


def _check(rc):
    if rc != 0:
        raise RsError(rc)


# ------------------------------------------------------------------ buffers
def _is_torch_cuda(x) -> bool:
    t = type(x)
    return t.__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _buffer_info(shards):
    """Return (mem, ptr array, lens array, stream, keepalive) for a shard list."""
    devs = [s is not None and _is_torch_cuda(s) for s in shards]
    mem = MEM_DEVICE if any(devs) else MEM_HOST
    ptrs = (ctypes.c_void_p * len(shards))()
    lens = (ctypes.c_size_t * len(shards))()
    keep = []
    for i, s in enumerate(shards):
        if s is None:
            ptrs[i] = None
            lens[i] = 0
            continue
        if mem == MEM_DEVICE:
            if not _is_torch_cuda(s):
                raise TypeError("mixing host and device shards in one call")
            assert s.is_contiguous()
            ptrs[i] = s.data_ptr()
            lens[i] = s.numel() * s.element_size()
        else:
            a = s if isinstance(s, np.ndarray) else np.frombuffer(s, np.uint8)
            if not a.flags.c_contiguous:
                raise TypeError("host shards must be C-contiguous")
            ptrs[i] = a.ctypes.data
            lens[i] = a.nbytes
            keep.append(a)
    stream = None
    if mem == MEM_DEVICE:
        import torch

        stream = torch.cuda.current_stream().cuda_stream
    return mem, ptrs, lens, stream, keep


def _slice_ptrs(ptrs, lens, start, n):
    """Pointer and length arrays of entries start .. start+n of _buffer_info's arrays."""
    p = (ctypes.c_void_p * max(1, n))(*ptrs[start:start + n])
    ln = (ctypes.c_size_t * max(1, n))(*lens[start:start + n])
    return p, ln


def _stripe_block(stripes):
    """(mem, ptr array, shard length, stream, keepalive) when `stripes` is one
    C-contiguous (stripes, shards, length) uint8 block -- a numpy array or a
    CUDA tensor -- with the pointers computed in one vectorised step; None for
    any other form (lists of shards take the per-shard path)."""
    if isinstance(stripes, np.ndarray):
        if stripes.ndim != 3 or stripes.dtype != np.uint8 or not stripes.flags.c_contiguous:
            return None
        mem, stream, base = MEM_HOST, None, stripes.__array_interface__["data"][0]
    elif _is_torch_cuda(stripes):
        import torch

        if stripes.dim() != 3 or stripes.dtype != torch.uint8 or not stripes.is_contiguous():
            return None
        mem, stream, base = MEM_DEVICE, torch.cuda.current_stream().cuda_stream, stripes.data_ptr()
    else:
        return None
    n, t, length = stripes.shape
    ptrs = np.uint64(base) + np.arange(max(1, n * t), dtype=np.uint64) * np.uint64(length)
    return mem, ptrs.ctypes.data_as(PP), int(length), stream, (stripes, ptrs)


def _check_stripe_widths(widths, total):
    """Every stripe holds exactly k + m shards (TooFewShards / TooManyShards
    otherwise, as the reference's per-call piece-count check)."""
    for w in widths:
        if w != total:
            raise RsError(1 if w < total else 2)


def _present_flags(present, n_stripes, n_shards):
    """Presence flags as a uint8 array of n_stripes * n_shards entries."""
    a = np.ascontiguousarray(np.asarray(present, dtype=bool), dtype=np.uint8).reshape(-1)
    if a.size != n_stripes * n_shards:
        raise ValueError("present must hold one flag per shard of every stripe")
    return a, a.ctypes.data_as(U8P)


def _flags(v, n):
    arr = (ctypes.c_uint8 * n)()
    for i, b in enumerate(v):
        arr[i] = 1 if b else 0
    return arr


@dataclass
class CodecOptions:
    """src/core/options.rs:97-146."""

    fast_one_parity: bool = False
    inversion_cache: bool = True
    inversion_cache_capacity: int = 0
    inversion_cache_max_bytes: int = 0
    codec_family: str = "classic"
    leopard_mode: str = "disabled"
    matrix_mode: str = "vandermonde"
    max_parallel_jobs: int = 0

    def _c(self):
        o = _Options()
        o.fast_one_parity = int(self.fast_one_parity)
        o.inversion_cache = int(self.inversion_cache)
        o.inversion_cache_capacity = self.inversion_cache_capacity
        o.inversion_cache_max_bytes = self.inversion_cache_max_bytes
        o.codec_family = FAMILY[self.codec_family]
        o.leopard_mode = LEOPARD_MODE[self.leopard_mode]
        o.matrix_mode = MATRIX_MODE[self.matrix_mode]
        o.max_parallel_jobs = self.max_parallel_jobs
        return o


class VerifyWorkspace:
    """src/core/workspace.rs:16-69."""

    def __init__(self, codec: "ReedSolomon", shard_len: int):
        h = ctypes.c_void_p()
        _check(_lib().rsgpu_verify_ws_new(codec._h, shard_len, ctypes.byref(h)))
        self._h = h

    def __del__(self, _free=_free_handle):
        _free(self, "rsgpu_verify_ws_free")


class ReconstructWorkspace:
    """src/core/workspace.rs:70-112."""

    def __init__(self, h):
        self._h = h
        self.goal = "all"
        self.required = None

    def targets(self) -> List[int]:
        n = _lib().rsgpu_reconstruct_ws_targets(self._h, None, 0)
        out = (ctypes.c_size_t * max(1, n))()
        _lib().rsgpu_reconstruct_ws_targets(self._h, out, n)
        return list(out)[:n]

    def __del__(self, _free=_free_handle):
        _free(self, "rsgpu_reconstruct_ws_free")


OP = {"encode": 0, "reconstruct": 1, "verify": 2}


def device_pointer_table(base_ptr: int, offsets) -> np.ndarray:
    """uint64 array of base_ptr + offsets (stripe-major shard pointers)."""
    return (np.uint64(base_ptr) + np.asarray(offsets, dtype=np.uint64)).astype(np.uint64)


class PreparedBatch:
    """Device-resident batch (see rsgpu_batch_prepare in include/rsgpu.h):
    launch() is a bare kernel launch on the current torch stream."""

    def __init__(self, codec: "ReedSolomon", op: str, ptr_table: np.ndarray, shard_len: int,
                 present: Optional[np.ndarray] = None, goal: str = "all"):
        self._codec = codec  # keep the codec alive
        self.op = op
        n = ptr_table.size // codec.total_shard_count()
        self.n_stripes = n
        self._ptrs = np.ascontiguousarray(ptr_table, np.uint64)
        self._present = None if present is None else np.ascontiguousarray(present, np.uint8)
        h = ctypes.c_void_p()
        _check(_lib().rsgpu_batch_prepare(
            codec._h, OP[op], n, self._ptrs.ctypes.data,
            None if self._present is None else self._present.ctypes.data, shard_len, GOAL[goal],
            ctypes.byref(h)))
        self._h = h

    def _stream(self):
        import torch

        return torch.cuda.current_stream().cuda_stream

    def launch(self, stream=None) -> None:
        _check(_lib().rsgpu_batch_launch(self._h, self._stream() if stream is None else stream))

    def verify_result(self) -> np.ndarray:
        ok = np.zeros(max(1, self.n_stripes), np.uint8)
        _check(_lib().rsgpu_batch_verify_result(self._h, ok.ctypes.data_as(U8P), self._stream()))
        return ok[: self.n_stripes].astype(bool)

    def kernel_count(self) -> int:
        return int(_lib().rsgpu_batch_kernel_count(self._h))

    def __del__(self, _free=_free_handle):
        _free(self, "rsgpu_batch_free")


def _mix_ops(ops, keep):
    """ctypes array of rsgpu_mix_op for a list of op dicts (see MixedBatch)."""
    n = len(ops)
    arr = (MixOp * max(n, 1))()
    for i, o in enumerate(ops):
        codec = o["codec"]
        ptrs = np.array([s.data_ptr() if hasattr(s, "data_ptr") else int(s) for s in o["shards"]], np.uint64)
        keep += [codec, ptrs, o["shards"]]
        arr[i].codec = codec._h
        arr[i].op = OP[o["op"]]
        arr[i].goal = GOAL[o.get("goal", "all")]
        arr[i].shards = ptrs.ctypes.data
        if o["op"] == "reconstruct":
            pres = np.ascontiguousarray(np.asarray(o["present"], dtype=np.uint8))
            keep.append(pres)
            arr[i].present = pres.ctypes.data
        arr[i].shard_len = int(o["shard_len"])
    return arr


class MixedBatch:
    """A mixed batch (rsgpu_mix_prepare in include/rsgpu.h): operations of
    different codecs, shard lengths and kinds in one persistent kernel.

    ``ops`` is a list of dicts with keys ``codec`` (ReedSolomon), ``op``
    ("encode" / "reconstruct" / "verify"), ``shards`` (k + m device pointers,
    or torch CUDA tensors), ``shard_len``, and for reconstruct ``present`` (k + m
    flags) and ``goal`` ("all" / "data").  ``plans`` optionally forces a plan
    (algo, tile) per operation."""

    def __init__(self, ops, planner: str = "fixed", order: str = "cost", graph: bool = True, ctas_per_sm: int = 0,
                 plans=None):
        self._keep = []
        n = len(ops)
        arr = _mix_ops(ops, self._keep)
        self._arr = arr
        self.n_ops = n
        opts = MixOptions()
        _lib().rsgpu_mix_options_default(ctypes.byref(opts))
        opts.planner = PLANNER[planner]
        opts.order = ORDER[order]
        opts.graph = 1 if graph else 0
        opts.ctas_per_sm = int(ctas_per_sm)
        h = ctypes.c_void_p()
        if plans is None:
            rc = _lib().rsgpu_mix_prepare(ctypes.addressof(arr), n, ctypes.byref(opts), ctypes.byref(h))
        else:
            parr = (Plan * max(n, 1))(*[Plan(int(a), int(t)) for a, t in plans])
            rc = _lib().rsgpu_mix_prepare_planned(ctypes.addressof(arr), n, ctypes.addressof(parr),
                                                  ctypes.byref(opts), ctypes.byref(h))
        _check(rc)
        self._h = h

    @staticmethod
    def _stream():
        import torch

        return torch.cuda.current_stream().cuda_stream

    def launch(self, stream=None) -> None:
        _check(_lib().rsgpu_mix_launch(self._h, self._stream() if stream is None else stream))

    def results(self) -> np.ndarray:
        ok = np.zeros(max(1, self.n_ops), np.uint8)
        _check(_lib().rsgpu_mix_results(self._h, ok.ctypes.data_as(U8P), self._stream()))
        return ok[: self.n_ops].astype(bool)

    def info(self) -> MixInfo:
        out = MixInfo()
        _check(_lib().rsgpu_mix_get_info(self._h, ctypes.byref(out)))
        return out

    def plans(self) -> List[tuple]:
        parr = (Plan * max(self.n_ops, 1))()
        _check(_lib().rsgpu_mix_get_plans(self._h, ctypes.addressof(parr), self.n_ops))
        return [parr[i].tuple() for i in range(self.n_ops)]

    def __del__(self, _free=_free_handle):
        _free(self, "rsgpu_mix_free")


class _StreamIO:
    """ctypes read / write callbacks over Python file-like objects; the first
    exception a callback raises is kept and re-raised as a StreamError."""

    def __init__(self, readers=None, writers=None):
        self.readers = readers
        self.writers = writers
        self.exc = None

        def read(ctx, shard, buf, cap):
            try:
                r = self.readers[shard]
                mv = memoryview((ctypes.c_uint8 * cap).from_address(buf)).cast("B")
                if hasattr(r, "readinto"):
                    n = r.readinto(mv)
                else:
                    data = r.read(cap)
                    n = len(data)
                    mv[:n] = data
                return int(n or 0)
            except Exception as e:  # noqa: BLE001 - handed back to the caller
                if self.exc is None:
                    self.exc = (shard, e)
                return -1

        def write(ctx, shard, buf, n):
            try:
                data = bytes((ctypes.c_uint8 * n).from_address(buf)) if n else b""
                w = self.writers[shard]
                view = memoryview(data)
                while view:
                    k = w.write(view)
                    if k is None:
                        break
                    if k == 0:
                        raise OSError("write returned 0")
                    view = view[k:]
                return 0
            except Exception as e:  # noqa: BLE001
                if self.exc is None:
                    self.exc = (shard, e)
                return -1

        self.read_fn = _READFN(read)
        self.write_fn = _WRITEFN(write)

    def check(self, rc, status):
        if rc == 0:
            return
        kind = STREAM_KINDS.get(status.kind, "codec")
        if rc == 106 and self.exc is not None:
            raise StreamError(kind, self.exc[0], self.exc[1])
        raise StreamError(kind, status.shard_index, RsError(rc))


def _stream_opts(block_size):
    o = StreamOptions()
    _lib().rsgpu_stream_options_default(ctypes.byref(o))
    if block_size is not None:
        o.block_size = int(block_size)
    return o


class Server:
    """The request server (rsgpu_server_* in include/rsgpu.h): continuous
    batching of requests onto the GPU.  Shards are NumPy uint8 arrays (host
    memory, staged through the device; pinned memory, e.g. torch tensors
    created with pin_memory=True and passed as .numpy(), is fastest), torch
    CUDA tensors, or raw device pointers (ints).  Buffers are kept alive by
    this object until their completion has been polled."""

    def __init__(self, device_budget=0, max_inflight=0, max_batch=0, streams=0, planner="model"):
        o = ServerOptions()
        _lib().rsgpu_server_options_default(ctypes.byref(o))
        o.device_budget = int(device_budget)
        o.max_inflight = int(max_inflight)
        o.max_batch = int(max_batch)
        o.streams = int(streams)
        o.planner = PLANNER[planner]
        h = ctypes.c_void_p()
        _check(_lib().rsgpu_server_new(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self._keep = {}
        self._next = 1

    def submit(self, codec: "ReedSolomon", op: str, shards, shard_len: int, present=None, goal="all",
               tag=None) -> int:
        first = shards[0]
        if isinstance(first, (int, np.integer)):
            mem, ptrs = MEM_DEVICE, np.array([int(x) for x in shards], np.uint64)
        elif _is_torch_cuda(first):
            mem, ptrs = MEM_DEVICE, np.array([x.data_ptr() for x in shards], np.uint64)
        else:
            mem, ptrs = MEM_HOST, np.array([x.ctypes.data for x in shards], np.uint64)
        if tag is None:
            tag = self._next
            self._next += 1
        pres = None
        if op == "reconstruct":
            pres = np.ascontiguousarray(np.asarray(present, dtype=np.uint8))
        r = Request()
        r.codec = codec._h
        r.op = OP[op]
        r.goal = GOAL[goal]
        r.shards = ptrs.ctypes.data
        r.present = None if pres is None else pres.ctypes.data
        r.shard_len = int(shard_len)
        r.mem = mem
        r.tag = int(tag)
        _check(_lib().rsgpu_server_submit(self._h, ctypes.byref(r)))
        self._keep[int(tag)] = (codec, shards)
        return int(tag)

    def poll(self, max_n: int = 4096, timeout_ms: int = 0):
        arr = (Completion * max_n)()
        n = int(_lib().rsgpu_server_poll(self._h, ctypes.addressof(arr), max_n, int(timeout_ms)))
        out = []
        for i in range(n):
            c = arr[i]
            self._keep.pop(int(c.tag), None)
            out.append(dict(tag=int(c.tag), status=int(c.status), ok=bool(c.ok), submit_s=c.submit_s,
                            admit_s=c.admit_s, done_s=c.done_s))
        return out

    def wait(self, n: int, timeout_ms: int = 60000):
        """Poll until n completions have arrived."""
        out = []
        while len(out) < n:
            got = self.poll(timeout_ms=timeout_ms)
            if not got:
                raise TimeoutError(f"{len(out)} of {n} completions")
            out += got
        return out

    def stats(self) -> dict:
        s = ServerStats()
        _check(_lib().rsgpu_server_get_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_ if f != "pad"}

    def close(self) -> None:
        if getattr(self, "_h", None) and _L is not None and getattr(_L, "rsgpu_server_free", None) is not None:
            _L.rsgpu_server_free(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        self.close()


class Tuner:
    """The process-wide plan table and cost model (rsgpu_tune, rsgpu_model_*
    in include/rsgpu.h).  Every call runs on the GPU through librsgpu.so."""

    @staticmethod
    def features(op: dict) -> np.ndarray:
        keep = []
        arr = _mix_ops([op], keep)
        out = np.zeros(MODEL_FEATURES, np.float32)
        _check(_lib().rsgpu_plan_features(ctypes.addressof(arr), out.ctypes.data))
        return out

    @staticmethod
    def tune(ops, target_bytes: int = 0, repeats: int = 0) -> int:
        keep = []
        arr = _mix_ops(ops, keep)
        o = TuneOptions(int(target_bytes), int(repeats), 0)
        done = ctypes.c_size_t()
        _check(_lib().rsgpu_tune(ctypes.addressof(arr), len(ops), ctypes.byref(o), ctypes.byref(done)))
        return int(done.value)

    @staticmethod
    def lookup(op: dict):
        keep = []
        arr = _mix_ops([op], keep)
        p = Plan()
        rc = _lib().rsgpu_tuner_lookup(ctypes.addressof(arr), ctypes.byref(p))
        if rc == 13:
            return None
        _check(rc)
        return p.tuple()

    @staticmethod
    def samples():
        n = int(_lib().rsgpu_tuner_samples(None, 0))
        arr = (TuneSample * max(n, 1))()
        n = int(_lib().rsgpu_tuner_samples(ctypes.addressof(arr), n))
        return [(np.array(arr[i].features[:], np.float32), arr[i].plan.tuple(), float(arr[i].gbps)) for i in range(n)]

    @staticmethod
    def table_size() -> int:
        return int(_lib().rsgpu_tuner_table_size())

    @staticmethod
    def save(path: str) -> None:
        _check(_lib().rsgpu_tuner_save(path.encode()))

    @staticmethod
    def load(path: str) -> None:
        _check(_lib().rsgpu_tuner_load(path.encode()))

    @staticmethod
    def clear() -> None:
        _lib().rsgpu_tuner_clear()

    # ---- cost model
    @staticmethod
    def param_count() -> int:
        return int(_lib().rsgpu_model_param_count())

    @staticmethod
    def model_ready() -> bool:
        return bool(_lib().rsgpu_model_ready())

    @staticmethod
    def get_params() -> np.ndarray:
        out = np.zeros(Tuner.param_count(), np.float32)
        _check(_lib().rsgpu_model_get_params(out.ctypes.data, out.size))
        return out

    @staticmethod
    def set_params(w) -> None:
        w = np.ascontiguousarray(w, np.float32)
        _check(_lib().rsgpu_model_set_params(w.ctypes.data, w.size))

    @staticmethod
    def train(x, y, mask, epochs=0, lr=0.0, seed=1) -> float:
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        mask = np.ascontiguousarray(mask, np.uint8)
        loss = ctypes.c_float()
        o = TrainOptions(int(epochs), float(lr), int(seed))
        _check(_lib().rsgpu_model_train(x.ctypes.data, y.ctypes.data, mask.ctypes.data, x.shape[0], ctypes.byref(o),
                                        ctypes.byref(loss)))
        return float(loss.value)

    @staticmethod
    def train_from_tuner(epochs=0, lr=0.0, seed=1) -> float:
        loss = ctypes.c_float()
        o = TrainOptions(int(epochs), float(lr), int(seed))
        _check(_lib().rsgpu_model_train_from_tuner(ctypes.byref(o), ctypes.byref(loss)))
        return float(loss.value)

    @staticmethod
    def predict(x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros((x.shape[0], MODEL_PLANS), np.float32)
        _check(_lib().rsgpu_model_predict(x.ctypes.data, x.shape[0], out.ctypes.data))
        return out

    @staticmethod
    def gradients(params, x, y, mask):
        params = np.ascontiguousarray(params, np.float32)
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        mask = np.ascontiguousarray(mask, np.uint8)
        loss = ctypes.c_float()
        g = np.zeros_like(params)
        _check(_lib().rsgpu_model_gradients(params.ctypes.data, x.ctypes.data, y.ctypes.data, mask.ctypes.data,
                                            x.shape[0], ctypes.byref(loss), g.ctypes.data))
        return float(loss.value), g


class ReedSolomon:
    """GPU drop-in for ``galois_8::ReedSolomon`` (and, with ``field='gf16'``,
    ``galois_16::ReedSolomon``)."""

    def __init__(self, data_shards: int, parity_shards: int, options: Optional[CodecOptions] = None,
                 *, field: str = "gf8", _custom=None):
        h = ctypes.c_void_p()
        L = _lib()
        if field == "gf16" and _custom is not None:
            rows = np.ascontiguousarray(np.array(_custom, np.uint8).reshape(-1))
            _check(L.rsgpu_codec_gf16_with_custom_matrix(data_shards, parity_shards, rows.ctypes.data_as(U8P),
                                                         ctypes.byref(h)))
        elif field == "gf16":
            _check(L.rsgpu_codec_new_gf16(data_shards, parity_shards, ctypes.byref(h)))
        elif _custom is not None:
            o = (options or CodecOptions())._c()
            rows = np.ascontiguousarray(np.array(_custom, np.uint8).reshape(-1))
            _check(L.rsgpu_codec_with_custom_matrix(data_shards, parity_shards,
                                                    rows.ctypes.data_as(U8P), ctypes.byref(o), ctypes.byref(h)))
        else:
            o = (options or CodecOptions())._c()
            _check(L.rsgpu_codec_new(data_shards, parity_shards, ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.field = field

    # src/core/codec.rs:264-266
    @classmethod
    def new(cls, data_shards, parity_shards):
        return cls(data_shards, parity_shards)

    # src/core/codec.rs:269-349
    @classmethod
    def with_options(cls, data_shards, parity_shards, options: CodecOptions):
        return cls(data_shards, parity_shards, options)

    # src/core/codec.rs:546-615
    @classmethod
    def with_custom_matrix(cls, data_shards, parity_shards, rows, options: Optional[CodecOptions] = None,
                           field: str = "gf8"):
        """rows: parity_shards x data_shards coefficients (galois_16: pairs
        [X coefficient, constant])."""
        return cls(data_shards, parity_shards, options, field=field, _custom=rows)

    def __del__(self, _free=_free_handle):
        _free(self, "rsgpu_codec_free")

    def data_shard_count(self) -> int:
        return _lib().rsgpu_data_shard_count(self._h)

    def parity_shard_count(self) -> int:
        return _lib().rsgpu_parity_shard_count(self._h)

    def total_shard_count(self) -> int:
        return _lib().rsgpu_total_shard_count(self._h)

    def codec_family(self) -> str:
        return {0: "classic", 1: "leopard_gf8", 2: "leopard_gf16"}[_lib().rsgpu_codec_family(self._h)]

    def encoding_matrix(self) -> np.ndarray:
        k, t = self.data_shard_count(), self.total_shard_count()
        es = 2 if self.field == "gf16" else 1
        out = np.zeros(t * k * es, np.uint8)
        _check(_lib().rsgpu_encoding_matrix(self._h, out.ctypes.data_as(U8P), out.size))
        return out.reshape((t, k, 2) if es == 2 else (t, k))

    def cache_stats(self) -> CacheStats:
        st = CacheStats()
        _check(_lib().rsgpu_get_cache_stats(self._h, ctypes.byref(st)))
        return st

    # ---------------------------------------------------------- encode
    def encode(self, shards: Sequence) -> None:
        """src/core/encode.rs:935-947."""
        mem, ptrs, lens, stream, keep = _buffer_info(list(shards))
        _check(_lib().rsgpu_encode(self._h, ptrs, lens, len(shards), mem, stream))

    def encode_sep(self, data: Sequence, parity: Sequence) -> None:
        """src/core/encode.rs:950-972."""
        mem, dp, dl, stream, k1 = _buffer_info(list(data))
        mem2, pp, pl, _, k2 = _buffer_info(list(parity))
        _check(_lib().rsgpu_encode_sep(self._h, dp, dl, len(data), pp, pl, len(parity), mem, stream))

    # ---------------------------------------------------------- verify
    def verify(self, shards: Sequence) -> bool:
        """src/core/verify.rs:72-94."""
        mem, ptrs, lens, stream, keep = _buffer_info(list(shards))
        ok = ctypes.c_int32(0)
        _check(_lib().rsgpu_verify(self._h, ptrs, lens, len(shards), ctypes.byref(ok), mem, stream))
        return bool(ok.value)

    def verify_with_workspace(self, shards: Sequence, ws: VerifyWorkspace) -> bool:
        """src/core/verify.rs:96-115."""
        mem, ptrs, lens, stream, keep = _buffer_info(list(shards))
        ok = ctypes.c_int32(0)
        _check(_lib().rsgpu_verify_with_workspace(self._h, ptrs, lens, len(shards), ws._h, ctypes.byref(ok), mem,
                                                  stream))
        return bool(ok.value)

    def verify_with_buffer(self, shards: Sequence, buffer: Sequence) -> bool:
        """src/core/verify.rs:157-176: the recomputed parity is left in `buffer`
        (m buffers of the shard length, host or device like the shards)."""
        shards, buffer = list(shards), list(buffer)
        mem, ptrs, lens, stream, keep = _buffer_info(shards + buffer)
        n = len(shards)
        ok = ctypes.c_int32(0)
        sp, sl = _slice_ptrs(ptrs, lens, 0, n)
        bp, bl = _slice_ptrs(ptrs, lens, n, len(buffer))
        _check(_lib().rsgpu_verify_with_buffer(self._h, sp, sl, n, bp, bl, len(buffer), ctypes.byref(ok), mem,
                                               stream))
        return bool(ok.value)

    # ---------------------------------------------------------- progressive recovery
    def decode_idx(self, dst: List, expect_input: Optional[Sequence[bool]], inputs: Sequence) -> None:
        """src/galois_8/policy.rs:543-700: XOR-accumulate into the non-None
        entries of `dst` (changed in place) the contributions of the non-None
        entries of `inputs`; expect_input=None merges partial results."""
        dst, inputs = list(dst), list(inputs)
        mem, ptrs, lens, stream, keep = _buffer_info(dst + inputs)
        nd = len(dst)
        dp, dl = _slice_ptrs(ptrs, lens, 0, nd)
        ip, il = _slice_ptrs(ptrs, lens, nd, len(inputs))
        if expect_input is None:
            ex, nex = None, 0
        else:
            ex, nex = _flags(expect_input, max(1, len(expect_input))), len(expect_input)
        _check(_lib().rsgpu_decode_idx(self._h, dp, dl, nd, ex, nex, ip, il, len(inputs), mem, stream))

    # ---------------------------------------------------------- reconstruct
    def _fill_targets(self, shards: List, goal: str, required=None) -> List:
        """Option<Vec<u8>> semantics: None entries are missing; they receive a
        freshly allocated buffer when they are recovery targets."""
        present = [s is not None for s in shards]
        filled = list(shards)
        known = [s for s in shards if s is not None]
        if len(shards) == self.total_shard_count() and known and sum(present) < len(shards):
            proto = known[0]
            n = self.data_shard_count()
            for i, s in enumerate(shards):
                if s is not None:
                    continue
                target = goal == "all" or (goal == "data" and i < n) or (
                    goal == "required" and required is not None and i < len(required) and required[i])
                if not target:
                    continue
                if _is_torch_cuda(proto):
                    import torch

                    filled[i] = torch.empty_like(proto)
                else:
                    filled[i] = np.zeros_like(proto)
        return filled

    def _reconstruct(self, shards: List, goal: str, required=None):
        present = [s is not None for s in shards]
        filled = self._fill_targets(shards, goal, required)
        mem, ptrs, lens, stream, keep = _buffer_info(filled)
        pres = _flags(present, len(shards))
        req = _flags(required or [], max(1, len(required or [])))
        _check(_lib().rsgpu_reconstruct(self._h, ptrs, lens, pres, len(shards), GOAL[goal], req,
                                        len(required or []), mem, stream))
        for i in range(len(shards)):
            shards[i] = filled[i]

    def reconstruct(self, shards: List) -> None:
        """src/core/reconstruct.rs:731-739: fills every missing entry (None) in place."""
        self._reconstruct(shards, "all")

    def reconstruct_data(self, shards: List) -> None:
        """src/core/reconstruct.rs:742-750."""
        self._reconstruct(shards, "data")

    def reconstruct_some(self, shards: List, required: Sequence[bool]) -> None:
        """src/core/reconstruct.rs:753-790."""
        self._reconstruct(shards, "required", list(required))

    def prepare_reconstruct_workspace(self, present: Sequence[bool], shard_len: int, goal: str = "all",
                                      required=None) -> ReconstructWorkspace:
        """src/core/reconstruct.rs:539-616: a plan for the erasure layout
        `present` (one flag per shard) at `shard_len` bytes."""
        h = ctypes.c_void_p()
        req = list(required or [])
        _check(_lib().rsgpu_prepare_reconstruct_ws(self._h, _flags(present, max(1, len(present))), len(present),
                                                   shard_len, GOAL[goal], _flags(req, max(1, len(req))), len(req),
                                                   ctypes.byref(h)))
        ws = ReconstructWorkspace(h)
        ws.goal, ws.required = goal, (list(required) if required is not None else None)
        return ws

    def prepare_reconstruct_data_workspace(self, present: Sequence[bool], shard_len: int) -> ReconstructWorkspace:
        """src/core/reconstruct.rs:546-555."""
        return self.prepare_reconstruct_workspace(present, shard_len, "data")

    def prepare_reconstruct_some_workspace(self, present: Sequence[bool], shard_len: int,
                                           required: Sequence[bool]) -> ReconstructWorkspace:
        """src/core/reconstruct.rs:557-590."""
        return self.prepare_reconstruct_workspace(present, shard_len, "required", list(required))

    def reconstruct_with_workspace(self, shards: List, ws: ReconstructWorkspace, present=None) -> None:
        """src/core/reconstruct.rs:618-640.  None entries are missing and
        receive new buffers when the plan targets them; with `present`, every
        entry is a buffer and the missing ones are outputs (ShardSlot)."""
        if present is None:
            present = [s is not None for s in shards]
            filled = self._fill_targets(shards, ws.goal, ws.required)
        else:
            filled = list(shards)
        mem, ptrs, lens, stream, keep = _buffer_info(filled)
        _check(_lib().rsgpu_reconstruct_with_ws(self._h, ws._h, ptrs, lens, _flags(present, max(1, len(present))),
                                                len(filled), mem, stream))
        for i in range(len(shards)):
            shards[i] = filled[i]

    # ---------------------------------------------------------- batched
    def encode_batch(self, stripes: Sequence[Sequence]) -> None:
        """Encode every stripe.  `stripes` is a list of shard lists, or one
        contiguous (stripes, k + m, length) uint8 array / CUDA tensor."""
        blk = _stripe_block(stripes)
        if blk is not None:
            mem, ptrs, length, stream, keep = blk
            _check_stripe_widths([stripes.shape[1]], self.total_shard_count())
            _check(_lib().rsgpu_encode_batch(self._h, len(stripes), ptrs, length, mem, stream))
            return
        _check_stripe_widths([len(st) for st in stripes], self.total_shard_count())
        flat = [s for st in stripes for s in st]
        mem, ptrs, lens, stream, keep = _buffer_info(flat)
        _check(_lib().rsgpu_encode_batch(self._h, len(stripes), ptrs, lens[0] if flat else 0, mem, stream))

    def reconstruct_batch(self, stripes: Sequence[Sequence], present: Sequence[Sequence[bool]], goal="all") -> None:
        blk = _stripe_block(stripes)
        if blk is not None:
            mem, ptrs, length, stream, keep = blk
            _check_stripe_widths([stripes.shape[1]], self.total_shard_count())
            n = len(stripes)
            flags, pres = _present_flags(present, n, self.total_shard_count())
            _check(_lib().rsgpu_reconstruct_batch(self._h, n, ptrs, pres, length, GOAL[goal], mem, stream))
            return
        _check_stripe_widths([len(st) for st in stripes], self.total_shard_count())
        flat = [s for st in stripes for s in st]
        mem, ptrs, lens, stream, keep = _buffer_info(flat)
        pres = _flags([p for row in present for p in row], len(flat))
        _check(_lib().rsgpu_reconstruct_batch(self._h, len(stripes), ptrs, pres, lens[0] if flat else 0,
                                              GOAL[goal], mem, stream))

    def prepare_batch(self, op: str, ptr_table: np.ndarray, shard_len: int, present=None,
                      goal: str = "all") -> PreparedBatch:
        return PreparedBatch(self, op, ptr_table, shard_len, present, goal)

    def verify_batch(self, stripes: Sequence[Sequence]) -> List[bool]:
        blk = _stripe_block(stripes)
        if blk is not None:
            mem, ptrs, length, stream, keep = blk
            _check_stripe_widths([stripes.shape[1]], self.total_shard_count())
            n = len(stripes)
            ok = np.zeros(max(1, n), dtype=np.uint8)
            _check(_lib().rsgpu_verify_batch(self._h, n, ptrs, length, ok.ctypes.data_as(U8P), mem, stream))
            return [bool(v) for v in ok[:n]]
        _check_stripe_widths([len(st) for st in stripes], self.total_shard_count())
        flat = [s for st in stripes for s in st]
        mem, ptrs, lens, stream, keep = _buffer_info(flat)
        ok = (ctypes.c_uint8 * max(1, len(stripes)))()
        _check(_lib().rsgpu_verify_batch(self._h, len(stripes), ptrs, lens[0] if flat else 0, ok, mem, stream))
        return [bool(v) for v in list(ok)[: len(stripes)]]

    # ---- block streaming (src/core/stream.rs:650-1000)
    def encode_stream(self, data, parity, block_size=None) -> None:
        """Read data shards from `data` (file-like objects) block by block
        and write the parity to `parity` (file-like objects)."""
        k = self.data_shard_count()
        io = _StreamIO(readers=list(data), writers={k + i: w for i, w in enumerate(parity)})
        st = StreamStatus()
        rc = _lib().rsgpu_encode_stream(self._h, len(data), io.read_fn, None, len(parity), io.write_fn, None,
                                        ctypes.byref(_stream_opts(block_size)), ctypes.byref(st))
        io.check(rc, st)

    def verify_stream(self, shards, block_size=None) -> bool:
        io = _StreamIO(readers=list(shards))
        ok = I32()
        st = StreamStatus()
        rc = _lib().rsgpu_verify_stream(self._h, len(shards), io.read_fn, None, ctypes.byref(_stream_opts(block_size)),
                                        ctypes.byref(ok), ctypes.byref(st))
        io.check(rc, st)
        return bool(ok.value)

    def reconstruct_stream_from(self, readers, writers, block_size=None) -> None:
        """readers[i] / writers[i]: a file-like object or None; exactly one of
        the two per shard (present shards have a reader)."""
        total = self.total_shard_count()
        for cnt in (len(readers), len(writers)):
            if cnt != total:
                raise StreamError("codec", 0, RsError(1 if cnt < total else 2))
        has_r = np.array([r is not None for r in readers], np.uint8)
        has_w = np.array([w is not None for w in writers], np.uint8)
        io = _StreamIO(readers=list(readers), writers=list(writers))
        st = StreamStatus()
        rc = _lib().rsgpu_reconstruct_stream_from(self._h, total, has_r.ctypes.data_as(U8P), io.read_fn, None,
                                                  has_w.ctypes.data_as(U8P), io.write_fn, None,
                                                  ctypes.byref(_stream_opts(block_size)), ctypes.byref(st))
        io.check(rc, st)

    def reconstruct_stream(self, shards, block_size=None) -> None:
        """shards: one io.BytesIO per shard (src/core/stream.rs:839-946);
        empty ones are missing and receive the recovered bytes, present ones
        are read from the start."""
        total = self.total_shard_count()
        if len(shards) != total:
            raise StreamError("codec", 0, RsError(1 if len(shards) < total else 2))
        if self.codec_family() != "classic" or self.field != "gf8":
            raise StreamError("codec", 0, RsError(15))
        present = [len(s.getbuffer()) > 0 for s in shards]
        if not any(present):
            return
        for s, p in zip(shards, present):
            if p:
                s.seek(0)
        self.reconstruct_stream_from([s if p else None for s, p in zip(shards, present)],
                                     [None if p else s for s, p in zip(shards, present)], block_size)

    # ---- incremental parity (src/core/encode.rs:889-930, 1048-1120)
    def encode_single(self, i_data: int, shards: Sequence) -> None:
        mem, ptrs, lens, stream, keep = _buffer_info(shards)
        _check(_lib().rsgpu_encode_single(self._h, int(i_data), ptrs, lens, len(shards), mem, stream))

    def encode_single_sep(self, i_data: int, data, parity: Sequence) -> None:
        mem, ptrs, lens, stream, keep = _buffer_info(list(parity) + [data])
        n = len(parity)
        _check(_lib().rsgpu_encode_single_sep(self._h, int(i_data), ptrs[n], lens[n], ptrs, lens, n, mem, stream))

    def update(self, old_data: Sequence, new_data: Sequence, parity: Sequence) -> None:
        """new_data[j] is None for an unchanged data shard."""
        changed = [x for x in new_data if x is not None]
        mem, ptrs, lens, stream, keep = _buffer_info(list(old_data) + changed + list(parity))
        no, nc, npar = len(old_data), len(changed), len(parity)
        new_ptrs = (ctypes.c_void_p * max(1, len(new_data)))()
        new_lens = (ctypes.c_size_t * max(1, len(new_data)))()
        c = 0
        for j, x in enumerate(new_data):
            if x is not None:
                new_ptrs[j] = ptrs[no + c]
                new_lens[j] = lens[no + c]
                c += 1
        par_ptrs = (ctypes.c_void_p * max(1, npar))(*[ptrs[no + nc + r] for r in range(npar)])
        par_lens = (ctypes.c_size_t * max(1, npar))(*[lens[no + nc + r] for r in range(npar)])
        _check(_lib().rsgpu_update(self._h, ptrs, lens, no, new_ptrs, new_lens, len(new_data), par_ptrs, par_lens,
                                   npar, mem, stream))

    # ---- layout and format (src/core/codec.rs:476-538, src/core/format.rs:168-220)
    def split(self, data) -> List[np.ndarray]:
        """Data shards of `data` (bytes / uint8 array), zero-padded."""
        buf = np.frombuffer(bytes(data), np.uint8) if not isinstance(data, np.ndarray) else np.ascontiguousarray(data)
        sl = int(_lib().rsgpu_split_shard_len(self._h, buf.size))
        k = self.data_shard_count()
        out = np.zeros(k * sl, np.uint8)
        _check(_lib().rsgpu_split(self._h, buf.ctypes.data if buf.size else None, buf.size,
                                  out.ctypes.data if out.size else None, out.size))
        return [out[i * sl:(i + 1) * sl] for i in range(k)]

    def join(self, shards: Sequence, out_len: int) -> bytes:
        arrs = [np.ascontiguousarray(np.asarray(s, np.uint8)) for s in shards]
        ptrs = (ctypes.c_void_p * max(1, len(arrs)))(*[a.ctypes.data for a in arrs])
        lens = (ctypes.c_size_t * max(1, len(arrs)))(*[a.size for a in arrs])
        cap = min(out_len, sum(a.size for a in arrs))
        out = np.zeros(max(cap, 1), np.uint8)
        wrote = ctypes.c_size_t()
        _check(_lib().rsgpu_join(self._h, ptrs, lens, len(arrs), out.ctypes.data, out_len, ctypes.byref(wrote)))
        return out[: wrote.value].tobytes()

    def stable_id_bytes(self) -> bytes:
        n = ctypes.c_size_t()
        _check(_lib().rsgpu_format_id(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, np.uint8)
        _check(_lib().rsgpu_format_id(self._h, out.ctypes.data, out.size, ctypes.byref(n)))
        return out.tobytes()


class SBSError(Exception):
    """src/errors.rs SBSError: TooManyCalls, LeftoverShards or an RSError."""

    def __init__(self, kind: str, rs_error: Optional[RsError] = None):
        self.kind = kind
        self.rs_error = rs_error
        super().__init__(kind if rs_error is None else f"{kind}: {rs_error}")


class ShardByShard:
    """src/core/shard_by_shard.rs: encode the data shards one at a time."""

    def __init__(self, codec: ReedSolomon):
        self.codec = codec
        self.cur_input = 0

    def parity_ready(self) -> bool:
        return self.cur_input == self.codec.data_shard_count()

    def reset(self) -> None:
        if self.cur_input > 0 and not self.parity_ready():
            raise SBSError("LeftoverShards")
        self.cur_input = 0

    def reset_force(self) -> None:
        self.cur_input = 0

    def cur_input_index(self) -> int:
        return self.cur_input

    def encode(self, shards: Sequence) -> None:
        if self.parity_ready():
            raise SBSError("TooManyCalls")
        try:
            self.codec.encode_single(self.cur_input, shards)
        except RsError as e:
            raise SBSError("RSError", e) from None
        self.cur_input += 1

    def encode_sep(self, data: Sequence, parity: Sequence) -> None:
        if self.parity_ready():
            raise SBSError("TooManyCalls")
        k, m = self.codec.data_shard_count(), self.codec.parity_shard_count()
        # sbs_encode_sep_checks: data and parity piece counts, equal slices
        try:
            if len(data) != k:
                raise RsError(3 if len(data) < k else 4)
            if len(parity) != m:
                raise RsError(5 if len(parity) < m else 6)
            # check_slices!(multi => data, multi => parity), src/macros.rs:172-178
            for group in (data, parity):
                if len(group[0]) == 0:
                    raise RsError(11)
                if any(len(x) != len(group[0]) for x in group):
                    raise RsError(9)
            if len(data[0]) != len(parity[0]):
                raise RsError(9)
            self.codec.encode_single_sep(self.cur_input, data[self.cur_input], parity)
        except RsError as e:
            raise SBSError("RSError", e) from None
        self.cur_input += 1
