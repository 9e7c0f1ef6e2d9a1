"""Python binding of libtoposzp_b200.so (the B200 topology path).

Mirrors the reference's CUDA topology interface (SZp/include/szp_cuda_topology.cuh,
szp_cuda_topology_3d.cuh, szp_cuda_decompress.cuh): the same entry points, the
same argument meaning, the same CriticalPoint layouts and compressed bytes.
The device-pointer functions take torch CUDA tensors.

The library is required: importing this module on a machine without the
built library raises, there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtoposzp_b200.so")

CP2_DT = np.dtype([("x", "<i4"), ("y", "<i4"), ("type", "<i4"),
                   ("quantized_bin", "<i4"), ("sort_position", "<i4")])
CP3_DT = np.dtype([("x", "<i4"), ("y", "<i4"), ("z", "<i4"), ("type", "<i4"),
                   ("quantized_bin", "<i4"), ("sort_position", "<i4")])

EXPORTS = [
    "szp_cuda_find_critical_points",
    "szp_cuda_sort_critical_points_by_original_data",
    "szp_cuda_compress_sort_positions",
    "szp_cuda_float_compress_randomaccess_topology_preserved",
    "szp_cuda_find_critical_points_3d",
    "szp_cuda_sort_critical_points_3d",
    "szp_cuda_compress_sort_positions_3d",
    "szp_cuda_float_compress_topology_3d",
    "szp_cuda_double_compress_topology_3d",
    "szp_cuda_float_decompress_randomaccess_topology_preserved",
    "szp_cuda_decompress_sort_positions",
    "szp_b200_last_error",
    "szp_b200_version",
    "szp_b200_ctx_create",
    "szp_b200_ctx_destroy",
    "szp_b200_topo_bound",
    "szp_b200_sort_bound",
    "szp_b200_topo_compress_dev",
    "szp_b200_topo_decompress_dev",
    "szp_b200_topo_postprocess_dev",
    "szp_b200_ctx_stage_times",
    "szp_b200_ctx_launches",
    "szp_b200_topo_compress_host",
    "szp_b200_topo_decompress_host",
    "szp_b200_topo_encode_noalloc",
    "szp_b200_topo_check",
    "szp_b200_double_compress_topology_3d_dev",
    "szp_b200_f64_topo_scratch_bytes",
    "szp_cuda_float_compress_randomaccess",
    "szp_cuda_float_compress_randomaccess_arg",
    "szp_cuda_double_compress_randomaccess",
    "szp_cuda_double_compress_randomaccess_arg",
    "szp_cuda_float_compress_threadblock",
    "szp_cuda_float_compress_threadblock_arg",
    "szp_cuda_double_compress_threadblock",
    "szp_cuda_double_compress_threadblock_arg",
    "szp_cuda_float_direct_predict_quantization",
    "szp_cuda_float_threadblock_predict_quantization",
    "szp_cuda_float_decompress_randomaccess",
    "szp_cuda_float_decompress_randomaccess_arg",
    "szp_cuda_double_decompress_randomaccess",
    "szp_cuda_double_decompress_randomaccess_arg",
    "szp_cuda_float_decompress_threadblock",
    "szp_cuda_float_decompress_threadblock_arg",
    "szp_cuda_double_decompress_threadblock",
    "szp_cuda_double_decompress_threadblock_arg",
    "szp_b200_plain_bound",
    "szp_b200_plain_compress_dev",
    "szp_b200_plain_decompress_dev",
    "szp_b200_topo_encode_slab_dev",
    "szp_b200_pair_bins_dev",
    "szp_b200_rank_pairs_dev",
    "szp_b200_encode_ints_dev",
    "szp_b200_selftest_bounded_wait",
    "szp_b200_container_bound",
    "szp_b200_container_from_streams_dev",
    "szp_b200_container_decompress_dev",
    "szp_b200_batch_create",
    "szp_b200_batch_destroy",
    "szp_b200_batch_configure",
    "szp_b200_batch_compress",
    "szp_b200_batch_reserve",
    "szp_b200_batch_tuning",
    "szp_b200_batch_ctx",
    "szp_b200_server_create",
    "szp_b200_server_destroy",
    "szp_b200_server_now",
    "szp_b200_server_reserve",
    "szp_b200_server_submit",
    "szp_b200_server_wait",
    "szp_b200_server_drain",
    "szp_b200_server_run_trace",
    "szp_b200_server_stats",
]

OP_COMPRESS = 0
OP_DECOMPRESS = 1


class ToposzpError(RuntimeError):
    pass


class Geom(C.Structure):
    _fields_ = [("nd", C.c_int), ("dims", C.c_int * 3)]


class Sizes(C.Structure):
    _fields_ = [("topo_bytes", C.c_size_t), ("sort_bytes", C.c_size_t),
                ("cp_count", C.c_size_t), ("extrema_count", C.c_size_t)]


class SlabSizes(C.Structure):
    _fields_ = [("payload_bytes", C.c_size_t), ("cp_count", C.c_size_t), ("extrema_count", C.c_size_t)]


class ServerConfig(C.Structure):
    _fields_ = [("slots", C.c_int), ("max_batch", C.c_int), ("blockSize", C.c_int),
                ("hbm_budget", C.c_size_t)]


class Request(C.Structure):
    _fields_ = [("op", C.c_int), ("blockSize", C.c_int), ("geom", Geom), ("errBound", C.c_float),
                ("rel", C.c_int), ("postprocess", C.c_int), ("d_data", C.c_void_p), ("d_out", C.c_void_p),
                ("d_topo", C.c_void_p), ("topo_bytes", C.c_size_t), ("d_sort", C.c_void_p),
                ("sort_bytes", C.c_size_t), ("sizes", Sizes), ("abs_eb", C.c_float), ("status", C.c_int),
                ("done", C.c_int), ("t_arrival", C.c_double), ("t_start", C.c_double),
                ("t_done", C.c_double), ("message", C.c_char * 96)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_ulonglong), ("completed", C.c_ulonglong), ("failed", C.c_ulonglong),
                ("batches", C.c_ulonglong), ("batched_requests", C.c_ulonglong),
                ("max_inflight_bytes", C.c_size_t), ("max_concurrent", C.c_int)]


class TopoReport(C.Structure):
    _fields_ = [("orig_cps", C.c_uint64 * 4), ("dec_cps", C.c_uint64 * 4), ("preserved", C.c_uint64),
                ("lost", C.c_uint64), ("changed", C.c_uint64), ("new_cps", C.c_uint64),
                ("lost_by_type", C.c_uint64 * 4), ("pairs", C.c_uint64 * 4), ("violations", C.c_uint64 * 4),
                ("over_1eb", C.c_uint64), ("over_2eb", C.c_uint64), ("max_err", C.c_double)]

    def as_dict(self) -> dict:
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if hasattr(v, "__len__") else v
        return d


class BatchField(C.Structure):
    _fields_ = [("d_data", C.c_void_p), ("geom", Geom), ("errBound", C.c_float), ("rel", C.c_int),
                ("d_topo", C.c_void_p), ("topo_cap", C.c_size_t), ("d_sort", C.c_void_p),
                ("sort_cap", C.c_size_t), ("sizes", Sizes), ("abs_eb", C.c_float)]


def build() -> str:
    """Compile the library in place (nvcc, sm_100a)."""
    subprocess.run(["make", "-s", "-C", HERE, "-j8"], check=True)
    return LIB_PATH


_lib = None
_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ToposzpError("libtoposzp_b200.so is not built (run build())")
        L = C.CDLL(LIB_PATH)
        vp, sz, i, f = C.c_void_p, C.c_size_t, C.c_int, C.c_float
        sig = {
            "szp_cuda_find_critical_points": (vp, [vp, C.POINTER(sz), i, i, f]),
            "szp_cuda_find_critical_points_3d": (vp, [vp, C.POINTER(sz), i, i, i, f]),
            "szp_cuda_sort_critical_points_by_original_data": (None, [vp, sz, vp, i]),
            "szp_cuda_sort_critical_points_3d": (None, [vp, sz, vp, i, i]),
            "szp_cuda_compress_sort_positions": (vp, [vp, sz, C.POINTER(sz), i]),
            "szp_cuda_compress_sort_positions_3d": (vp, [vp, sz, C.POINTER(sz), i]),
            "szp_cuda_float_compress_randomaccess_topology_preserved":
                (vp, [vp, C.POINTER(sz), f, sz, i, vp, i, i, i]),
            "szp_cuda_float_compress_topology_3d": (vp, [vp, C.POINTER(sz), f, sz, i, vp, i, i, i, i]),
            "szp_cuda_double_compress_topology_3d": (vp, [vp, C.POINTER(sz), C.c_double, sz, i, vp, i, i, i,
                                                          i]),
            "szp_cuda_float_decompress_randomaccess_topology_preserved":
                (None, [C.POINTER(vp), sz, f, i, vp, C.POINTER(vp)]),
            "szp_cuda_decompress_sort_positions": (vp, [vp, sz, i]),
            "szp_b200_last_error": (C.c_char_p, []),
            "szp_b200_version": (C.c_char_p, []),
            "szp_b200_ctx_create": (vp, [vp]),
            "szp_b200_ctx_destroy": (None, [vp]),
            "szp_b200_topo_bound": (sz, [sz, i]),
            "szp_b200_sort_bound": (sz, [sz, i]),
            "szp_b200_topo_compress_dev": (i, [vp, vp, Geom, f, i, vp, vp, vp, C.POINTER(Sizes)]),
            "szp_b200_topo_decompress_dev": (i, [vp, vp, sz, vp, sz, vp, Geom, f, i, vp, vp, i]),
            "szp_b200_topo_postprocess_dev": (i, [vp, vp, vp, vp, vp, sz, Geom, f, i]),
            "szp_b200_ctx_stage_times": (i, [vp, C.POINTER(C.c_char_p), C.POINTER(C.c_float), i]),
            "szp_b200_ctx_launches": (C.c_ulonglong, [vp]),
            "szp_b200_topo_compress_host": (i, [vp, vp, Geom, f, i, vp, sz, vp, sz, C.POINTER(Sizes)]),
            "szp_b200_topo_decompress_host": (i, [vp, vp, sz, vp, sz, Geom, f, i, vp, i]),
            "szp_b200_topo_encode_noalloc": (i, [vp, Geom, f, i, vp, sz, C.POINTER(sz), vp]),
            "szp_b200_topo_check": (i, [vp, vp, vp, Geom, f, C.POINTER(TopoReport)]),
            "szp_b200_selftest_bounded_wait": (i, [i, i, C.POINTER(i), C.POINTER(f)]),
            "szp_b200_double_compress_topology_3d_dev": (i, [vp, vp, Geom, C.c_double, i, vp, sz, i, vp, sz,
                                                             C.POINTER(sz), vp]),
            "szp_b200_f64_topo_scratch_bytes": (sz, [sz, sz, i]),
            "szp_cuda_float_compress_randomaccess": (vp, [vp, C.POINTER(sz), f, sz, i]),
            "szp_cuda_float_compress_randomaccess_arg": (None, [vp, vp, C.POINTER(sz), f, sz, i]),
            "szp_cuda_double_compress_randomaccess": (vp, [vp, C.POINTER(sz), C.c_double, sz, i]),
            "szp_cuda_double_compress_randomaccess_arg": (None, [vp, vp, C.POINTER(sz), C.c_double, sz, i]),
            "szp_cuda_float_compress_threadblock": (vp, [vp, C.POINTER(sz), f, sz, i]),
            "szp_cuda_float_compress_threadblock_arg": (None, [vp, vp, C.POINTER(sz), f, sz, i]),
            "szp_cuda_double_compress_threadblock": (vp, [vp, C.POINTER(sz), C.c_double, sz, i]),
            "szp_cuda_double_compress_threadblock_arg": (None, [vp, vp, C.POINTER(sz), C.c_double, sz, i]),
            "szp_cuda_float_direct_predict_quantization": (vp, [vp, C.POINTER(sz), f, sz, i]),
            "szp_cuda_float_threadblock_predict_quantization": (vp, [vp, C.POINTER(sz), f, sz, i]),
            "szp_cuda_float_decompress_randomaccess": (vp, [sz, f, i, vp]),
            "szp_cuda_float_decompress_randomaccess_arg": (None, [vp, sz, f, i, vp]),
            "szp_cuda_double_decompress_randomaccess": (vp, [sz, C.c_double, i, vp]),
            "szp_cuda_double_decompress_randomaccess_arg": (None, [vp, sz, C.c_double, i, vp]),
            "szp_cuda_float_decompress_threadblock": (vp, [sz, f, i, vp]),
            "szp_cuda_float_decompress_threadblock_arg": (None, [vp, sz, f, i, vp]),
            "szp_cuda_double_decompress_threadblock": (vp, [sz, C.c_double, i, vp]),
            "szp_cuda_double_decompress_threadblock_arg": (None, [vp, sz, C.c_double, i, vp]),
            "szp_b200_topo_encode_slab_dev": (i, [vp, vp, sz, Geom, f, i, sz, sz, vp, sz, vp, sz,
                                                  C.POINTER(SlabSizes)]),
            "szp_b200_pair_bins_dev": (i, [vp, vp, sz, f, vp]),
            "szp_b200_rank_pairs_dev": (i, [vp, vp, sz, sz, f, vp]),
            "szp_b200_encode_ints_dev": (i, [vp, vp, sz, i, vp, sz, C.POINTER(sz)]),
            "szp_b200_plain_bound": (sz, [sz, i, i, i]),
            "szp_b200_plain_compress_dev": (i, [vp, vp, i, sz, C.c_double, i, i, vp, sz, C.POINTER(sz)]),
            "szp_b200_plain_decompress_dev": (i, [vp, vp, sz, i, sz, C.c_double, i, vp]),
            "szp_b200_container_bound": (sz, [sz, i, i]),
            "szp_b200_container_from_streams_dev": (i, [vp, vp, sz, vp, sz, Geom, i, sz, i, vp, sz,
                                                        C.POINTER(sz)]),
            "szp_b200_container_decompress_dev": (i, [vp, vp, sz, Geom, f, i, vp, vp, i]),
            "szp_b200_batch_create": (vp, [vp, i]),
            "szp_b200_batch_destroy": (None, [vp]),
            "szp_b200_batch_configure": (i, [vp, i, i]),
            "szp_b200_batch_compress": (i, [vp, C.POINTER(BatchField), i]),
            "szp_b200_batch_reserve": (i, [vp, i, sz]),
            "szp_b200_batch_tuning": (i, [vp, C.POINTER(C.c_int), C.POINTER(C.c_float), i]),
            "szp_b200_batch_ctx": (vp, [vp]),
            "szp_b200_server_create": (vp, [C.POINTER(ServerConfig)]),
            "szp_b200_server_destroy": (None, [vp]),
            "szp_b200_server_now": (C.c_double, [vp]),
            "szp_b200_server_reserve": (i, [vp, sz]),
            "szp_b200_server_submit": (i, [vp, C.POINTER(Request)]),
            "szp_b200_server_wait": (i, [vp, C.POINTER(Request), C.c_double]),
            "szp_b200_server_drain": (i, [vp, C.c_double]),
            "szp_b200_server_run_trace": (i, [vp, C.POINTER(Request), i, C.POINTER(C.c_double), C.c_double]),
            "szp_b200_server_stats": (i, [vp, C.POINTER(ServerStats)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().szp_b200_last_error().decode()


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _take(ptr, nbytes, dtype):
    if not ptr:
        return None
    buf = (C.c_char * nbytes).from_address(ptr)
    out = np.frombuffer(bytes(buf), dtype=dtype).copy()
    _libc.free(ptr)
    return out


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ---------------------------------------------------------------------------
# reference entry points (host buffers)
# ---------------------------------------------------------------------------

def find_critical_points(data: np.ndarray, eb: float) -> np.ndarray:
    """szp_cuda_find_critical_points[_3d]: CPs in raster order."""
    d = _f32(data)
    k = C.c_size_t(0)
    if d.ndim == 2:
        ptr = lib().szp_cuda_find_critical_points(_p(d), C.byref(k), d.shape[0], d.shape[1], eb)
        dt = CP2_DT
    else:
        ptr = lib().szp_cuda_find_critical_points_3d(_p(d), C.byref(k), *d.shape, eb)
        dt = CP3_DT
    if not ptr:
        err = last_error()
        if err:
            raise ToposzpError(err)
        return np.zeros(0, dtype=dt)
    return _take(ptr, k.value * dt.itemsize, dt)


def sort_critical_points(cps: np.ndarray, data: np.ndarray) -> np.ndarray:
    """szp_cuda_sort_critical_points_by_original_data / _3d (returns a sorted copy)."""
    cp = np.ascontiguousarray(cps).copy()
    d = _f32(data)
    if len(cp) == 0:
        return cp
    if cp.dtype == CP2_DT:
        lib().szp_cuda_sort_critical_points_by_original_data(_p(cp), len(cp), _p(d), d.shape[-1])
    else:
        lib().szp_cuda_sort_critical_points_3d(_p(cp), len(cp), _p(d), d.shape[1], d.shape[2])
    err = last_error()
    if err:
        raise ToposzpError(err)
    return cp


def compress_sort_positions(cps: np.ndarray, block_size: int) -> bytes:
    cp = np.ascontiguousarray(cps)
    sz = C.c_size_t(0)
    if cp.dtype == CP2_DT:
        ptr = lib().szp_cuda_compress_sort_positions(_p(cp), len(cp), C.byref(sz), block_size)
    else:
        ptr = lib().szp_cuda_compress_sort_positions_3d(_p(cp), len(cp), C.byref(sz), block_size)
    if not ptr:
        err = last_error()
        if err:
            raise ToposzpError(err)
        return b""
    return _take(ptr, sz.value, np.uint8).tobytes()


def compress_topology(data: np.ndarray, eb: float, block_size: int, cps: np.ndarray) -> bytes:
    """szp_cuda_float_compress_randomaccess_topology_preserved (2D) or
    szp_cuda_float_compress_topology_3d (3D)."""
    d = _f32(data)
    cp = np.ascontiguousarray(cps)
    sz = C.c_size_t(0)
    if d.ndim == 2:
        ptr = lib().szp_cuda_float_compress_randomaccess_topology_preserved(
            _p(d), C.byref(sz), eb, d.size, block_size, _p(cp) if len(cp) else None, len(cp),
            d.shape[0], d.shape[1])
    else:
        ptr = lib().szp_cuda_float_compress_topology_3d(
            _p(d), C.byref(sz), eb, d.size, block_size, _p(cp) if len(cp) else None, len(cp),
            *d.shape)
    if not ptr:
        raise ToposzpError(last_error() or "compression returned NULL")
    return _take(ptr, sz.value, np.uint8).tobytes()


def double_compress_topology_3d(data: np.ndarray, eb: float, block_size: int, cps: np.ndarray) -> bytes:
    """szp_cuda_double_compress_topology_3d: a 3D float64 field, the critical
    points that mark its types (CP3_DT records), the topology stream."""
    d = np.ascontiguousarray(data, dtype=np.float64)
    if d.ndim != 3:
        raise ValueError("a 3D field is required")
    cp = np.ascontiguousarray(cps)
    sz = C.c_size_t(0)
    ptr = lib().szp_cuda_double_compress_topology_3d(
        _p(d), C.byref(sz), float(eb), d.size, block_size, _p(cp) if len(cp) else None, len(cp), *d.shape)
    if not ptr:
        raise ToposzpError(last_error() or "compression returned NULL")
    return _take(ptr, sz.value, np.uint8).tobytes()


def plain_compress(data: np.ndarray, eb: float, block_size: int, threadblock: bool = False) -> bytes:
    """szp_cuda_{float,double}_compress_{randomaccess,threadblock}: the whole
    stream [T eb][u64 0][body] (T the dtype of data)."""
    dbl = np.asarray(data).dtype == np.float64
    d = np.ascontiguousarray(data, dtype=np.float64 if dbl else np.float32).reshape(-1)
    kind = ("double" if dbl else "float") + ("_compress_threadblock" if threadblock else "_compress_randomaccess")
    sz = C.c_size_t(0)
    ptr = getattr(lib(), "szp_cuda_" + kind)(_p(d), C.byref(sz), float(eb), d.size, block_size)
    if not ptr:
        raise ToposzpError(last_error() or "compression returned NULL")
    return _take(ptr, sz.value, np.uint8).tobytes()


def plain_decompress(stream: bytes, n: int, eb: float, block_size: int, dtype=np.float32,
                     threadblock: bool = False) -> np.ndarray:
    """szp_cuda_{float,double}_decompress_*: stream is the compressor's whole
    output; the entry point receives it after its T header, as the
    reference's callers pass it."""
    dbl = np.dtype(dtype) == np.float64
    es = 8 if dbl else 4
    s = np.frombuffer(stream, dtype=np.uint8)[es:].copy()
    out = np.zeros(n, dtype=np.float64 if dbl else np.float32)
    kind = ("double" if dbl else "float") + ("_decompress_threadblock_arg" if threadblock
                                             else "_decompress_randomaccess_arg")
    getattr(lib(), "szp_cuda_" + kind)(_p(out), n, float(eb), block_size, _p(s))
    err = last_error()
    if err:
        raise ToposzpError(err)
    return out


def predict_quantization(data: np.ndarray, eb: float, threadblock: bool = False) -> np.ndarray:
    d = _f32(data).reshape(-1)
    name = "szp_cuda_float_threadblock_predict_quantization" if threadblock else \
        "szp_cuda_float_direct_predict_quantization"
    ptr = getattr(lib(), name)(_p(d), None, float(eb), d.size, 64)
    if not ptr:
        raise ToposzpError(last_error() or "quantization returned NULL")
    return _take(ptr, 4 * d.size, np.int32)


def decompress_topology(stream: bytes, n: int, eb: float, block_size: int):
    """szp_cuda_float_decompress_randomaccess_topology_preserved -> (data, FN)."""
    s = np.frombuffer(stream, dtype=np.uint8)
    outp, fnp = C.c_void_p(), C.c_void_p()
    lib().szp_cuda_float_decompress_randomaccess_topology_preserved(
        C.byref(outp), n, eb, block_size, _p(s), C.byref(fnp))
    if not outp.value:
        raise ToposzpError(last_error() or "decompression returned NULL")
    return _take(outp.value, 4 * n, np.float32), _take(fnp.value, 4 * n, np.int32)


def decompress_sort_positions(stream: bytes, count: int, block_size: int) -> np.ndarray:
    s = np.frombuffer(stream, dtype=np.uint8)
    ptr = lib().szp_cuda_decompress_sort_positions(_p(s), count, block_size)
    if not ptr:
        raise ToposzpError(last_error() or "sort-position decompression returned NULL")
    return _take(ptr, 4 * count, np.int32)


# ---------------------------------------------------------------------------
# device-pointer entry points (torch CUDA tensors)
# ---------------------------------------------------------------------------

def geom_of(shape) -> Geom:
    g = Geom()
    g.nd = len(shape)
    for i, v in enumerate(shape):
        g.dims[i] = int(v)
    return g


def encode_noalloc(d_data, shape, eb: float, block_size: int, d_topo, stream_handle: int = 0) -> int:
    """Topology stream of a device field into the caller's uint8 device
    tensor d_topo, with no allocation inside the library; returns the stream
    length in bytes.  Calls on one device must not overlap."""
    import torch
    n = int(np.prod(shape))
    if not (d_data.is_cuda and d_data.dtype == torch.float32 and d_data.is_contiguous()):
        raise ToposzpError("encode_noalloc: d_data must be a contiguous float32 CUDA tensor")
    if d_data.numel() != n:
        raise ToposzpError("encode_noalloc: d_data holds %d elements, the shape %s needs %d"
                           % (d_data.numel(), tuple(shape), n))
    if not (d_topo.is_cuda and d_topo.dtype == torch.uint8 and d_topo.is_contiguous()):
        raise ToposzpError("encode_noalloc: d_topo must be a contiguous uint8 CUDA tensor")
    if d_topo.device != d_data.device:
        raise ToposzpError("encode_noalloc: d_data and d_topo are on different devices")
    nbytes = C.c_size_t(0)
    rc = lib().szp_b200_topo_encode_noalloc(
        C.c_void_p(d_data.data_ptr()), geom_of(shape), eb, block_size, C.c_void_p(d_topo.data_ptr()),
        d_topo.numel(), C.byref(nbytes), C.c_void_p(stream_handle) if stream_handle else None)
    if rc:
        raise ToposzpError(last_error())
    return int(nbytes.value)


class Context:
    """A reusable device workspace bound to a CUDA stream (0 = own stream)."""

    def __init__(self, stream_handle: int = 0):
        self.ptr = lib().szp_b200_ctx_create(C.c_void_p(stream_handle) if stream_handle else None)
        if not self.ptr:
            raise ToposzpError(last_error())

    def close(self):
        if self.ptr:
            lib().szp_b200_ctx_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def compress(self, d_data, shape, eb: float, block_size: int = 64, index=True):
        """Fused compression of a device field -> (topo, sort, index, sizes).
        topo / sort are uint8 device tensors sized to the streams."""
        import torch
        n = int(np.prod(shape))
        L = lib()
        topo = torch.empty(L.szp_b200_topo_bound(n, block_size), dtype=torch.uint8, device=d_data.device)
        sort = torch.empty(L.szp_b200_sort_bound(n, block_size), dtype=torch.uint8, device=d_data.device)
        nb = (n + block_size - 1) // block_size
        idx = torch.empty(2 * nb, dtype=torch.int64, device=d_data.device) if index else None
        sizes = Sizes()
        rc = L.szp_b200_topo_compress_dev(
            self.ptr, C.c_void_p(d_data.data_ptr()), geom_of(shape), eb, block_size,
            C.c_void_p(topo.data_ptr()), C.c_void_p(sort.data_ptr()),
            C.c_void_p(idx.data_ptr()) if idx is not None else None, C.byref(sizes))
        if rc:
            raise ToposzpError(last_error())
        return topo, sort, idx, sizes

    def decompress(self, topo, topo_bytes, sort, sort_bytes, index, shape, eb: float,
                   block_size: int = 64, postprocess: int = 1, out=None, types=None):
        """Fused decompression of device streams.  index: the block index from
        compress(), or None to parse the block offsets on the device."""
        import torch
        n = int(np.prod(shape))
        if out is None:
            out = torch.empty(n, dtype=torch.float32, device=topo.device)
        rc = lib().szp_b200_topo_decompress_dev(
            self.ptr, C.c_void_p(topo.data_ptr()), topo_bytes,
            C.c_void_p(sort.data_ptr()) if sort is not None else None, sort_bytes,
            C.c_void_p(index.data_ptr()) if index is not None else None, geom_of(shape), eb, block_size,
            C.c_void_p(out.data_ptr()), C.c_void_p(types.data_ptr()) if types is not None else None,
            postprocess)
        if rc:
            raise ToposzpError(last_error())
        return out

    def stage_times(self):
        """[(stage, ms)] of the last call, from CUDA events on the workspace stream."""
        names = (C.c_char_p * 24)()
        ms = (C.c_float * 24)()
        k = lib().szp_b200_ctx_stage_times(self.ptr, names, ms, 24)
        return [(names[i].decode(), float(ms[i])) for i in range(k)]

    def launches(self) -> int:
        return int(lib().szp_b200_ctx_launches(self.ptr))

    def compress_host(self, h_data: np.ndarray, eb: float, block_size: int, h_topo: np.ndarray,
                      h_sort: np.ndarray) -> Sizes:
        """Host-buffer fused compression (h_* may be pinned numpy views)."""
        sizes = Sizes()
        rc = lib().szp_b200_topo_compress_host(
            self.ptr, h_data.ctypes.data_as(C.c_void_p), geom_of(h_data.shape), eb, block_size,
            h_topo.ctypes.data_as(C.c_void_p), h_topo.nbytes, h_sort.ctypes.data_as(C.c_void_p),
            h_sort.nbytes, C.byref(sizes))
        if rc:
            raise ToposzpError(last_error())
        return sizes

    def decompress_host(self, h_topo: np.ndarray, topo_bytes: int, h_sort: np.ndarray, sort_bytes: int,
                        shape, eb: float, block_size: int, h_out: np.ndarray, postprocess: int = 1):
        rc = lib().szp_b200_topo_decompress_host(
            self.ptr, h_topo.ctypes.data_as(C.c_void_p), topo_bytes,
            h_sort.ctypes.data_as(C.c_void_p) if sort_bytes else None, sort_bytes, geom_of(shape), eb,
            block_size, h_out.ctypes.data_as(C.c_void_p), postprocess)
        if rc:
            raise ToposzpError(last_error())
        return h_out

    def to_container(self, topo, topo_bytes, sort, sort_bytes, shape, block_size, extrema, threads=1):
        """.SZp container (OpenMP layout, `threads` chunks) of device streams -> uint8 device tensor."""
        import torch
        n = int(np.prod(shape))
        L = lib()
        out = torch.empty(L.szp_b200_container_bound(n, block_size, threads), dtype=torch.uint8, device=topo.device)
        nb = C.c_size_t(0)
        rc = L.szp_b200_container_from_streams_dev(
            self.ptr, C.c_void_p(topo.data_ptr()), topo_bytes,
            C.c_void_p(sort.data_ptr()) if sort is not None and sort_bytes else None, sort_bytes,
            geom_of(shape), block_size, extrema, threads, C.c_void_p(out.data_ptr()), out.numel(), C.byref(nb))
        if rc:
            raise ToposzpError(last_error())
        return out[: nb.value]

    def decompress_container(self, cont, shape, eb: float, block_size: int = 64, postprocess: int = 1,
                             out=None, types=None):
        import torch
        n = int(np.prod(shape))
        if out is None:
            out = torch.empty(n, dtype=torch.float32, device=cont.device)
        rc = lib().szp_b200_container_decompress_dev(
            self.ptr, C.c_void_p(cont.data_ptr()), cont.numel(), geom_of(shape), eb, block_size,
            C.c_void_p(out.data_ptr()), C.c_void_p(types.data_ptr()) if types is not None else None, postprocess)
        if rc:
            raise ToposzpError(last_error())
        return out

    def topo_check(self, d_orig, d_dec, shape, eb: float) -> dict:
        """Topology report of a decompressed device field against the original."""
        rep = TopoReport()
        rc = lib().szp_b200_topo_check(self.ptr, C.c_void_p(d_orig.data_ptr()), C.c_void_p(d_dec.data_ptr()),
                                       geom_of(shape), eb, C.byref(rep))
        if rc:
            raise ToposzpError(last_error())
        return rep.as_dict()

    def compress_f64(self, d_data, shape, eb: float, block_size: int, d_cps, count: int, d_out,
                     passes: int = 3, d_q=None) -> int:
        """fp64 3D topology compression of device memory (d_cps: CriticalPoint3D
        records on the device, or None); returns the stream length in d_out."""
        out_len = C.c_size_t(0)
        rc = lib().szp_b200_double_compress_topology_3d_dev(
            self.ptr, C.c_void_p(d_data.data_ptr()), geom_of(shape), float(eb), block_size,
            C.c_void_p(d_cps.data_ptr()) if d_cps is not None else None, count, passes,
            C.c_void_p(d_out.data_ptr()), d_out.numel() * d_out.element_size(), C.byref(out_len),
            C.c_void_p(d_q.data_ptr()) if d_q is not None else None)
        if rc:
            raise ToposzpError(last_error())
        return out_len.value

    def plain_compress(self, d_data, eb: float, block_size: int, d_out, threadblock: bool = False) -> int:
        """Plain-codec stream of a device tensor (float32 or float64) into d_out
        (uint8 device tensor); returns its length."""
        import torch
        dbl = d_data.dtype == torch.float64
        out_len = C.c_size_t(0)
        rc = lib().szp_b200_plain_compress_dev(self.ptr, C.c_void_p(d_data.data_ptr()), int(dbl), d_data.numel(),
                                               float(eb), block_size, int(threadblock), C.c_void_p(d_out.data_ptr()),
                                               d_out.numel(), C.byref(out_len))
        if rc:
            raise ToposzpError(last_error())
        return out_len.value

    def plain_decompress(self, d_stream, length: int, n: int, eb: float, block_size: int, d_out) -> None:
        """Random-access decode of a device stream written by plain_compress
        (the whole stream, T header included) into d_out."""
        import torch
        dbl = d_out.dtype == torch.float64
        es = 8 if dbl else 4
        rc = lib().szp_b200_plain_decompress_dev(self.ptr, C.c_void_p(d_stream.data_ptr() + es), length - es,
                                                 int(dbl), n, float(eb), block_size, C.c_void_p(d_out.data_ptr()))
        if rc:
            raise ToposzpError(last_error())

    def postprocess(self, d_data, d_orig, d_types_int, d_sp, shape, eb: float, axis_stencil=False):
        rc = lib().szp_b200_topo_postprocess_dev(
            self.ptr, C.c_void_p(d_data.data_ptr()), C.c_void_p(d_orig.data_ptr()),
            C.c_void_p(d_types_int.data_ptr()),
            C.c_void_p(d_sp.data_ptr()) if d_sp is not None and d_sp.numel() else None,
            0 if d_sp is None else d_sp.numel(), geom_of(shape), eb, int(axis_stencil))
        if rc:
            raise ToposzpError(last_error())
        return d_data


class Batch:
    """Batched compression of many device fields (one persistent launch per
    codec pass, CUDA-graph replay, autotuned CTA shapes)."""

    def __init__(self, block_size: int = 64, stream_handle: int = 0):
        self.B = block_size
        self.ptr = lib().szp_b200_batch_create(C.c_void_p(stream_handle) if stream_handle else None, block_size)
        if not self.ptr:
            raise ToposzpError(last_error())
        self._bufs = []

    def close(self):
        if self.ptr:
            lib().szp_b200_batch_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def configure(self, use_graphs: bool = True, autotune: int = 1):
        if lib().szp_b200_batch_configure(self.ptr, int(use_graphs), int(autotune)):
            raise ToposzpError(last_error())

    def buffers(self, items):
        """Device output buffers sized for items [(tensor, shape, err, rel)]."""
        import torch
        L = lib()
        out = []
        for t, shape, _, _ in items:
            n = int(np.prod(shape))
            out.append((torch.empty(L.szp_b200_topo_bound(n, self.B), dtype=torch.uint8, device=t.device),
                        torch.empty(L.szp_b200_sort_bound(n, self.B), dtype=torch.uint8, device=t.device)))
        return out

    def compress(self, items, bufs=None):
        """items: [(device float tensor, shape, err, rel)].  Returns
        [(topo, sort, Sizes, abs_eb)] with topo / sort the device buffers."""
        if bufs is None:
            bufs = self.buffers(items)
        arr = (BatchField * len(items))()
        for k, ((t, shape, err, rel), (tb, sb)) in enumerate(zip(items, bufs)):
            arr[k].d_data = t.data_ptr()
            arr[k].geom = geom_of(shape)
            arr[k].errBound = err
            arr[k].rel = int(bool(rel))
            arr[k].d_topo = tb.data_ptr()
            arr[k].topo_cap = tb.numel()
            arr[k].d_sort = sb.data_ptr()
            arr[k].sort_cap = sb.numel()
        if lib().szp_b200_batch_compress(self.ptr, arr, len(items)):
            raise ToposzpError(last_error())
        return [(tb, sb, arr[k].sizes, float(arr[k].abs_eb)) for k, (tb, sb) in enumerate(bufs)]

    def tuning(self):
        shape = (C.c_int * 4)()
        ms = (C.c_float * 16)()
        tuned = lib().szp_b200_batch_tuning(self.ptr, shape, ms, 16)
        return {"tuned": bool(tuned), "topo_threads": shape[0], "topo_ctas_per_sm": shape[1],
                "sort_threads": shape[2], "sort_ctas_per_sm": shape[3],
                "topo_candidates_ms": [round(float(x), 4) for x in ms if x > 0]}

    def stage_times(self):
        c = lib().szp_b200_batch_ctx(self.ptr)
        names = (C.c_char_p * 24)()
        ms = (C.c_float * 24)()
        k = lib().szp_b200_ctx_stage_times(c, names, ms, 24)
        return [(names[i].decode(), float(ms[i])) for i in range(k)]

    def launches(self) -> int:
        return int(lib().szp_b200_ctx_launches(lib().szp_b200_batch_ctx(self.ptr)))


class Server:
    """Request server with continuous batching (compress / decompress of
    device-resident fields, HBM admission budget, per-request timing)."""

    def __init__(self, slots: int = 4, max_batch: int = 64, block_size: int = 64, hbm_budget: int = 0):
        cfg = ServerConfig(slots, max_batch, block_size, hbm_budget)
        self.B = block_size
        self.ptr = lib().szp_b200_server_create(C.byref(cfg))
        if not self.ptr:
            raise ToposzpError(last_error())

    def close(self):
        if self.ptr:
            lib().szp_b200_server_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reserve(self, max_elements: int):
        """Grows every worker's workspace for requests of up to max_elements."""
        if lib().szp_b200_server_reserve(self.ptr, int(max_elements)):
            raise ToposzpError(last_error())

    def compress_request(self, d_data, shape, err, rel, d_topo, d_sort) -> Request:
        r = Request()
        r.op, r.blockSize, r.geom = OP_COMPRESS, self.B, geom_of(shape)
        r.errBound, r.rel = err, int(bool(rel))
        r.d_data = d_data.data_ptr()
        r.d_topo, r.topo_bytes = d_topo.data_ptr(), d_topo.numel()
        r.d_sort, r.sort_bytes = d_sort.data_ptr(), d_sort.numel()
        return r

    def decompress_request(self, d_topo, topo_bytes, d_sort, sort_bytes, shape, abs_eb, d_out,
                           postprocess: int = 1) -> Request:
        r = Request()
        r.op, r.blockSize, r.geom = OP_DECOMPRESS, self.B, geom_of(shape)
        r.errBound, r.postprocess = abs_eb, postprocess
        r.d_topo, r.topo_bytes = d_topo.data_ptr(), topo_bytes
        r.d_sort, r.sort_bytes = (d_sort.data_ptr() if d_sort is not None else None), sort_bytes
        r.d_out = d_out.data_ptr()
        return r

    def run_trace(self, reqs, arrivals=None, timeout: float = 600.0):
        """Submits the Request array reqs (a ctypes array) at the given arrival
        offsets in seconds (None: all at once) and waits for all of them."""
        arr = (C.c_double * len(reqs))(*arrivals) if arrivals is not None else None
        rc = lib().szp_b200_server_run_trace(self.ptr, reqs, len(reqs), arr, timeout)
        if rc < 0:
            raise ToposzpError(last_error())
        if rc > 0:
            raise ToposzpError("server trace timed out")
        for r in reqs:
            if r.status != 0:
                raise ToposzpError(r.message.decode())
        return reqs

    def stats(self) -> dict:
        st = ServerStats()
        lib().szp_b200_server_stats(self.ptr, C.byref(st))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}
