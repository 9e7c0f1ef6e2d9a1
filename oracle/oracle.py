"""TEST INFRASTRUCTURE ONLY: ctypes bindings for the C oracle (liboracle.so)
and for the reference CPU library built from the reference sources
(_ref/libszp_ref.so).  Only tests, the smoke check and the benchmark's
CPU-baseline / reference legs import this module; the product library never
does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libszp_ref.so")
# the reference's CUDA library for the path (runs on a GPU; fixtures and the
# reference GPU timing only)
REF_CUDA_SO = os.path.join(HERE, "_ref", "libszp_ref_cuda.so")
# reference source tree: the build argument, else $TOPOSZP_REF_SRC (no default:
# without either, an already built _ref/libszp_ref.so is used as it is)
REF_SRC = os.environ.get("TOPOSZP_REF_SRC")


class CP2(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("type", C.c_int),
                ("quantized_bin", C.c_int), ("sort_position", C.c_int)]


class CP3(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("z", C.c_int), ("type", C.c_int),
                ("quantized_bin", C.c_int), ("sort_position", C.c_int)]


CP2_DT = np.dtype([("x", "<i4"), ("y", "<i4"), ("type", "<i4"),
                   ("quantized_bin", "<i4"), ("sort_position", "<i4")])
CP3_DT = np.dtype([("x", "<i4"), ("y", "<i4"), ("z", "<i4"), ("type", "<i4"),
                   ("quantized_bin", "<i4"), ("sort_position", "<i4")])


def build(ref: bool = True, ref_src: str | None = None) -> None:
    """Compile liboracle.so (always) and the reference library from the
    reference sources at ref_src (or $TOPOSZP_REF_SRC) when they are there."""
    src = ref_src or REF_SRC
    targets = ["oracle"]
    args = []
    if ref and src and os.path.isdir(os.path.join(src, "SZp")):
        targets += ["ref", "refcpu2d", "refcuda"]
        args = ["REF=" + src]
    subprocess.run(["make", "-s", "-C", HERE] + args + targets, check=True)


_ora = None
_ref = None


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def lib():
    global _ora
    if _ora is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        L = C.CDLL(ORACLE_SO)
        vp, sz, i, f, d = C.c_void_p, C.c_size_t, C.c_int, C.c_float, C.c_double
        sig = {
            "ora_quantize": (i, [f, d]),
            "ora_bitcount": (C.c_uint, [C.c_uint]),
            "ora_block_bytes": (sz, [sz, C.c_uint, i, i]),
            "ora_find_cp_2d": (sz, [vp, i, i, f, vp]),
            "ora_find_cp_3d": (sz, [vp, i, i, i, f, vp]),
            "ora_sort_cp_2d": (None, [vp, sz, vp, i]),
            "ora_sort_cp_3d": (None, [vp, sz, vp, i, i]),
            "ora_mark_types_2d": (None, [vp, sz, i, i, vp]),
            "ora_mark_types_3d": (None, [vp, sz, i, i, i, vp]),
            "ora_extract_sp_2d": (sz, [vp, sz, vp]),
            "ora_extract_sp_3d": (sz, [vp, sz, vp]),
            "ora_encode_topo": (sz, [vp, sz, f, i, vp, i, vp]),
            "ora_encode_ints": (sz, [vp, sz, i, i, vp]),
            "ora_double_compress_topo_3d": (sz, [vp, sz, d, i, vp, i, i, i, i, vp, vp]),
            "ora_plain_compress": (sz, [vp, i, sz, d, i, i, vp]),
            "ora_plain_bound": (sz, [sz, i, i]),
            "ora_plain_decompress_ra": (i, [vp, sz, sz, d, i, i, vp, C.POINTER(sz)]),
            "ora_plain_decompress_tb": (i, [vp, sz, sz, d, i, i, vp, C.POINTER(sz)]),
            "ora_topo_bound": (sz, [sz, i]),
            "ora_ints_bound": (sz, [sz, i]),
            "ora_decode_topo": (i, [vp, sz, sz, f, i, vp, vp, C.POINTER(sz)]),
            "ora_decode_ints": (i, [vp, sz, sz, i, vp, C.POINTER(sz)]),
            "ora_post_2d": (i, [vp, vp, vp, vp, sz, i, i, f, C.POINTER(i)]),
            "ora_post_3d": (i, [vp, vp, vp, vp, sz, i, i, i, f, i, C.POINTER(i)]),
            "ora_stencils_2d": (None, [vp, vp, vp, vp, sz, i, i, f]),
            "ora_enforce_2d": (None, [vp, vp, vp, i, i, f, f]),
            "ora_rbf_2d": (i, [vp, vp, vp, i, i, f, f]),
            "ora_stencils_3d": (None, [vp, vp, vp, vp, sz, i, i, i, f]),
            "ora_enforce_3d": (None, [vp, vp, vp, i, i, i, f, f]),
            "ora_rbf_3d": (i, [vp, vp, vp, i, i, i, f, f]),
            "ora_axis_saddles_3d": (i, [vp, vp, vp, i, i, i, f]),
            "ora_rel_to_abs": (f, [vp, sz, f]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _ora = L
    return _ora


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def reflib():
    """The reference's OpenMP library + driver post-processing."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            build(ref=True)
        L = C.CDLL(REF_SO)
        vp, sz, i, f = C.c_void_p, C.c_size_t, C.c_int, C.c_float
        sig = {
            "szp_find_critical_points": (vp, [vp, C.POINTER(sz), i, i, f]),
            "szp_find_critical_points_3d": (vp, [vp, C.POINTER(sz), i, i, i, f]),
            "szp_sort_critical_points_by_original_data": (None, [vp, sz, vp, i]),
            "szp_sort_critical_points_3d": (None, [vp, sz, vp, i, i]),
            "szp_compress_sort_positions": (vp, [vp, sz, C.POINTER(sz), i]),
            "szp_compress_sort_positions_3d": (vp, [vp, sz, C.POINTER(sz), i]),
            "szp_float_openmp_threadblock_randomaccess_topology_preserved":
                (vp, [vp, C.POINTER(sz), f, sz, i, vp, i, i, i]),
            "szp_float_compress_topology_3d": (vp, [vp, C.POINTER(sz), f, sz, i, vp, i, i, i, i]),
            "szp_float_decompress_openmp_threadblock_randomaccess_topology_preserved":
                (None, [C.POINTER(vp), sz, f, i, vp, C.POINTER(vp)]),
            "szp_decompress_sort_positions": (vp, [vp, sz, i]),
            "ref2d_stencils": (None, [vp, vp, vp, vp, i, i, f, sz]),
            "ref2d_enforce": (None, [vp, vp, vp, i, i, f, f]),
            "ref2d_rbf": (i, [vp, vp, vp, i, i, f, f]),
            "ref3d_stencils": (None, [vp, vp, vp, vp, i, i, i, f, sz]),
            "ref3d_enforce": (None, [vp, vp, vp, i, i, i, f, f]),
            "ref3d_rbf": (i, [vp, vp, vp, i, i, i, f, f]),
            "ref3d_axis_saddles": (i, [vp, vp, vp, i, i, i, f]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _ref = L
    return _ref


_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]


def _take(ptr, nbytes, dtype):
    """Copy a malloc'd reference buffer into numpy and free it."""
    if not ptr:
        return np.zeros(0, dtype=dtype)
    buf = (C.c_char * nbytes).from_address(ptr)
    out = np.frombuffer(bytes(buf), dtype=dtype).copy()
    _libc.free(ptr)
    return out


def set_ref_threads(n: int) -> None:
    """Set the OpenMP thread count used by the reference library."""
    gomp = C.CDLL("libgomp.so.1")
    gomp.omp_set_num_threads(C.c_int(int(n)))


# ---------------------------------------------------------------------------
# oracle wrappers (numpy in, numpy out)
# ---------------------------------------------------------------------------

def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def find_cp(data: np.ndarray, eb: float) -> np.ndarray:
    d = f32(data)
    L = lib()
    if d.ndim == 2:
        cap = max(1, (d.shape[0] - 2) * (d.shape[1] - 2))
        out = np.zeros(cap, dtype=CP2_DT)
        k = L.ora_find_cp_2d(_p(d), d.shape[0], d.shape[1], eb, _p(out))
    else:
        cap = max(1, (d.shape[0] - 2) * (d.shape[1] - 2) * (d.shape[2] - 2))
        out = np.zeros(cap, dtype=CP3_DT)
        k = L.ora_find_cp_3d(_p(d), d.shape[0], d.shape[1], d.shape[2], eb, _p(out))
    return out[:k].copy()


def sort_cp(cp: np.ndarray, data: np.ndarray) -> np.ndarray:
    cp = cp.copy()
    d = f32(data)
    if len(cp) == 0:
        return cp
    if d.ndim == 2:
        lib().ora_sort_cp_2d(_p(cp), len(cp), _p(d), d.shape[1])
    else:
        lib().ora_sort_cp_3d(_p(cp), len(cp), _p(d), d.shape[1], d.shape[2])
    return cp


def mark_types(cp: np.ndarray, dims) -> np.ndarray:
    n = int(np.prod(dims))
    t = np.zeros(n, dtype=np.uint8)
    if len(cp):
        if len(dims) == 2:
            lib().ora_mark_types_2d(_p(cp), len(cp), dims[0], dims[1], _p(t))
        else:
            lib().ora_mark_types_3d(_p(cp), len(cp), dims[0], dims[1], dims[2], _p(t))
    return t


def extract_sp(cp: np.ndarray) -> np.ndarray:
    sp = np.zeros(max(1, len(cp)), dtype=np.int32)
    if cp.dtype == CP2_DT:
        e = lib().ora_extract_sp_2d(_p(cp), len(cp), _p(sp))
    else:
        e = lib().ora_extract_sp_3d(_p(cp), len(cp), _p(sp))
    return sp[:e].copy()


def encode_topo(data: np.ndarray, eb: float, B: int, types=None, cpu_layout=False) -> bytes:
    d = f32(data).reshape(-1)
    n = d.size
    out = np.zeros(lib().ora_topo_bound(n, B), dtype=np.uint8)
    t = None if types is None else np.ascontiguousarray(types, dtype=np.uint8).reshape(-1)
    m = lib().ora_encode_topo(_p(d), n, eb, B, _p(t), int(cpu_layout), _p(out))
    return out[:m].tobytes()


def double_compress_topo_3d(data: np.ndarray, eb: float, B: int, types, dims, passes: int = 3,
                            with_q: bool = False):
    """fp64 3D topology stream: double quantization, `passes` saddle-repair
    passes in q-space, int blocks with 2-bit tags (CUDA layout).  With with_q,
    also returns the repaired ints."""
    d = np.ascontiguousarray(data, dtype=np.float64).reshape(-1)
    n = d.size
    t = np.ascontiguousarray(types, dtype=np.uint8).reshape(-1)
    assert t.size == n
    out = np.zeros(lib().ora_topo_bound(n, B), dtype=np.uint8)
    q = np.zeros(n, dtype=np.int32)
    m = lib().ora_double_compress_topo_3d(_p(d), n, float(eb), B, _p(t), dims[0], dims[1], dims[2],
                                          passes, _p(q), _p(out))
    return (out[:m].tobytes(), q) if with_q else out[:m].tobytes()


def plain_compress(data: np.ndarray, eb: float, B: int, threadblock: bool = False) -> bytes:
    """Plain-codec stream [T eb][u64 0][body] of the CUDA compressors (T: the
    dtype of data, float32 or float64).  eb is the caller's bound (a float32
    value for float32 data)."""
    dbl = np.asarray(data).dtype == np.float64
    d = np.ascontiguousarray(data, dtype=np.float64 if dbl else np.float32).reshape(-1)
    ebv = float(eb) if dbl else float(np.float32(eb))
    out = np.zeros(lib().ora_plain_bound(d.size, B, int(dbl)), dtype=np.uint8)
    m = lib().ora_plain_compress(_p(d), int(dbl), d.size, ebv, B, int(threadblock), _p(out))
    return out[:m].tobytes()


def plain_decompress(stream: bytes, n: int, eb: float, B: int, dtype=np.float32, threadblock: bool = False,
                     pad: int = 4096):
    """Values of a plain stream (the compressor's whole output; decoded from
    after its T header, as the reference's callers pass it)."""
    dbl = np.dtype(dtype) == np.float64
    es = 8 if dbl else 4
    body = np.frombuffer(stream, dtype=np.uint8)[es:]
    buf = np.zeros(body.size + pad, dtype=np.uint8)
    buf[: body.size] = body
    out = np.zeros(max(1, n), dtype=np.float64 if dbl else np.float32)
    used = C.c_size_t(0)
    fn = lib().ora_plain_decompress_tb if threadblock else lib().ora_plain_decompress_ra
    ebv = float(eb) if dbl else float(np.float32(eb))
    rc = fn(_p(buf), buf.size, n, ebv, B, int(dbl), _p(out), C.byref(used))
    if rc:
        raise ValueError("malformed plain stream")
    return out[:n], used.value


def encode_ints(v: np.ndarray, B: int, cpu_layout=False) -> bytes:
    a = np.ascontiguousarray(v, dtype=np.int32)
    out = np.zeros(lib().ora_ints_bound(a.size, B), dtype=np.uint8)
    m = lib().ora_encode_ints(_p(a), a.size, B, int(cpu_layout), _p(out))
    return out[:m].tobytes()


def decode_topo(stream: bytes, n: int, eb: float, B: int):
    pad = np.zeros(8 * n + 1024 + 64, dtype=np.uint8)
    s = np.frombuffer(stream, dtype=np.uint8)
    pad[: s.size] = s
    out = np.zeros(n, dtype=np.float32)
    fn = np.zeros(n, dtype=np.int32)
    used = C.c_size_t(0)
    rc = lib().ora_decode_topo(_p(pad), pad.size, n, eb, B, _p(out), _p(fn), C.byref(used))
    if rc:
        raise ValueError("malformed topology stream")
    return out, fn, used.value


def decode_ints(stream: bytes, n: int, B: int):
    pad = np.zeros(4 * n + 4 + 1024, dtype=np.uint8)
    s = np.frombuffer(stream, dtype=np.uint8)
    pad[: s.size] = s
    out = np.zeros(max(1, n), dtype=np.int32)
    used = C.c_size_t(0)
    rc = lib().ora_decode_ints(_p(pad), pad.size, n, B, _p(out), C.byref(used))
    if rc:
        raise ValueError("malformed sort-position stream")
    return out[:n], used.value


def post(data: np.ndarray, orig: np.ndarray, fn: np.ndarray, sp, eb: float,
         axis_stencil=False):
    """Full post-processing (stencils, enforcement, RBF [, axis pattern])."""
    d = f32(data).copy()
    o = f32(orig)
    t = np.ascontiguousarray(fn, dtype=np.int32)
    s = None if sp is None or len(sp) == 0 else np.ascontiguousarray(sp, dtype=np.int32)
    ns = 0 if s is None else s.size
    r = C.c_int(0)
    if d.ndim == 2:
        lib().ora_post_2d(_p(d), _p(o), _p(t), _p(s), ns, d.shape[0], d.shape[1], eb,
                          C.byref(r))
    else:
        lib().ora_post_3d(_p(d), _p(o), _p(t), _p(s), ns, d.shape[0], d.shape[1],
                          d.shape[2], eb, int(axis_stencil), C.byref(r))
    return d, r.value


def rel_to_abs(data: np.ndarray, rel: float) -> float:
    d = f32(data).reshape(-1)
    return float(lib().ora_rel_to_abs(_p(d), d.size, rel))


# ---------------------------------------------------------------------------
# reference wrappers (the reference's own code, one OpenMP thread unless set)
# ---------------------------------------------------------------------------

def ref_find_cp(data: np.ndarray, eb: float) -> np.ndarray:
    d = f32(data)
    L = reflib()
    k = C.c_size_t(0)
    if d.ndim == 2:
        ptr = L.szp_find_critical_points(_p(d), C.byref(k), d.shape[0], d.shape[1], eb)
        return _take(ptr, k.value * CP2_DT.itemsize, CP2_DT)
    ptr = L.szp_find_critical_points_3d(_p(d), C.byref(k), d.shape[0], d.shape[1],
                                        d.shape[2], eb)
    return _take(ptr, k.value * CP3_DT.itemsize, CP3_DT)


def ref_sort_cp(cp: np.ndarray, data: np.ndarray) -> np.ndarray:
    cp = cp.copy()
    d = f32(data)
    if len(cp) == 0:
        return cp
    if d.ndim == 2:
        reflib().szp_sort_critical_points_by_original_data(_p(cp), len(cp), _p(d), d.shape[1])
    else:
        reflib().szp_sort_critical_points_3d(_p(cp), len(cp), _p(d), d.shape[1], d.shape[2])
    return cp


def ref_compress_sp(cp: np.ndarray, B: int) -> bytes:
    sz = C.c_size_t(0)
    if cp.dtype == CP2_DT:
        ptr = reflib().szp_compress_sort_positions(_p(cp), len(cp), C.byref(sz), B)
    else:
        ptr = reflib().szp_compress_sort_positions_3d(_p(cp), len(cp), C.byref(sz), B)
    return _take(ptr, sz.value, np.uint8).tobytes()


def ref_compress_topo(data: np.ndarray, eb: float, B: int, cp: np.ndarray) -> bytes:
    d = f32(data)
    sz = C.c_size_t(0)
    if d.ndim == 2:
        ptr = reflib().szp_float_openmp_threadblock_randomaccess_topology_preserved(
            _p(d), C.byref(sz), eb, d.size, B, _p(cp), len(cp), d.shape[0], d.shape[1])
    else:
        ptr = reflib().szp_float_compress_topology_3d(
            _p(d), C.byref(sz), eb, d.size, B, _p(cp), len(cp), *d.shape)
    return _take(ptr, sz.value, np.uint8).tobytes()


def ref_decompress_topo(stream: bytes, n: int, eb: float, B: int):
    s = np.frombuffer(stream + b"\0" * 64, dtype=np.uint8).copy()
    outp, fnp = C.c_void_p(), C.c_void_p()
    reflib().szp_float_decompress_openmp_threadblock_randomaccess_topology_preserved(
        C.byref(outp), n, eb, B, _p(s), C.byref(fnp))
    return _take(outp.value, 4 * n, np.float32), _take(fnp.value, 4 * n, np.int32)


def ref_decompress_sp(stream_after_count: bytes, e: int, B: int) -> np.ndarray:
    s = np.frombuffer(stream_after_count + b"\0" * 64, dtype=np.uint8).copy()
    ptr = reflib().szp_decompress_sort_positions(_p(s), e, B)
    return _take(ptr, 4 * e, np.int32)


REF_CPU2D_SO = os.path.join(HERE, "_ref", "libszp_ref_cpu2d.so")
_ref_cpu2d = None


def ref_cpu2d_available() -> bool:
    return os.path.exists(REF_CPU2D_SO)


def ref_post_cpu2d(data, fn, sp, eb: float):
    """The reference CPU decompress driver's own 2D post-processing sequence
    (example/testfloat_decompress_fastmode1_topology.cc:826-966) on a copy of
    data: returns (field, false-negative saddles, sigma, ksize, eps)."""
    global _ref_cpu2d
    if _ref_cpu2d is None:
        L = C.CDLL(REF_CPU2D_SO)
        L.ref2dcpu_post.restype = C.c_int
        L.ref2dcpu_post.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_float,
                                    C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_float)]
        _ref_cpu2d = L
    d = f32(data).copy()
    t = np.ascontiguousarray(fn, dtype=np.int32)
    s = None if sp is None or len(sp) == 0 else np.ascontiguousarray(sp, dtype=np.int32)
    sig, ks, ep = C.c_double(0), C.c_int(0), C.c_float(0)
    r, c = d.shape
    fnc = _ref_cpu2d.ref2dcpu_post(_p(d), _p(t), _p(s), 0 if s is None else s.size, r, c, eb, C.byref(sig),
                                   C.byref(ks), C.byref(ep))
    return d, fnc, sig.value, ks.value, ep.value


def ref_post(data, orig, fn, sp, eb: float, axis_stencil=False):
    """The reference drivers' post-processing sequence on copies."""
    d = f32(data).copy()
    o = f32(orig)
    t = np.ascontiguousarray(fn, dtype=np.int32)
    s = None if sp is None or len(sp) == 0 else np.ascontiguousarray(sp, dtype=np.int32)
    eps = float(max(np.float32(1e-6), np.float32(np.float32(0.1) * np.float32(eb))))
    L = reflib()
    if d.ndim == 2:
        r, c = d.shape
        if s is not None:
            L.ref2d_stencils(_p(d), _p(o), _p(t), _p(s), r, c, eb, s.size)
        L.ref2d_enforce(_p(t), _p(d), _p(o), r, c, eps, eb)
        rest = L.ref2d_rbf(_p(d), _p(t), _p(o), r, c, eps, eb)
    else:
        a, b, c = d.shape
        if s is not None:
            L.ref3d_stencils(_p(d), _p(o), _p(t), _p(s), a, b, c, eb, s.size)
        L.ref3d_enforce(_p(t), _p(d), _p(o), a, b, c, eps, eb)
        rest = L.ref3d_rbf(_p(d), _p(t), _p(o), a, b, c, eps, eb)
        if axis_stencil:
            rest += L.ref3d_axis_saddles(_p(d), _p(t), _p(o), a, b, c, eb)
    return d, rest


# ---------------------------------------------------------------------------
# topology report (restates the reference drivers' verification steps)
# ---------------------------------------------------------------------------

def _classify(f: np.ndarray) -> np.ndarray:
    """Types of every point (0 on the boundary): 4-neighbour in 2D
    (SZp/src/szp_cuda_topology.cu:57-64), 6-neighbour in 3D
    (example/test_cuda_topology_3d.cu:52-73)."""
    f = f32(f)
    t = np.zeros(f.shape, dtype=np.int8)
    inner = tuple(slice(1, -1) for _ in f.shape)
    c = f[inner]
    hi, lo = [], []
    for ax in range(f.ndim):
        m = [slice(1, -1)] * f.ndim
        p = [slice(1, -1)] * f.ndim
        m[ax] = slice(0, -2)
        p[ax] = slice(2, None)
        a, b = f[tuple(m)], f[tuple(p)]
        hi.append((c > a) & (c > b))
        lo.append((c < a) & (c < b))
    if f.ndim == 2:
        mx = hi[0] & hi[1]
        mn = lo[0] & lo[1] & ~mx
        sd = ((lo[0] & hi[1]) | (hi[0] & lo[1])) & ~mx & ~mn
    else:
        mx = hi[0] & hi[1] & hi[2]
        mn = lo[0] & lo[1] & lo[2] & ~mx
        sd = (hi[0] | hi[1] | hi[2]) & (lo[0] | lo[1] | lo[2]) & ~mx & ~mn
    ti = np.zeros(c.shape, dtype=np.int8)
    ti[mx] = 1
    ti[mn] = 2
    ti[sd] = 3
    t[inner] = ti
    return t


def topo_report(orig: np.ndarray, dec: np.ndarray, eb: float) -> dict:
    """Critical-point preservation, error bound and local order of a
    decompressed field (example/test_cuda_topology.cu:540-602, 636-660,
    800-868; example/test_cuda_topology_3d.cu:636-730; the order check is
    applied to every axis in 3D)."""
    o, d = f32(orig), f32(dec)
    to, td = _classify(o), _classify(d)
    r = {}
    r["orig_cps"] = [int(np.count_nonzero(to))] + [int(np.count_nonzero(to == k)) for k in (1, 2, 3)]
    r["dec_cps"] = [int(np.count_nonzero(td))] + [int(np.count_nonzero(td == k)) for k in (1, 2, 3)]
    cp = to != 0
    r["preserved"] = int(np.count_nonzero(cp & (td == to)))
    lost = cp & (td == 0)
    r["lost"] = int(np.count_nonzero(lost))
    r["changed"] = int(np.count_nonzero(cp & (td != 0) & (td != to)))
    r["new_cps"] = int(np.count_nonzero((td != 0) & ~cp))
    r["lost_by_type"] = [0] + [int(np.count_nonzero(lost & (to == k))) for k in (1, 2, 3)]
    err = np.abs(o.astype(np.float64) - d.astype(np.float64))
    ok = ~np.isnan(err)
    r["max_err"] = float(err[ok].max()) if ok.any() else 0.0
    r["over_1eb"] = int(np.count_nonzero(err > float(eb) * 1.01))
    r["over_2eb"] = int(np.count_nonzero(err > float(eb) * 2.0))
    pairs, viol = [0] * 4, [0] * 4
    inner = tuple(slice(1, -1) for _ in o.shape)
    for ax in range(o.ndim):
        # a interior, b = a + 1 along ax, b interior too
        sa = list(inner)
        sb = list(inner)
        sa[ax] = slice(1, -2)
        sb[ax] = slice(2, -1)
        sa, sb = tuple(sa), tuple(sb)
        oo = np.sign(o[sa].astype(np.float64) - o[sb].astype(np.float64))
        do = np.sign(d[sa].astype(np.float64) - d[sb].astype(np.float64))
        oo = np.where(np.isnan(oo), 0, oo)
        do = np.where(np.isnan(do), 0, do)
        keep = oo != 0
        v = keep & (oo != do)
        ta, tb = to[sa], to[sb]
        cats = [np.ones_like(keep), (ta != 0) | (tb != 0), (ta != 0) & (tb != 0),
                (ta == 1) | (ta == 2) | (tb == 1) | (tb == 2)]
        for k, m in enumerate(cats):
            pairs[k] += int(np.count_nonzero(keep & m))
            viol[k] += int(np.count_nonzero(v & m))
    r["pairs"], r["violations"] = pairs, viol
    return r
