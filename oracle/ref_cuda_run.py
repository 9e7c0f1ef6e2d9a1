"""TEST AND BASELINE INFRASTRUCTURE ONLY -- never imported by the product.

Runs the reference's own CUDA implementation of the topology path
(oracle/_ref/libszp_ref_cuda.so, compiled from the reference's CUDA sources by
`make -C oracle refcuda REF=<tree>`) on one fp32 field, in a child process
(the reference exits the process on any CUDA error), with the call sequence
of the reference's drivers (example/test_cuda_topology.cu,
example/test_cuda_topology_3d.cu:498-615):

  compress    find CPs -> sort (sort positions) -> sort-position stream ->
              topology stream
  decompress  topology stream -> raw field + per-element types (FN);
              sort-position stream -> sort positions

Each step is timed by wall clock around the host-pointer call, as the drivers
time them (the reference's own device allocations and host<->device copies
fall inside every call).  Every output is reported as a SHA-256 digest.  The
reference's CUDA finder appends critical points with an atomic counter, so
its CP list order -- and with it the sort-position stream, which follows list
order -- changes from run to run; the order-free digest reported for the
sort positions is that of the extrema's positions in raster order.

Sort positions of the reference's CUDA sort (szp_cuda_topology.cu:253,
szp_cuda_topology_3d.cu:362-395): the CPs are sorted by (bin, value) with an
unstable sort, a flag marks each CP whose value differs from its predecessor
in the same bin, and an EXCLUSIVE scan of the flags per bin gives the
position.  A CP's position is therefore its dense rank r in the bin when it is
not the first of its run of equal values, and r - 1 when it is (the first run
of a bin keeps 0), and which CP of a tied run counts as "first" follows the
unstable sort.  The reference's OpenMP sort (szp_float.cc:345-356,
szp_topology_3d.cc:223-232) writes the dense rank itself.  The child checks
this relation on the reference's own CP list and reports the dense ranks of
its extrema in raster order beside the positions the CUDA sort wrote.
"""
import ctypes as C
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_CUDA_SO = os.path.join(HERE, "_ref", "libszp_ref_cuda.so")

CP2 = np.dtype([("x", "<i4"), ("y", "<i4"), ("type", "<i4"), ("quantized_bin", "<i4"), ("sort_position", "<i4")])
CP3 = np.dtype([("x", "<i4"), ("y", "<i4"), ("z", "<i4"), ("type", "<i4"), ("quantized_bin", "<i4"),
                ("sort_position", "<i4")])


def available() -> bool:
    return os.path.exists(REF_CUDA_SO)


def sha(b) -> str:
    return hashlib.sha256(b).hexdigest()


def _lib():
    L = C.CDLL(REF_CUDA_SO)
    vp, sz, i, f = C.c_void_p, C.c_size_t, C.c_int, C.c_float
    sig = {
        "szp_cuda_find_critical_points": (vp, [vp, C.POINTER(sz), i, i, f]),
        "szp_cuda_find_critical_points_3d": (vp, [vp, C.POINTER(sz), i, i, i, f]),
        "szp_cuda_sort_critical_points_by_original_data": (None, [vp, sz, vp, i]),
        "szp_cuda_sort_critical_points_3d": (None, [vp, sz, vp, i, i]),
        "szp_cuda_compress_sort_positions": (vp, [vp, sz, C.POINTER(sz), i]),
        "szp_cuda_compress_sort_positions_3d": (vp, [vp, sz, C.POINTER(sz), i]),
        "szp_cuda_float_compress_randomaccess_topology_preserved": (vp, [vp, C.POINTER(sz), f, sz, i, vp, i, i, i]),
        "szp_cuda_float_compress_topology_3d": (vp, [vp, C.POINTER(sz), f, sz, i, vp, i, i, i, i]),
        "szp_cuda_float_decompress_randomaccess_topology_preserved": (None, [C.POINTER(vp), sz, f, i, vp,
                                                                             C.POINTER(vp)]),
        "szp_cuda_decompress_sort_positions": (vp, [vp, sz, i]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def _dense_rank_relation(rec, vals):
    """Dense rank of every CP in its bin (values vals, one per record), and
    whether the positions in rec match the reference CUDA sort's rule: each
    position equals the dense rank except for exactly one CP of every run of
    equal values with rank >= 1, whose position is one less."""
    k = len(rec)
    if k == 0:
        return np.zeros(0, np.int64), True
    bins = rec["quantized_bin"].astype(np.int64)
    order = np.lexsort((vals, bins))
    sb, sv = bins[order], vals[order]
    newbin = np.r_[True, sb[1:] != sb[:-1]]
    newrun = newbin | np.r_[True, sv[1:] != sv[:-1]]
    flag = (newrun & ~newbin).astype(np.int64)
    cum = np.cumsum(flag)
    start = np.maximum.accumulate(np.where(newbin, np.arange(k), 0))
    r_sorted = cum - cum[start]
    dense = np.empty(k, np.int64)
    dense[order] = r_sorted
    diff = r_sorted - rec["sort_position"][order].astype(np.int64)
    runs = np.nonzero(newrun)[0]
    per_run = np.add.reduceat(diff, runs)
    ok = bool(((diff == 0) | (diff == 1)).all() and (per_run == (r_sorted[runs] >= 1)).all())
    return dense, ok


def _child(path, dims, eb, B, reps, warmup, dump):
    dims = tuple(dims)
    n = int(np.prod(dims))
    data = np.fromfile(path, dtype=np.float32, count=n)
    assert data.size == n
    L = _lib()
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    dp = data.ctypes.data_as(C.c_void_p)
    nd = len(dims)
    dt = CP2 if nd == 2 else CP3
    times = {}
    res = {}

    def tick(name, t0):
        times.setdefault(name, []).append((time.perf_counter() - t0) * 1e3)

    for it in range(warmup + reps):
        keep = it == warmup + reps - 1
        cnt = C.c_size_t(0)
        t0 = time.perf_counter()
        if nd == 2:
            cps = L.szp_cuda_find_critical_points(dp, C.byref(cnt), dims[0], dims[1], eb)
        else:
            cps = L.szp_cuda_find_critical_points_3d(dp, C.byref(cnt), dims[0], dims[1], dims[2], eb)
        tick("find", t0)
        k = cnt.value
        t0 = time.perf_counter()
        if nd == 2:
            L.szp_cuda_sort_critical_points_by_original_data(cps, k, dp, dims[1])
        else:
            L.szp_cuda_sort_critical_points_3d(cps, k, dp, dims[1], dims[2])
        tick("sort", t0)
        rec = np.frombuffer(C.string_at(cps, k * dt.itemsize), dtype=dt).copy() if k else np.zeros(0, dt)
        ssz = C.c_size_t(0)
        t0 = time.perf_counter()
        if nd == 2:
            sp_s = L.szp_cuda_compress_sort_positions(cps, k, C.byref(ssz), B)
        else:
            sp_s = L.szp_cuda_compress_sort_positions_3d(cps, k, C.byref(ssz), B)
        tick("sort_stream", t0)
        tsz = C.c_size_t(0)
        t0 = time.perf_counter()
        if nd == 2:
            topo = L.szp_cuda_float_compress_randomaccess_topology_preserved(dp, C.byref(tsz), eb, n, B, cps, k,
                                                                             dims[0], dims[1])
        else:
            topo = L.szp_cuda_float_compress_topology_3d(dp, C.byref(tsz), eb, n, B, cps, k, *dims)
        tick("topo_stream", t0)
        out = C.c_void_p()
        fn = C.c_void_p()
        t0 = time.perf_counter()
        L.szp_cuda_float_decompress_randomaccess_topology_preserved(C.byref(out), n, eb, B, topo, C.byref(fn))
        tick("decode_topo", t0)
        ext = int(np.count_nonzero((rec["type"] == 1) | (rec["type"] == 2)))
        t0 = time.perf_counter()
        sp = L.szp_cuda_decompress_sort_positions(sp_s, ext, B) if (sp_s and ext) else None
        tick("decode_sort", t0)
        if keep:
            topo_b = C.string_at(topo, tsz.value)
            raw = np.frombuffer(C.string_at(out, 4 * n), dtype=np.float32)
            fnv = np.frombuffer(C.string_at(fn, 4 * n), dtype=np.int32).astype(np.uint8)
            if nd == 2:
                flat = rec["x"].astype(np.int64) * dims[1] + rec["y"]
            else:
                flat = (rec["x"].astype(np.int64) * dims[1] + rec["y"]) * dims[2] + rec["z"]
            order = np.argsort(flat, kind="stable")
            r = rec[order]
            ex = (r["type"] == 1) | (r["type"] == 2)
            sp_raster = np.ascontiguousarray(r["sort_position"][ex], dtype=np.int32)
            dense, relation = _dense_rank_relation(r, data[np.sort(flat)])
            dec_sp = (np.frombuffer(C.string_at(sp, 4 * ext), dtype=np.int32) if sp is not None
                      else np.zeros(0, np.int32))
            res = {"cp_count": k, "extrema": ext, "topo_bytes": tsz.value, "topo": sha(topo_b),
                   "sort_bytes": ssz.value, "raw": sha(raw.tobytes()), "types": sha(fnv.tobytes()),
                   "sp_raster": sha(sp_raster.tobytes()),
                   "sp_dense_raster": sha(np.ascontiguousarray(dense[ex], dtype=np.int32).tobytes()),
                   "cuda_sort_relation": relation,
                   "sort_stream_round_trip": bool(np.array_equal(
                       dec_sp, rec["sort_position"][(rec["type"] == 1) | (rec["type"] == 2)]))}
            if dump:
                np.save(os.path.join(dump, "raw.npy"), raw)
                np.save(os.path.join(dump, "types.npy"), fnv)
                np.save(os.path.join(dump, "sp_raster.npy"), sp_raster)
                with open(os.path.join(dump, "topo.bin"), "wb") as fh:
                    fh.write(topo_b)
        for p in (cps, sp_s, topo, out.value, fn.value, sp):
            if p:
                libc.free(p)
    med = {k: statistics.median(v[warmup:]) for k, v in times.items()}
    med["compress"] = med["find"] + med["sort"] + med["sort_stream"] + med["topo_stream"]
    med["decompress"] = med["decode_topo"] + med["decode_sort"]
    res["ms"] = med
    res["reps"] = reps
    print(json.dumps(res))


def _plain_child(path, n, dtype, eb, B, tb, reps, warmup):
    x = np.fromfile(path, dtype=np.dtype(dtype), count=n)
    L = C.CDLL(REF_CUDA_SO)
    vp, sz, i = C.c_void_p, C.c_size_t, C.c_int
    dbl = x.dtype == np.float64
    ft = C.c_double if dbl else C.c_float
    T = "double" if dbl else "float"
    comp = getattr(L, "szp_cuda_%s_compress_%s" % (T, "threadblock" if tb else "randomaccess"))
    comp.restype, comp.argtypes = vp, [vp, C.POINTER(sz), ft, sz, i]
    dec = getattr(L, "szp_cuda_%s_decompress_%s_arg" % (T, "threadblock" if tb else "randomaccess"))
    dec.restype, dec.argtypes = None, [vp, sz, ft, i, vp]
    libc = C.CDLL(None)
    libc.free.argtypes = [vp]
    out = np.zeros(n, dtype=x.dtype)
    tc, td = [], []
    es = 8 if dbl else 4
    for it in range(warmup + reps):
        m = C.c_size_t(0)
        t0 = time.perf_counter()
        ptr = comp(x.ctypes.data_as(vp), C.byref(m), eb, n, B)
        t1 = time.perf_counter()
        s = C.string_at(ptr, m.value)
        libc.free(ptr)
        buf = np.zeros(len(s) - es + 4096, dtype=np.uint8)
        buf[: len(s) - es] = np.frombuffer(s, dtype=np.uint8)[es:]
        t2 = time.perf_counter()
        dec(out.ctypes.data_as(vp), n, eb, B, buf.ctypes.data_as(vp))
        t3 = time.perf_counter()
        if it >= warmup:
            tc.append((t1 - t0) * 1e3)
            td.append((t3 - t2) * 1e3)
    print(json.dumps({"bytes": len(s), "stream": sha(s), "values": sha(out.tobytes()),
                      "ms": {"compress": statistics.median(tc), "decompress": statistics.median(td)}}))


def run_plain(x: np.ndarray, eb: float, B: int, threadblock: bool = False, reps: int = 1, warmup: int = 0,
              timeout: float = 1200.0) -> dict:
    """The reference's CUDA plain codec (host-pointer compress, then its
    decompressor on that stream) on a 1-D array, in a child process; digests
    and median wall-clock milliseconds per call."""
    d = np.ascontiguousarray(x)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "field.bin")
        d.tofile(path)
        cmd = [sys.executable, os.path.abspath(__file__), "--plain", path, str(d.size), d.dtype.str, repr(float(eb)),
               str(B), str(int(threadblock)), str(reps), str(warmup)]
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if p.returncode:
        raise RuntimeError("reference CUDA plain run failed (%d): %s" % (p.returncode, p.stderr[-2000:]))
    return json.loads(p.stdout.strip().splitlines()[-1])


def run(field: np.ndarray, eb: float, B: int, reps: int = 1, warmup: int = 0, dump: str = None,
        timeout: float = 1200.0) -> dict:
    """The reference's CUDA path on `field` (fp32, 2D or 3D) in a child
    process; returns digests, counts and median milliseconds per step."""
    d = np.ascontiguousarray(field, dtype=np.float32)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "field.f32")
        d.tofile(path)
        cmd = [sys.executable, os.path.abspath(__file__), path, ",".join(map(str, d.shape)), repr(float(eb)),
               str(B), str(reps), str(warmup), dump or ""]
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if p.returncode:
        raise RuntimeError("reference CUDA run failed (%d): %s" % (p.returncode, p.stderr[-2000:]))
    return json.loads(p.stdout.strip().splitlines()[-1])


if __name__ == "__main__":
    a = sys.argv[1:]
    if a and a[0] == "--plain":
        _plain_child(a[1], int(a[2]), a[3], float(a[4]), int(a[5]), int(a[6]), int(a[7]), int(a[8]))
        sys.exit(0)
    _child(a[0], [int(x) for x in a[1].split(",")], float(a[2]), int(a[3]), int(a[4]), int(a[5]),
           a[6] if len(a) > 6 and a[6] else None)
