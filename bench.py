#!/usr/bin/env python
"""Benchmark of the TopoSZp topology path on B200.

One step = one pass of the hot path over one field: fused compression
(classification + sort positions + topology stream + sort-position stream)
followed by fused decompression with post-processing (extremum stencils,
enforcement, RBF saddle restoration).  Workload: the 512^3 band-limited fp32
field (power spectrum k^-3, [0,1], seed 2), absolute error bound 1e-4,
blockSize 64 -- the single-field bandwidth/roofline case.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1: one process per GPU under torch.distributed.run, each rank processes
its own replica of the field (weak scaling, no data-path collective); the
timed region is bracketed by barriers and the reported time is the max over
ranks.  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "toposzp-cuda_b200")
for _p in (PKG, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

import synth  # noqa: E402

METRIC = "topo-compress+decompress GB/s of fp32 input (fused round trip)"
UNIT = "GB/s"


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and clock-event (throttle) reasons during the timed
    region: NVML polled every 10 ms from a thread (the GPU is matched by UUID),
    else nvidia-smi at its 100 ms minimum interval."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, device_index: int, period_s: float = 0.01):
        self.dev = device_index
        self.period = period_s
        self.samples = []          # (sm_mhz, reason_bits)
        self.sm_max = None
        self.source = None
        self.proc = None
        self.lines = []
        self._stop = threading.Event()
        self._nvml = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        self._nvml = pynvml
        try:
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def _poll(self, h):
        N = self._nvml
        while not self._stop.is_set():
            try:
                sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                bits = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), int(bits)))
            except Exception:
                pass
            self._stop.wait(self.period)

    def __enter__(self):
        try:
            h = self._nvml_handle()
            self.sm_max = float(self._nvml.nvmlDeviceGetMaxClockInfo(h, self._nvml.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, args=(h,), daemon=True)
            self.t.start()
            self.source = "nvml"
            return self
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.source = "nvidia-smi"
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        self._stop.set()
        if self.source == "nvml":
            self.t.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, reasons = [], set()
        mx = self.sm_max
        if self.source == "nvml":
            for mhz, bits in self.samples:
                sm.append(mhz)
                for b, nm in self.REASONS.items():
                    if bits & b:
                        reasons.add(nm)
        else:
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for ln in self.lines:
                parts = [p.strip() for p in ln.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "source": self.source}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    # NCCL reduces device tensors; gloo (host-only runs) host tensors
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# CPU reference leg: the reference's OpenMP library + driver post-processing
# ---------------------------------------------------------------------------

def cpu_reference_run(field: np.ndarray, eb: float, B: int, threads: int):
    """One round trip of the reference's own CPU implementation on `field`
    (3D): find -> sort -> sort-position stream -> topology stream ->
    decompress -> sort-position decode -> stencils -> enforcement -> RBF."""
    import oracle as O
    O.set_ref_threads(threads)
    d = np.ascontiguousarray(field, dtype=np.float32)
    t0 = time.perf_counter()
    cp = O.ref_sort_cp(O.ref_find_cp(d, eb), d)
    # The reference's sort-position compressor frees its per-thread offset
    # table inside `omp single` with no barrier before it, while other threads
    # may still copy with it (SZp/src/szp_topology_3d.cc:405-416,
    # SZp/src/szp_float.cc:850-864): a use after free that crashes now and
    # then with several threads.  That call (a small share of the work) runs on
    # one thread; every other call uses all of them.
    O.set_ref_threads(1)
    sp_stream = O.ref_compress_sp(cp, B)
    O.set_ref_threads(threads)
    topo = O.ref_compress_topo(d, eb, B, cp)
    raw, fn = O.ref_decompress_topo(topo, d.size, eb, B)
    e = int(np.count_nonzero((cp["type"] == 1) | (cp["type"] == 2)))
    sp = O.ref_decompress_sp(sp_stream[8:], e, B) if e else None
    out, _ = O.ref_post(raw.reshape(d.shape), raw.reshape(d.shape), fn.reshape(d.shape), sp, eb)
    return time.perf_counter() - t0, len(topo), len(sp_stream)


def cpu_port_run(field: np.ndarray, eb: float, B: int):
    import oracle as O
    d = np.ascontiguousarray(field, dtype=np.float32)
    t0 = time.perf_counter()
    cp = O.sort_cp(O.find_cp(d, eb), d)
    topo = O.encode_topo(d, eb, B, O.mark_types(cp, d.shape))
    sp = O.extract_sp(cp)
    srt = O.encode_ints(sp, B) if len(sp) else b""
    raw, fn, _ = O.decode_topo(topo, d.size, eb, B)
    O.post(raw.reshape(d.shape), raw.reshape(d.shape), fn.reshape(d.shape), sp, eb)
    return time.perf_counter() - t0, len(topo), len(srt)


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_leg(f, planes, threads):
    import oracle as O
    planes = min(planes, f.dims[0])
    sample = np.ascontiguousarray(f.data[:planes])
    eb = f.abs_eb()
    kind = "reference" if O.ref_available() else "port"
    if kind == "reference":
        t, _, _ = cpu_reference_run(sample, eb, f.block_size, threads)
    else:
        t, _, _ = cpu_port_run(sample, eb, f.block_size)
        threads = 1
    gbs = 4.0 * sample.size / t / 1e9
    what = ("the whole %s field" % f.name if planes == f.dims[0]
            else "first %d of %d planes of the %s field" % (planes, f.dims[0], f.name))
    return {"value": gbs, "unit": UNIT, "cores": threads, "kind": kind, "cpu": cpu_model(),
            "seconds": t,
            "sample": "%s (%d elements), full round trip incl. post-processing, %.2f s"
                      % (what, sample.size, t)}


def cpu_reference_run_2d(field: np.ndarray, eb: float, B: int, threads: int):
    """One round trip of the reference's own CPU path on a 2D field, with the
    CPU decompress driver's own post-processing (its a15 variant): find ->
    sort -> sort-position stream -> topology stream -> decompress ->
    sort-position decode -> locks, false-negative saddles, adaptive RBF,
    stencils, extremum restoration.  Returns (compress s, decompress s)."""
    import oracle as O
    O.set_ref_threads(threads)
    d = np.ascontiguousarray(field, dtype=np.float32)
    t0 = time.perf_counter()
    cp = O.ref_sort_cp(O.ref_find_cp(d, eb), d)
    O.set_ref_threads(1)   # the sort-position compressor's use after free (see cpu_reference_run)
    sp_stream = O.ref_compress_sp(cp, B)
    O.set_ref_threads(threads)
    topo = O.ref_compress_topo(d, eb, B, cp)
    t1 = time.perf_counter()
    raw, fn = O.ref_decompress_topo(topo, d.size, eb, B)
    e = int(np.count_nonzero((cp["type"] == 1) | (cp["type"] == 2)))
    sp = O.ref_decompress_sp(sp_stream[8:], e, B) if e else None
    O.ref_post_cpu2d(raw.reshape(d.shape), fn.reshape(d.shape), sp, eb)
    return t1 - t0, time.perf_counter() - t1


def c1_leg(T, dev, steps, threads, rank0):
    """C1, the 2D 1800x3600 bump field (abs eb 1e-3, blockSize 64): this
    library's fused round trip on the device (each step timed by CUDA events
    on the library's stream, L2 flushed between steps: the field, 26 MB, fits
    in L2) and through the host-buffer C ABI, and the reference's CPU path with
    its CPU driver's post-processing at all host threads and at one thread."""
    import ctypes as C
    import torch
    f = synth.config1()
    eb, B, dims, n = f.abs_eb(), f.block_size, f.dims, f.n
    stream = torch.cuda.Stream(device=dev)
    ctx = T.Context(stream.cuda_stream)
    L = T.lib()
    d = torch.from_numpy(f.data.reshape(-1)).to(dev)
    topo = torch.empty(L.szp_b200_topo_bound(n, B), dtype=torch.uint8, device=dev)
    sort = torch.empty(L.szp_b200_sort_bound(n, B), dtype=torch.uint8, device=dev)
    idx = torch.empty(2 * ((n + B - 1) // B), dtype=torch.int64, device=dev)
    out = torch.empty(n, dtype=torch.float32, device=dev)
    flush = torch.empty(64 << 22, dtype=torch.float32, device=dev)   # 256 MiB > L2
    sizes = T.Sizes()

    def step():
        if L.szp_b200_topo_compress_dev(ctx.ptr, C.c_void_p(d.data_ptr()), T.geom_of(dims), eb, B,
                                        C.c_void_p(topo.data_ptr()), C.c_void_p(sort.data_ptr()),
                                        C.c_void_p(idx.data_ptr()), C.byref(sizes)):
            raise T.ToposzpError(T.last_error())
        if L.szp_b200_topo_decompress_dev(ctx.ptr, C.c_void_p(topo.data_ptr()), sizes.topo_bytes,
                                          C.c_void_p(sort.data_ptr()), sizes.sort_bytes,
                                          C.c_void_p(idx.data_ptr()), T.geom_of(dims), eb, B,
                                          C.c_void_p(out.data_ptr()), None, 1):
            raise T.ToposzpError(T.last_error())

    for _ in range(3):
        step()
    tot = 0.0
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    ms = tot / steps
    rep = ctx.topo_check(d, out, dims, eb)
    # end to end through the host-buffer calls (pinned buffers)
    h_f = torch.from_numpy(f.data.reshape(dims)).pin_memory().numpy()
    h_t = torch.empty(L.szp_b200_topo_bound(n, B), dtype=torch.uint8).pin_memory().numpy()
    h_s = torch.empty(L.szp_b200_sort_bound(n, B), dtype=torch.uint8).pin_memory().numpy()
    h_o = torch.empty(dims, dtype=torch.float32).pin_memory().numpy()
    for _ in range(2):
        sz = ctx.compress_host(h_f, eb, B, h_t, h_s)
        ctx.decompress_host(h_t, sz.topo_bytes, h_s, sz.sort_bytes, dims, eb, B, h_o, 1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        sz = ctx.compress_host(h_f, eb, B, h_t, h_s)
        ctx.decompress_host(h_t, sz.topo_bytes, h_s, sz.sort_bytes, dims, eb, B, h_o, 1)
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / steps
    res = {"workload": "c1: 2D %dx%d fp32 bump field, abs eb %g, blockSize %d, fused compress + decompress + "
                       "post-processing" % (dims[0], dims[1], eb, B),
           "value": 4.0 * n / (ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": ms,
           "l2": "flushed between steps (256 MiB write outside the timed region)",
           "e2e": {"value": 4.0 * n / (e2e_ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": e2e_ms,
                   "timing": "wall clock around the host-buffer calls"},
           "cps": sizes.cp_count, "extrema": sizes.extrema_count,
           "topology": {"preserved": rep["preserved"], "orig_cps": rep["orig_cps"][0],
                        "max_err_over_eb": rep["max_err"] / eb, "over_2eb": rep["over_2eb"]}}
    ctx.close()
    if rank0:
        import oracle as O
        if O.ref_available() and O.ref_cpu2d_available():
            cpu = {}
            for th, key in ((threads, "all_threads"), (1, "one_thread")):
                tc, td = cpu_reference_run_2d(f.data, eb, B, th)
                cpu[key] = {"threads": th, "compress_s": tc, "decompress_s": td,
                            "value": 4.0 * n / (tc + td) / 1e9, "unit": UNIT}
            cpu["what"] = ("the reference's OpenMP library (find, sort, both streams, decode) and its CPU "
                           "decompress driver's own post-processing, whole C1 field")
            cpu["cpu"] = cpu_model()
            res["cpu_reference"] = cpu
    return res


def plain_leg(T, dev, f, steps, rank0):
    """The plain (non-topology) codec, random-access mode, on the 512^3 field:
    device compress + decompress through the device entry points (CUDA events
    on the library's stream, input larger than L2), the same through the
    reference-compatible host entry points, and the reference's own CUDA codec
    on the same field (host-pointer calls, wall clock), with the streams
    compared byte for byte."""
    import hashlib
    import torch
    eb, B, n = f.abs_eb(), f.block_size, f.n
    stream = torch.cuda.Stream(device=dev)
    ctx = T.Context(stream.cuda_stream)
    L = T.lib()
    x = torch.from_numpy(f.data.reshape(-1)).to(dev)
    buf = torch.empty(L.szp_b200_plain_bound(n, B, 0, 0), dtype=torch.uint8, device=dev)
    y = torch.empty_like(x)
    m = 0
    for _ in range(2):
        m = ctx.plain_compress(x, eb, B, buf)
        ctx.plain_decompress(buf, m, n, eb, B, y)
    tc = td = 0.0
    for _ in range(steps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        m = ctx.plain_compress(x, eb, B, buf)
        e[1].record(stream)
        ctx.plain_decompress(buf, m, n, eb, B, y)
        e[2].record(stream)
        torch.cuda.synchronize()
        tc += e[0].elapsed_time(e[1])
        td += e[1].elapsed_time(e[2])
    tc /= steps
    td /= steps
    stream_bytes = m
    ours_sha = hashlib.sha256(buf[:m].cpu().numpy().tobytes()).hexdigest()
    ctx.close()
    peak, _ = peaks()
    ac = (4.0 * n + stream_bytes) / (tc * 1e-3) / 1e9
    ad = (4.0 * n + stream_bytes) / (td * 1e-3) / 1e9
    res = {"workload": "plain codec, random access, float: the %s field, abs eb %g, blockSize %d" % (f.name, eb, B),
           "compress_ms": tc, "decompress_ms": td,
           "value": 4.0 * n / ((tc + td) * 1e-3) / 1e9, "unit": UNIT, "stream_bytes": stream_bytes,
           "roofline": {"compress_gbs": ac, "compress_frac": ac / peak, "decompress_gbs": ad,
                        "decompress_frac": ad / peak, "algorithmic_bytes": 4.0 * n + stream_bytes}}
    # host entry points (the reference's signatures), wall clock around each
    # call as the reference run below is timed: one warm-up, median of two
    import ctypes as C
    h = np.ascontiguousarray(f.data.reshape(-1))
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    v = np.zeros(n, dtype=np.float32)
    tcs, tds = [], []
    s = b""
    for it in range(3):
        sz = C.c_size_t(0)
        t0 = time.perf_counter()
        ptr = L.szp_cuda_float_compress_randomaccess(h.ctypes.data_as(C.c_void_p), C.byref(sz), eb, n, B)
        t1 = time.perf_counter()
        if not ptr:
            raise T.ToposzpError(T.last_error())
        s = C.string_at(ptr, sz.value)
        libc.free(ptr)
        body = np.zeros(len(s) - 4 + 4096, dtype=np.uint8)
        body[: len(s) - 4] = np.frombuffer(s, dtype=np.uint8)[4:]
        t2 = time.perf_counter()
        L.szp_cuda_float_decompress_randomaccess_arg(v.ctypes.data_as(C.c_void_p), n, eb, B,
                                                     body.ctypes.data_as(C.c_void_p))
        t3 = time.perf_counter()
        if it:
            tcs.append((t1 - t0) * 1e3)
            tds.append((t3 - t2) * 1e3)
    tc_h, td_h = statistics.median(tcs), statistics.median(tds)
    res["host_api"] = {"compress_ms": tc_h, "decompress_ms": td_h,
                       "value": 4.0 * n / ((tc_h + td_h) * 1e-3) / 1e9, "unit": UNIT,
                       "max_err_over_eb": float(np.abs(v - h).max() / eb),
                       "timing": "wall clock around each host-pointer call, one warm-up, median of two"}
    if rank0:
        import ref_cuda_run as R
        if R.available():
            r = R.run_plain(h, eb, B, reps=2, warmup=1)
            res["reference_gpu"] = {"compress_ms": r["ms"]["compress"], "decompress_ms": r["ms"]["decompress"],
                                    "value": 4.0 * n / ((r["ms"]["compress"] + r["ms"]["decompress"]) * 1e-3) / 1e9,
                                    "unit": UNIT, "identical_stream": r["stream"] == hashlib.sha256(s).hexdigest()
                                    and ours_sha == r["stream"],
                                    "what": "the reference's CUDA plain codec, host-pointer calls, wall clock"}
    return res


# ---------------------------------------------------------------------------
# reference GPU leg: the reference's own CUDA path on the same GPU and field
# ---------------------------------------------------------------------------

def reference_gpu_leg(T, f, eb, B, dims, topo, sort, sizes, ctx, reps=2):
    """The reference's CUDA implementation (compiled from its sources into
    oracle/_ref) run by its drivers' call sequence on the same field, timed by
    wall clock per host-pointer call as its drivers do, in a child process;
    with a bit-for-bit comparison of its outputs and this library's.  Its
    post-processing is host code (the drivers') and is not part of these
    times."""
    import hashlib
    import torch
    import ref_cuda_run as R
    if not R.available():
        return None
    n = f.n
    r = R.run(f.data, eb, B, reps=reps, warmup=1)
    tys = torch.empty(n, dtype=torch.uint8, device=topo.device)
    raw = ctx.decompress(topo, sizes.topo_bytes, sort, sizes.sort_bytes, None, dims, eb, B, postprocess=0, types=tys)
    sort_b = sort[: sizes.sort_bytes].cpu().numpy().tobytes()
    sp = T.decompress_sort_positions(sort_b, sizes.extrema_count, B)

    def sha(b):
        return hashlib.sha256(b).hexdigest()
    same = {"topo_stream": sha(topo[: sizes.topo_bytes].cpu().numpy().tobytes()) == r["topo"],
            "raw_field": sha(raw.cpu().numpy().tobytes()) == r["raw"],
            "types": sha(tys.cpu().numpy().tobytes()) == r["types"],
            # the reference's CUDA sort writes dense rank - 1 for the first CP of
            # each run of equal values (exclusive scan); its OpenMP sort, which
            # this library follows, writes the dense rank
            "sort_positions_equal_dense_rank_of_reference_cps":
                sha(np.ascontiguousarray(sp, dtype=np.int32).tobytes()) == r["sp_dense_raster"],
            "reference_cuda_sort_is_dense_rank_minus_run_start": r["cuda_sort_relation"],
            "sort_positions_bitwise": sha(np.ascontiguousarray(sp, dtype=np.int32).tobytes()) == r["sp_raster"],
            "cp_count": r["cp_count"] == sizes.cp_count}
    ms = r["ms"]
    return {"compress_ms": ms["compress"], "decompress_ms": ms["decompress"],
            "round_trip_ms": ms["compress"] + ms["decompress"],
            "value": 4.0 * n / ((ms["compress"] + ms["decompress"]) * 1e-3) / 1e9, "unit": UNIT,
            "steps_ms": {k: v for k, v in ms.items() if k not in ("compress", "decompress")},
            "identical_outputs": same, "reps": r["reps"],
            "what": "the reference's CUDA path (find, sort, sort-position and topology streams; topology and "
                    "sort-position decode) built from its sources for sm_100a, host-pointer calls timed by "
                    "wall clock as its drivers do; its post-processing runs on the host in its drivers and "
                    "is not included"}


# ---------------------------------------------------------------------------
# batched leg: 256 mixed fields (seed 3) in one batch vs back-to-back plain calls
# ---------------------------------------------------------------------------

def batch_leg(T, dev, steps, warmup, count=256):
    """Aggregate compress throughput of the mixed-size batch: the batched
    compressor (one persistent launch per codec pass, graph replay, autotuned
    shapes) against back-to-back per-field fused calls on the same stream.
    Inputs resident in HBM; relative bounds are resolved on the device inside
    the batched timed region, and handed to the plain calls precomputed."""
    import torch
    specs = synth.batch_specs(count, 3)
    fields = [synth.batch_field(sp, k) for k, sp in enumerate(specs)]
    items = [(torch.from_numpy(fl.data.reshape(-1)).to(dev), fl.dims, float(sp[2]), sp[1] == "rel")
             for fl, sp in zip(fields, specs)]
    elems = sum(int(np.prod(fl.dims)) for fl in fields)
    stream = torch.cuda.Stream(device=dev)
    b = T.Batch(64, stream.cuda_stream)
    bufs = b.buffers(items)
    res = None
    for _ in range(max(2, warmup)):
        res = b.compress(items, bufs)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    l0 = b.launches()
    ev0.record(stream)
    for _ in range(steps):
        res = b.compress(items, bufs)
    ev1.record(stream)
    torch.cuda.synchronize()
    t_batch = ev0.elapsed_time(ev1) / steps
    launches_batch = (b.launches() - l0) / steps
    stages = b.stage_times()
    # back-to-back plain calls, same buffers, bounds precomputed
    ctx = T.Context(stream.cuda_stream)
    L = T.lib()
    import ctypes as C
    sizes = T.Sizes()
    abs_eb = [r[3] for r in res]

    def plain():
        for (t, dims, _, _), (tb, sb), eb in zip(items, bufs, abs_eb):
            if L.szp_b200_topo_compress_dev(ctx.ptr, C.c_void_p(t.data_ptr()), T.geom_of(dims), eb, 64,
                                            C.c_void_p(tb.data_ptr()), C.c_void_p(sb.data_ptr()), None,
                                            C.byref(sizes)):
                raise T.ToposzpError(T.last_error())
    ref = [(r[2].topo_bytes, r[2].sort_bytes, r[0][: r[2].topo_bytes].clone(),
            r[1][: r[2].sort_bytes].clone()) for r in res]
    for _ in range(max(2, warmup)):
        plain()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        plain()
    ev1.record(stream)
    torch.cuda.synchronize()
    t_plain = ev0.elapsed_time(ev1) / steps
    # the plain calls rewrote the same buffers: the streams must be identical
    same = all(torch.equal(tb[:tn], rt) and torch.equal(sb[:sn], rs)
               for (tb, sb), (tn, sn, rt, rs) in zip(bufs, ref))
    out = {"workload": "c4 batch: %d fields (%d 2D, %d 3D), %.1f M elements, eb log-U[1e-5,1e-2] half abs / "
                       "half rel, blockSize 64, seed 3" % (count, count // 2, count - count // 2, elems / 1e6),
           "batched_gbs": 4.0 * elems / (t_batch * 1e-3) / 1e9, "batched_ms": t_batch,
           "plain_gbs": 4.0 * elems / (t_plain * 1e-3) / 1e9, "plain_ms": t_plain,
           "batched_over_plain": t_plain / t_batch, "streams_identical": bool(same),
           "launches_per_batch": launches_batch, "stages_ms": dict(stages), "tuning": b.tuning()}
    ctx.close()
    b.close()
    return out


# ---------------------------------------------------------------------------
# served leg: Poisson request stream with continuous batching vs plain calls
# ---------------------------------------------------------------------------

def serve_pool(count=32, seed=4):
    """Fields of the request stream: sizes log-uniform over 16 KB - 256 MB of
    fp32, 2D or 3D, Gaussian-bump generator; generated once and cached."""
    import math
    rng = np.random.default_rng(seed)
    pool = []
    for k in range(count):
        nbytes = math.exp(rng.uniform(math.log(16e3), math.log(256e6)))
        n = max(4096, int(nbytes / 4))
        if rng.random() < 0.5:
            a = int(round(math.sqrt(n) * math.exp(rng.uniform(-0.3, 0.3))))
            dims = (max(3, a), max(3, n // max(3, a)))
        else:
            a = int(round(n ** (1 / 3)))
            dims = (max(3, a), max(3, a), max(3, n // max(3, a) // max(3, a)))
        nb = 20 if len(dims) == 2 else 40
        side = min(dims)
        data = synth._cached("serve_%d_%d" % (seed, k), dims,
                             lambda dims=dims, nb=nb, side=side, k=k: synth.gaussian_bumps(
                                 dims, nb, max(1.0, 0.03 * side), max(2.0, 0.25 * side), 1e-3, 1000 + k))
        pool.append((dims, data))
    return pool


def serve_leg(T, dev, nreq=600, slots=4, rate=2000.0, seed=4):
    """Served mode against back-to-back plain calls on the same requests.
    Served: requests submitted at their Poisson arrival times to the server
    (continuous batching, HBM budget 120 GiB); latency = completion - arrival.
    Plain: the same requests one after another on one stream, each timed with
    CUDA events; its latencies follow from the same arrivals through a FIFO
    queue (start = max(arrival, previous completion))."""
    import torch
    rng = np.random.default_rng(seed)
    pool = serve_pool(seed=seed)
    L = T.lib()
    d_pool = [torch.from_numpy(d.reshape(-1)).to(dev) for _, d in pool]
    stream = torch.cuda.Stream(device=dev)
    ctx = T.Context(stream.cuda_stream)
    # streams of every pool field for the decompress requests (untimed setup)
    pre = []
    for (dims, _), d in zip(pool, d_pool):
        eb = float(10 ** rng.uniform(-4, -2))
        topo, sort, _, sz = ctx.compress(d, dims, eb, 64, index=False)
        pre.append((topo, sz.topo_bytes, sort, sz.sort_bytes, eb))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=nreq))
    ops = rng.random(nreq) < 0.7
    picks = rng.integers(0, len(pool), size=nreq)
    ebs = 10 ** rng.uniform(-4, -2, size=nreq)
    srv = T.Server(slots=slots, max_batch=64, block_size=64, hbm_budget=120 << 30)
    spec = []
    for i in range(nreq):
        dims = pool[picks[i]][0]
        n = int(np.prod(dims))
        if ops[i]:
            spec.append(("c", picks[i], float(ebs[i]),
                         torch.empty(L.szp_b200_topo_bound(n, 64), dtype=torch.uint8, device=dev),
                         torch.empty(L.szp_b200_sort_bound(n, 64), dtype=torch.uint8, device=dev)))
        else:
            spec.append(("d", picks[i], torch.empty(n, dtype=torch.float32, device=dev)))

    def requests(sel):
        arr = (T.Request * len(sel))()
        for j, i in enumerate(sel):
            sp = spec[i]
            dims = pool[sp[1]][0]
            if sp[0] == "c":
                arr[j] = srv.compress_request(d_pool[sp[1]], dims, sp[2], False, sp[3], sp[4])
            else:
                topo, tn, sort, sn, eb = pre[sp[1]]
                arr[j] = srv.decompress_request(topo, tn, sort if sn else None, sn, dims, eb, sp[2], 1)
        return arr
    # warm-up: every worker's workspace sized for the largest field (no
    # allocation while serving), autotuning of the batch compressors
    srv.reserve(max(int(np.prod(dims)) for dims, _ in pool))
    warm = list(range(min(nreq, 160)))
    srv.run_trace(requests(warm))
    srv.run_trace(requests(warm))
    torch.cuda.synchronize()
    arr = requests(list(range(nreq)))
    st0 = srv.stats()
    srv.run_trace(arr, arrivals.tolist())
    st = srv.stats()
    lat = np.array([r.t_done - r.t_arrival for r in arr]) * 1e3
    span = max(r.t_done for r in arr) - min(r.t_arrival for r in arr)
    nbytes = np.array([4.0 * np.prod(pool[sp[1]][0]) for sp in spec])
    import ctypes as C
    sizes = T.Sizes()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    svc = np.zeros(nreq)
    stage_rows = [None] * nreq
    for rep in range(2):
        for i, sp in enumerate(spec):
            dims = pool[sp[1]][0]
            ev[0].record(stream)
            if sp[0] == "c":
                rc = L.szp_b200_topo_compress_dev(ctx.ptr, C.c_void_p(d_pool[sp[1]].data_ptr()), T.geom_of(dims),
                                                  sp[2], 64, C.c_void_p(sp[3].data_ptr()),
                                                  C.c_void_p(sp[4].data_ptr()), None, C.byref(sizes))
            else:
                topo, tn, sort, sn, eb = pre[sp[1]]
                rc = L.szp_b200_topo_decompress_dev(ctx.ptr, C.c_void_p(topo.data_ptr()), tn,
                                                    C.c_void_p(sort.data_ptr()) if sn else None, sn, None,
                                                    T.geom_of(dims), eb, 64, C.c_void_p(sp[2].data_ptr()), None, 1)
            if rc:
                raise T.ToposzpError(T.last_error())
            ev[1].record(stream)
            ev[1].synchronize()
            svc[i] = ev[0].elapsed_time(ev[1]) * 1e-3
            stage_rows[i] = ctx.stage_times()
    # where the plain calls spend their device time: per op and size decile,
    # the summed stage times (CUDA events on the workspace stream)
    sizes_b = np.array([4.0 * np.prod(pool[sp[1]][0]) for sp in spec])
    edges = np.quantile(sizes_b, np.linspace(0, 1, 11))
    breakdown = []
    for op in ("c", "d"):
        for k in range(10):
            sel = [i for i, sp in enumerate(spec) if sp[0] == op and
                   edges[k] <= sizes_b[i] <= edges[k + 1] and (k == 9 or sizes_b[i] < edges[k + 1])]
            if not sel:
                continue
            acc = {}
            for i in sel:
                for name, ms in stage_rows[i]:
                    acc[name] = acc.get(name, 0.0) + ms
            mb = float(sizes_b[sel].sum() / 1e6)
            tsum = float(svc[sel].sum())
            breakdown.append({"op": "compress" if op == "c" else "decompress", "decile": k,
                              "requests": len(sel), "mb": round(mb, 1), "device_s": round(tsum, 4),
                              "gbs": round(mb / 1e3 / tsum, 2) if tsum > 0 else None,
                              "stages_ms": {kk: round(v, 2) for kk, v in sorted(acc.items(), key=lambda x: -x[1])}})
    t = 0.0
    plat = np.zeros(nreq)
    for i in range(nreq):
        t = max(t, arrivals[i]) + svc[i]
        plat[i] = (t - arrivals[i]) * 1e3
    pspan = t - arrivals[0]
    out = {"workload": "c5 served: %d requests, Poisson %.0f req/s (seed %d), 70%% compress / 30%% decompress "
                       "(with post-processing), fields 16 KB-256 MB log-uniform (pool of %d 2D/3D bump fields), "
                       "abs eb log-U[1e-4,1e-2], HBM budget 120 GiB, %d slots" % (nreq, rate, seed, len(pool), slots),
           "served_gbs": float(nbytes.sum() / span / 1e9), "served_p50_ms": float(np.percentile(lat, 50)),
           "served_p99_ms": float(np.percentile(lat, 99)),
           "plain_gbs": float(nbytes.sum() / pspan / 1e9), "plain_p50_ms": float(np.percentile(plat, 50)),
           "plain_p99_ms": float(np.percentile(plat, 99)),
           "plain_busy_s": float(svc.sum()), "served_span_s": float(span),
           "batches": st["batches"] - st0["batches"],
           "batched_requests": st["batched_requests"] - st0["batched_requests"],
           "max_concurrent": st["max_concurrent"], "max_inflight_gb": st["max_inflight_bytes"] / 1e9,
           "plain_breakdown": breakdown}
    srv.close()
    ctx.close()
    return out


# ---------------------------------------------------------------------------
# main
# ---------------------------------------------------------------------------

def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--side", type=int, default=512, help="edge of the cubic field")
    ap.add_argument("--cpu-planes", type=int, default=0,
                    help="planes in the CPU baseline sample (0: the whole field)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-c1", action="store_true", help="skip the 2D 1800x3600 leg")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-codec leg")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own CUDA path on the same field")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-e2e-pipelined", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-vs-plain leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-vs-plain leg")
    ap.add_argument("--serve-requests", type=int, default=600, help="requests of the served leg")
    ap.add_argument("--serve-slots", type=int, default=4, help="server worker slots")
    return ap.parse_args()


def run_reference_arm(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    f = synth.config3(args.side)
    threads = os.cpu_count() or 1
    # The reference ranks critical points by an insertion sort inside every
    # quantization bin (SZp/src/szp_topology_3d.cc:190-209), so its cost per
    # element grows with the number of critical points per bin, i.e. with the
    # size of the field: a slab of the field runs several times faster per
    # byte than the whole field.  The line's value is therefore one round trip
    # of the WHOLE field (the GPU arm's workload; about half a minute on 16
    # host threads).  The K steps beside it are bounded 32-plane slabs, timed
    # as the bench contract asks and reported as `slab_value`; warm-up steps
    # use 4-plane slabs.  One slab on one thread is reported as `one_thread`.
    for _ in range(args.warmup):
        reference_leg(f, 4, threads)
    vals, secs = [], []
    slab = min(32, f.dims[0])
    for _ in range(args.steps):
        r = reference_leg(f, slab, threads)
        vals.append(r["value"])
        secs.append(round(r["seconds"], 2))
    full = reference_leg(f, f.dims[0], threads)
    v = full["value"]
    one = reference_leg(f, slab, 1)
    info = dict(full, slab_value=statistics.median(vals), slab_step_seconds=secs,
                one_thread={"value": one["value"], "sample": one["sample"]})
    planes = f.dims[0]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 4.0 * planes * args.side * args.side / v / 1e6,
        "cpu": cpu_model(),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded band-limited field)",
        "config": {"workload": "%s: %d^3 band-limited fp32 field, abs eb 1e-4, blockSize 64, "
                               "round trip with post-processing; every step is the whole field (%d planes)"
                               % (f.name, args.side, planes),
                   "threads": threads},
        "cpu_baseline": info,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0



def e2e_pipelined(T, f, dims, eb, B, steps, out, world, streams=2):
    """Round trips of independent fields through the same host-buffer C ABI
    calls as the e2e leg, from `streams` host threads, each with its own
    workspace (own CUDA stream) and pinned buffers: one field's output copy
    (device to host) overlaps the next field's input copy (host to device),
    which the serial e2e leg cannot do.  Every field still crosses PCIe both
    ways inside the timed region; the figure is fields x 4n bytes over the
    wall time from the start barrier to the last result on the host."""
    import torch
    n = int(np.prod(dims))
    L = T.lib()
    workers = []
    for _ in range(streams):
        h_field = torch.from_numpy(f.data.reshape(dims)).pin_memory()
        h_topo = torch.empty(L.szp_b200_topo_bound(n, B), dtype=torch.uint8).pin_memory()
        h_sort = torch.empty(L.szp_b200_sort_bound(n, B), dtype=torch.uint8).pin_memory()
        h_out = torch.empty(dims, dtype=torch.float32).pin_memory()
        workers.append({"bufs": (h_field, h_topo, h_sort, h_out), "ctx": T.Context(), "err": None})

    dev = out.device

    def run(w, k, start):
        # a new host thread starts on device 0: select this rank's device,
        # on which the workspaces were created
        torch.cuda.set_device(dev)
        hf, ht, hs, ho = (x.numpy() for x in w["bufs"])
        start.wait()
        try:
            for _ in range(k):
                sz = w["ctx"].compress_host(hf, eb, B, ht, hs)
                w["ctx"].decompress_host(ht, sz.topo_bytes, hs, sz.sort_bytes, dims, eb, B, ho, 1)
        except Exception as e:  # reported below; the other threads finish their fields
            w["err"] = e

    def round_of(k):
        start = threading.Barrier(streams + 1)
        th = [threading.Thread(target=run, args=(w, k, start)) for w in workers]
        for t in th:
            t.start()
        start.wait()
        t0 = time.perf_counter()
        for t in th:
            t.join()
        return (time.perf_counter() - t0) * 1e3

    round_of(1)  # warm-up: workspaces grow, weights upload
    torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(round_of(steps), world)
    for w in workers:
        if w["err"] is not None:
            raise w["err"]
    same = all(bool(np.array_equal(w["bufs"][3].numpy().reshape(-1).view(np.int32),
                                   out.cpu().numpy().view(np.int32))) for w in workers)
    fields = streams * steps
    for w in workers:
        w["ctx"].close()
    return {"value": world * fields * 4.0 * n / (ms * 1e-3) / 1e9, "unit": UNIT, "streams": streams,
            "fields": fields, "ms_per_field": ms / fields, "matches_device_path": same,
            "timing": "wall clock, start barrier to the last field's output in host memory"}

def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch

    import toposzp_b200 as T

    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    f = synth.config3(args.side)
    eb = f.abs_eb()
    B = f.block_size
    dims = f.dims
    n = f.n
    d_field = torch.from_numpy(f.data.reshape(-1)).to(dev)

    # the library runs on this stream; every CUDA event below is recorded on it
    stream = torch.cuda.Stream(device=dev)
    ctx = T.Context(stream.cuda_stream)
    L = T.lib()
    topo = torch.empty(L.szp_b200_topo_bound(n, B), dtype=torch.uint8, device=dev)
    sort = torch.empty(L.szp_b200_sort_bound(n, B), dtype=torch.uint8, device=dev)
    idx = torch.empty(2 * ((n + B - 1) // B), dtype=torch.int64, device=dev)
    out = torch.empty(n, dtype=torch.float32, device=dev)
    import ctypes as C
    sizes = T.Sizes()

    def step():
        rc = L.szp_b200_topo_compress_dev(ctx.ptr, C.c_void_p(d_field.data_ptr()), T.geom_of(dims), eb, B,
                                          C.c_void_p(topo.data_ptr()), C.c_void_p(sort.data_ptr()),
                                          C.c_void_p(idx.data_ptr()), C.byref(sizes))
        if rc:
            raise T.ToposzpError(T.last_error())
        st_c = ctx.stage_times()
        rc = L.szp_b200_topo_decompress_dev(ctx.ptr, C.c_void_p(topo.data_ptr()), sizes.topo_bytes,
                                            C.c_void_p(sort.data_ptr()), sizes.sort_bytes,
                                            C.c_void_p(idx.data_ptr()), T.geom_of(dims), eb, B,
                                            C.c_void_p(out.data_ptr()), None, 1)
        if rc:
            raise T.ToposzpError(T.last_error())
        return st_c + ctx.stage_times()

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    stage_acc = {}
    l0 = ctx.launches()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            for name, ms in step():
                stage_acc.setdefault(name, []).append(ms)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ms_local = ev0.elapsed_time(ev1) / args.steps
    launches = ctx.launches() - l0
    ms_step = max_over_ranks(ms_local, world)
    value = world * 4.0 * n / (ms_step * 1e-3) / 1e9

    # check the last output against the error bound (cheap, after timing)
    err = (out - d_field).abs().max().item()
    # topology of the last output against the original, on the device, with
    # the reference drivers' acceptance rule (max error <= 2 eb and more than
    # 90 % of the critical points preserved)
    rep = ctx.topo_check(d_field, out, dims, eb)
    ncp = max(1, rep["orig_cps"][0])
    topology = {"orig_cps": rep["orig_cps"][0], "preserved": rep["preserved"],
                "cp_preserved_frac": rep["preserved"] / ncp, "lost": rep["lost"], "changed": rep["changed"],
                "false_negatives": rep["lost"] + rep["changed"], "false_positives": rep["new_cps"],
                "order_pairs": rep["pairs"][0], "order_violations": rep["violations"][0],
                "order_violations_at_cps": rep["violations"][1],
                "order_violations_at_extrema": rep["violations"][3],
                "max_err_over_eb": rep["max_err"] / eb, "over_2eb": rep["over_2eb"],
                "accepted": bool(rep["max_err"] <= 2 * eb and rep["preserved"] > 0.9 * ncp)}

    stages = {k: statistics.mean(v) for k, v in stage_acc.items()}
    peak, peak_kind = peaks()
    s_topo, s_sort = sizes.topo_bytes, sizes.sort_bytes
    alg = {"encode_topo": 4.0 * n + s_topo, "decode_topo": s_topo + 4.0 * n,
           "encode_sort": 4.0 * sizes.extrema_count + s_sort,
           "decode_sort": s_sort + 4.0 * sizes.extrema_count}
    dom = max(stages, key=stages.get)
    # roofline of the dominant codec kernel (the stage with algorithmic bytes
    # and the largest share); the dominant stage overall is reported beside it
    codec = max([k for k in alg if k in stages], key=lambda k: stages[k])
    achieved = alg[codec] / (stages[codec] * 1e-3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "traffic.txt")
    if os.path.exists(prof):
        with open(prof) as fh:
            for ln in fh:
                parts = ln.split("#")[0].split()
                if len(parts) == 2 and parts[0] == codec and args.side == 512:
                    traffic = float(parts[1])
    rt_bytes = 2.0 * (4.0 * n + s_topo + s_sort)
    roofline = {"bound": "hbm", "kernel": codec, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": alg[codec], "ms_per_launch": stages[codec],
                "round_trip": {"algorithmic_bytes": rt_bytes,
                               "achieved": rt_bytes / (ms_step * 1e-3) / 1e9,
                               "frac": rt_bytes / (ms_step * 1e-3) / 1e9 / peak},
                "dominant_stage": dom}

    # end to end through the host-buffer C ABI: pinned field in, streams out,
    # streams in, post-processed field out
    e2e = None
    if not args.no_e2e:
        h_field = torch.from_numpy(f.data.reshape(dims)).pin_memory()
        h_topo = torch.empty(L.szp_b200_topo_bound(n, B), dtype=torch.uint8).pin_memory()
        h_sort = torch.empty(L.szp_b200_sort_bound(n, B), dtype=torch.uint8).pin_memory()
        h_out = torch.empty(dims, dtype=torch.float32).pin_memory()
        hf, ht, hs, ho = (h_field.numpy(), h_topo.numpy(), h_sort.numpy(), h_out.numpy())
        ectx = T.Context(stream.cuda_stream)

        def e2e_step():
            sz = ectx.compress_host(hf, eb, B, ht, hs)
            ectx.decompress_host(ht, sz.topo_bytes, hs, sz.sort_bytes, dims, eb, B, ho, 1)
            return sz
        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ke = max(2, min(args.steps, 3))
        for _ in range(ke):
            sz = e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        wall_ms = (time.perf_counter() - t0) * 1e3 / ke
        e_ms = max_over_ranks(e0.elapsed_time(e1) / ke, world)
        same = bool(np.array_equal(ho.reshape(-1).view(np.int32), out.cpu().numpy().view(np.int32)))
        e2e = {"value": world * 4.0 * n / (e_ms * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": 4 * n + sz.topo_bytes + sz.sort_bytes,
               "d2h_bytes_per_step": sz.topo_bytes + sz.sort_bytes + 4 * n,
               "ms_per_step": e_ms, "matches_device_path": same,
               "wall_ms_per_step": wall_ms}
        ectx.close()
        if not args.no_e2e_pipelined:
            e2e["pipelined"] = e2e_pipelined(T, f, dims, eb, B, ke, out, world)

    batched = None
    if not args.no_batch:
        batched = batch_leg(T, dev, max(3, min(args.steps, 5)), args.warmup)

    served = None
    if not args.no_serve:
        served = serve_leg(T, dev, nreq=args.serve_requests, slots=args.serve_slots)

    c1 = None
    if world == 1 and not args.no_c1:
        c1 = c1_leg(T, dev, max(3, min(args.steps, 10)), os.cpu_count() or 1, rank == 0)

    plain = None
    if world == 1 and not args.no_plain:
        plain = plain_leg(T, dev, f, max(3, min(args.steps, 10)), rank == 0)

    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        ref_gpu = reference_gpu_leg(T, f, eb, B, dims, topo, sort, sizes, ctx)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = reference_leg(f, args.cpu_planes or f.dims[0], os.cpu_count() or 1)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded band-limited field, FFT-filtered noise k^-3, seed 2)",
            "config": {"workload": "%s: %dx%dx%d fp32, abs eb %g, blockSize %d, fused compress + "
                                   "decompress + post-processing per step"
                                   % (f.name, dims[0], dims[1], dims[2], eb, B),
                       "l2": "input (%.0f MB) larger than L2 (126 MB)" % (4 * n / 1e6),
                       "parallelism": "replicas (one field per GPU)" if world > 1 else "single GPU",
                       "cps": sizes.cp_count, "extrema": sizes.extrema_count,
                       "topo_bytes": s_topo, "sort_bytes": s_sort,
                       "compression_ratio": 4.0 * n / (s_topo + s_sort),
                       "max_abs_err_over_eb": err / eb},
            "topology": topology,
            "clocks": clk.summary(),
            "gpu_launches": launches,
            "stages_ms": stages,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "c1": c1,
            "plain": plain,
            "e2e": e2e,
            "batched": batched,
            "served": served,
        }
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
