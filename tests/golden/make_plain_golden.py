"""Generates tests/golden/plain.json: SHA-256 digests of the reference's own
CUDA plain codec (SZp/src/szp_cuda_compress.cu, szp_cuda_decompress.cu, built
into oracle/_ref/libszp_ref_cuda.so by `make -C oracle refcuda REF=<tree>`)
on the plain-codec cases (toposzp-cuda_b200/synth.py: plain_cases): per case
the compressed stream of szp_cuda_{float,double}_compress_{randomaccess,
threadblock} and the values its decompressor returns for that stream, plus
szp_cuda_float_direct_predict_quantization on the float cases.  Each case runs
in a child process (the reference exits on a CUDA error).  The oracle is
checked against the reference's bytes before anything is written, except on
cases where the reference's own decompressor does not reproduce its input
within the bound: those are recorded (`reference_round_trip` false) and pin
nothing.  The one such case family is the threadblock mode at blockSize 1025:
its packing kernel keeps the B deltas of a block in arrays of
SZP_CUDA_MAX_BLOCK = 1024 entries (SZp/src/szp_cuda_compress.cu:296-357, the
arrays at :315-316), one past their end, so its output is undefined there.
Run from the repository root on a machine with a GPU:

    python tests/golden/make_plain_golden.py
"""
import ctypes as C
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "toposzp-cuda_b200")]
OUT = os.path.join(ROOT, "tests", "golden", "plain.json")


def sha(b):
    return hashlib.sha256(b).hexdigest()


def child(name):
    import oracle
    import synth
    x, eb, B, tb = synth.plain_case(name)
    dbl = x.dtype == np.float64
    L = C.CDLL(oracle.REF_CUDA_SO)
    vp, sz, i = C.c_void_p, C.c_size_t, C.c_int
    ft = C.c_double if dbl else C.c_float
    T = "double" if dbl else "float"
    comp = getattr(L, "szp_cuda_%s_compress_%s" % (T, "threadblock" if tb else "randomaccess"))
    comp.restype, comp.argtypes = vp, [vp, C.POINTER(sz), ft, sz, i]
    dec = getattr(L, "szp_cuda_%s_decompress_%s_arg" % (T, "threadblock" if tb else "randomaccess"))
    dec.restype, dec.argtypes = None, [vp, sz, ft, i, vp]
    libc = C.CDLL(None)
    libc.free.argtypes = [vp]
    n = C.c_size_t(0)
    ptr = comp(x.ctypes.data_as(vp), C.byref(n), eb, x.size, B)
    if not ptr:
        raise SystemExit("%s: reference returned NULL" % name)
    s = C.string_at(ptr, n.value)
    libc.free(ptr)
    es = 8 if dbl else 4
    # the decompressor reads its offset table (up to 256 words) past short streams: pad
    buf = np.zeros(len(s) - es + 4096, dtype=np.uint8)
    buf[: len(s) - es] = np.frombuffer(s, dtype=np.uint8)[es:]
    out = np.zeros(x.size, dtype=x.dtype)
    dec(out.ctypes.data_as(vp), x.size, eb, B, buf.ctypes.data_as(vp))
    res = {"bytes": len(s), "stream": sha(s), "values": sha(out.tobytes())}
    with np.errstate(invalid="ignore"):
        fin = np.isfinite(x) & (np.abs(x.astype(np.float64)) * (1.0 / eb) < 2.0 ** 31 - 2)
        err = np.abs(out.astype(np.float64) - x.astype(np.float64))[fin]
    res["round_trip_within_bound"] = bool(err.size == 0 or err.max() <= eb * 1.01)
    if not dbl and not tb:
        pq = L.szp_cuda_float_direct_predict_quantization
        pq.restype, pq.argtypes = vp, [vp, C.POINTER(sz), C.c_float, sz, i]
        p = pq(x.ctypes.data_as(vp), None, eb, x.size, B)
        res["predict"] = sha(C.string_at(p, 4 * x.size))
        libc.free(p)
    print(json.dumps(res))


def main():
    import oracle
    import synth
    out, bad = {}, []
    for name in synth.plain_cases():
        p = subprocess.run([sys.executable, os.path.abspath(__file__), "--child", name],
                           capture_output=True, text=True, timeout=900)
        if p.returncode:
            raise SystemExit("%s: child failed (%d): %s" % (name, p.returncode, p.stderr[-2000:]))
        r = json.loads(p.stdout.strip().splitlines()[-1])
        x, eb, B, tb = synth.plain_case(name)
        so = oracle.plain_compress(x, eb, B, tb)
        ok = sha(so) == r["stream"] and len(so) == r["bytes"]
        vals, _ = oracle.plain_decompress(so, x.size, eb, B, x.dtype, tb)
        okv = sha(vals.tobytes()) == r["values"]
        print("%-40s %9d B stream %s  values %s  ref round trip %s" % (
            name, r["bytes"], "oracle ok" if ok else "ORACLE DIFFERS", "oracle ok" if okv else "ORACLE DIFFERS",
            "ok" if r["round_trip_within_bound"] else "OUTSIDE BOUND (not a pin)"))
        r["reference_round_trip"] = r.pop("round_trip_within_bound")
        if not ok and r["reference_round_trip"]:
            bad.append(name)
        r["values_oracle_agrees"] = okv
        r["field"] = sha(np.ascontiguousarray(x).tobytes())
        out[name] = r
    if bad:
        raise SystemExit("oracle stream disagrees with the reference on " + ", ".join(bad))
    with open(OUT, "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print("wrote", OUT)


if __name__ == "__main__":
    if len(sys.argv) == 3 and sys.argv[1] == "--child":
        child(sys.argv[2])
    else:
        main()
