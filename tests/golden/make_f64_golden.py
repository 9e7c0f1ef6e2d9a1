"""Generates tests/golden/f64_topo.json: SHA-256 digests of the reference's
own CUDA 3D topology compressors on the fp64 parity cases
(toposzp-cuda_b200/synth.py: f64_cases):

  f64  szp_cuda_double_compress_topology_3d(field, eb, blockSize, CP list)
  f32  szp_cuda_float_compress_topology_3d(float32 cast of the field,
       float32 eb, blockSize, the same CP list)

The reference library is oracle/_ref/libszp_ref_cuda.so, compiled from the
reference's CUDA sources by `make -C oracle refcuda REF=<tree>`; it runs on a
GPU.  Each call runs in a child process (the reference exits the
process on a CUDA error).  The oracle's restatement of both compressors is
checked against the reference's bytes on every case before anything is
written.  Run from the repository root on a machine with a GPU:

    python tests/golden/make_f64_golden.py
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
OUT = os.path.join(ROOT, "tests", "golden", "f64_topo.json")


def sha(b):
    return hashlib.sha256(b).hexdigest()


def child(name):
    import oracle
    import synth
    d, cp, eb, B = synth.f64_case(name)
    L = C.CDLL(oracle.REF_CUDA_SO)
    vp, sz, i = C.c_void_p, C.c_size_t, C.c_int
    L.szp_cuda_double_compress_topology_3d.restype = vp
    L.szp_cuda_double_compress_topology_3d.argtypes = [vp, C.POINTER(sz), C.c_double, sz, i, vp, i, i, i, i]
    L.szp_cuda_float_compress_topology_3d.restype = vp
    L.szp_cuda_float_compress_topology_3d.argtypes = [vp, C.POINTER(sz), C.c_float, sz, i, vp, i, i, i, i]
    libc = C.CDLL(None)
    libc.free.argtypes = [vp]
    res = {}
    cpp = cp.ctypes.data_as(vp) if len(cp) else None
    for tag, arr, fn in (("f64", np.ascontiguousarray(d, dtype=np.float64), L.szp_cuda_double_compress_topology_3d),
                         ("f32", np.ascontiguousarray(d, dtype=np.float32), L.szp_cuda_float_compress_topology_3d)):
        n = C.c_size_t(0)
        ebv = float(eb) if tag == "f64" else float(np.float32(eb))
        ptr = fn(arr.ctypes.data_as(vp), C.byref(n), ebv, arr.size, B, cpp, len(cp), *arr.shape)
        if not ptr:
            raise SystemExit("%s %s: reference returned NULL" % (name, tag))
        b = C.string_at(ptr, n.value)
        libc.free(ptr)
        if os.environ.get("F64_GOLDEN_DUMP"):
            with open(os.path.join(os.environ["F64_GOLDEN_DUMP"], "%s.%s.bin" % (name, tag)), "wb") as fh:
                fh.write(b)
        res[tag + "_sha"] = sha(b)
        res[tag + "_bytes"] = n.value
    print(json.dumps(res))


def main():
    import oracle
    import synth
    out = {}
    bad = []
    for name in synth.f64_cases():
        p = subprocess.run([sys.executable, os.path.abspath(__file__), "--child", name],
                           capture_output=True, text=True, timeout=600)
        if p.returncode:
            raise SystemExit("%s: child failed (%d): %s" % (name, p.returncode, p.stderr[-2000:]))
        r = json.loads(p.stdout.strip().splitlines()[-1])
        d, cp, eb, B = synth.f64_case(name)
        types = oracle.mark_types(cp.view(oracle.CP3_DT).reshape(-1), d.shape)
        o64 = oracle.double_compress_topo_3d(d, eb, B, types, d.shape)
        o32 = oracle.encode_topo(d.astype(np.float32), float(np.float32(eb)), B, types)
        ok64 = sha(o64) == r["f64_sha"] and len(o64) == r["f64_bytes"]
        ok32 = sha(o32) == r["f32_sha"] and len(o32) == r["f32_bytes"]
        print("%-26s f64 %8d B %s   f32 %8d B %s" % (name, r["f64_bytes"], "oracle ok" if ok64 else "ORACLE DIFFERS",
                                                    r["f32_bytes"], "oracle ok" if ok32 else "ORACLE DIFFERS"))
        if not (ok64 and ok32):
            bad.append(name)
            continue
        out[name] = {"field": sha(np.ascontiguousarray(d).tobytes()), "cps": sha(cp.tobytes()),
                     "f64_bytes": r["f64_bytes"], "f64": r["f64_sha"],
                     "f32_bytes": r["f32_bytes"], "f32": r["f32_sha"]}
    if bad:
        raise SystemExit("oracle disagrees with the reference on " + ", ".join(bad))
    with open(OUT, "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print("wrote", OUT)


if __name__ == "__main__":
    if len(sys.argv) == 3 and sys.argv[1] == "--child":
        child(sys.argv[2])
    else:
        main()
