"""Generates tests/golden/configs.json: SHA-256 digests of the reference CPU
library's outputs (built from the reference sources into oracle/_ref, run at
one OpenMP thread) on the full-size benchmark workloads:

  c1  2D 1800x3600 Gaussian-bump field, seed 0, abs eb 1e-3, blockSize 64
  c2  3D 100x500x500 Gaussian-bump field, seed 1, rel eb 1e-4, blockSize 64
  c3  3D 512^3 band-limited field, seed 2, abs eb 1e-4, blockSize 64
  c4  the 256-field mixed batch, seed 3 (compression only, per field)

Per single-field workload: the field, the sorted critical-point list, the
topology stream and the sort-position stream in the CUDA layout (the OpenMP
layout at one thread with its extrema-count word dropped, and without the
bit-count byte of an anchor-only tail block), the raw decode, the tags, and
the post-processed field of the reference drivers' sequence (stencils,
enforcement, RBF; the 3D axis-pattern stencil is not part of the drivers'
sequence).  Run from the repository root (takes several minutes: the
reference is serial here):

    python tests/golden/make_config_golden.py [c1 c2 c3 c4]
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "toposzp-cuda_b200")]

import oracle as O  # noqa: E402
import synth  # noqa: E402

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "configs.json")


def digest(b):
    return hashlib.sha256(b).hexdigest()


def cuda_layout_topo(cpu: bytes, n: int, B: int) -> bytes:
    # the OpenMP layout writes a bit-count byte for an anchor-only tail block
    # (SZp/src/szp_float.cc:1239-1242); the CUDA layout omits it
    if n % B == 1:
        return cpu[:-2] + cpu[-1:]
    return cpu


def cuda_layout_sort(cpu: bytes, e: int, B: int) -> bytes:
    # OpenMP: [u64 E][u64 offset][blocks] (SZp/src/szp_float.cc:605-621);
    # CUDA: [u64 0][blocks].  At one thread the offset word is 0.
    s = cpu[8:]
    if e % B == 1:
        s = s[:-1]   # anchor-only tail block: no bit-count byte (it is the last byte)
    return s


def single(f):
    t0 = time.time()
    d = f.data
    eb = f.abs_eb()
    B = f.block_size
    cp = O.ref_sort_cp(O.ref_find_cp(d, eb), d)
    t1 = time.time()
    topo_cpu = O.ref_compress_topo(d, eb, B, cp)
    sort_cpu = O.ref_compress_sp(cp, B)
    ext = (cp["type"] == 1) | (cp["type"] == 2)
    sp = np.ascontiguousarray(cp["sort_position"][ext], dtype=np.int32)
    t2 = time.time()
    topo = cuda_layout_topo(topo_cpu, d.size, B)
    raw, fn, _ = O.decode_topo(topo, d.size, eb, B)
    if d.size % B != 1:
        rraw, rfn = O.ref_decompress_topo(topo_cpu, d.size, eb, B)
        assert (rraw.view(np.int32) == raw.view(np.int32)).all() and (rfn == fn).all()
    if len(sp):
        rsp = O.ref_decompress_sp(sort_cpu[8:], len(sp), B)
        assert (rsp == sp).all()
    t3 = time.time()
    post, restored = O.ref_post(raw.reshape(f.dims), raw.reshape(f.dims), fn.reshape(f.dims), sp, eb)
    t4 = time.time()
    print("  %s: find+sort %.1f s, streams %.1f s, decode %.1f s, post %.1f s" %
          (f.name, t1 - t0, t2 - t1, t3 - t2, t4 - t3), flush=True)
    return dict(dims=list(f.dims), abs_eb=float(np.float32(eb)), block_size=B,
                field=digest(d.tobytes()), cp=digest(cp.tobytes()), cp_count=int(len(cp)),
                extrema=int(len(sp)), topo=digest(topo), topo_bytes=len(topo),
                sort=digest(cuda_layout_sort(sort_cpu, len(sp), B)) if len(sp) else None,
                sort_bytes=len(cuda_layout_sort(sort_cpu, len(sp), B)) if len(sp) else 0,
                sp=digest(sp.tobytes()), raw=digest(raw.tobytes()),
                types=digest(fn.astype(np.uint8).tobytes()), post=digest(post.tobytes()),
                restored=int(restored))


def batch(count=256, seed=3):
    out = []
    t0 = time.time()
    for k, spec in enumerate(synth.batch_specs(count, seed)):
        f = synth.batch_field(spec, k)
        d = f.data
        eb = f.abs_eb()
        cp = O.ref_sort_cp(O.ref_find_cp(d, eb), d)
        topo = cuda_layout_topo(O.ref_compress_topo(d, eb, 64, cp), d.size, 64)
        e = int(np.count_nonzero((cp["type"] == 1) | (cp["type"] == 2)))
        srt = cuda_layout_sort(O.ref_compress_sp(cp, 64), e, 64) if e else b""
        out.append(dict(dims=list(f.dims), abs_eb=float(np.float32(eb)), field=digest(d.tobytes()),
                        topo=digest(topo), topo_bytes=len(topo), sort=digest(srt), sort_bytes=len(srt),
                        cp_count=int(len(cp)), extrema=e))
    print("  c4: %d fields, %.1f s" % (count, time.time() - t0), flush=True)
    return out


def main(which):
    O.build(ref=True)
    O.set_ref_threads(1)
    gold = {}
    if os.path.exists(PATH):
        with open(PATH) as fh:
            gold = json.load(fh)
    makers = {"c1": lambda: single(synth.config1()), "c2": lambda: single(synth.config2()),
              "c3": lambda: single(synth.config3()), "c4": batch}
    for key in which:
        gold[key] = makers[key]()
        with open(PATH, "w") as fh:
            json.dump(gold, fh, indent=1, sort_keys=True)
    print("wrote", PATH, sorted(gold))


if __name__ == "__main__":
    main(sys.argv[1:] or ["c1", "c2", "c3", "c4"])
