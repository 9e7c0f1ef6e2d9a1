"""Generates the .SZp container fixtures in tests/golden/containers/: the
bytes the reference's own CPU path writes (built from the reference sources
into oracle/_ref) for small seeded fields, at one and at eight OpenMP threads.

The critical-point list is found and ranked at one thread (raster order, the
order the fused GPU path emits); the topology and sort-position streams are
then written with T threads and joined with the drivers' footer
(example/testfloat_compress_fastmode1_topology.cc:105-125).  The reference's
multi-threaded sort-position writer frees its offset table while other
threads may still read it (SZp/src/szp_topology_3d.cc:405-416,
SZp/src/szp_float.cc:850-864), so it runs in a child process that is retried
when it crashes.  Run from the repository root:

    python tests/golden/make_container_golden.py
"""
import json
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "toposzp-cuda_b200")]

import oracle as O  # noqa: E402
import synth  # noqa: E402

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "containers")

CASES = [
    # name, dims, eb, B, kind, scale, seed
    ("bumps_60x90_B16", (60, 90), 1e-2, 16, "bumps", 1.0, 5),
    ("noise_37x53_B64", (37, 53), 1e-2, 64, "noise", 0.1, 5),
    ("tail_5x13_B64", (5, 13), 1e-3, 64, "noise", 1.0, 5),          # 65 % 64 == 1
    ("tail_9x9x9_B8", (9, 9, 9), 1e-4, 8, "bumps", 1.0, 5),          # 729 % 8 == 1
    ("band_20x24x28_B64", (20, 24, 28), 1e-3, 64, "band", 1.0, 5),
]
THREADS = [1, 8]

CHILD = r"""
import sys, numpy as np
sys.path[:0] = [%r]
import oracle as O
cp = np.load(sys.argv[1])
O.set_ref_threads(int(sys.argv[3]))
open(sys.argv[2], "wb").write(O.ref_compress_sp(cp, int(sys.argv[4])))
"""


def field(dims, kind, scale, seed):
    return (synth.small_field(dims, seed=seed, kind=kind) * np.float32(scale)).astype(np.float32)


def sort_stream(cp, B, T):
    if T == 1:
        O.set_ref_threads(1)
        return O.ref_compress_sp(cp, B)
    with tempfile.TemporaryDirectory() as td:
        cpf, out = os.path.join(td, "cp.npy"), os.path.join(td, "sp.bin")
        np.save(cpf, cp)
        for _ in range(50):
            r = subprocess.run([sys.executable, "-c", CHILD % os.path.join(ROOT, "oracle"), cpf, out, str(T), str(B)])
            if r.returncode == 0:
                return open(out, "rb").read()
    raise RuntimeError("the reference's sort-position writer crashed 50 times")


def main():
    O.build(ref=True)
    os.makedirs(HERE, exist_ok=True)
    manifest = {}
    for name, dims, eb, B, kind, scale, seed in CASES:
        d = field(dims, kind, scale, seed)
        O.set_ref_threads(1)
        cp = O.ref_sort_cp(O.ref_find_cp(d, eb), d)
        for T in THREADS:
            O.set_ref_threads(T)
            topo = O.ref_compress_topo(d, eb, B, cp)
            srt = sort_stream(cp, B, T)
            blob = topo + srt + struct.pack("<QQ", len(topo), len(srt))
            fn = "%s_T%d.szp" % (name, T)
            with open(os.path.join(HERE, fn), "wb") as fh:
                fh.write(blob)
            manifest[fn] = dict(case=name, dims=list(dims), eb=eb, block_size=B, kind=kind, scale=scale,
                                seed=seed, threads=T, topo_bytes=len(topo), sort_bytes=len(srt))
    with open(os.path.join(HERE, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)
    print("wrote", len(manifest), "containers to", HERE)


if __name__ == "__main__":
    main()
