"""Generates tests/golden/golden.json: SHA-256 digests of the reference CPU
library's outputs (built from the reference sources into oracle/_ref, run at
one OpenMP thread) on seeded synthetic fields.  Run from the repository root:

    python tests/golden/make_golden.py

The digests pin the oracle on machines where the reference is absent.
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "toposzp-cuda_b200"),
                os.path.join(ROOT, "tests")]

import oracle as O  # noqa: E402
from test_oracle_pin import CASES, case_id, field  # noqa: E402


def digest(b):
    return hashlib.sha256(b).hexdigest()


def main():
    O.build(ref=True)
    O.set_ref_threads(1)
    out = {}
    for case in CASES:
        dims, eb, B, kind, scale = case
        d = field(dims, kind, scale)
        cp = O.ref_sort_cp(O.ref_find_cp(d, eb), d)
        topo_cpu = O.ref_compress_topo(d, eb, B, cp)
        sp = np.array([c["sort_position"] for c in cp if c["type"] in (1, 2)], dtype=np.int32)
        raw, fn = O.ref_decompress_topo(topo_cpu, d.size, eb, B)
        if d.size % B == 1:
            # the reference CUDA layout drops the tail bit-count byte; decode that layout
            cu = topo_cpu[:-2] + topo_cpu[-1:]
            raw, fn, _ = O.decode_topo(cu, d.size, eb, B)
        post, restored = O.ref_post(raw.reshape(dims), raw.reshape(dims), fn.reshape(dims), sp, eb,
                                    axis_stencil=len(dims) == 3)
        out[case_id(case)] = dict(field=digest(d.tobytes()), cp=digest(cp.tobytes()),
                                  topo_cpu=digest(topo_cpu), sp=digest(sp.tobytes()),
                                  post=digest(post.tobytes()), restored=int(restored))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", path, len(out), "cases")


if __name__ == "__main__":
    main()
