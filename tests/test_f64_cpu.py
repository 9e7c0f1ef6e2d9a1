"""The oracle's fp64 3D topology compressor (double quantization, three
saddle-repair passes in q-space, int blocks with 2-bit tags;
SZp/src/szp_cuda_topology_3d.cu:641-646, 736-826, 836-958, 1066-1188):

* pinned against the reference's own CUDA library on every fp64 case
  (tests/golden/f64_topo.json, made by tests/golden/make_f64_golden.py on a
  GPU from the reference's szp_cuda_topology_3d.cu), together with the
  reference's fp32 3D compressor on the float32 cast of the same fields;
* checked against a loop-by-loop Python restatement of the repair on small
  fields, pass by pass;
* repair properties: only interior saddles change, by at most one step per
  pass, and zero passes is the plain quantization."""
import hashlib
import json
import os

import numpy as np
import pytest

import synth

GOLD = os.path.join(os.path.dirname(__file__), "golden", "f64_topo.json")


def sha(b):
    return hashlib.sha256(b).hexdigest()


def gold():
    with open(GOLD) as fh:
        return json.load(fh)


def types_of(ora, cp, dims):
    return ora.mark_types(cp.view(ora.CP3_DT).reshape(-1), dims)


SMALL = [k for k, v in synth.f64_cases().items() if np.prod(v[0]) < 100000]


@pytest.mark.parametrize("name", list(synth.f64_cases()))
def test_oracle_matches_reference_cuda(ora, name):
    g = gold()[name]
    d, cp, eb, B = synth.f64_case(name)
    assert sha(np.ascontiguousarray(d).tobytes()) == g["field"], "field generator changed"
    assert sha(cp.tobytes()) == g["cps"], "critical-point list changed"
    t = types_of(ora, cp, d.shape)
    s64 = ora.double_compress_topo_3d(d, eb, B, t, d.shape)
    assert len(s64) == g["f64_bytes"] and sha(s64) == g["f64"]
    s32 = ora.encode_topo(d.astype(np.float32), float(np.float32(eb)), B, t)
    assert len(s32) == g["f32_bytes"] and sha(s32) == g["f32"]


def _trunc(v):
    if v != v:
        return -2147483648
    if v >= 2147483647.0:
        return 2147483647
    if v <= -2147483648.0:
        return -2147483648
    return int(v)


def _wrap(v):
    return ((v + 2**31) % 2**32) - 2**31


def _repair_loops(q, t, dims, passes):
    """One thread's view of each pass: reads the snapshot, writes the copy."""
    d1, d2, d3 = dims
    q = q.reshape(dims).astype(np.int64).copy()
    t = t.reshape(dims)
    for _ in range(passes):
        src = q.copy()
        for x in range(1, d1 - 1):
            for y in range(1, d2 - 1):
                for z in range(1, d3 - 1):
                    if t[x, y, z] != 3:
                        continue
                    c = src[x, y, z]
                    nb = [(x - 1, y, z), (x + 1, y, z), (x, y - 1, z), (x, y + 1, z), (x, y, z - 1), (x, y, z + 1)]
                    v = [src[p] for p in nb]
                    tt = [t[p] for p in nb]
                    pairs = [(v[0], v[1]), (v[2], v[3]), (v[4], v[5])]
                    high = sum(c > max(a, b) for a, b in pairs)
                    low = sum(c < min(a, b) for a, b in pairs)
                    if high and low:
                        continue
                    for trial in (c, _wrap(c - 1), _wrap(c + 1)):
                        th = sum(trial > max(a, b) for a, b in pairs)
                        tl = sum(trial < min(a, b) for a, b in pairs)
                        if not (th and tl):
                            continue
                        if any(tk == 1 and vk <= trial for tk, vk in zip(tt, v)):
                            continue
                        if any(tk == 2 and vk >= trial for tk, vk in zip(tt, v)):
                            continue
                        q[x, y, z] = trial
                        break
    return q.reshape(-1).astype(np.int32)


@pytest.mark.parametrize("name", [n for n in SMALL if np.prod(synth.f64_cases()[n][0]) <= 20000])
@pytest.mark.parametrize("passes", [1, 2, 3])
def test_repair_matches_loops(ora, name, passes):
    d, cp, eb, B = synth.f64_case(name)
    t = types_of(ora, cp, d.shape)
    _, q = ora.double_compress_topo_3d(d, eb, B, t, d.shape, passes=passes, with_q=True)
    inv = 1.0 / eb
    q0 = np.array([_trunc(v * inv) for v in d.reshape(-1)], dtype=np.int64)
    ql = _repair_loops(q0, t, d.shape, passes)
    assert (q == ql).all()


@pytest.mark.parametrize("name", SMALL)
def test_repair_properties(ora, name):
    d, cp, eb, B = synth.f64_case(name)
    dims = d.shape
    t = types_of(ora, cp, dims)
    s0, q0 = ora.double_compress_topo_3d(d, eb, B, t, dims, passes=0, with_q=True)
    # zero passes: the plain quantization, encoded with the tags
    with np.errstate(invalid="ignore", over="ignore"):
        p = d.reshape(-1) * (1.0 / eb)
    plain = np.trunc(np.where(np.isnan(p), -2147483648.0, np.clip(p, -2147483648.0, 2147483647.0))).astype(np.int64)
    assert (q0 == plain).all()
    inner = np.zeros(dims, bool)
    if min(dims) >= 3:
        inner[1:-1, 1:-1, 1:-1] = True
    inner = inner.reshape(-1)
    for passes in (1, 3):
        _, q = ora.double_compress_topo_3d(d, eb, B, t, dims, passes=passes, with_q=True)
        ch = q != q0
        assert (t[ch] == 3).all() and inner[ch].all()
        assert (np.abs(q.astype(np.int64) - q0)[ch] <= passes).all()
    # the stream carries the types as its tags
    s3 = ora.double_compress_topo_3d(d, eb, B, t, dims)
    _, fn, used = ora.decode_topo(s3, d.size, float(np.float32(eb)), B)
    assert used == len(s3)
    assert (fn == t).all()
