"""The oracle is pinned against the reference's own CPU code, built from the
reference sources (oracle/_ref), at one OpenMP thread, and against the
committed golden fixtures generated from that build.

Layout differences between the reference's OpenMP and CUDA paths are known
and covered: the OpenMP layout writes a bit-count byte for an anchor-only
tail block and prefixes the sort stream with the extrema count.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import synth

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden.json")

CASES = [
    ((37, 53), 1e-3, 64, "bumps", 1.0),
    ((60, 90), 1e-2, 16, "bumps", 1.0),
    ((64, 80), 1e-2, 64, "noise", 0.1),
    ((40, 45), 0.05, 64, "noise", 0.1),
    ((5, 13), 1e-3, 64, "noise", 1.0),
    ((33, 31), 1e-3, 7, "bumps", 1.0),
    ((12, 20, 17), 1e-3, 64, "bumps", 1.0),
    ((16, 18, 20), 0.02, 64, "noise", 1.0),
    ((20, 24, 28), 1e-3, 64, "band", 1.0),
    ((9, 9, 9), 1e-4, 8, "bumps", 1.0),
    ((7, 5, 13), 1e-2, 64, "noise", 0.1),
]


def case_id(c):
    return "%s_%s_B%d_%s" % ("x".join(map(str, c[0])), c[1], c[2], c[3])


def field(dims, kind, scale, seed=5):
    return (synth.small_field(dims, seed=seed, kind=kind) * np.float32(scale)).astype(np.float32)


def digest(b):
    return hashlib.sha256(b).hexdigest()


def oracle_artifacts(ora, dims, eb, B, kind, scale):
    d = field(dims, kind, scale)
    cp = ora.sort_cp(ora.find_cp(d, eb), d)
    types = ora.mark_types(cp, dims)
    topo = ora.encode_topo(d, eb, B, types)
    sp = ora.extract_sp(cp)
    sort = ora.encode_ints(sp, B) if len(sp) else b""
    raw, fn, _ = ora.decode_topo(topo, d.size, eb, B)
    post, restored = ora.post(raw.reshape(dims), raw.reshape(dims), fn.reshape(dims), sp, eb,
                              axis_stencil=len(dims) == 3)
    return dict(d=d, cp=cp, types=types, topo=topo, sp=sp, sort=sort, raw=raw, fn=fn, post=post,
                restored=restored)


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_oracle_matches_reference_cpu(ref, case):
    ora = ref
    dims, eb, B, kind, scale = case
    a = oracle_artifacts(ora, dims, eb, B, kind, scale)
    d = a["d"]
    rcp = ora.ref_sort_cp(ora.ref_find_cp(d, eb), d)
    assert (rcp == a["cp"]).all()
    # streams: the OpenMP layout at one thread
    assert ora.encode_topo(d, eb, B, a["types"], cpu_layout=True) == ora.ref_compress_topo(d, eb, B, rcp)
    if len(a["sp"]):
        assert ora.encode_ints(a["sp"], B, cpu_layout=True) == ora.ref_compress_sp(rcp, B)
    # the CUDA layout differs only by the tail bit-count byte
    cpu = ora.encode_topo(d, eb, B, a["types"], cpu_layout=True)
    if d.size % B == 1:
        assert len(cpu) == len(a["topo"]) + 1
    else:
        assert cpu == a["topo"]
    # decoders
    rraw, rfn = ora.ref_decompress_topo(cpu, d.size, eb, B)
    if d.size % B != 1:
        assert (rraw.view(np.int32) == a["raw"].view(np.int32)).all()
        assert (rfn == a["fn"]).all()
    if len(a["sp"]):
        ref_sp = ora.ref_decompress_sp(ora.ref_compress_sp(rcp, B)[8:], len(a["sp"]), B)
        assert (ref_sp == a["sp"]).all()
    # post-processing of the reference drivers
    rpost, rrest = ora.ref_post(a["raw"].reshape(dims), a["raw"].reshape(dims),
                                a["fn"].reshape(dims), a["sp"], eb, axis_stencil=len(dims) == 3)
    assert (rpost.view(np.int32) == a["post"].view(np.int32)).all()
    assert rrest == a["restored"]


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_oracle_matches_golden(ora, case):
    """Golden digests generated from the reference CPU build
    (tests/golden/make_golden.py)."""
    with open(GOLDEN) as f:
        gold = json.load(f)
    g = gold[case_id(case)]
    a = oracle_artifacts(ora, *case)
    assert digest(a["d"].tobytes()) == g["field"]
    assert digest(a["cp"].tobytes()) == g["cp"]
    assert digest(ora.encode_topo(a["d"], case[1], case[2], a["types"], cpu_layout=True)) == g["topo_cpu"]
    assert digest(a["sp"].astype(np.int32).tobytes()) == g["sp"]
    assert digest(a["post"].tobytes()) == g["post"]
    assert a["restored"] == g["restored"]


def test_round_trip_error_bound(ora):
    d = field((90, 110), "bumps", 1.0)
    eb = 1e-3
    cp = ora.sort_cp(ora.find_cp(d, eb), d)
    topo = ora.encode_topo(d, eb, 64, ora.mark_types(cp, d.shape))
    raw, fn, _ = ora.decode_topo(topo, d.size, eb, 64)
    assert np.abs(raw.astype(np.float64) - d.reshape(-1)).max() <= 1.01 * eb
    post, _ = ora.post(raw.reshape(d.shape), raw.reshape(d.shape), fn.reshape(d.shape),
                       ora.extract_sp(cp), eb)
    assert np.abs(post.astype(np.float64) - d).max() <= 2.0 * eb


def test_rel_error_bound_matches_float_arithmetic(ora):
    d = field((40, 50), "bumps", 3.0)
    f = synth.Field("t", d.shape, d, "rel", 1e-4)
    assert np.float32(f.abs_eb()) == np.float32(ora.rel_to_abs(d, 1e-4))


def test_bitcount_rule(ora):
    L = ora.lib()
    for m in [1, 2, 3, 7, 8, 255, 256, 65535, 65536, (1 << 24) - 1, 1 << 24, (1 << 31) - 1]:
        assert L.ora_bitcount(m) == int(np.floor(np.log2(np.float32(m)))) + 1 or m >= (1 << 17)
    assert L.ora_bitcount(0) == 0
