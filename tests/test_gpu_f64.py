"""GPU parity of the fp64 3D topology compressor
(szp_cuda_double_compress_topology_3d, SZp/include/szp_cuda_topology_3d.cuh:34)
through the C ABI, bit for bit:

* the reference-compatible host entry point against the oracle and against
  the reference's own CUDA library (tests/golden/f64_topo.json) on every fp64
  case, and the fp32 3D compressor on the float32 cast of the same fields
  against the reference's fp32 CUDA compressor;
* the device entry point at 0..5 repair passes against the oracle, with the
  repaired integers compared as well, on aligned and unaligned inputs;
* a 256^3 field (16.8 M elements, 163 k repaired saddles) against the oracle;
* the reference's argument handling: NULL for a non-positive bound, no data
  or no elements; errors for block sizes outside [1, 257] and bad extents."""
import hashlib
import json
import os

import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "f64_topo.json")


def sha(b):
    return hashlib.sha256(b).hexdigest()


@pytest.fixture(scope="module")
def T(ora):
    import torch
    import toposzp_b200
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    toposzp_b200.lib()
    return toposzp_b200


def types_of(ora, cp, dims):
    return ora.mark_types(cp.view(ora.CP3_DT).reshape(-1), dims)


@pytest.mark.parametrize("name", list(synth.f64_cases()))
def test_host_entry_point(T, ora, name):
    with open(GOLD) as fh:
        g = json.load(fh)[name]
    d, cp, eb, B = synth.f64_case(name)
    s = T.double_compress_topology_3d(d, eb, B, cp.view(T.CP3_DT).reshape(-1))
    assert len(s) == g["f64_bytes"] and sha(s) == g["f64"]
    assert s == ora.double_compress_topo_3d(d, eb, B, types_of(ora, cp, d.shape), d.shape)
    s32 = T.compress_topology(d.astype(np.float32), float(np.float32(eb)), B, cp.view(T.CP3_DT).reshape(-1))
    assert len(s32) == g["f32_bytes"] and sha(s32) == g["f32"]


@pytest.mark.parametrize("name", ["noise_32x33x35", "noise_tail_17x19x23_B7", "special_20x21x22", "thin_3x40x50"])
@pytest.mark.parametrize("offset", [0, 1])
def test_device_entry_point_passes(T, ora, name, offset):
    import torch
    d, cp, eb, B = synth.f64_case(name)
    t = types_of(ora, cp, d.shape)
    n = d.size
    # offset 1: the field starts 8 bytes past a 16-byte boundary (scalar loads)
    buf = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
    buf[offset: offset + n] = torch.from_numpy(d.reshape(-1))
    dd = buf[offset: offset + n]
    dcp = torch.from_numpy(cp.reshape(-1).copy()).cuda()
    out = torch.zeros(T.lib().szp_b200_topo_bound(n, B), dtype=torch.uint8, device="cuda")
    q = torch.zeros(n, dtype=torch.int32, device="cuda")
    ctx = T.Context()
    for passes in range(6):
        m = ctx.compress_f64(dd, d.shape, eb, B, dcp, len(cp), out, passes=passes, d_q=q)
        so, qo = ora.double_compress_topo_3d(d, eb, B, t, d.shape, passes=passes, with_q=True)
        assert out[:m].cpu().numpy().tobytes() == so, passes
        assert (q.cpu().numpy() == qo).all(), passes
    # no critical points: plain quantization, all tags 0
    m = ctx.compress_f64(dd, d.shape, eb, B, None, 0, out)
    assert out[:m].cpu().numpy().tobytes() == ora.double_compress_topo_3d(d, eb, B, np.zeros(n, np.uint8), d.shape)
    ctx.close()


def test_large_field(T, ora):
    import torch
    dims = (256, 256, 256)
    d = synth.f64_field(dims, seed=21, kind="noise")
    cp = synth.f64_critical_points(d)
    eb, B = 0.05, 64
    t = types_of(ora, cp, dims)
    so, qo = ora.double_compress_topo_3d(d, eb, B, t, dims, with_q=True)
    _, q0 = ora.double_compress_topo_3d(d, eb, B, t, dims, passes=0, with_q=True)
    assert (qo != q0).sum() > 100000
    ctx = T.Context()
    dd = torch.from_numpy(d.reshape(-1)).cuda()
    dcp = torch.from_numpy(cp.reshape(-1).copy()).cuda()
    out = torch.zeros(T.lib().szp_b200_topo_bound(d.size, B), dtype=torch.uint8, device="cuda")
    m = ctx.compress_f64(dd, dims, eb, B, dcp, len(cp), out)
    assert m == len(so)
    assert out[:m].cpu().numpy().tobytes() == so
    ctx.close()


def test_argument_handling(T):
    import ctypes as C
    L = T.lib()
    d = np.ones((4, 5, 6))
    sz = C.c_size_t(123)
    p = d.ctypes.data_as(C.c_void_p)
    # the reference returns NULL with *outSize 0 for these, without a message
    for eb, ptr, n in ((0.0, p, d.size), (-1.0, p, d.size), (1e-3, None, d.size), (1e-3, p, 0)):
        sz.value = 123
        assert not L.szp_cuda_double_compress_topology_3d(ptr, C.byref(sz), eb, n, 64, None, 0, 4, 5, 6)
        assert sz.value == 0
    for B in (0, 258):
        assert not L.szp_cuda_double_compress_topology_3d(p, C.byref(sz), 1e-3, d.size, B, None, 0, 4, 5, 6)
        assert "blockSize" in T.last_error()
    assert not L.szp_cuda_double_compress_topology_3d(p, C.byref(sz), 1e-3, d.size, 64, None, 0, 0, 5, 6)
    assert "dimensions" in T.last_error()
    # the extreme block sizes compress
    for B in (1, 257):
        assert T.double_compress_topology_3d(d, 1e-3, B, np.zeros(0, T.CP3_DT))
