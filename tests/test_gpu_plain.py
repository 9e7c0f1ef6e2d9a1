"""GPU parity of the plain (non-topology) codec through the C ABI
(SZp/include/szp_cuda_compress.cuh:22-64, szp_cuda_decompress.cuh:23-57),
bit for bit:

* the reference-compatible entry points against the reference's own CUDA
  codec (tests/golden/plain.json) and the oracle on 36 cases: float and
  double, random-access and threadblock modes, blockSize 1/7/64/256/1025,
  one- and two-element fields, a tail block of one element, +-inf / NaN /
  values beyond the int range;
* the predict-quantization helpers against the reference;
* multi-chunk offset tables (the layout of the reference's OpenMP
  compressors) decoded with the reference's thread-count detection;
* the device entry points (compress both modes, random-access decompress with
  the device parser) on a 64 M-element field against the oracle;
* the reference's argument handling."""
import ctypes as C
import hashlib
import json
import os

import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "plain.json")


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


def gold():
    with open(GOLD) as fh:
        return json.load(fh)


@pytest.mark.parametrize("name", list(synth.plain_cases()))
def test_reference_entry_points(T, ora, name):
    g = gold()[name]
    x, eb, B, tb = synth.plain_case(name)
    assert sha(np.ascontiguousarray(x).tobytes()) == g["field"]
    s = T.plain_compress(x, eb, B, tb)
    assert s == ora.plain_compress(x, eb, B, tb)
    if g["reference_round_trip"]:
        assert len(s) == g["bytes"] and sha(s) == g["stream"]
    else:
        # the reference's output is undefined here (threadblock mode at
        # blockSize 1025 overruns its 1024-entry delta arrays)
        assert tb and B == 1025
    v = T.plain_decompress(s, x.size, eb, B, x.dtype, tb)
    vo, _ = ora.plain_decompress(s, x.size, eb, B, x.dtype, tb)
    assert v.tobytes() == vo.tobytes()
    if g["values_oracle_agrees"] and g["reference_round_trip"]:
        assert sha(v.tobytes()) == g["values"]
    with np.errstate(invalid="ignore"):
        fin = np.isfinite(x) & (np.abs(x.astype(np.float64)) / eb < 2.0 ** 31 - 2)
    assert np.abs(v.astype(np.float64) - x)[fin].max(initial=0.0) <= eb * 1.01
    if "predict" in g:
        assert sha(T.predict_quantization(x, eb).tobytes()) == g["predict"]
        assert sha(T.predict_quantization(x, eb, threadblock=True).tobytes()) == g["predict"]


def _multi_chunk(ora, x, eb, B, tb, chunks):
    """A T-chunk stream: chunk c holds x[lo:hi] as its own one-chunk body."""
    dbl = x.dtype == np.float64
    es = 8 if dbl else 4
    n = x.size
    tbs = n // chunks
    bodies = []
    for c in range(chunks):
        lo, hi = c * tbs, (n if c == chunks - 1 else (c + 1) * tbs)
        bodies.append(ora.plain_compress(x[lo:hi], eb, B, tb)[es + 8:])
    offs, o = [], 0
    for b in bodies:
        offs.append(o)
        o += len(b)
    head = ora.plain_compress(x[:1], eb, B, tb)[:es]
    return head + np.array(offs, dtype=np.uint64).tobytes() + b"".join(bodies)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("tb", [False, True])
@pytest.mark.parametrize("chunks,B", [(3, 64), (8, 7), (5, 1025)])
def test_multi_chunk_tables(T, ora, dtype, tb, chunks, B):
    x = synth.plain_field(20011, seed=31, kind="walk", dtype=dtype)
    eb = 1e-3
    s = _multi_chunk(ora, x, eb, B, tb, chunks)
    v = T.plain_decompress(s, x.size, eb, B, dtype, tb)
    vo, _ = ora.plain_decompress(s, x.size, eb, B, dtype, tb)
    assert v.tobytes() == vo.tobytes()
    assert np.abs(v.astype(np.float64) - x).max() <= eb * 1.01


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_device_entry_points_large(T, ora, dtype):
    import torch
    n = 1 << 26
    x = synth.plain_field(n, seed=41, kind="wave", dtype=dtype)
    eb, B = 1e-4, 64
    ctx = T.Context()
    dx = torch.from_numpy(x).cuda()
    cap = T.lib().szp_b200_plain_bound(n, B, int(dtype == np.float64), 0)
    out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    m = ctx.plain_compress(dx, eb, B, out)
    so = ora.plain_compress(x, eb, B)
    assert m == len(so) and out[:m].cpu().numpy().tobytes() == so
    y = torch.empty_like(dx)
    ctx.plain_decompress(out, m, n, eb, B, y)
    vo, _ = ora.plain_decompress(so, n, eb, B, dtype)
    assert y.cpu().numpy().tobytes() == vo.tobytes()
    # threadblock mode through the device compressor
    m2 = ctx.plain_compress(dx[:1000003], eb, B, out, threadblock=True)
    assert out[:m2].cpu().numpy().tobytes() == ora.plain_compress(x[:1000003], eb, B, True)
    ctx.close()


def test_argument_handling(T):
    L = T.lib()
    x = np.ones(100, np.float32)
    sz = C.c_size_t(7)
    p = x.ctypes.data_as(C.c_void_p)
    for eb, ptr, n in ((0.0, p, 100), (-1.0, p, 100), (1e-3, p, 0)):
        sz.value = 7
        assert not L.szp_cuda_float_compress_randomaccess(ptr, C.byref(sz), eb, n, 64)
        assert sz.value == 0
    for B in (0, 1026):
        assert not L.szp_cuda_float_compress_threadblock(p, C.byref(sz), 1e-3, 100, B)
        assert "blockSize" in T.last_error()
    sz.value = 7
    L.szp_cuda_float_compress_randomaccess_arg(None, p, C.byref(sz), 1e-3, 100, 64)
    assert sz.value == 0
    # the largest block size compresses and decompresses
    y = synth.plain_field(5000, seed=3, kind="walk")
    s = T.plain_compress(y, 1e-3, 1025)
    assert np.abs(T.plain_decompress(s, y.size, 1e-3, 1025) - y).max() <= 1.01e-3
