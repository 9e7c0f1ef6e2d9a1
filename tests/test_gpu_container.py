""".SZp containers in the reference's OpenMP layout, on the GPU.

tests/golden/containers/ holds containers written by the reference's own CPU
path at one and eight OpenMP threads (tests/golden/make_container_golden.py).
Read: every container is decompressed on the device (thread counts detected,
every chunk parsed on the device) and compared bit for bit with the oracle's
raw decode and post-processing.  Write: the fused GPU compressor's streams,
repacked with the same thread count, are the reference's bytes."""
import json
import os

import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(__file__), "golden", "containers")
MANIFEST = json.load(open(os.path.join(HERE, "manifest.json")))


@pytest.fixture(scope="module")
def T(ora):
    import torch
    import toposzp_b200
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    toposzp_b200.lib()
    return toposzp_b200


def _field(m):
    d = synth.small_field(tuple(m["dims"]), seed=m["seed"], kind=m["kind"])
    return (d * np.float32(m["scale"])).astype(np.float32)


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_container_read(T, ora, name):
    import torch
    m = MANIFEST[name]
    dims, eb, B = tuple(m["dims"]), m["eb"], m["block_size"]
    d = _field(m)
    blob = open(os.path.join(HERE, name), "rb").read()
    cont = torch.from_numpy(np.frombuffer(blob, dtype=np.uint8).copy()).cuda()
    cp = ora.sort_cp(ora.find_cp(d, eb), d)
    topo = ora.encode_topo(d, eb, B, ora.mark_types(cp, dims))
    sp = ora.extract_sp(cp)
    raw, fn, _ = ora.decode_topo(topo, d.size, eb, B)
    if ora.ref_available():
        # the reference's own reader of its container is the expectation: its
        # thread-count rule can take a multi-chunk table of a stream of two
        # blocks for one chunk and read the table as data
        # (SZp/include/szp_detect_threads.h:282-309); the device reader applies
        # the same rule and must return the same values
        ora.set_ref_threads(1)
        ts, ss = m["topo_bytes"], m["sort_bytes"]
        raw, fn = ora.ref_decompress_topo(blob[:ts], d.size, eb, B)
        e = int(np.frombuffer(blob[ts:ts + 8], dtype=np.uint64)[0]) if ss else 0
        sp = ora.ref_decompress_sp(blob[ts + 8:ts + ss], e, B) if e else np.zeros(0, np.int32)
    ctx = T.Context()
    tys = torch.empty(d.size, dtype=torch.uint8, device="cuda")
    got = ctx.decompress_container(cont, dims, eb, B, postprocess=0, types=tys)
    assert (got.cpu().numpy().view(np.int32) == raw.view(np.int32)).all()
    assert (tys.cpu().numpy() == fn.astype(np.uint8)).all()
    post = ctx.decompress_container(cont, dims, eb, B, postprocess=1).cpu().numpy()
    ref, _ = ora.post(raw.reshape(dims), raw.reshape(dims), fn.reshape(dims), sp, eb)
    assert (post.view(np.int32) == ref.reshape(-1).view(np.int32)).all()
    ctx.close()


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_container_write(T, name):
    import torch
    m = MANIFEST[name]
    dims, eb, B = tuple(m["dims"]), m["eb"], m["block_size"]
    d = _field(m)
    ctx = T.Context()
    topo, sort, _, sizes = ctx.compress(torch.from_numpy(d.reshape(-1).copy()).cuda(), dims, eb, B, index=False)
    cont = ctx.to_container(topo, sizes.topo_bytes, sort, sizes.sort_bytes, dims, B, sizes.extrema_count,
                            threads=m["threads"])
    assert cont.cpu().numpy().tobytes() == open(os.path.join(HERE, name), "rb").read()
    ctx.close()


def test_container_round_trip_many_threads(T, ora):
    """Write with 1..40 chunks and read back: the reader finds every count."""
    import torch
    dims, eb, B = (70, 90), 1e-2, 16
    d = synth.small_field(dims, seed=11, kind="noise")
    ctx = T.Context()
    dd = torch.from_numpy(d.reshape(-1).copy()).cuda()
    topo, sort, _, sizes = ctx.compress(dd, dims, eb, B, index=False)
    ref = ctx.decompress(topo, sizes.topo_bytes, sort, sizes.sort_bytes, None, dims, eb, B, postprocess=1)
    for threads in (1, 2, 3, 7, 16, 40):
        cont = ctx.to_container(topo, sizes.topo_bytes, sort, sizes.sort_bytes, dims, B, sizes.extrema_count,
                                threads=threads)
        out = ctx.decompress_container(cont, dims, eb, B, postprocess=1)
        assert torch.equal(out.view(torch.int32), ref.view(torch.int32)), threads
    ctx.close()
