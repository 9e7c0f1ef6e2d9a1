"""Bit-exact parity with the reference's own CUDA implementation, run on the
same GPU (oracle/_ref/libszp_ref_cuda.so, compiled from the reference's CUDA
sources; each reference run is a child process, oracle/ref_cuda_run.py).

Per field, the reference's driver sequence (find CPs, sort, sort-position
stream, topology stream, decode) against the fused device path of this
library:

* topology stream: identical bytes
* raw decoded field and per-element types: identical
* sort positions: the reference's CUDA sort writes the dense rank of a CP in
  its bin minus one for the first CP of every run of equal values (an
  exclusive scan of the new-value flags, szp_cuda_topology.cu:253,
  szp_cuda_topology_3d.cu:387), with the tie order of an unstable sort; its
  OpenMP sort, which this library follows, writes the dense rank.  Checked:
  the reference's CUDA positions obey that rule exactly on its own CP list,
  and this library's positions of the extrema, in raster order, equal the
  dense ranks of that same list (the reference's CUDA finder appends CPs in
  atomic order, so its sort-position stream itself changes from run to run;
  this library emits raster order, the order of the reference's OpenMP path
  at one thread)
* the reference's own sort-position stream round-trips through its decoder
"""
import hashlib

import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu


def sha(b):
    return hashlib.sha256(b).hexdigest()


@pytest.fixture(scope="module")
def R(ora):
    import ref_cuda_run
    if not ref_cuda_run.available():
        pytest.skip("reference CUDA library not built (reference sources absent at build time)")
    return ref_cuda_run


@pytest.fixture(scope="module")
def T():
    import torch
    import toposzp_b200
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    toposzp_b200.lib()
    return toposzp_b200


def ours(T, d, eb, B):
    import torch
    dims = d.shape
    ctx = T.Context()
    dd = torch.from_numpy(d.reshape(-1).copy()).cuda()
    topo, sort, idx, sizes = ctx.compress(dd, dims, eb, B)
    tys = torch.empty(d.size, dtype=torch.uint8, device="cuda")
    raw = ctx.decompress(topo, sizes.topo_bytes, sort, sizes.sort_bytes, None, dims, eb, B, postprocess=0, types=tys)
    topo_b = topo[: sizes.topo_bytes].cpu().numpy().tobytes()
    sort_b = sort[: sizes.sort_bytes].cpu().numpy().tobytes()
    sp = (T.decompress_sort_positions(sort_b, sizes.extrema_count, B) if sizes.extrema_count
          else np.zeros(0, np.int32))
    out = {"cp_count": sizes.cp_count, "extrema": sizes.extrema_count, "topo_bytes": sizes.topo_bytes,
           "topo": sha(topo_b), "raw": sha(raw.cpu().numpy().tobytes()), "types": sha(tys.cpu().numpy().tobytes()),
           "sp_raster": sha(np.ascontiguousarray(sp, dtype=np.int32).tobytes())}
    ctx.close()
    return out


CASES = {
    "2d_37x53_B64": lambda: (synth.small_field((37, 53), seed=7), 1e-3, 64),
    "2d_33x31_B7": lambda: (synth.small_field((33, 31), seed=8), 1e-3, 7),
    "2d_noise_64x80": lambda: (synth.small_field((64, 80), seed=9, kind="noise") * np.float32(0.1), 1e-2, 64),
    "3d_40x50x60": lambda: (synth.small_field((40, 50, 60), seed=10), 1e-3, 64),
    "3d_noise_16x18x20_B257": lambda: (synth.small_field((16, 18, 20), seed=11, kind="noise"), 0.02, 257),
    "3d_band_7x5x13_B1": lambda: (synth.small_field((7, 5, 13), seed=12, kind="noise"), 1e-2, 1),
}


@pytest.mark.parametrize("name", list(CASES))
def test_small_fields(T, R, name):
    d, eb, B = CASES[name]()
    d = np.ascontiguousarray(d, dtype=np.float32)
    check(R.run(d, eb, B), ours(T, d, eb, B))


def check(r, o):
    for k in o:
        assert o[k] == (r["sp_dense_raster"] if k == "sp_raster" else r[k]), k
    assert r["cuda_sort_relation"]
    assert r["sort_stream_round_trip"]


@pytest.mark.parametrize("which", ["c1", "c2"])
def test_configs(T, R, which):
    f = synth.config1() if which == "c1" else synth.config2()
    eb = f.abs_eb()
    check(R.run(f.data, eb, f.block_size), ours(T, f.data, eb, f.block_size))
