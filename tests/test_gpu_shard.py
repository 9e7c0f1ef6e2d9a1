"""The sharded compression on the GPU: two or three processes share the one
device of this run (each with its own context and workspace, collectives over
gloo on the host; no kernel waits on another process), each encodes its
block-aligned slab with the library's slab encoder and ranks the pairs of the
bins it owns on the device.  The assembled streams must equal the single-
device fused compression's streams byte for byte, and every process's slab
must decode to the single-device raw decode of that slab."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, case, q):
    import sys
    for p in (ROOT, os.path.join(ROOT, "toposzp-cuda_b200")):
        sys.path.insert(0, p)
    import torch
    import torch.distributed as dist
    import shard
    import synth
    import toposzp_b200 as T
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        dims, kind, eb = case
        field = synth.small_field(dims, seed=9, kind=kind) if kind != "c3" else synth.band_limited(dims, 2)
        n = field.size
        bounds = shard.slab_bounds(n, world)
        begin, end = bounds[rank], bounds[rank + 1]
        lo, hi = shard.halo_of(dims, begin, end, n)
        d = torch.from_numpy(field.reshape(-1).copy())
        ctx = T.Context()
        slab = d[begin - lo: end + hi].cuda()
        res = shard.compress_slab(shard.CudaBackend(T, ctx), slab, lo, dims, eb, begin, end)
        raw = shard.decompress_slab_raw(T, ctx, res, begin, end, eb).cpu().numpy() if end > begin else None
        topo, sort = shard.gather_streams(res)
        single = T.Context()
        dd = d.cuda()
        t, s, _, sz = single.compress(dd, dims, eb, 64, index=False)
        ok_slab = True
        if raw is not None:
            full = single.decompress(t, sz.topo_bytes, s, sz.sort_bytes, None, dims, eb, 64, postprocess=0)
            ok_slab = bool(np.array_equal(raw.view(np.int32), full[begin:end].cpu().numpy().view(np.int32)))
        allok = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(allok, torch.tensor([int(ok_slab)], dtype=torch.int64))
        if rank == 0:
            want_t = t[: sz.topo_bytes].cpu().numpy().tobytes()
            want_s = s[: sz.sort_bytes].cpu().numpy().tobytes()
            q.put((topo == want_t, sort == want_s, res.cp_count == sz.cp_count, res.extrema == sz.extrema_count,
                   all(int(x) for x in allok)))
        ctx.close()
        single.close()
    finally:
        dist.destroy_process_group()


CASES = [
    ((300, 500), "bumps", 1e-3),
    ((64, 70, 90), "bumps", 1e-3),
    ((40, 45, 50), "noise", 0.02),
    ((128, 128, 128), "c3", 1e-4),
]


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[0])) + "_" + c[1])
def test_sharded_streams_on_gpu(world, case):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert q.get(timeout=5) == (True, True, True, True, True)
