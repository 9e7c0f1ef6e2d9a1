"""The sharded compression's exchange protocol (toposzp-cuda_b200/shard.py) on
gloo ranks on the host: offsets, the bin-owner all-to-all of the critical-
point pairs, the sort-position blocks that straddle slabs.  The local steps
run through a test backend built on the oracle (slab blocks from the oracle's
encoder, pairs from its CP list, dense ranks in numpy), so the assembled
streams must equal the oracle's single-field streams byte for byte -- at 2
and 3 ranks, with slab boundaries inside rows and planes, empty slabs and
bins spread over several owners."""
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _code(v):
    b = np.asarray(v, dtype=np.float32).view(np.uint32).astype(np.int64)
    b = np.where(b == 0x80000000, 0, b)
    return np.where(b & 0x80000000, (~b) & 0xFFFFFFFF, b | 0x80000000)


def _value(code):
    c = np.asarray(code, dtype=np.int64)
    bits = np.where(c & 0x80000000, c & 0x7FFFFFFF, (~c) & 0xFFFFFFFF).astype(np.uint32)
    return bits.view(np.float32)


def _bins(vals, eb):
    s = (vals.astype(np.float32) + np.float32(eb)).astype(np.float64)
    return np.trunc(s * (1.0 / np.float64(np.float32(eb)))).astype(np.int64)


class OracleBackend:
    """Local steps from the oracle, on host tensors."""

    def __init__(self, ora, field, eb):
        self.ora, self.field, self.eb = ora, field, eb
        cp = ora.find_cp(field, eb)
        self.types = ora.mark_types(cp, field.shape)
        d = field.reshape(-1)
        self.flat = np.nonzero(self.types)[0]
        self.vals = d[self.flat]
        self.is_ext = (self.types[self.flat] == 1) | (self.types[self.flat] == 2)

    def encode_slab(self, d_slab, halo_lo, shape, eb, begin, end):
        import torch
        d = self.field.reshape(-1)
        # the slab buffer carries the field from begin - halo_lo on
        assert np.array_equal(d_slab.numpy()[halo_lo: halo_lo + end - begin], d[begin:end])
        payload = self.ora.encode_topo(d[begin:end], eb, 64, self.types[begin:end])[8:]
        sel = (self.flat >= begin) & (self.flat < end)
        ext = self.is_ext[sel]
        loc = np.where(ext, np.cumsum(ext) - 1, 0xFFFFFFFF)
        pairs = np.stack([_code(self.vals[sel]), loc], 1).astype(np.int64)
        pairs = np.where(pairs >= 2 ** 31, pairs - 2 ** 32, pairs).astype(np.int32)
        return (torch.from_numpy(np.frombuffer(payload, dtype=np.uint8).copy()), torch.from_numpy(pairs),
                int(ext.sum()))

    def pair_bins(self, pairs, eb):
        import torch
        codes = pairs[:, 0].numpy().astype(np.int64) & 0xFFFFFFFF
        return torch.from_numpy(_bins(_value(codes), eb).astype(np.int32))

    def rank_pairs(self, pairs, E, eb):
        import torch
        p = pairs.numpy().astype(np.int64) & 0xFFFFFFFF
        codes, ext = p[:, 0], p[:, 1]
        vals = _value(codes)
        bins = _bins(vals, eb)
        order = np.lexsort((vals, bins))
        sp = np.zeros(E, dtype=np.int32)
        r, pb, pv = -1, None, None
        for k in order:
            if bins[k] != pb:
                r, pb, pv = 0, bins[k], vals[k]
            elif vals[k] != pv:
                r, pv = r + 1, vals[k]
            if ext[k] != 0xFFFFFFFF:
                sp[ext[k]] = r
        return torch.from_numpy(sp)

    def encode_ints(self, vals):
        import torch
        return torch.from_numpy(np.frombuffer(self.ora.encode_ints(vals.numpy(), 64)[8:], dtype=np.uint8).copy())


def _worker(rank, world, port, case, q):
    import sys
    for p in (ROOT, os.path.join(ROOT, "toposzp-cuda_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import torch
    import torch.distributed as dist
    import oracle as ora
    import shard
    import synth as sy
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        dims, kind, eb, cuts = case
        field = sy.small_field(dims, seed=5, kind=kind)
        n = field.size
        bounds = cuts if cuts else shard.slab_bounds(n, world)
        begin, end = bounds[rank], bounds[rank + 1]
        be = OracleBackend(ora, field, eb)
        lo, hi = shard.halo_of(dims, begin, end, n)
        d = field.reshape(-1)
        slab = torch.from_numpy(d[begin - lo: end + hi].copy())
        res = shard.compress_slab(be, slab, lo, dims, eb, begin, end)
        topo, sort = shard.gather_streams(res)
        if rank == 0:
            cp = ora.sort_cp(ora.find_cp(field, eb), field)
            want_t = ora.encode_topo(field, eb, 64, ora.mark_types(cp, dims))
            sp = ora.extract_sp(cp)
            want_s = ora.encode_ints(sp, 64) if len(sp) else b""
            q.put((topo == want_t, sort == want_s, res.cp_count == len(cp), res.extrema == len(sp)))
    finally:
        dist.destroy_process_group()


CASES = [
    ((37, 53), "bumps", 1e-3, None),
    ((64, 80), "noise", 1e-2, None),
    ((12, 20, 17), "bumps", 1e-3, None),
    ((16, 18, 20), "noise", 0.02, None),
    ((16, 18, 20), "noise", 0.02, [0, 64, 64, 16 * 18 * 20]),    # an empty middle slab
    ((9, 9, 9), "noise", 1e-3, [0, 128, 320, 729]),              # cuts inside rows and planes
]


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[0])) + "_" + c[1] + ("_cuts" if c[3] else ""))
def test_sharded_streams_equal_single_field(world, case):
    import torch.multiprocessing as mp
    if case[3] and len(case[3]) != world + 1:
        pytest.skip("explicit cuts for another process count")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert q.get(timeout=5) == (True, True, True, True)
