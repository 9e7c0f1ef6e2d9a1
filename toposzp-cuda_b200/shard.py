"""One field compressed across several processes (one per device).

The field is split into block-aligned flat-index slabs (multiples of the
blockSize, 64); each process holds its slab plus a halo of one plane (one row
in 2D) + 1 element on either side, encodes its topology blocks and critical-
point pairs on its own device, and the processes then exchange what the
single-device path computes globally:

  1. stream offsets: an all-gather of every slab's payload bytes, critical
     points and extrema (exclusive prefixes give each slab's place);
  2. sort positions: a critical point's sort position is its dense rank among
     the critical points of its quantization bin over the WHOLE field, so the
     pairs {value code, global extremum index} go to the process that owns
     their bin (bins split into equal ranges over the global bin span), which
     ranks them and sends each extremum's position back (two all-to-alls);
  3. sort-position blocks: blocks of 64 positions may straddle slabs; each
     block belongs to the process holding its first extremum, which receives
     the up to 63 following positions from the first positions every process
     shares (an all-gather of at most 63 ints each).

The topology payload and the sort-position payload of the slabs, concatenated
in slab order after the 8-byte header, are the single-device streams byte for
byte.  Decompression is per slab (blocks are self-contained); the post-
processing, whose serial raster order spans the whole field, runs on one
device.

The local steps go through a backend object (``CudaBackend`` here: the
library's slab encoder, bins, rank and integer encoder), so the exchange
protocol is the same whatever computes the local steps.  Collectives use the
process group's backend: device tensors with NCCL, host tensors with gloo.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch
import torch.distributed as dist

B = 64
NO_EXT = 0xFFFFFFFF


def slab_bounds(n: int, world: int, B: int = B):
    """Block-aligned slab boundaries: world + 1 increasing offsets, 0 and n at
    the ends, equal shares rounded to blocks (a slab may be empty)."""
    cuts = [0]
    for r in range(1, world):
        c = (n * r // world) // B * B
        cuts.append(max(cuts[-1], min(c, n)))
    cuts.append(n)
    return cuts


def halo_of(shape, begin: int, end: int, n: int):
    """(halo_lo, halo_hi): elements the slab's buffer holds before begin and
    after end -- one plane (one row) + 1, the low side rounded up to a
    multiple of 4 so the slab keeps the field's 16-byte alignment."""
    reach = (shape[1] * shape[2] if len(shape) == 3 else shape[1]) + 1
    lo = min(begin, (reach + 3) // 4 * 4)
    hi = min(n - end, reach)
    return lo, hi


# ---------------------------------------------------------------------------
# collectives (device tensors with NCCL, host tensors with gloo)
# ---------------------------------------------------------------------------

class Exchange:
    def __init__(self, group=None):
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.host = dist.get_backend(group) == "gloo"

    def allgather_i64(self, vals, device) -> torch.Tensor:
        """[world, len(vals)] int64 of every process's values."""
        t = torch.tensor(vals, dtype=torch.int64, device="cpu" if self.host else device)
        out = [torch.empty_like(t) for _ in range(self.world)]
        dist.all_gather(out, t, group=self.group)
        return torch.stack(out).to(device)

    def alltoallv(self, send: torch.Tensor, counts: torch.Tensor):
        """Variable all-to-all of a 1-D int64 tensor grouped by destination
        (counts[d] items for process d); returns (received, counts per source)."""
        dev = send.device
        cnt = counts.to(torch.int64)
        cin = cnt.cpu() if self.host else cnt
        cout = torch.empty_like(cin)
        dist.all_to_all_single(cout, cin, group=self.group)
        cout_h = cout.cpu()
        s = send.cpu() if self.host else send
        r = torch.empty(int(cout_h.sum()), dtype=torch.int64, device=s.device)
        dist.all_to_all_single(r, s.contiguous(), output_split_sizes=cout_h.tolist(),
                               input_split_sizes=cnt.cpu().tolist(), group=self.group)
        return r.to(dev), cout_h.to(dev)

    def gather_bytes(self, part: torch.Tensor, dst: int = 0):
        """Concatenation, in process order, of every process's uint8 part on
        process dst (None elsewhere)."""
        dev = part.device
        sizes = self.allgather_i64([part.numel()], dev)[:, 0].cpu().tolist()
        m = max(sizes + [1])
        buf = torch.zeros(m, dtype=torch.uint8, device="cpu" if self.host else dev)
        buf[: part.numel()] = part.to(buf.device)
        out = [torch.empty_like(buf) for _ in range(self.world)]
        dist.all_gather(out, buf, group=self.group)
        if self.rank != dst:
            return None
        return b"".join(out[r][: sizes[r]].cpu().numpy().tobytes() for r in range(self.world))


# ---------------------------------------------------------------------------
# local steps on this process's device
# ---------------------------------------------------------------------------

class CudaBackend:
    """The library's slab encoder, pair bins, rank and integer encoder."""

    def __init__(self, T, ctx):
        self.T, self.ctx, self.L = T, ctx, T.lib()

    def encode_slab(self, d_slab, halo_lo, shape, eb, begin, end):
        m = end - begin
        dev = d_slab.device
        cap = self.L.szp_b200_topo_bound(m, B)
        payload = torch.empty(cap, dtype=torch.uint8, device=dev)
        pairs = torch.empty(2 * max(m, 1), dtype=torch.int32, device=dev)
        sz = self.T.SlabSizes()
        rc = self.L.szp_b200_topo_encode_slab_dev(
            self.ctx.ptr, C.c_void_p(d_slab.data_ptr()), halo_lo, self.T.geom_of(shape), float(eb), B, begin, end,
            C.c_void_p(payload.data_ptr()), cap, C.c_void_p(pairs.data_ptr()), m, C.byref(sz))
        if rc:
            raise self.T.ToposzpError(self.T.last_error())
        return payload[: sz.payload_bytes], pairs[: 2 * sz.cp_count].view(-1, 2), int(sz.extrema_count)

    def pair_bins(self, pairs, eb):
        K = pairs.shape[0]
        bins = torch.empty(K, dtype=torch.int32, device=pairs.device)
        pc = pairs.contiguous()
        if K and self.L.szp_b200_pair_bins_dev(self.ctx.ptr, C.c_void_p(pc.data_ptr()), K, float(eb),
                                               C.c_void_p(bins.data_ptr())):
            raise self.T.ToposzpError(self.T.last_error())
        return bins

    def rank_pairs(self, pairs, E, eb):
        sp = torch.empty(max(E, 1), dtype=torch.int32, device=pairs.device)
        K = pairs.shape[0]
        pc = pairs.contiguous()
        if K and E and self.L.szp_b200_rank_pairs_dev(self.ctx.ptr, C.c_void_p(pc.data_ptr()), K, E, float(eb),
                                                      C.c_void_p(sp.data_ptr())):
            raise self.T.ToposzpError(self.T.last_error())
        return sp[:E]

    def encode_ints(self, vals):
        n = vals.numel()
        cap = self.L.szp_b200_sort_bound(n, B)
        out = torch.empty(cap, dtype=torch.uint8, device=vals.device)
        nb = C.c_size_t(0)
        vc = vals.contiguous()
        if self.L.szp_b200_encode_ints_dev(self.ctx.ptr, C.c_void_p(vc.data_ptr()), n, B,
                                           C.c_void_p(out.data_ptr()), cap, C.byref(nb)):
            raise self.T.ToposzpError(self.T.last_error())
        return out[8: nb.value]


# ---------------------------------------------------------------------------
# the sharded compression
# ---------------------------------------------------------------------------

@dataclass
class ShardResult:
    topo_part: torch.Tensor     # this slab's topology blocks (uint8)
    topo_offset: int            # their payload offset in the whole stream
    topo_payload: int           # payload bytes of the whole stream
    sort_part: torch.Tensor     # the sort-position blocks this process owns (uint8)
    sort_offset: int
    sort_payload: int
    cp_count: int               # critical points of the whole field
    extrema: int                # extrema of the whole field
    slab_extrema: int
    sort_positions: torch.Tensor  # this slab's extrema, raster order


def _u32(t: torch.Tensor) -> torch.Tensor:
    return t.to(torch.int64) & 0xFFFFFFFF


def compress_slab(backend, d_slab, halo_lo: int, shape, eb: float, begin: int, end: int,
                  group=None) -> ShardResult:
    """This process's part of the compression of the field `shape` (see the
    module docstring).  d_slab holds elements begin - halo_lo .. min(n, end +
    one plane (row) + 1) of the field.  Every process takes every collective
    step, an empty slab (begin == end) included."""
    ex = Exchange(group)
    world, rank = ex.world, ex.rank
    dev = d_slab.device
    if end > begin:
        payload, pairs, E_r = backend.encode_slab(d_slab, halo_lo, shape, eb, begin, end)
    else:
        payload = torch.zeros(0, dtype=torch.uint8, device=dev)
        pairs = torch.zeros((0, 2), dtype=torch.int32, device=dev)
        E_r = 0
    K_r = pairs.shape[0]
    # 1. offsets and totals
    stats = ex.allgather_i64([payload.numel(), K_r, E_r], dev).cpu()
    pb, Ks, Es = stats[:, 0].tolist(), stats[:, 1].tolist(), stats[:, 2].tolist()
    topo_offset, topo_payload = sum(pb[:rank]), sum(pb)
    e_pref, e_tot = sum(Es[:rank]), sum(Es)
    # 2. global ranks: pairs to the owners of their bins
    bins = backend.pair_bins(pairs, eb).to(torch.int64)
    big = 1 << 40
    lo = int(bins.min()) if K_r else big
    hi = int(bins.max()) if K_r else -big
    span = ex.allgather_i64([lo, hi], dev).cpu()
    bmin, bmax = int(span[:, 0].min()), int(span[:, 1].max())
    width = max(bmax - bmin + 1, 1)
    empty = torch.zeros(0, dtype=torch.int64, device=dev)
    owner = ((bins - bmin) * world) // width if K_r else empty
    code = _u32(pairs[:, 0]) if K_r else empty
    ext = _u32(pairs[:, 1]) if K_r else empty
    gext = torch.where(ext == NO_EXT, torch.full_like(ext, NO_EXT), ext + e_pref)
    rec = code | (gext << 32)
    order = torch.argsort(owner, stable=True)
    counts = torch.bincount(owner, minlength=world)
    recv, rcounts = ex.alltoallv(rec[order], counts)
    rg = (recv >> 32) & 0xFFFFFFFF
    is_ext = rg != NO_EXT
    E_o = int(is_ext.sum())
    loc = torch.cumsum(is_ext.to(torch.int64), 0) - 1
    loc = torch.where(is_ext, loc, torch.full_like(loc, NO_EXT))
    pairs_o = torch.stack([(recv & 0xFFFFFFFF), loc], 1)
    pairs_o = torch.where(pairs_o >= 2 ** 31, pairs_o - 2 ** 32, pairs_o).to(torch.int32).contiguous()
    sp_o = backend.rank_pairs(pairs_o, E_o, eb).to(torch.int64)
    src = torch.repeat_interleave(torch.arange(world, device=dev), rcounts.to(torch.int64))
    ext_src = src[is_ext]
    reply = rg[is_ext] | (sp_o << 32)
    back, _ = ex.alltoallv(reply[torch.argsort(ext_src, stable=True)], torch.bincount(ext_src, minlength=world))
    sp_local = torch.empty(E_r, dtype=torch.int64, device=dev)
    if E_r:
        sp_local[(back & 0xFFFFFFFF) - e_pref] = back >> 32
    sp_local = sp_local.to(torch.int32)
    # 3. sort-position blocks owned here: those whose first extremum is here
    h = min(E_r, B - 1)
    head = torch.zeros(B - 1, dtype=torch.int64, device=dev)
    head[:h] = sp_local[:h].to(torch.int64)
    heads = ex.allgather_i64(head.cpu().tolist() + [h], dev).cpu()
    s0 = -(-e_pref // B) * B
    sort_part = torch.zeros(0, dtype=torch.uint8, device=dev)
    if s0 < e_pref + E_r:
        s_end = min(e_tot, -(-(e_pref + E_r) // B) * B)
        vals = [sp_local[s0 - e_pref:]]
        need = s_end - (e_pref + E_r)
        r = rank + 1
        while need > 0 and r < world:
            take = min(need, int(heads[r, B - 1]))
            if take:
                vals.append(heads[r, :take].to(torch.int32).to(dev))
            need -= take
            r += 1
        sort_part = backend.encode_ints(torch.cat(vals))
    ss = ex.allgather_i64([sort_part.numel()], dev)[:, 0].cpu().tolist()
    return ShardResult(payload, topo_offset, topo_payload, sort_part, sum(ss[:rank]), sum(ss), sum(Ks), e_tot, E_r,
                       sp_local)


def gather_streams(res: ShardResult, group=None, dst: int = 0):
    """(topology stream, sort-position stream) of the whole field on process
    dst -- the single-device streams' bytes -- and (None, None) elsewhere."""
    ex = Exchange(group)
    topo = ex.gather_bytes(res.topo_part, dst)
    sort = ex.gather_bytes(res.sort_part, dst)
    if ex.rank != dst:
        return None, None
    hdr = bytes(8)
    return hdr + topo, (hdr + sort) if res.extrema else b""


def decompress_slab_raw(T, ctx, res: ShardResult, begin: int, end: int, eb: float, types=None):
    """Decoded values (no post-processing) of this process's slab from its own
    topology blocks: the blocks are self-contained, so the slab decodes as a
    stream of its own."""
    m = end - begin
    dev = res.topo_part.device
    s = torch.zeros(8 + res.topo_part.numel() + 64, dtype=torch.uint8, device=dev)
    s[8: 8 + res.topo_part.numel()] = res.topo_part
    return ctx.decompress(s, 8 + res.topo_part.numel(), None, 0, None, (1, m), eb, B, postprocess=0, types=types)
