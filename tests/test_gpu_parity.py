"""GPU parity of the C ABI against the oracle (bit-exact).

Every check goes through libtoposzp_b200.so: the reference-compatible entry
points (host buffers) and the fused device entry points (torch CUDA tensors).
Integer / byte outputs and decoded / post-processed floats must be identical
to the oracle's, bit for bit.
"""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu

CASES_2D = [
    # dims, eb, B, kind, scale
    ((37, 53), 1e-3, 64, "bumps", 1.0),
    ((64, 80), 1e-2, 64, "noise", 0.1),
    ((60, 90), 1e-2, 16, "bumps", 1.0),
    ((33, 31), 1e-3, 7, "bumps", 1.0),
    ((5, 13), 1e-3, 64, "noise", 1.0),        # n % B == 1: anchor-only tail block
    ((40, 45), 0.05, 1, "noise", 0.1),        # blockSize 1
    ((41, 47), 1e-3, 257, "noise", 1.0),      # largest blockSize
    ((3, 3), 1e-3, 64, "noise", 1.0),
    ((50, 70), 1e-5, 64, "noise", 1e3),       # wide deltas: bit counts > 24
    ((30, 30), 1e-9, 32, "noise", 1e3),       # quantization saturates the int range
    ((180, 360), 1e-3, 64, "bumps", 1.0),
]

CASES_3D = [
    ((12, 20, 17), 1e-3, 64, "bumps", 1.0),
    ((16, 18, 20), 0.02, 64, "noise", 1.0),
    ((20, 24, 28), 1e-3, 64, "band", 1.0),
    ((9, 9, 9), 1e-4, 8, "bumps", 1.0),
    ((3, 3, 3), 1e-3, 64, "noise", 1.0),
    ((7, 5, 13), 1e-2, 64, "noise", 0.1),     # 455 % 64 == 7
    ((40, 50, 60), 1e-3, 64, "bumps", 1.0),   # the reference's own 3D test shape
]


def field(dims, kind, scale, seed=7):
    d = synth.small_field(dims, seed=seed, kind=kind)
    return (d * np.float32(scale)).astype(np.float32)


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.int32)


@pytest.fixture(scope="module")
def T(ora):
    import torch
    import toposzp_b200
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    toposzp_b200.lib()
    return toposzp_b200


@pytest.mark.parametrize("case", CASES_2D + CASES_3D, ids=lambda c: "x".join(map(str, c[0])) + "_B%d" % c[2])
def test_reference_api_parity(T, ora, case):
    dims, eb, B, kind, scale = case
    d = field(dims, kind, scale)
    # find
    cp = T.find_critical_points(d, eb)
    ocp = ora.find_cp(d, eb)
    assert len(cp) == len(ocp)
    assert (cp == ocp).all()
    if len(ocp) == 0:
        return
    # sort positions (of the oracle's list: the entry point ranks any list)
    scp = T.sort_critical_points(ocp, d)
    oscp = ora.sort_cp(ocp, d)
    assert (scp == oscp).all()
    # topology stream
    types = ora.mark_types(oscp, dims)
    s_gpu = T.compress_topology(d, eb, B, oscp)
    s_ora = ora.encode_topo(d, eb, B, types)
    assert s_gpu == s_ora
    # sort-position stream
    sp = ora.extract_sp(oscp)
    sp_gpu = T.compress_sort_positions(oscp, B)
    sp_ora = ora.encode_ints(sp, B) if len(sp) else b""
    assert sp_gpu == sp_ora
    # decode
    out, fn = T.decompress_topology(s_gpu, d.size, eb, B)
    oout, ofn, used = ora.decode_topo(s_ora, d.size, eb, B)
    assert used == len(s_ora)
    assert (bits(out) == bits(oout)).all()
    assert (fn == ofn).all()
    if len(sp):
        dsp = T.decompress_sort_positions(sp_gpu, len(sp), B)
        assert (dsp == sp).all()
    # raw error bound (reference tests use 1.01 eb) where float32 can resolve eb
    if np.abs(d).max() * (1.0 / eb) < 2e9 and np.spacing(np.float32(np.abs(d).max())) < 0.01 * eb:
        assert np.abs(out.astype(np.float64) - d.reshape(-1)).max() <= 1.01 * eb


@pytest.mark.parametrize("case", CASES_2D + CASES_3D, ids=lambda c: "x".join(map(str, c[0])) + "_B%d" % c[2])
def test_fused_device_parity(T, ora, case):
    import torch
    dims, eb, B, kind, scale = case
    d = field(dims, kind, scale)
    ctx = T.Context()
    dd = torch.from_numpy(d.reshape(-1).copy()).cuda()
    topo, sort, idx, sizes = ctx.compress(dd, dims, eb, B)
    ocp = ora.sort_cp(ora.find_cp(d, eb), d)
    types = ora.mark_types(ocp, dims)
    s_ora = ora.encode_topo(d, eb, B, types)
    sp = ora.extract_sp(ocp)
    assert sizes.cp_count == len(ocp)
    assert sizes.extrema_count == len(sp)
    assert sizes.topo_bytes == len(s_ora)
    assert topo[: sizes.topo_bytes].cpu().numpy().tobytes() == s_ora
    if len(sp):
        assert sort[: sizes.sort_bytes].cpu().numpy().tobytes() == ora.encode_ints(sp, B)
    else:
        assert sizes.sort_bytes == 0
    # raw decode
    raw = ctx.decompress(topo, sizes.topo_bytes, sort, sizes.sort_bytes, idx, dims, eb, B,
                         postprocess=0)
    oraw, ofn, _ = ora.decode_topo(s_ora, d.size, eb, B)
    assert (bits(raw.cpu().numpy()) == bits(oraw)).all()
    # decode + post-processing
    for mode in ([1, 2] if len(dims) == 3 else [1]):
        tys = torch.empty(d.size, dtype=torch.uint8, device="cuda")
        post = ctx.decompress(topo, sizes.topo_bytes, sort, sizes.sort_bytes, idx, dims, eb, B,
                              postprocess=mode, types=tys)
        ref, _ = ora.post(oraw.reshape(dims), oraw.reshape(dims), ofn.reshape(dims), sp, eb,
                          axis_stencil=(mode == 2))
        got = post.cpu().numpy()
        mism = np.nonzero(bits(got) != bits(ref.reshape(-1)))[0]
        assert mism.size == 0, "post mode %d: %d mismatches, first %s" % (mode, mism.size, mism[:5])
        assert (tys.cpu().numpy() == ofn.astype(np.uint8)).all()
    ctx.close()


@pytest.mark.parametrize("case", [c for c in CASES_2D + CASES_3D if np.prod(c[0]) >= 27],
                         ids=lambda c: "x".join(map(str, c[0])))
def test_postprocess_entry_parity(T, ora, case):
    """szp_b200_topo_postprocess_dev on the reference decoder's outputs."""
    import torch
    dims, eb, B, kind, scale = case
    d = field(dims, kind, scale, seed=11)
    ocp = ora.sort_cp(ora.find_cp(d, eb), d)
    types = ora.mark_types(ocp, dims)
    raw, fn, _ = ora.decode_topo(ora.encode_topo(d, eb, B, types), d.size, eb, B)
    sp = ora.extract_sp(ocp)
    ctx = T.Context()
    for axis in ([False, True] if len(dims) == 3 else [False]):
        f = torch.from_numpy(raw.copy()).cuda()
        o = torch.from_numpy(raw.copy()).cuda()
        t = torch.from_numpy(fn.copy()).cuda()
        s = torch.from_numpy(sp.copy()).cuda() if len(sp) else None
        ctx.postprocess(f, o, t, s, dims, eb, axis_stencil=axis)
        ref, _ = ora.post(raw.reshape(dims), raw.reshape(dims), fn.reshape(dims), sp, eb,
                          axis_stencil=axis)
        assert (bits(f.cpu().numpy()) == bits(ref.reshape(-1))).all()
    ctx.close()


def test_bitcount_matches_host_log2f(T, ora):
    """The device bit count floor(log2f(m))+1 equals the host one for every
    magnitude of a full block sweep (both through the codec)."""
    # magnitudes around every power of two up to 2^31, packed as consecutive deltas
    mags = []
    for k in range(1, 32):
        for dm in (-3, -2, -1, 0, 1, 2):
            m = (1 << k) + dm
            if 0 < m < 2**31:
                mags.append(m)
    v = np.zeros(2 * len(mags), dtype=np.int64)
    v[1::2] = mags
    v = v.astype(np.int32)
    import oracle as O
    cp = np.zeros(len(v), dtype=O.CP2_DT)
    cp["type"] = 1
    cp["sort_position"] = v
    got = T.compress_sort_positions(cp, 2)
    assert got == O.encode_ints(v, 2)


def test_errors_do_not_exit(T):
    """Invalid arguments return NULL with a message instead of exiting."""
    d = np.zeros((8, 8), dtype=np.float32)
    with pytest.raises(T.ToposzpError):
        T.compress_topology(d, 1e-3, 300, np.zeros(0, dtype=T.CP2_DT))
    with pytest.raises(T.ToposzpError):
        T.compress_topology(d, -1.0, 64, np.zeros(0, dtype=T.CP2_DT))


def _oracle_round_trip(ora, d, dims, eb, B):
    ocp = ora.sort_cp(ora.find_cp(d, eb), d)
    s_ora = ora.encode_topo(d, eb, B, ora.mark_types(ocp, dims))
    sp = ora.extract_sp(ocp)
    s_sp = ora.encode_ints(sp, B) if len(sp) else b""
    oraw, ofn, _ = ora.decode_topo(s_ora, d.size, eb, B)
    ref, _ = ora.post(oraw.reshape(dims), oraw.reshape(dims), ofn.reshape(dims), sp, eb)
    return s_ora, s_sp, oraw, ref


def _dev_bytes(b):
    import torch
    return torch.from_numpy(np.frombuffer(b, dtype=np.uint8).copy()).cuda() if b else None


@pytest.mark.parametrize("case", CASES_2D + CASES_3D, ids=lambda c: "x".join(map(str, c[0])) + "_B%d" % c[2])
def test_device_parse_and_host_buffers(T, ora, case):
    """Streams without a block index (offsets parsed on the device) and the
    host-buffer entry points give the oracle's bytes and values."""
    dims, eb, B, kind, scale = case
    d = field(dims, kind, scale)
    s_ora, s_sp, oraw, ref = _oracle_round_trip(ora, d, dims, eb, B)
    ctx = T.Context()
    dt, ds = _dev_bytes(s_ora), _dev_bytes(s_sp)
    raw = ctx.decompress(dt, len(s_ora), ds, len(s_sp), None, dims, eb, B, postprocess=0)
    assert (bits(raw.cpu().numpy()) == bits(oraw)).all()
    post = ctx.decompress(dt, len(s_ora), ds, len(s_sp), None, dims, eb, B, postprocess=1)
    assert (bits(post.cpu().numpy()) == bits(ref.reshape(-1))).all()
    n = d.size
    L = T.lib()
    h_topo = np.zeros(L.szp_b200_topo_bound(n, B), dtype=np.uint8)
    h_sort = np.zeros(L.szp_b200_sort_bound(n, B), dtype=np.uint8)
    sz = ctx.compress_host(d, eb, B, h_topo, h_sort)
    assert h_topo[: sz.topo_bytes].tobytes() == s_ora
    assert h_sort[: sz.sort_bytes].tobytes() == s_sp
    out = np.full(dims, np.nan, dtype=np.float32)
    ctx.decompress_host(h_topo, sz.topo_bytes, h_sort, sz.sort_bytes, dims, eb, B, out, 1)
    assert (bits(out) == bits(ref)).all()
    ctx.close()


def test_device_parse_many_segments(T, ora):
    """A stream long enough for three composition levels of the parser."""
    import torch
    dims, eb, B = (96, 128, 160), 1e-4, 64
    d = synth.small_field(dims, seed=9, kind="band")
    ctx = T.Context()
    dd = torch.from_numpy(d.reshape(-1).copy()).cuda()
    topo, sort, idx, sizes = ctx.compress(dd, dims, eb, B)
    assert sizes.topo_bytes > 32 * 16384
    a = ctx.decompress(topo, sizes.topo_bytes, sort, sizes.sort_bytes, idx, dims, eb, B, postprocess=1)
    b = ctx.decompress(topo, sizes.topo_bytes, sort, sizes.sort_bytes, None, dims, eb, B, postprocess=1)
    assert torch.equal(a.view(torch.int32), b.view(torch.int32))
    ctx.close()


def test_truncated_stream_is_an_error(T, ora):
    dims, eb, B = (60, 90), 1e-2, 16
    d = field(dims, "bumps", 1.0)
    s_ora, s_sp, _, _ = _oracle_round_trip(ora, d, dims, eb, B)
    ctx = T.Context()
    cut = s_ora[: len(s_ora) - 5]
    with pytest.raises(T.ToposzpError):
        ctx.decompress(_dev_bytes(cut), len(cut), _dev_bytes(s_sp), len(s_sp), None, dims, eb, B,
                       postprocess=0)
    h = np.frombuffer(cut, dtype=np.uint8).copy()
    out = np.zeros(dims, dtype=np.float32)
    with pytest.raises(T.ToposzpError):
        ctx.decompress_host(h, len(cut), np.frombuffer(s_sp, np.uint8).copy(), len(s_sp), dims, eb, B,
                            out, 1)
    ctx.close()


def test_host_decompress_two_chunk_table(T, ora):
    """A stream with a two-entry offset table (the reference's OpenMP layout)
    is detected on the host, as the reference decoder does."""
    import torch
    dims, eb, B = (60, 90), 1e-2, 16
    d = field(dims, "bumps", 1.0)
    s_ora, s_sp, oraw, ref = _oracle_round_trip(ora, d, dims, eb, B)
    ctx = T.Context()
    dd = torch.from_numpy(d.reshape(-1).copy()).cuda()
    _, _, idx, _ = ctx.compress(dd, dims, eb, B)
    nb = (d.size + B - 1) // B
    bpt = (nb + 1) // 2
    off1 = int(idx[bpt].item())
    s2 = np.zeros(8, np.uint8).tobytes() + np.array([off1], dtype="<u8").tobytes() + s_ora[8:]
    oraw2, _, _ = ora.decode_topo(s2, d.size, eb, B)
    assert (bits(oraw2) == bits(oraw)).all()
    out = np.zeros(dims, dtype=np.float32)
    ctx.decompress_host(np.frombuffer(s2, np.uint8).copy(), len(s2), np.frombuffer(s_sp, np.uint8).copy(),
                        len(s_sp), dims, eb, B, out, 1)
    assert (bits(out) == bits(ref)).all()
    ctx.close()


def test_host_compress_in_parts_matches_device(T):
    """From 2^24 elements the host-buffer compressor copies the field in parts
    that overlap the encoder; its streams equal the device-resident call's."""
    import torch
    dims = (256, 256, 256)
    d = synth.small_field(dims, seed=12, kind="band")
    eb, B = 1e-4, 64
    ctx = T.Context()
    dd = torch.from_numpy(d.reshape(-1).copy()).cuda()
    topo, sort, _, sz = ctx.compress(dd, dims, eb, B, index=False)
    L = T.lib()
    n = d.size
    h_topo = torch.empty(L.szp_b200_topo_bound(n, B), dtype=torch.uint8).pin_memory().numpy()
    h_sort = torch.empty(L.szp_b200_sort_bound(n, B), dtype=torch.uint8).pin_memory().numpy()
    hf = torch.from_numpy(d).pin_memory().numpy()
    hz = ctx.compress_host(hf, eb, B, h_topo, h_sort)
    assert (hz.topo_bytes, hz.sort_bytes, hz.cp_count, hz.extrema_count) == \
        (sz.topo_bytes, sz.sort_bytes, sz.cp_count, sz.extrema_count)
    assert h_topo[: hz.topo_bytes].tobytes() == topo[: sz.topo_bytes].cpu().numpy().tobytes()
    assert h_sort[: hz.sort_bytes].tobytes() == sort[: sz.sort_bytes].cpu().numpy().tobytes()
    ctx.close()


@pytest.mark.parametrize("dims", [(128, 128, 128), (224, 224, 224)], ids=["sort_tier", "radix_tier"])
def test_rank_fallback_tiers(T, ora, dims):
    """Values up to 1e3 at eb 1e-6 give bins far wider than the shared bitmap
    of a bucket: at 128^3 every bucket (about 1.7 K points) is ranked by the
    in-CTA sort, at 224^3 (about 9 K points per bucket) most go to the
    device-wide radix fallback.  Sort positions must still be bit-exact."""
    import torch
    eb = 1e-6
    d = (synth.small_field(dims, seed=3, kind="noise") * np.float32(1e3)).astype(np.float32)
    ctx = T.Context()
    topo, sort, idx, sizes = ctx.compress(torch.from_numpy(d.reshape(-1).copy()).cuda(), dims, eb, 64)
    ocp = ora.sort_cp(ora.find_cp(d, eb), d)
    sp = ora.extract_sp(ocp)
    assert sizes.cp_count == len(ocp)
    assert sizes.extrema_count == len(sp)
    assert sort[: sizes.sort_bytes].cpu().numpy().tobytes() == ora.encode_ints(sp, 64)
    ctx.close()


def test_decompress_unaligned_streams(T):
    """Device streams may start at any byte for blockSize <= 256 (the decoder
    stages them through aligned vector loads); blockSize 257 needs 4-byte
    alignment and reports an error, not a fault, without it."""
    import torch
    dims, eb = (40, 50, 60), 1e-3
    d = torch.from_numpy(field(dims, "bumps", 1.0).reshape(-1).copy()).cuda()
    ctx = T.Context()
    topo, sort, idx, sz = ctx.compress(d, dims, eb, 64)
    ref = ctx.decompress(topo, sz.topo_bytes, sort, sz.sort_bytes, idx, dims, eb, 64).clone()
    for off in (1, 2, 3, 5, 13):
        tb = torch.zeros(sz.topo_bytes + 32, dtype=torch.uint8, device="cuda")
        sb = torch.zeros(sz.sort_bytes + 32, dtype=torch.uint8, device="cuda")
        tb[off:off + sz.topo_bytes] = topo[:sz.topo_bytes]
        sb[off:off + sz.sort_bytes] = sort[:sz.sort_bytes]
        for index in (idx, None):
            got = ctx.decompress(tb[off:], sz.topo_bytes, sb[off:], sz.sort_bytes, index, dims, eb, 64)
            assert torch.equal(got.view(torch.int32), ref.view(torch.int32)), (off, index is None)
    topo3, sort3, idx3, sz3 = ctx.compress(d, dims, eb, 257)
    tb = torch.zeros(sz3.topo_bytes + 32, dtype=torch.uint8, device="cuda")
    tb[1:1 + sz3.topo_bytes] = topo3[:sz3.topo_bytes]
    with pytest.raises(T.ToposzpError):
        ctx.decompress(tb[1:], sz3.topo_bytes, None, 0, idx3, dims, eb, 257, postprocess=0)
    ok = ctx.decompress(topo3, sz3.topo_bytes, sort3, sz3.sort_bytes, idx3, dims, eb, 257)
    assert torch.isfinite(ok).all()
    ctx.close()


def test_concurrent_contexts_on_host_threads(T):
    """Workspaces are independent: host threads that each drive their own
    context through the host-buffer calls, at the same time, get exactly the
    bytes and fields that one thread gets alone (the first call of a fresh
    device also uploads the post-processing weights from several threads)."""
    import threading
    jobs = [((40, 50, 60), "bumps", 1e-3), ((180, 360), "noise", 1e-3), ((20, 24, 28), "band", 1e-4),
            ((96, 64, 48), "bumps", 1e-2)]

    def run(job, ctx):
        dims, kind, eb = job
        d = field(dims, kind, 1.0, seed=11)
        n = d.size
        L = T.lib()
        ht = np.empty(L.szp_b200_topo_bound(n, 64), dtype=np.uint8)
        hs = np.empty(L.szp_b200_sort_bound(n, 64), dtype=np.uint8)
        sz = ctx.compress_host(d, eb, 64, ht, hs)
        out = np.empty(dims, dtype=np.float32)
        ctx.decompress_host(ht, sz.topo_bytes, hs, sz.sort_bytes, dims, eb, 64, out, 1)
        return ht[:sz.topo_bytes].tobytes(), hs[:sz.sort_bytes].tobytes(), out.view(np.int32).copy()

    ctxs = [T.Context() for _ in jobs]
    alone = [run(j, c) for j, c in zip(jobs, ctxs)]
    for _ in range(2):
        res = [None] * len(jobs)
        errs = []

        def work(i):
            try:
                res[i] = run(jobs[i], ctxs[i])
            except Exception as e:
                errs.append(e)
        th = [threading.Thread(target=work, args=(i,)) for i in range(len(jobs))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert not errs, errs
        for a, r in zip(alone, res):
            assert a[0] == r[0] and a[1] == r[1]
            assert np.array_equal(a[2], r[2])
    for c in ctxs:
        c.close()
