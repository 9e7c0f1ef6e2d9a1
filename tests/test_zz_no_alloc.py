"""szp_b200_topo_encode_noalloc (fixed device scratch, no allocation) against
the workspace encoder szp_b200_topo_compress_dev: identical topology streams,
call after call, so nothing left in the shared scratch leaks into the next
call.  Collected last so it also runs after every other GPU test."""
import ctypes as C

import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu

CASES = [
    # dims, eb, B, kind
    ((180, 360), 1e-3, 64, "bumps"),
    ((33, 31), 1e-3, 7, "noise"),
    ((41, 47), 1e-3, 257, "noise"),
    ((40, 50, 60), 1e-3, 64, "bumps"),
    ((5, 13), 1e-3, 64, "noise"),         # anchor-only tail block
    ((96, 128, 160), 1e-4, 64, "band"),   # 1.97 M elements, 961 tiles
]


@pytest.fixture(scope="module")
def T():
    import torch
    import toposzp_b200
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    toposzp_b200.lib()
    return toposzp_b200


def _workspace_stream(T, ctx, d, dims, eb, B):
    topo, _, _, sizes = ctx.compress(d, dims, eb, B, index=False)
    return topo[: sizes.topo_bytes].cpu().numpy().tobytes()


def _noalloc_stream(T, d, dims, eb, B):
    import torch
    n = int(np.prod(dims))
    cap = T.lib().szp_b200_topo_bound(n, B)
    out = torch.full((cap,), 0xAB, dtype=torch.uint8, device="cuda")
    nbytes = T.encode_noalloc(d, dims, eb, B, out)
    return out[:nbytes].cpu().numpy().tobytes()


@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[0])) + "_B%d" % c[2])
def test_noalloc_matches_workspace_encoder(T, case):
    import torch
    dims, eb, B, kind = case
    a = torch.from_numpy(synth.small_field(dims, seed=3, kind=kind).reshape(-1).copy()).cuda()
    b = torch.from_numpy(synth.small_field(dims, seed=4, kind=kind).reshape(-1).copy()).cuda()
    ctx = T.Context()
    ref_a = _workspace_stream(T, ctx, a, dims, eb, B)
    ref_b = _workspace_stream(T, ctx, b, dims, eb, B)
    ctx.close()
    # calls in a row on the shared scratch: a, b, a
    assert _noalloc_stream(T, a, dims, eb, B) == ref_a
    assert _noalloc_stream(T, b, dims, eb, B) == ref_b
    assert _noalloc_stream(T, a, dims, eb, B) == ref_a


def _raw_call(T, d, dims, eb, B, out, cap):
    n = C.c_size_t(0)
    rc = T.lib().szp_b200_topo_encode_noalloc(C.c_void_p(d.data_ptr()), T.geom_of(dims), eb, B,
                                              C.c_void_p(out.data_ptr()), cap, C.byref(n), None)
    return rc, n.value


def test_noalloc_rejects_fields_beyond_the_scratch(T):
    """A field needing more tile descriptors than the fixed scratch holds is
    rejected on the host before anything is launched or read (the C ABI is
    called directly with a small buffer: nothing may touch it)."""
    import torch
    tiny = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(64, dtype=torch.uint8, device="cuda")
    # 2^28 + 2048 elements: one tile of 2048 beyond the limit at blockSize 64
    rc, _ = _raw_call(T, tiny, (131073, 2048), 1e-3, 64, out, 64)
    assert rc == -1 and "fixed scratch" in T.last_error()
    rc, _ = _raw_call(T, tiny, (1024, 1024, 1024), 1e-3, 64, out, 64)
    assert rc == -1 and "fixed scratch" in T.last_error()
    rc, _ = _raw_call(T, tiny, (4, 4), 1e-3, 300, out, 64)
    assert rc == -1 and "blockSize" in T.last_error()
    # extents whose product overflows are invalid geometry, not a small field
    rc, _ = _raw_call(T, tiny, (2**31 - 1, 2**31 - 1, 2**31 - 1), 1e-3, 64, out, 64)
    assert rc == -1 and "geometry" in T.last_error()
    assert (out.cpu().numpy() == 0).all()


def test_noalloc_accepts_the_largest_field(T):
    """Exactly 2^28 elements at blockSize 64 fill the fixed scratch and are
    accepted (a constant field: no critical points, 21-byte blocks)."""
    import torch
    dims = (512, 512, 1024)
    d = torch.zeros(int(np.prod(dims)), dtype=torch.float32, device="cuda")
    nblk = d.numel() // 64
    cap = 8 + 21 * nblk + 64
    out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    nbytes = T.encode_noalloc(d, dims, 1e-3, 64, out)
    assert nbytes == 8 + 21 * nblk
    head = out[:8 + 21 * 2].cpu().numpy()
    assert (head[:8] == 0).all()
    # block: anchor 0, bit count 0, 16 tag bytes 0
    assert (head[8:] == 0).all()
    del d, out
    torch.cuda.empty_cache()


def test_noalloc_wrapper_checks_tensors(T):
    import torch
    d = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(4096, dtype=torch.uint8, device="cuda")
    with pytest.raises(T.ToposzpError, match="elements"):
        T.encode_noalloc(d, (1024, 1024, 512), 1e-3, 64, out)
    with pytest.raises(T.ToposzpError, match="float32"):
        T.encode_noalloc(d.double(), (4, 4), 1e-3, 64, out)
    with pytest.raises(T.ToposzpError, match="uint8"):
        T.encode_noalloc(d, (4, 4), 1e-3, 64, out.int())


def test_noalloc_output_too_small_is_an_error(T):
    """An undersized output buffer is reported by the encoder's own bounds
    check (no byte is written past topo_cap), and the next call still works."""
    import torch
    dims, eb, B = (64, 80), 1e-2, 64
    d = torch.from_numpy(synth.small_field(dims, seed=5, kind="noise").reshape(-1).copy()).cuda()
    guard = torch.full((4096,), 0x5A, dtype=torch.uint8, device="cuda")
    n = C.c_size_t(0)
    rc = T.lib().szp_b200_topo_encode_noalloc(
        C.c_void_p(d.data_ptr()), T.geom_of(dims), eb, B, C.c_void_p(guard.data_ptr()), 64,
        C.byref(n), None)
    assert rc == -1 and "too small" in T.last_error()
    assert (guard[64:].cpu().numpy() == 0x5A).all()
    ctx = T.Context()
    ref = _workspace_stream(T, ctx, d, dims, eb, B)
    ctx.close()
    assert _noalloc_stream(T, d, dims, eb, B) == ref
