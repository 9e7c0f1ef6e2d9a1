"""Request server: every result is the same served alone and in a mix of
overlapping requests (bit-exact), compressions are merged into batched
launches, requests overlap on the device, and the HBM budget is honoured."""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu

SHAPES = [((180, 360), "bumps"), ((40, 50, 60), "bumps"), ((64, 80), "noise"), ((20, 24, 28), "band"),
          ((300, 257), "bumps"), ((9, 9, 9), "noise"), ((5, 13), "noise"), ((96, 64, 48), "band")]


@pytest.fixture(scope="module")
def T():
    import torch
    import toposzp_b200
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    toposzp_b200.lib()
    return toposzp_b200


def build_mix(T, seed=5):
    """Two compress requests for every decompress request over SHAPES, each
    with fresh output buffers; the decompress inputs are compressed first."""
    import torch
    L = T.lib()
    ctx = T.Context()
    rng = np.random.default_rng(seed)
    spec, keep = [], []
    for k, (dims, kind) in enumerate(SHAPES * 2):
        d = torch.from_numpy(synth.small_field(dims, seed=100 + k, kind=kind).reshape(-1).copy()).cuda()
        n = d.numel()
        err = float(10 ** rng.uniform(-4, -2))
        if k % 3 != 2:
            tb = torch.empty(L.szp_b200_topo_bound(n, 64), dtype=torch.uint8, device="cuda")
            sb = torch.empty(L.szp_b200_sort_bound(n, 64), dtype=torch.uint8, device="cuda")
            spec.append(("c", dims, d, err, bool(k % 2), tb, sb))
        else:
            topo, sort, _, sz = ctx.compress(d, dims, err, 64, index=False)
            out = torch.empty(n, dtype=torch.float32, device="cuda")
            spec.append(("d", dims, topo, sz.topo_bytes, sort, sz.sort_bytes, err, out))
        keep.append(d)
    ctx.close()
    return spec, keep


def to_requests(T, srv, spec):
    arr = (T.Request * len(spec))()
    for i, s in enumerate(spec):
        if s[0] == "c":
            _, dims, d, err, rel, tb, sb = s
            arr[i] = srv.compress_request(d, dims, err, rel, tb, sb)
        else:
            _, dims, topo, tbytes, sort, sbytes, abs_eb, out = s
            arr[i] = srv.decompress_request(topo, tbytes, sort if sbytes else None, sbytes, dims, abs_eb, out, 1)
    return arr


def results(spec, arr):
    res = []
    for s, r in zip(spec, arr):
        if s[0] == "c":
            res.append((s[5][: r.sizes.topo_bytes].clone(), s[6][: r.sizes.sort_bytes].clone(), r.abs_eb))
        else:
            res.append((s[7].clone(),))
    return res


def same(x, y):
    import torch
    if isinstance(x, float):
        return np.float32(x) == np.float32(y)
    if x.dtype != torch.uint8:
        x, y = x.view(torch.uint8), y.view(torch.uint8)
    return bool(torch.equal(x, y))


def test_same_alone_and_in_mix(T):
    srv = T.Server(slots=4, max_batch=16)
    spec, keep = build_mix(T)
    # alone: one request at a time
    alone = []
    for s in spec:
        arr = to_requests(T, srv, [s])
        srv.run_trace(arr)
        alone.append(results([s], arr)[0])
    st0 = srv.stats()
    # in the mix: all at once, so requests overlap and compressions merge
    for s in spec:
        if s[0] == "c":
            s[5].zero_()
            s[6].zero_()
        else:
            s[7].zero_()
    arr = to_requests(T, srv, spec)
    srv.run_trace(arr)
    mixed = results(spec, arr)
    st = srv.stats()
    for a, m in zip(alone, mixed):
        for x, y in zip(a, m):
            assert same(x, y)
    ncomp = sum(1 for s in spec if s[0] == "c")
    assert st["completed"] - st0["completed"] == len(spec)
    assert st["batches"] - st0["batches"] < ncomp            # compressions were merged
    assert st["max_concurrent"] > 1                          # requests overlapped
    for r in arr:
        assert r.t_arrival <= r.t_start <= r.t_done
    srv.close()


def test_served_compressions_match_oracle(T, ora):
    srv = T.Server(slots=2, max_batch=8)
    spec, keep = build_mix(T, seed=6)
    spec = [s for s in spec if s[0] == "c"][:6]
    arr = to_requests(T, srv, spec)
    srv.run_trace(arr)
    for s, r in zip(spec, arr):
        _, dims, d, err, rel, tb, sb = s
        host = d.cpu().numpy().reshape(dims)
        eb = np.float32(ora.rel_to_abs(host, np.float32(err))) if rel else np.float32(err)
        assert np.float32(r.abs_eb) == eb
        cp = ora.sort_cp(ora.find_cp(host, float(eb)), host)
        topo = ora.encode_topo(host, float(eb), 64, ora.mark_types(cp, dims))
        assert tb[: r.sizes.topo_bytes].cpu().numpy().tobytes() == topo
    srv.close()


def test_hbm_budget_limits_admission(T):
    """With a budget that holds about one request at a time, the admitted
    working set never exceeds it unless a single request is larger."""
    budget = 64 << 20
    srv = T.Server(slots=4, max_batch=16, hbm_budget=budget)
    spec, keep = build_mix(T, seed=7)
    arr = to_requests(T, srv, spec)
    srv.run_trace(arr)
    st = srv.stats()
    costs = [(40 if s[0] == "c" else 32) * int(np.prod(s[1])) + (1 << 20) for s in spec]
    assert st["max_inflight_bytes"] <= max(budget, max(costs))
    srv.close()


def test_poisson_trace(T):
    srv = T.Server(slots=3, max_batch=8)
    spec, keep = build_mix(T, seed=8)
    rng = np.random.default_rng(4)
    arrivals = np.cumsum(rng.exponential(1.0 / 2000.0, size=len(spec)))
    arr = to_requests(T, srv, spec)
    srv.run_trace(arr, arrivals.tolist())
    lat = np.array([r.t_done - r.t_arrival for r in arr])
    assert (lat > 0).all() and np.isfinite(lat).all()
    srv.close()


def test_large_compressions_run_alone_and_match(T):
    """Compressions of at least 2^21 elements take the fused single-field path
    inside the server (not the batched one); their streams equal the plain
    call's, alone and beside small merged requests, after a workspace
    reserve."""
    import torch
    L = T.lib()
    big = (160, 128, 128)
    d = torch.from_numpy(synth.small_field(big, seed=42, kind="band").reshape(-1).copy()).cuda()
    ctx = T.Context()
    ref_t, ref_s, _, ref_sz = ctx.compress(d, big, 1e-4, 64, index=False)
    ref = (ref_t[:ref_sz.topo_bytes].cpu().numpy().tobytes(), ref_s[:ref_sz.sort_bytes].cpu().numpy().tobytes())
    ctx.close()
    srv = T.Server(slots=3, max_batch=8, block_size=64)
    srv.reserve(d.numel())
    spec = []
    n = d.numel()
    for k in range(2):
        tb = torch.empty(L.szp_b200_topo_bound(n, 64), dtype=torch.uint8, device="cuda")
        sb = torch.empty(L.szp_b200_sort_bound(n, 64), dtype=torch.uint8, device="cuda")
        spec.append(("c", big, d, 1e-4, False, tb, sb))
    small, keep = build_mix(T, seed=9)
    arr = to_requests(T, srv, spec + small)
    srv.run_trace(arr)
    for k in range(2):
        r = arr[k]
        assert r.status == 0, r.message
        got = (spec[k][5][:r.sizes.topo_bytes].cpu().numpy().tobytes(),
               spec[k][6][:r.sizes.sort_bytes].cpu().numpy().tobytes())
        assert got == ref
    assert all(arr[i].status == 0 for i in range(len(arr)))
    srv.close()


def test_served_decompressions_match_single_workspace(T):
    """Server workers run the post-processing rounds as ordinary launches in
    bursts (their streams share the GPU, so no cooperative launch); the
    decompressed fields equal those of a single workspace, whose round tails
    run in one cooperative launch."""
    import torch
    spec, keep = build_mix(T, seed=7)
    spec = [s for s in spec if s[0] == "d"]
    assert len(spec) >= 4
    srv = T.Server(slots=3, max_batch=8)
    arr = to_requests(T, srv, spec)
    srv.run_trace(arr)
    ctx = T.Context()
    for s, r in zip(spec, arr):
        assert r.status == 0
        _, dims, topo, tbytes, sort, sbytes, abs_eb, out = s
        ref = ctx.decompress(topo, tbytes, sort if sbytes else None, sbytes, None, dims, abs_eb, 64, postprocess=1)
        assert torch.equal(out.view(torch.int32), ref.view(torch.int32))
    ctx.close()
    srv.close()
