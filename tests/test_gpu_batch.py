"""Batched compression (one persistent launch per codec pass over many
fields) against the oracle, field by field: bit-exact streams and sizes,
relative bounds resolved on the device exactly as the reference does."""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu

FIELDS = [
    # dims, err, rel, kind
    ((180, 360), 1e-3, False, "bumps"),
    ((64, 80), 1e-2, True, "noise"),
    ((3, 3), 1e-3, False, "noise"),
    ((5, 13), 1e-3, True, "noise"),           # n % 64 == 1
    ((1, 200), 1e-3, False, "noise"),         # no interior: no critical points
    ((40, 50, 60), 1e-3, False, "bumps"),
    ((16, 18, 20), 0.02, True, "noise"),
    ((20, 24, 28), 1e-4, True, "band"),
    ((9, 9, 9), 1e-4, False, "bumps"),
    ((300, 257), 1e-5, True, "bumps"),
    ((7, 5, 13), 1e-2, False, "noise"),
    ((64, 64, 64), 1e-3, True, "band"),
]


@pytest.fixture(scope="module")
def T():
    import torch
    import toposzp_b200
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    toposzp_b200.lib()
    return toposzp_b200


def expected(ora, d, dims, err, rel, B=64):
    eb = np.float32(ora.rel_to_abs(d, np.float32(err))) if rel else np.float32(err)
    cp = ora.sort_cp(ora.find_cp(d, float(eb)), d)
    topo = ora.encode_topo(d, float(eb), B, ora.mark_types(cp, dims))
    sp = ora.extract_sp(cp)
    sort = ora.encode_ints(sp, B) if len(sp) else b""
    return float(eb), topo, sort, len(cp), len(sp)


def make_items(specs, seed0=21):
    import torch
    items, host = [], []
    for k, (dims, err, rel, kind) in enumerate(specs):
        d = synth.small_field(dims, seed=seed0 + k, kind=kind)
        host.append(d)
        items.append((torch.from_numpy(d.reshape(-1).copy()).cuda(), dims, err, rel))
    return items, host


def check(ora, specs, host, res):
    for (dims, err, rel, _), d, (tb, sb, sz, abs_eb) in zip(specs, host, res):
        eb, topo, sort, K, E = expected(ora, d, dims, err, rel)
        assert np.float32(abs_eb) == np.float32(eb), (dims, abs_eb, eb)
        assert sz.cp_count == K and sz.extrema_count == E, dims
        assert sz.topo_bytes == len(topo) and tb[: sz.topo_bytes].cpu().numpy().tobytes() == topo, dims
        assert sz.sort_bytes == len(sort), dims
        if len(sort):
            assert sb[: sz.sort_bytes].cpu().numpy().tobytes() == sort, dims


@pytest.mark.parametrize("graphs", [True, False])
def test_batch_matches_oracle(T, ora, graphs):
    b = T.Batch(64)
    b.configure(use_graphs=graphs, autotune=1)
    items, host = make_items(FIELDS)
    check(ora, FIELDS, host, b.compress(items))
    # a second batch of other fields and order replays the same graphs
    specs2 = FIELDS[::-1][:7]
    items2, host2 = make_items(specs2, seed0=40)
    check(ora, specs2, host2, b.compress(items2))
    tun = b.tuning()
    assert tun["tuned"] and tun["topo_threads"] in (128, 256)
    b.close()


def test_batch_grows_and_matches_plain_calls(T, ora):
    """A batch larger than the previous capacity regrows its buffers; every
    field equals the per-field fused call with the batch's absolute bound."""
    b = T.Batch(64)
    items, host = make_items(FIELDS[:3])
    check(ora, FIELDS[:3], host, b.compress(items))
    specs = FIELDS * 3
    items, host = make_items(specs, seed0=60)
    res = b.compress(items)
    ctx = T.Context()
    for (t, dims, err, rel), (tb, sb, sz, abs_eb) in zip(items, res):
        topo, sort, _, psz = ctx.compress(t, dims, abs_eb, 64, index=False)
        assert psz.topo_bytes == sz.topo_bytes and psz.sort_bytes == sz.sort_bytes
        assert torch_equal(topo[: sz.topo_bytes], tb[: sz.topo_bytes])
        if sz.sort_bytes:
            assert torch_equal(sort[: sz.sort_bytes], sb[: sz.sort_bytes])
    ctx.close()
    b.close()


def torch_equal(a, b):
    import torch
    return bool(torch.equal(a, b))


def test_batch_reports_small_buffers(T):
    import torch
    b = T.Batch(64)
    items, _ = make_items(FIELDS[:2])
    bufs = b.buffers(items)
    bufs[1] = (bufs[1][0][:16], bufs[1][1])
    with pytest.raises(T.ToposzpError, match="too small"):
        b.compress(items, bufs)
    # the batch object stays usable
    items, host = make_items(FIELDS[:2])
    res = b.compress(items)
    assert res[0][2].topo_bytes > 8
    b.close()
