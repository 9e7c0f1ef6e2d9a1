"""Every device wait of the library is bounded: a wait that can never be
satisfied gives up after its poll limit, records its error status and lets
the kernel finish, so the GPU and the context stay usable.  Both probes run a
wait with a short limit through the C ABI and check the status and that the
call returned within milliseconds."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu

LOOKBACK_TIMEOUT = 1
WAIT_TIMEOUT = 5


@pytest.fixture(scope="module")
def T():
    import torch
    import toposzp_b200
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    toposzp_b200.lib()
    return toposzp_b200


def _probe(T, which, limit):
    st, ms = C.c_int(-1), C.c_float(-1.0)
    rc = T.lib().szp_b200_selftest_bounded_wait(which, limit, C.byref(st), C.byref(ms))
    assert rc == 0, T.last_error()
    return st.value, ms.value


@pytest.mark.parametrize("limit", [64, 4096])
def test_lookback_gives_up(T, limit):
    st, ms = _probe(T, 0, limit)
    assert st == LOOKBACK_TIMEOUT
    assert 0.0 <= ms < 1000.0


@pytest.mark.parametrize("limit", [64, 4096])
def test_grid_barrier_gives_up(T, limit):
    st, ms = _probe(T, 1, limit)
    assert st == WAIT_TIMEOUT
    assert 0.0 <= ms < 1000.0


def test_context_usable_after_timeouts(T):
    """A normal call right after the probes works (nothing left hanging)."""
    import numpy as np
    import torch
    import synth
    _probe(T, 0, 32)
    _probe(T, 1, 32)
    d = synth.small_field((40, 50), seed=1, kind="bumps")
    ctx = T.Context()
    topo, sort, idx, sizes = ctx.compress(torch.from_numpy(d.reshape(-1).copy()).cuda(), d.shape, 1e-3, 64)
    out = ctx.decompress(topo, sizes.topo_bytes, sort, sizes.sort_bytes, idx, d.shape, 1e-3, 64, postprocess=0)
    assert np.abs(out.cpu().numpy() - d.reshape(-1)).max() <= 1.01e-3
    ctx.close()


def test_probe_arguments_checked(T):
    st, ms = C.c_int(0), C.c_float(0)
    assert T.lib().szp_b200_selftest_bounded_wait(2, 64, C.byref(st), C.byref(ms)) == -1
    assert T.lib().szp_b200_selftest_bounded_wait(0, 0, C.byref(st), C.byref(ms)) == -1
