"""The oracle's topology report (numpy) against a loop-by-loop restatement of
the reference drivers' verification steps on small fields
(example/test_cuda_topology.cu:540-602, 636-660, 800-868)."""
import numpy as np
import pytest

import synth


def _cls2(f, i, j):
    c, up, dn, lf, rt = f[i, j], f[i - 1, j], f[i + 1, j], f[i, j - 1], f[i, j + 1]
    if c > up and c > dn and c > lf and c > rt:
        return 1
    if c < up and c < dn and c < lf and c < rt:
        return 2
    if (c < up and c < dn and c > lf and c > rt) or (c > up and c > dn and c < lf and c < rt):
        return 3
    return 0


def _loops_2d(o, d, eb):
    rows, cols = o.shape
    to = np.zeros(o.shape, int)
    td = np.zeros(o.shape, int)
    for i in range(1, rows - 1):
        for j in range(1, cols - 1):
            to[i, j] = _cls2(o, i, j)
            td[i, j] = _cls2(d, i, j)
    preserved = lost = changed = new = 0
    for i in range(rows):
        for j in range(cols):
            if to[i, j]:
                if td[i, j] == to[i, j]:
                    preserved += 1
                elif td[i, j] == 0:
                    lost += 1
                else:
                    changed += 1
            if td[i, j] and not to[i, j]:
                new += 1
    max_err, e1, e2 = 0.0, 0, 0
    for v, w in zip(o.reshape(-1), d.reshape(-1)):
        e = abs(float(v) - float(w))
        max_err = max(max_err, e)
        e1 += e > eb * 1.01
        e2 += e > eb * 2.0
    pairs, viol = [0] * 4, [0] * 4
    for i in range(1, rows - 1):
        for j in range(1, cols - 1):
            for di, dj in ((0, 1), (1, 0)):
                ni, nj = i + di, j + dj
                if ni >= rows - 1 or nj >= cols - 1:
                    continue
                oa, ob, da, db = o[i, j], o[ni, nj], d[i, j], d[ni, nj]
                oo = -1 if oa < ob else (1 if oa > ob else 0)
                if oo == 0:
                    continue
                do = -1 if da < db else (1 if da > db else 0)
                v = oo != do
                ta, tb = to[i, j], to[ni, nj]
                for k, m in enumerate([True, bool(ta or tb), bool(ta and tb), ta in (1, 2) or tb in (1, 2)]):
                    if m:
                        pairs[k] += 1
                        viol[k] += v
    return dict(preserved=preserved, lost=lost, changed=changed, new_cps=new, max_err=max_err,
                over_1eb=e1, over_2eb=e2, pairs=pairs, violations=viol)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_topo_report_matches_reference_loops(ora, seed):
    o = synth.small_field((23, 29), seed=seed, kind="bumps")
    eb = 1e-3
    rng = np.random.default_rng(seed)
    d = (o + rng.uniform(-2.2 * eb, 2.2 * eb, size=o.shape)).astype(np.float32)
    d[3, 4] = o[3, 4]
    got = ora.topo_report(o, d, eb)
    ref = _loops_2d(o, d, np.float32(eb))
    for k, v in ref.items():
        assert got[k] == pytest.approx(v) if k == "max_err" else got[k] == v, k


def test_topo_report_identity_3d(ora):
    o = synth.small_field((9, 10, 11), seed=3, kind="noise")
    r = ora.topo_report(o, o, 1e-3)
    assert r["preserved"] == r["orig_cps"][0] and r["lost"] == r["changed"] == r["new_cps"] == 0
    assert r["violations"] == [0, 0, 0, 0] and r["max_err"] == 0.0
    assert r["pairs"][0] > 0
