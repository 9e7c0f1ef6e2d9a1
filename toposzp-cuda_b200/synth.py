"""Seeded synthetic scalar fields that stand in for the SDRBench / CESM inputs.

The reference publishes its timings on SDRBench fields that are not available
offline, so every workload here is generated from a seed.  Choices that the
workload descriptions leave open are fixed as follows:

* Gaussian-bump fields: bump centres are uniform over the grid, sigma is
  uniform in the stated range, amplitudes are N(0, 1).  Each bump is evaluated
  separably (a rank-1 tensor per bump), summed in float64, and the low-frequency
  term ``0.3*sin(2*pi*x/W)*cos(2*pi*y/H)`` (times ``cos(2*pi*z/D)`` in 3D) plus
  N(0, noise) white noise is added before the cast to float32.
* Band-limited field: white noise -> real FFT -> amplitude scaled by
  ``k**-1.5`` (power spectrum k^-3), DC set to 0 -> inverse FFT -> min-max
  normalised to [0, 1] -> float32.

Arrays are row-major (C order); axis 0 is the slowest.  Generated fields are
cached as raw ``.f32`` files under ``$TOPOSZP_CACHE`` (default
``/tmp/toposzp_fields``) so that repeated runs on one machine read identical
bytes.
"""

from __future__ import annotations

import hashlib
import math
import os
from dataclasses import dataclass, field

import numpy as np

CACHE_DIR = os.environ.get("TOPOSZP_CACHE", "/tmp/toposzp_fields")


def _cache_path(tag: str) -> str:
    return os.path.join(CACHE_DIR, tag + ".f32")


def _cached(tag: str, shape, make):
    path = _cache_path(tag)
    n = int(np.prod(shape))
    if os.path.exists(path) and os.path.getsize(path) == 4 * n:
        return np.fromfile(path, dtype=np.float32).reshape(shape)
    arr = np.ascontiguousarray(make(), dtype=np.float32).reshape(shape)
    try:
        os.makedirs(CACHE_DIR, exist_ok=True)
        tmp = path + ".%d.tmp" % os.getpid()
        arr.tofile(tmp)
        os.replace(tmp, path)
    except OSError:
        pass
    return arr


def gaussian_bumps(shape, n_bumps, sigma_lo, sigma_hi, noise, seed,
                   lowfreq=0.3) -> np.ndarray:
    """Sum of separable Gaussian bumps + low-frequency trig term + noise."""
    rng = np.random.default_rng(seed)
    shape = tuple(int(s) for s in shape)
    nd = len(shape)
    centers = np.stack([rng.uniform(0, s, size=n_bumps) for s in shape], 1)
    sigmas = rng.uniform(sigma_lo, sigma_hi, size=n_bumps)
    amps = rng.standard_normal(n_bumps)
    axes = [np.arange(s, dtype=np.float64) for s in shape]
    # per-axis factor matrices G[a] of shape (s_a, n_bumps)
    G = [np.exp(-((ax[:, None] - centers[None, :, a]) ** 2) /
                (2.0 * sigmas[None, :] ** 2)) for a, ax in enumerate(axes)]
    if nd == 2:
        out = (G[0] * amps[None, :]) @ G[1].T
    else:
        out = np.empty(shape, dtype=np.float64)
        A = G[0] * amps[None, :]
        for x in range(shape[0]):
            out[x] = (G[1] * A[x][None, :]) @ G[2].T
    # low-frequency term: 0.3 sin(2 pi x / W) cos(2 pi y / H) [cos(2 pi z / D)]
    trig = [np.sin(2 * np.pi * axes[-1] / shape[-1]),
            np.cos(2 * np.pi * axes[-2] / shape[-2])]
    if nd == 2:
        out += lowfreq * trig[1][:, None] * trig[0][None, :]
    else:
        cz = np.cos(2 * np.pi * axes[0] / shape[0])
        out += lowfreq * (cz[:, None, None] * trig[1][None, :, None] *
                          trig[0][None, None, :])
    if noise > 0:
        out += rng.normal(0.0, noise, size=shape)
    return out.astype(np.float32)


def band_limited(shape, seed, slope=-1.5) -> np.ndarray:
    """FFT-filtered white noise with power spectrum k^(2*slope), in [0, 1]."""
    import scipy.fft as sfft
    rng = np.random.default_rng(seed)
    shape = tuple(int(s) for s in shape)
    white = rng.standard_normal(shape)
    spec = sfft.rfftn(white, workers=-1)
    del white
    freqs = [np.fft.fftfreq(s) * s for s in shape[:-1]]
    freqs.append(np.fft.rfftfreq(shape[-1]) * shape[-1])
    k2 = np.zeros(spec.shape, dtype=np.float64)
    for a, f in enumerate(freqs):
        sl = [None] * len(shape)
        sl[a] = slice(None)
        k2 = k2 + (f[tuple(sl)] ** 2)
    k2.flat[0] = 1.0
    amp = k2 ** (slope / 2.0)
    amp.flat[0] = 0.0
    spec *= amp
    del k2, amp
    out = sfft.irfftn(spec, s=shape, workers=-1)
    del spec
    lo, hi = out.min(), out.max()
    out = (out - lo) / (hi - lo)
    return out.astype(np.float32)


@dataclass
class Field:
    name: str
    dims: tuple            # (rows, cols) or (d1, d2, d3)
    data: np.ndarray       # float32, C order, shape == dims
    eb_mode: str           # "abs" or "rel"
    eb_value: float        # as given (relative fraction for "rel")
    block_size: int = 64
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.data.size)

    def abs_eb(self) -> float:
        """Absolute error bound, computed like the reference's eb parser:
        relative bounds are ``rel * (max - min)`` in float32 arithmetic,
        with a zero range replaced by FLT_EPSILON."""
        if self.eb_mode == "abs":
            return float(np.float32(self.eb_value))
        mn = np.float32(self.data.min())
        mx = np.float32(self.data.max())
        rng_ = np.float32(mx - mn)
        if not rng_ > 0:
            rng_ = np.float32(np.finfo(np.float32).eps)
        return float(np.float32(np.float32(self.eb_value) * rng_))

    def digest(self) -> str:
        return hashlib.sha256(self.data.tobytes()).hexdigest()[:16]


def config1() -> Field:
    """2D 1800x3600, 40 bumps (sigma 20-200), +0.3 sin*cos, +N(0,1e-3), seed 0."""
    dims = (1800, 3600)
    data = _cached("c1_1800x3600_s0", dims,
                   lambda: gaussian_bumps(dims, 40, 20, 200, 1e-3, 0))
    return Field("c1_2d_1800x3600", dims, data, "abs", 1e-3)


def config2() -> Field:
    """3D 100x500x500, 200 bumps (sigma 5-60), +N(0,1e-4), seed 1, rel 1e-4."""
    dims = (100, 500, 500)
    data = _cached("c2_100x500x500_s1", dims,
                   lambda: gaussian_bumps(dims, 200, 5, 60, 1e-4, 1))
    return Field("c2_3d_100x500x500", dims, data, "rel", 1e-4)


def config3(side: int = 512) -> Field:
    """3D side^3 band-limited field (power k^-3) in [0,1], seed 2, abs 1e-4."""
    dims = (side, side, side)
    data = _cached("c3_%d_s2" % side, dims, lambda: band_limited(dims, 2))
    return Field("c3_3d_%d^3" % side, dims, data, "abs", 1e-4)


def batch_specs(count: int = 256, seed: int = 3):
    """Shapes and error bounds of the mixed-size batch (no data)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        if i < count // 2:
            dims = tuple(int(round(math.exp(rng.uniform(math.log(64), math.log(2048)))))
                         for _ in range(2))
        else:
            dims = tuple(int(round(math.exp(rng.uniform(math.log(32), math.log(256)))))
                         for _ in range(3))
        eb = float(math.exp(rng.uniform(math.log(1e-5), math.log(1e-2))))
        mode = "abs" if (i % 2 == 0) else "rel"
        specs.append((dims, mode, eb, int(rng.integers(0, 2**31 - 1))))
    return specs


def batch_field(spec, index: int) -> Field:
    dims, mode, eb, fseed = spec
    nd = len(dims)
    nb = 20 if nd == 2 else 40
    lo, hi = (0.02, 0.2) if nd == 2 else (0.05, 0.3)
    side = min(dims)
    data = gaussian_bumps(dims, nb, max(1.0, lo * side), max(2.0, hi * side),
                          1e-3, fseed)
    return Field("batch_%03d" % index, dims, data, mode, eb)


def small_field(dims, seed=0, kind="bumps", noise=1e-3) -> np.ndarray:
    """Small fields for parity tests (fast to generate)."""
    dims = tuple(int(d) for d in dims)
    if kind == "bumps":
        side = min(dims)
        return gaussian_bumps(dims, 6, max(1.0, 0.05 * side), max(2.0, 0.4 * side),
                              noise, seed)
    if kind == "noise":
        rng = np.random.default_rng(seed)
        return rng.standard_normal(dims).astype(np.float32)
    if kind == "band":
        return band_limited(dims, seed)
    raise ValueError(kind)


# ---------------------------------------------------------------------------
# float64 fields for the fp64 3D path
# ---------------------------------------------------------------------------

def f64_field(dims, seed=0, kind="smooth") -> np.ndarray:
    """Seeded float64 3D fields (computed in double, never cast to float32).

    smooth:  sum of 8 separable cosines (0.5..4 cycles per axis, random phase,
             amplitude N(0, 1)) plus N(0, 1e-4) noise
    noise:   N(0, 1) white noise (most interior points are critical and many
             saddles lose their shape under quantization)
    special: the smooth field with +-1e300, +-inf and NaN planted at seeded
             positions and a band of values just inside / outside the int32
             range of the quantizer (scaled by 1/eb = 1e3)
    """
    dims = tuple(int(d) for d in dims)
    rng = np.random.default_rng(seed)
    if kind == "noise":
        return rng.standard_normal(dims)
    out = np.zeros(dims, dtype=np.float64)
    axes = [np.arange(s, dtype=np.float64) / max(s, 1) for s in dims]
    for _ in range(8):
        term = rng.standard_normal()
        for a, ax in enumerate(axes):
            f = rng.uniform(0.5, 4.0)
            ph = rng.uniform(0.0, 2.0 * math.pi)
            shape = [1] * len(dims)
            shape[a] = dims[a]
            term = term * np.cos(2.0 * math.pi * f * ax + ph).reshape(shape)
        out += term
    out += rng.normal(0.0, 1e-4, size=dims)
    if kind == "special":
        flat = out.reshape(-1)
        pos = rng.choice(flat.size, size=min(flat.size, 64), replace=False)
        vals = [1e300, -1e300, np.inf, -np.inf, np.nan,
                2147483647.0 / 1e3, -2147483648.0 / 1e3, 2147483648.5 / 1e3, -2147483649.5 / 1e3]
        for k, p in enumerate(pos):
            flat[p] = vals[k % len(vals)]
    elif kind != "smooth":
        raise ValueError(kind)
    return out


def f64_critical_points(d: np.ndarray) -> np.ndarray:
    """CriticalPoint3D records (x, y, z, type, 0, 0) of the strict 6-neighbour
    classification of a float64 field, interior points only, raster order:
    1 maximum, 2 minimum, 3 saddle (higher than both neighbours along one axis
    and lower than both along another)."""
    c = d[1:-1, 1:-1, 1:-1]
    hi, lo = [], []
    for a in range(3):
        sl_m = [slice(1, -1)] * 3
        sl_p = [slice(1, -1)] * 3
        sl_m[a] = slice(0, -2)
        sl_p[a] = slice(2, None)
        m, p = d[tuple(sl_m)], d[tuple(sl_p)]
        hi.append((c > m) & (c > p))
        lo.append((c < m) & (c < p))
    mx = hi[0] & hi[1] & hi[2]
    mn = lo[0] & lo[1] & lo[2]
    anyh = hi[0] | hi[1] | hi[2]
    anyl = lo[0] | lo[1] | lo[2]
    sd = anyh & anyl
    t = np.zeros(c.shape, dtype=np.int32)
    t[sd] = 3
    t[mn] = 2
    t[mx] = 1
    x, y, z = np.nonzero(t)
    rec = np.zeros((x.size, 6), dtype=np.int32)
    rec[:, 0], rec[:, 1], rec[:, 2] = x + 1, y + 1, z + 1
    rec[:, 3] = t[x, y, z]
    return rec


def f64_cases():
    """The fp64 parity cases: name -> (dims, seed, kind, abs eb, blockSize,
    extra records).  Extra records (x, y, z, type) are appended to the
    classified list: points outside the grid, types outside 1..3 and saddles
    on the boundary (tagged, never repaired)."""
    edge = [(-1, 2, 2, 3), (2, 2, 99, 1), (0, 3, 3, 3), (3, 0, 4, 3), (4, 4, 0, 3), (5, 5, 5, 7), (6, 6, 6, 0)]
    return {
        "smooth_40x50x60": ((40, 50, 60), 11, "smooth", 1e-3, 64, []),
        "noise_32x33x35": ((32, 33, 35), 12, "noise", 5e-2, 64, []),
        "noise_tail_17x19x23_B7": ((17, 19, 23), 13, "noise", 2e-1, 7, edge),
        "smooth_B257_24x30x41": ((24, 30, 41), 14, "smooth", 1e-4, 257, edge),
        "special_20x21x22": ((20, 21, 22), 15, "special", 1e-3, 64, []),
        "noise_B1_9x10x11": ((9, 10, 11), 16, "noise", 1e-1, 1, []),
        "thin_3x40x50": ((3, 40, 50), 17, "noise", 1e-1, 32, []),
        "smooth_128x128x128": ((128, 128, 128), 18, "smooth", 1e-5, 64, []),
        "noise_96x96x96": ((96, 96, 96), 19, "noise", 5e-2, 64, []),
    }


def f64_case(name):
    """(field, CriticalPoint3D records as int32 rows of 6, abs eb, blockSize)."""
    dims, seed, kind, eb, B, extra = f64_cases()[name]
    d = f64_field(dims, seed, kind)
    cp = f64_critical_points(d)
    if extra:
        ex = np.zeros((len(extra), 6), dtype=np.int32)
        ex[:, :4] = np.array(extra, dtype=np.int32)
        # extra points replace none of the classified ones: skip duplicates
        have = {tuple(r[:3]) for r in cp}
        ex = np.array([r for r in ex if tuple(r[:3]) not in have], dtype=np.int32).reshape(-1, 6)
        cp = np.concatenate([cp, ex])
    return d, np.ascontiguousarray(cp, dtype=np.int32), eb, B


# ---------------------------------------------------------------------------
# 1-D inputs for the plain (non-topology) codec
# ---------------------------------------------------------------------------

def plain_field(n, seed=0, kind="wave", dtype=np.float32) -> np.ndarray:
    """Seeded 1-D inputs: wave (two sines of incommensurate periods, amplitude
    80), walk (a Gaussian random walk, step 0.3), uniform (U(-100, 100)),
    steps (constant runs of random length and level, then a ramp), special
    (the wave with +-inf, NaN, +-1e30 and values around the int32 range of
    the quantizer at 1/eb = 1e3 planted at seeded positions)."""
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.float64)
    if kind in ("wave", "special"):
        x = 80.0 * np.sin(i * 0.0123 + 0.4) + 20.0 * np.sin(i * 0.00071 + 1.3)
    elif kind == "walk":
        x = np.cumsum(rng.normal(0.0, 0.3, size=n))
    elif kind == "uniform":
        x = rng.uniform(-100.0, 100.0, size=n)
    elif kind == "steps":
        x = np.zeros(n)
        p = 0
        while p < n:
            r = int(rng.integers(1, 200))
            x[p:p + r] = rng.uniform(-50, 50)
            p += r
        x[n // 2:] += np.linspace(0.0, 10.0, n - n // 2)
    else:
        raise ValueError(kind)
    if kind == "special" and n > 16:
        pos = rng.choice(n, size=min(n, 32), replace=False)
        vals = [np.inf, -np.inf, np.nan, 1e30, -1e30, 2147483.0, -2147483.5, 2147484.0, -2147485.0]
        for k, p in enumerate(pos):
            x[p] = vals[k % len(vals)]
    return x.astype(dtype)


def plain_cases():
    """name -> (n, seed, kind, dtype, abs eb, blockSize, threadblock)."""
    cases = {}
    for dt in ("f32", "f64"):
        for tb in (0, 1):
            m = "tb" if tb else "ra"
            base = [
                ("wave_100k_B64", 100000, 21, "wave", 1e-3, 64),
                ("walk_65537_B64", 65537, 22, "walk", 1e-2, 64),
                ("uniform_3000_B7", 3000, 23, "uniform", 1e-4, 7),
                ("steps_20000_B1025", 20000, 24, "steps", 1e-3, 1025),
                ("special_5000_B64", 5000, 25, "special", 1e-3, 64),
                ("walk_2051_B1", 2051, 26, "walk", 1e-1, 1),
                ("wave_1_B64", 1, 27, "wave", 1e-3, 64),
                ("wave_2_B64", 2, 28, "wave", 1e-3, 64),
                ("walk_257_B256", 257, 29, "walk", 1e-3, 256),
            ]
            for name, n, seed, kind, eb, B in base:
                cases["%s_%s_%s" % (dt, m, name)] = (n, seed, kind, dt, eb, B, tb)
    return cases


def plain_case(name):
    """(field, abs eb, blockSize, threadblock)."""
    n, seed, kind, dt, eb, B, tb = plain_cases()[name]
    x = plain_field(n, seed, kind, np.float64 if dt == "f64" else np.float32)
    return x, eb, B, bool(tb)
