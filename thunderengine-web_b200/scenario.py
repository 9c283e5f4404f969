"""Synthetic CM1 scenarios for the large-step dynamics path.

Host-side restatement of the reference's scenario builders, restricted to what the
dynamics step needs.  All values are binary32, computed with numpy float32.  The
reference computes some base-state values with its own copies of the upstream libm
(web/core/libm.js); bit-identical initial states are not needed here because parity
is judged step by step on identical inputs, so numpy's float32 transcendental
functions are used.

* Grid layout: halo 3, ``strideJ = nx + 7`` (or, with ``align_rows``, rounded up to a
  multiple of 32 so that every row starts on a 128-byte boundary), ``strideK = ny + 7``,
  ``count = strideJ * strideK * (nz + 1)`` (web/core/grid.js:181-199); arena fields at
  ``n * fieldStride`` with fieldStride = count * 4 rounded up to 256 B
  (grid.js:322-331); ``hmetric`` = 9 strideJ + 3 strideK floats (grid.js:200-214).
* Vertical grid: uniform faces; mh, mf, c1, c2 and the surface/top extrapolation
  weights as ``VerticalGrid`` (grid.js:249-300).
* Base state: Weisman-Klemp thermodynamic sounding (base.js:181-216, 20 hydrostatic
  iterations, qv capped at 0.014), ``BaseState.tail`` (base.js:147-171), wind
  ``u = Us * tanh(z / 3 km)``, v = 0 (the base.js:383-385 form with 35 -> Us).
* Perturbation: cosine-squared warm bubble (``WarmBubble``, base.js:475-490) plus
  seeded +-0.1 K noise from ``HashRand`` (base.js:458-472) on interior points.
* Arena fill: scenario.js:234-296; step profiles rho0/rr0/rf0/th0/pi0/qv0
  (scenario.js:122-136).
"""
import functools
import math

import numpy as np

F = np.float32
HALO = 3

# CM1 constants (web/core/grid.js:13-40)
G, RD, CP, RV, P00 = 9.81, 287.04, 1005.7, 461.5, 1.0e5
EPS = RD / RV
REPS = RV / RD


def f(x):
    return F(x)


class Grid:
    """Uniform horizontal grid in the reference's arena layout (grid.js:181-199).
    ``align_rows``: the row pitch rounded up to 32 floats (the reference's ``alignRows``
    option, grid.js:184-191); the padding columns past i = nx + 3 belong to no point."""

    def __init__(self, nx, ny, nz, dx, dy, dz, align_rows=False):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)
        self.align_rows = bool(align_rows)
        raw = self.nx + 1 + 2 * HALO
        self.strideJ = (raw + 31) // 32 * 32 if self.align_rows else raw
        self.strideK = self.ny + 1 + 2 * HALO
        self.count = self.strideJ * self.strideK * (self.nz + 1)
        self.field_stride = int(math.ceil(self.count * 4 / 256) * 256)

    def index(self, i, j, k):
        return (i + HALO) + self.strideJ * ((j + HALO) + self.strideK * k)

    def axis(self, n, d):
        """Face and centre coordinates of a centred uniform axis (grid.js:75-83)."""
        idx = np.arange(-HALO, n + HALO + 1, dtype=np.float64)
        total = n * d
        xf = idx * d - 0.5 * total
        xh = (idx + 0.5) * d - 0.5 * total
        return xf, xh

    def metric_values(self):
        """``hmetric`` buffer (grid.js:200-214) for a uniform, non-axisymmetric grid."""
        sJ, sK = self.strideJ, self.strideK
        v = np.ones(9 * sJ + 3 * sK, dtype=F)
        xf, xh = self.axis(self.nx, self.dx)
        yf, _ = self.axis(self.ny, self.dy)
        # each plane takes its axis' values where it has them and keeps 1 beyond
        # (grid.js:200-214), which matters with aligned rows only
        x, y, h = xf[:sJ].astype(F), yf[:sK].astype(F), xh[:sJ].astype(F)
        v[2 * sJ + 2 * sK:2 * sJ + 2 * sK + len(x)] = x
        v[3 * sJ + 2 * sK:3 * sJ + 2 * sK + len(y)] = y
        base = 3 * sJ + 3 * sK
        v[base + 4 * sJ:base + 4 * sJ + len(x)] = 0.0          # rxh: 0 when not axisymmetric
        v[base + 5 * sJ:base + 5 * sJ + len(h)] = h
        return v


class VerticalGrid:
    """Uniform vertical grid (grid.js:249-300)."""

    def __init__(self, nz, dz):
        self.nz = nz
        zf = np.array([k * dz for k in range(nz + 1)], dtype=np.float64)
        self.zf = zf
        zh = np.array([f(0.5 * (zf[k] + zf[k + 1])) for k in range(nz)], dtype=F)
        self.zh = zh
        dz32 = f(dz)
        lo = -zh[0]
        hi = f(zh[nz - 1] + f(2.0 * f(f(zf[nz]) - zh[nz - 1])))
        mf = np.zeros(nz + 1, dtype=F)
        mf[0] = f(dz32 / f(zh[0] - lo))
        for k in range(1, nz):
            mf[k] = f(dz32 / f(zh[k] - zh[k - 1]))
        mf[nz] = f(dz32 / f(hi - zh[nz - 1]))
        w2 = np.zeros(nz + 1, dtype=F)
        w2[0] = f(f(f(zf[0]) - lo) / f(zh[0] - lo))
        for k in range(1, nz):
            w2[k] = f(f(f(zf[k]) - zh[k - 1]) / f(zh[k] - zh[k - 1]))
        w2[nz] = f(f(f(zf[nz]) - zh[nz - 1]) / f(hi - zh[nz - 1]))
        self.mh = np.array([f(dz32 / f(f(zf[k + 1]) - f(zf[k]))) for k in range(nz)], dtype=F)
        self.mf = mf
        self.c2 = w2
        self.c1 = (F(1.0) - w2).astype(F)
        d_bot = f(f(zf[1]) - f(zf[0]))
        d_top = f(f(zf[nz]) - f(zf[nz - 1]))
        self.surface = self._fornberg(f(f(zf[0]) / d_bot), [f(zh[0] / d_bot), f(zh[1] / d_bot), f(zh[2] / d_bot)])
        self.top = self._fornberg(f(f(zf[nz]) / d_top),
                                  [f(zh[nz - 1] / d_top), f(zh[nz - 2] / d_top), f(zh[nz - 3] / d_top)])

    @staticmethod
    def _fornberg(x0, alpha):
        """Three-point extrapolation weights (VerticalGrid.fornbergCM1, grid.js:220-234)."""
        x0 = float(x0)
        alpha = [float(a) for a in alpha]
        d = [[0.0] * 3 for _ in range(3)]
        d[0][0] = 1.0
        b1 = 1.0
        for n in range(1, 3):
            b2 = 1.0
            for nu in range(n):
                b3 = alpha[n] - alpha[nu]
                b2 = b2 * b3
                d[n][nu] = ((alpha[n] - x0) * d[n - 1][nu]) / b3
            d[n][n] = (b1 / b2) * (-((alpha[n - 1] - x0) * d[n - 1][n - 1]))
            b1 = b2
        return [f(d[2][0]), f(d[2][1]), f(d[2][2])]


def rslf32(p, t):
    esl = f(f(611.2) * np.exp(f(f(f(17.67) * f(t - f(273.15))) / f(t - f(29.65)))))
    esl = min(esl, f(p * F(0.5)))
    return f(f(F(EPS) * esl) / f(p - esl))


def fmaf(a, b, c):
    return f(float(a) * float(b) + float(c))   # product exact in double; one rounding suffices here


def weisman_klemp(zh, qv_pbl=0.014, iterations=20):
    """Weisman-Klemp thermodynamic profiles (base.js:181-216) + tail (base.js:147-171)."""
    nk = len(zh)
    z_trop, th_trop, t_trop = f(12000.0), f(343.0), f(213.0)
    th_sfc, prs_sfc = f(300.0), f(100000.0)
    cp, rd, g = f(CP), f(RD), f(G)
    reps = f(REPS)
    pi_sfc = f(np.power(f(prs_sfc / f(P00)), f(rd / cp)))
    qv_sfc = rslf32(prs_sfc, f(th_sfc * pi_sfc))
    thv_sfc = f(f(th_sfc * fmaf(qv_sfc, reps, 1.0)) / f(F(1.0) + qv_sfc))
    th = np.zeros(nk, F)
    rh = np.zeros(nk, F)
    for k in range(nk):
        z = zh[k]
        if z < z_trop:
            fr = f(np.power(f(z / z_trop), f(1.25)))
            th[k] = fmaf(f(th_trop - th_sfc), fr, th_sfc)
            rh[k] = fmaf(f(-0.75), fr, 1.0)
        else:
            th[k] = f(th_trop * np.exp(f(f(g / f(t_trop * cp)) * f(z - z_trop))))
            rh[k] = f(0.25)
    qv = np.zeros(nk, F)
    thv = np.zeros(nk, F)
    pi = np.zeros(nk, F)
    prs = np.zeros(nk, F)
    cp_over_rd = f(cp / rd)
    qv_pbl = f(qv_pbl)
    for _ in range(iterations):
        for k in range(nk):
            thv[k] = f(f(th[k] * fmaf(reps, qv[k], 1.0)) / f(F(1.0) + qv[k]))
        pi[0] = f(pi_sfc - f(f(g * zh[0]) / f(f(cp * F(0.5)) * f(thv_sfc + thv[0]))))
        for k in range(1, nk):
            pi[k] = f(pi[k - 1] - f(f(g * f(zh[k] - zh[k - 1])) / f(f(cp * F(0.5)) * f(thv[k] + thv[k - 1]))))
        for k in range(nk):
            prs[k] = f(F(P00) * np.power(pi[k], cp_over_rd))
        for k in range(nk):
            qv[k] = f(rh[k] * rslf32(prs[k], f(th[k] * pi[k])))
            if qv[k] > qv_pbl:
                qv[k] = qv_pbl
    cpdrd = f(cp / rd)
    prs = np.array([f(F(P00) * np.power(x, cpdrd)) for x in pi], F)
    rho = np.array([f(prs[k] / f(f(f(rd * th[k]) * pi[k]) * fmaf(qv[k], reps, 1.0))) for k in range(nk)], F)
    return {'th0': th, 'qv0': qv, 'pi0': pi, 'prs0': prs, 'rho0': rho}


def hash_rand(seed, i, j, k):
    """Deterministic hash RNG (HashRand.value, base.js:458-472)."""
    m = 0xFFFFFFFF
    x = (seed * 2654435761) & m
    x = (x + (i * 40503) & m) & m
    x = (x + (j * 1073741827) & m) & m
    x = (x + (k * 3145739) & m) & m
    x ^= x >> 16
    x = (x * 2246822519) & m
    x ^= x >> 13
    x = (x * 3266489917) & m
    x ^= x >> 16
    return f(f(x) / f(4294967296.0))


def hash_rand_grid(seed, ii, jj, kk):
    """Vectorised ``hash_rand`` over integer arrays."""
    m = np.uint64(0xFFFFFFFF)
    x = np.uint64((seed * 2654435761) & 0xFFFFFFFF)
    x = (x + ((ii.astype(np.uint64) * np.uint64(40503)) & m)) & m
    x = (x + ((jj.astype(np.uint64) * np.uint64(1073741827)) & m)) & m
    x = (x + ((kk.astype(np.uint64) * np.uint64(3145739)) & m)) & m
    x ^= x >> np.uint64(16)
    x = (x * np.uint64(2246822519)) & m
    x ^= x >> np.uint64(13)
    x = (x * np.uint64(3266489917)) & m
    x ^= x >> np.uint64(16)
    return (x.astype(np.float32) / F(4294967296.0)).astype(F)


class Config:
    """One synthetic run: grid, time step, acoustic substeps and perturbation."""

    def __init__(self, name, nx, ny, nz, dx, dz, dt, nsound, us, steps, amplitude=2.0, noise=0.1, seed=1,
                 bubbles=None, qv_pbl=0.014, align_rows=False):
        self.name = name
        self.align_rows = bool(align_rows)
        self.qv_pbl = float(qv_pbl)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dx = self.dy = float(dx)
        self.dz = float(dz)
        self.dt = float(dt)
        self.nsound = int(nsound)
        self.us = float(us)
        self.steps = int(steps)
        self.amplitude = amplitude
        self.noise = noise
        self.seed = seed
        self.bubbles = bubbles or [(0.0, 0.0)]

    def as_dict(self):
        return {'workload': self.name, 'nx': self.nx, 'ny': self.ny, 'nz': self.nz, 'dx': self.dx,
                'dz': self.dz, 'dt': self.dt, 'nsound': self.nsound}


# The synthetic workloads: small CPU-runnable case and the at-scale case.
SMALL = Config('cm1-dyn-64x64x40', 64, 64, 40, 1000.0, 500.0, 6.0, 6, 20.0, 50)
AT_SCALE = Config('cm1-dyn-256x256x80', 256, 256, 80, 500.0, 250.0, 3.0, 8, 25.0, 100)
# the large domain: 1024 x 1024 x 100 at dx = 250 m (dz = 200 m), dt = 1.5 s, nsound 8,
# a line of three bubbles 30 km apart in y (the BubbleLine spacing, base.js:522-539),
# domain-centred; ~21 GB of arena, memory offsets past 2^32 words
LARGE = Config('cm1-dyn-1024x1024x100', 1024, 1024, 100, 250.0, 200.0, 1.5, 8, 25.0, 20,
               bubbles=[(0.0, -30000.0), (0.0, 0.0), (0.0, 30000.0)])


def tiny(nx=12, ny=10, nz=8, dx=1000.0, dz=500.0, dt=6.0, nsound=6, us=20.0, align_rows=False):
    """A few-thousand-point case for fast oracle comparisons."""
    return Config('cm1-dyn-%dx%dx%d' % (nx, ny, nz), nx, ny, nz, dx, dz, dt, nsound, us, 1, align_rows=align_rows)


def profiles(cfg, dry=False):
    """Vertical profiles handed to the step (scenario.js:122-136); ``dry``: no water vapour
    (the sounding's moisture cap set to 0)."""
    vg = VerticalGrid(cfg.nz, cfg.dz)
    base = weisman_klemp(vg.zh, qv_pbl=0.0 if dry else getattr(cfg, 'qv_pbl', 0.014))
    nz = cfg.nz
    rho0 = base['rho0']
    cgs, cgt = vg.surface, vg.top
    rf0 = np.zeros(nz + 1, F)
    for k in range(nz + 1):
        if k == 0:
            rf0[k] = fmaf(cgs[2], rho0[2], fmaf(cgs[0], rho0[0], f(cgs[1] * rho0[1])))
        elif k == nz:
            rf0[k] = fmaf(cgt[2], rho0[nz - 3], fmaf(cgt[0], rho0[nz - 1], f(cgt[1] * rho0[nz - 2])))
        else:
            rf0[k] = fmaf(vg.c1[k], rho0[k - 1], f(vg.c2[k] * rho0[k]))
    u0 = np.array([f(f(cfg.us) * np.tanh(f(z / f(3000.0)))) for z in vg.zh], F)
    return {
        'vg': vg, 'rho0': rho0, 'rr0': (F(1.0) / rho0).astype(F), 'rf0': rf0,
        'th0': base['th0'], 'pi0': base['pi0'], 'qv0': base['qv0'],
        'qc0': np.zeros(nz, F), 'qi0': np.zeros(nz, F),
        'rth0': (F(1.0) / base['th0']).astype(F), 'u0': u0, 'v0': np.zeros(nz, F),
    }


def fill_arena(cfg, grid, prof, arena, fields):
    """Initial arena (scenario.js:234-296) with bubble + noise, halos periodic."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    sJ, sK = grid.strideJ, grid.strideK
    W = nx + 1 + 2 * HALO   # the columns of points; with aligned rows the rest is padding, left 0
    xf, xh = grid.axis(nx, grid.dx)
    yf, yh = grid.axis(ny, grid.dy)
    vg = prof['vg']
    pi0, th0, qv0, u0 = prof['pi0'], prof['th0'], prof['qv0'], prof['u0']
    p00 = f(P00)
    cpdrd = f(f(CP) / f(RD))
    rd, rv = f(RD), f(RV)

    def view(name):
        off = fields[name] // 4
        return arena[off:off + grid.count].reshape(nz + 1, sK, sJ)[:, :, :W]

    # bubble (+ noise on interior points, then periodic halos)
    X = xh[None, None, :W]
    Y = yh[None, :sK, None]
    Z = vg.zh.astype(np.float64)[:, None, None]
    tha = np.zeros((nz, sK, W), np.float64)
    for (ox, oy) in cfg.bubbles:
        bx = (X - ox) / 10000.0
        by = (Y - oy) / 10000.0
        bz = (Z - 1400.0) / 1400.0
        beta = np.sqrt(bx * bx + by * by + bz * bz)
        c = np.cos(0.5 * math.pi * beta)
        tha = np.maximum(tha, np.where(beta < 1.0, cfg.amplitude * c * c, 0.0))
    th = tha.astype(F)
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing='ij')
    r = hash_rand_grid(cfg.seed, ii + 1, jj + 1, kk + 1)
    noise = (F(cfg.noise) * ((F(2.0) * r) - F(1.0))).astype(F)
    th[:, HALO:HALO + ny, HALO:HALO + nx] = (th[:, HALO:HALO + ny, HALO:HALO + nx] + noise).astype(F)
    periodic_halos(th, nx, ny)
    for name in ('th', 'th_a'):
        view(name)[:nz] = th
    for name in ('qv', 'qv_a'):
        if name in fields:   # a dry run has no moisture fields
            view(name)[:nz] = qv0[:, None, None]
    for name in ('u', 'u_a'):
        view(name)[:nz] = u0[:, None, None]
    p = np.array([f(p00 * np.power(pi0[k], cpdrd)) for k in range(nz)], F)
    view('prs')[:nz] = p[:, None, None]
    qv = np.maximum(F(0.0), qv0).astype(F)
    rmix = (rd + (qv * rv).astype(F)).astype(F)
    th_full = (th0[:, None, None] + th).astype(F)
    view('rho')[:nz] = (p[:, None, None] / ((th_full * pi0[:, None, None]).astype(F) * rmix[:, None, None]).astype(F)).astype(F)


def periodic_halos(a, nx, ny):
    """Fill the 3-cell halos of a (k, j, i) array periodically."""
    h = HALO
    a[:, :, :h] = a[:, :, nx:nx + h]
    a[:, :, nx + h:nx + 2 * h + 1] = a[:, :, h:2 * h + 1]
    a[:, :h, :] = a[:, ny:ny + h, :]
    a[:, ny + h:ny + 2 * h + 1, :] = a[:, h:2 * h + 1, :]


# ---------------------------------------------------------------- ensembles

def cape(qv_pbl=0.014, dz=100.0, ztop=16000.0):
    """Surface-parcel CAPE (J/kg) of the Weisman-Klemp sounding with boundary-layer
    moisture capped at ``qv_pbl``: the parcel rises dry-adiabatically, then
    pseudo-adiabatically (condensate removed, saturation adjustment by Newton steps),
    CAPE = sum of g (thv_parcel - thv_env) / thv_env dz where positive.  Binary64, on a
    fine column of its own (dz), independent of any model grid."""
    zh = np.arange(0.5 * dz, ztop, dz)
    b = weisman_klemp(zh.astype(F), qv_pbl=qv_pbl)
    th_env = b['th0'].astype(np.float64)
    qv_env = b['qv0'].astype(np.float64)
    pi = b['pi0'].astype(np.float64)
    prs = b['prs0'].astype(np.float64)
    cp, rd, rv, lv = CP, RD, RV, 2.501e6
    eps = RD / RV

    def qsat(p, t):
        es = 611.2 * np.exp(17.67 * (t - 273.15) / (t - 29.65))
        es = min(es, 0.5 * p)
        return eps * es / (p - es)

    t = th_env[0] * pi[0]
    qv = qv_env[0]
    total = 0.0
    for k in range(1, len(zh)):
        t = t - G / cp * (zh[k] - zh[k - 1])        # dry ascent over the step
        for _ in range(20):                         # condense the excess (pseudo-adiabatic)
            qs = qsat(prs[k], t)
            if qv <= qs:
                break
            dq = (qv - qs) / (1.0 + lv * lv * qs / (cp * rv * t * t))
            qv -= dq
            t += lv / cp * dq
        thv_p = t / pi[k] * (1.0 + qv / eps) / (1.0 + qv)
        thv_e = th_env[k] * (1.0 + qv_env[k] / eps) / (1.0 + qv_env[k])
        buoy = G * (thv_p - thv_e) / thv_e
        if buoy > 0:
            total += buoy * (zh[k] - zh[k - 1])
    return total


_CAPE_TABLE = None


def _cape_table():
    """CAPE of moisture caps 0.0100, 0.0102, ..., 0.0200 (monotone; computed once)."""
    global _CAPE_TABLE
    if _CAPE_TABLE is None:
        q = np.linspace(0.010, 0.020, 51)
        _CAPE_TABLE = (q, np.array([cape(x) for x in q]))
    return _CAPE_TABLE


@functools.lru_cache(maxsize=None)
def qv_pbl_for_cape(target):
    """The boundary-layer moisture cap whose sounding has CAPE ``target``: bracketed in
    the table, then refined by bisection on the sounding itself."""
    q, c = _cape_table()
    k = int(np.clip(np.searchsorted(c, target), 1, len(q) - 1))
    lo, hi = q[k - 1], q[k]
    for _ in range(8):
        mid = 0.5 * (lo + hi)
        if cape(mid) < target:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def ensemble(n=64, seed=7, steps=50):
    """Members of the batched-ensemble workload: grids drawn from 64x64x40 to 192x192x64
    (nx, ny multiples of 8, nz multiple of 4), dx = 500 m with dt = 3 s or dx = 1000 m with
    dt = 6 s, nsound 6..8, shear Us ~ U[10, 30] m/s, CAPE ~ U[1000, 4000] J/kg through the
    boundary-layer moisture cap, each with its own noise seed."""
    rng = np.random.default_rng(seed)
    out = []
    caps = {}
    for m in range(n):
        nx = int(rng.integers(8, 25)) * 8
        ny = int(rng.integers(8, 25)) * 8
        nz = int(rng.integers(10, 17)) * 4
        fine = bool(rng.integers(0, 2))
        dx, dt = (500.0, 3.0) if fine else (1000.0, 6.0)
        dz = 16000.0 / nz if not fine else 12000.0 / nz
        nsound = int(rng.integers(6, 9))
        us = float(rng.uniform(10.0, 30.0))
        target = float(rng.uniform(1000.0, 4000.0))
        key = round(target, -2)
        if key not in caps:
            caps[key] = qv_pbl_for_cape(key)
        cfg = Config('member%02d-%dx%dx%d' % (m, nx, ny, nz), nx, ny, nz, dx, dz, dt, nsound, us, steps,
                     seed=1 + m, qv_pbl=caps[key])
        cfg.cape = key
        out.append(cfg)
    return out
