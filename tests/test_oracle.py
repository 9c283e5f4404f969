"""The CPU oracle: pinned to the reference's golden recording and to its own kernels."""
import ctypes
import math

import numpy as np
import pytest

from tests import helpers
from thunderengine_web_b200 import scenario, timestep


def test_div_cr_is_the_correctly_rounded_quotient(oracle_lib):
    f = oracle_lib.lib.te_div_cr
    f.restype = ctypes.c_float
    f.argtypes = [ctypes.c_float, ctypes.c_float]
    rng = np.random.default_rng(1)
    a = (rng.standard_normal(2000) * 10.0 ** rng.integers(-20, 20, 2000)).astype(np.float32)
    b = (rng.standard_normal(2000) * 10.0 ** rng.integers(-10, 10, 2000)).astype(np.float32)
    for x, y in zip(a, b):
        want = np.float32(np.float64(x) / np.float64(y))   # double quotient rounds correctly to f32 here
        assert f(float(x), float(y)) == want


def test_weno5_reproduces_smooth_data(oracle_lib):
    w = oracle_lib.lib.te_weno5
    w.restype = ctypes.c_float
    w.argtypes = [ctypes.c_float] * 6
    # the stencil weights are rounded binary32 quotients, so smooth data comes back
    # within a few ulps, not exactly
    assert abs(w(1.5, 1.5, 1.5, 1.5, 1.5, 1e-17) - 1.5) < 4e-7
    assert abs(w(1.0, 2.0, 3.0, 4.0, 5.0, 1e-17) - 3.5) < 1e-6      # linear: interface value 3.5
    assert abs(w(5.0, 4.0, 3.0, 2.0, 1.0, 1e-17) - 2.5) < 1e-6


def test_rr_pow_is_correctly_rounded(oracle_lib):
    # f_rr_pow_cr (update_rho_prs.wgsl, pressure_tendency.wgsl:114-226)
    p = oracle_lib.lib.te_rr_pow_cr
    p.restype = ctypes.c_float
    p.argtypes = [ctypes.c_float, ctypes.c_float]
    cpdrd = np.float32(np.float32(1005.7) / np.float32(287.04))
    xs = np.linspace(0.6, 1.05, 3001).astype(np.float32)
    bad = 0
    for x in xs:
        want = np.float32(math.pow(float(x), float(cpdrd)))
        bad += p(float(x), float(cpdrd)) != want
    assert bad <= 3



def test_wgsl_pow_is_correctly_rounded(oracle_lib):
    """te_pow_f64 (the WGSL pow builtin of turb_km_kh.wgsl) against x^y to 50 digits:
    correctly rounded on every sample, and exact on exact cubes."""
    from decimal import Decimal, getcontext
    getcontext().prec = 50
    p = oracle_lib.lib.te_pow_f64
    p.restype = ctypes.c_float
    p.argtypes = [ctypes.c_float, ctypes.c_float]

    def nearest(x, y):
        v = (Decimal(float(y)) * Decimal(float(x)).ln()).exp()
        f = np.float32(float(v))
        cands = [np.nextafter(f, np.float32(-np.inf)), f, np.nextafter(f, np.float32(np.inf))]
        return min(cands, key=lambda c: abs(Decimal(float(c)) - v))

    rng = np.random.default_rng(3)
    xs = (10.0 ** rng.uniform(-12, 12, 1500)).astype(np.float32)
    for y in (np.float32(0.33333334), np.float32(2.5), np.float32(-0.7)):
        for x in xs:
            assert p(float(x), float(y)) == nearest(x, y), (x, y)
    assert p(8.0, 0.33333334) == 2.0 and p(1.0, 0.33333334) == 1.0 and p(0.0, 0.33333334) == 0.0
    assert math.isnan(p(-1.0, 0.33333334))

def test_oracle_equals_reference_kernels_on_synthetic_step(oracle_lib, ref_lib, kernels_meta):
    """Hand-written oracle vs the reference's own kernels: every word after 2 steps."""
    run = timestep.Run(scenario.tiny(16, 12, 10))
    tape = run.tape(1)
    init = run.initial_buffers()
    a = helpers.cpu_run(tape, init, nsteps=2, hashes=True, kernels=ref_lib.get)
    b = helpers.cpu_run(tape, init, nsteps=2, hashes=True, kernels=oracle_lib.get)
    assert np.array_equal(a.hashes, b.hashes)
    assert np.array_equal(a.M, b.M)


@pytest.mark.slow
def test_oracle_pinned_to_golden_single_cell(oracle_lib, ref_lib):
    """Replay the recorded single_cell step 1 with the oracle on every in-scope dispatch.

    All 35 buffers' FNV-1a after step 1 equal the recording (step1.json).  Per-dispatch
    region hashes equal the recording except in the scratch fields tend/fpk, which the
    reference documents as not matching its recording (web/view.js:1047-1049).
    """
    from oracle.player import CpuPlayer, fnv1a
    tape, init, want, step1 = helpers.load_golden_scenario()
    p = CpuPlayer(tape, helpers.kernels_meta())
    p.plan(True)
    for i, b in init.items():
        p.upload(i, b)
    used = {o.name for o in p.ops if o.kind == 'k' and oracle_lib.has(o.name)}
    assert len(used) >= 36
    p.run(helpers.mixed, with_hashes=True)
    for b in tape['buffers']:
        assert fnv1a(p.buffer_words(b['id'])) == step1[b['id']], b['label']
    fields = {v // 4 + p.base[2]: k for k, v in tape['fields'].items()}
    slot_field = {s: fields.get(off) for o in p.ops if o.kind == 'k' for s, off, _ in o.hashes}
    bad = [s for s in range(want.size) if want[s] != p.hashes[s]]
    assert want.size == 1010 and len(bad) <= 40
    assert {slot_field[s] for s in bad} <= {'tend', 'fpk'}


@pytest.mark.slow
def test_column_kernels_on_branches_the_recording_does_not_take(oracle_lib, ref_lib):
    """turb_scalar_vert_implicit and mp_pdefq, oracle vs the reference's kernels, on the
    state of the recorded step at their first dispatch, with the flags of the branches the
    recording does not take: explicit vertical fluxes, surface flux, bcturbs = 2 and the
    three wall settings (turb_scalar_vert_implicit.wgsl lam_1), a clip threshold that
    zeroes part of every column (mp_pdefq.wgsl), the lateral sponge and level-average
    references of rayleigh_damping.wgsl, and a fixed km and the cmz floor of turb_km_kh.wgsl."""
    import itertools
    from oracle.player import CpuPlayer
    tape, init, want, step1 = helpers.load_golden_scenario()
    p = CpuPlayer(tape, helpers.kernels_meta())
    p.plan(False)
    for i, b in init.items():
        p.upload(i, b)
    fb = lambda x: int(np.float32(x).view(np.uint32))
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    done = set()
    compared = 0
    for o in p.ops:
        if o.kind == 'copy':
            p.M[o.dst:o.dst + o.n] = p.M[o.src:o.src + o.n]
            continue
        if o.name in ('turb_scalar_vert_implicit', 'mp_pdefq', 'rayleigh_damping', 'turb_km_kh') and o.name not in done:
            done.add(o.name)
            B = lambda n: int(o.arg[4 + n])
            sk = 127 * 127   # one level of the 120 x 120 recording (halo 3 on each side)
            if o.name == 'rayleigh_damping':
                variants = [{B(16): a, B(17): b} for a in (0, 1) for b in (0, 1)]
            elif o.name == 'turb_km_kh':
                variants = [{B(11): fb(5.0)}, {B(12): fb(0.001)}]
            elif o.name == 'mp_pdefq':
                q = p.M[B(2):B(2) + 8 * sk].view(np.float32)
                nz_q = np.abs(q[q != 0])
                variants = [{B(3): fb(np.median(nz_q) if nz_q.size else 1e-6)}, {B(3): fb(-1.0)}]
            else:
                variants = []
                for uf, ez, bt, ww in itertools.product([0, 1], [0, 1], [1, 2], [0.0, 1.0, 2.0]):
                    v = {B(15): uf, B(16): ez, B(18): bt}
                    v.update({B(17) + q: fb(x) for q, x in enumerate([0.37, 301.5, 290.25, ww])})
                    variants.append(v)
            for v in variants:
                E, F = p.M.copy(), p.M.copy()
                for X in (E, F):
                    for w, val in v.items():
                        X[w] = val
                    if o.name == 'turb_scalar_vert_implicit':
                        X[B(14):B(14) + sk] = fb(0.011)
                oracle_lib.get(o.name)(vp(E), vp(o.arg))
                ref_lib.get(o.name)(vp(F), vp(o.arg))
                assert np.array_equal(E, F), (o.name, v)
                compared += 1
        helpers.mixed(o.name)(vp(p.M), vp(o.arg))
        if len(done) == 4:
            break
    assert compared == 32
