"""Error of the binary32 step against the binary64 twin of the oracle.

The binary64 twin (oracle/liboracle64.so) evaluates the same kernels in the same order
in binary64.  The CUDA step equals the binary32 oracle bit for bit, so the binary32
oracle's error is the product's error; the GPU test measures it on the GPU's own state
at the benchmarked configuration.  Bounds: absolute, per prognostic field, from the
field's scale (K, kg/kg, m/s, nondimensional pi')."""
import numpy as np
import pytest

from tests import helpers
from thunderengine_web_b200 import scenario, timestep

# largest allowed |f32 - f64| per field after one large step
BOUND_1 = {'th': 1e-3, 'qv': 1e-8, 'u': 1e-4, 'v': 1e-4, 'w': 1e-4, 'pp3d': 1e-7}


def _interior(a, g):
    return a.reshape(g.nz + 1, g.strideK, g.strideJ)[:g.nz, 3:3 + g.ny, 3:3 + g.nx]


def _twin(run, init):
    from oracle.player import CpuPlayer64
    p = CpuPlayer64(run.tape(1), helpers.kernels_meta())
    p.plan()
    for i, b in init.items():
        p.upload(i, b)
    p.values_from_words()
    return p


def _errors(run, mem32, base, p):
    g = run.grid
    out = {}
    for f in BOUND_1:
        o = base + run.fields[f] // 4
        a = _interior(mem32[o:o + g.count].view(np.float32), g).astype(np.float64)
        b = _interior(p.field64(o, g.count), g)
        out[f] = float(np.abs(a - b).max())
    return out


def test_twin_equals_binary32_oracle_to_rounding_on_three_steps():
    """Tiny grid, three steps: the binary32 oracle stays within the bounds of the twin,
    and the twin is not the binary32 oracle (the errors are not all zero)."""
    run = timestep.Run(scenario.tiny(37, 29, 13, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0))
    tape = run.tape(1)
    init = run.initial_buffers()
    cpu = helpers.cpu_run(tape, init, nsteps=3, hashes=False)
    p = _twin(run, init)
    p.run64(3)
    err = _errors(run, cpu.M, cpu.base[run.rec.ids['arena']], p)
    for f, e in err.items():
        assert e <= 3 * BOUND_1[f], (f, e)
    assert any(e > 0 for e in err.values())


def test_twin_tracks_a_perturbation_linearly():
    """The twin is a binary64 evaluation of the same step: a 1e-6 K change of one th
    value moves the result by a finite, proportionate amount (no binary32 rounding
    floor), and the step of the unperturbed state is reproducible."""
    run = timestep.Run(scenario.tiny(16, 12, 10))
    run.tape(1)
    init = run.initial_buffers()
    p0 = _twin(run, init)
    p0.run64(1)
    p1 = _twin(run, init)
    for f in ('th', 'th_a'):     # the step's state and its start-of-step copy
        o = p1.base[run.rec.ids['arena']] + run.fields[f] // 4 + (3 + 6) + run.grid.strideJ * (3 + 5) \
            + run.grid.strideJ * run.grid.strideK * 4
        p1.D[o] += 1e-6
    p1.run64(1)
    g = run.grid
    base = p0.base[run.rec.ids['arena']]
    d = {f: np.abs(p1.field64(base + run.fields[f] // 4, g.count) - p0.field64(base + run.fields[f] // 4, g.count)).max()
         for f in ('th', 'w')}
    assert 1e-8 < d['th'] < 1e-5 and 0 < d['w'] < 1e-5
    p2 = _twin(run, init)
    p2.run64(1)
    assert np.array_equal(p2.D, p0.D)


@pytest.mark.gpu
def test_headline_config_error_against_binary64():
    """256x256x80, one large step on the GPU (fused mode, the benchmarked one) against
    the binary64 twin: every prognostic field within its bound."""
    from thunderengine_web_b200.replayer import TE_MODE_FUSED
    run = timestep.Run(scenario.AT_SCALE)
    tape = run.tape(1)
    init = run.initial_buffers()
    gpu = helpers.gpu_replayer(tape, init, hashes=False, mode=TE_MODE_FUSED)
    gpu.encode_steps(1)
    mem = gpu.read(gpu.buffers_end)
    base = gpu.base[run.rec.ids['arena']]
    gpu.close()
    p = _twin(run, init)
    p.run64(1)
    err = _errors(run, mem, base, p)
    for f, e in err.items():
        assert e <= BOUND_1[f], (f, e)
