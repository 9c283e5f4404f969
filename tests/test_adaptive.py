"""The dry step (update_diagnostics) and the adaptive time step (stability_max + the
host rule of web/core/adaptive.js)."""
import numpy as np
import pytest

from tests import helpers
from thunderengine_web_b200 import scenario, timestep


def _dry_run():
    cfg = scenario.tiny(20, 16, 12, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0)
    return timestep.Run(cfg, moist=False, adaptive=True)


def test_dry_adaptive_step_oracle_equals_reference_kernels():
    """The dry step with the stability reduction: the oracle and the reference's own
    kernels (oracle/_ref) leave the same memory, word for word (no shipped recording
    runs the dry step or stability_max)."""
    ref = helpers.reference()
    if ref is None:
        pytest.skip('oracle/_ref not built')
    run = _dry_run()
    tape = run.tape(1)
    names = {c['name'] for c in tape['steps'][0] if c['op'] == 'pipe'}
    assert {'update_diagnostics', 'stability_max'} <= names
    assert 'update_diagnostics_moist' not in names and 'apply_thterm' not in names
    init = run.initial_buffers()
    a = helpers.cpu_run(tape, init, nsteps=2, hashes=True)
    b = helpers.cpu_run(tape, init, nsteps=2, hashes=True, kernels=ref.get)
    assert np.array_equal(a.M, b.M)
    assert np.array_equal(a.hashes, b.hashes)


def test_adaptive_rule():
    """getnewdt / dtsmall (adaptive.js:59-101): CFL above 1 shrinks dt in proportion, a
    small CFL grows it by at most 10 %, the diffusion number caps it, dt never passes
    2 dtl, and the substep count is even, >= 4 and keeps dt / n <= dtsm."""
    a = timestep.AdaptiveTimeStep(3.0, 500.0)
    a.start(0.5, 0.0)
    assert abs(a.dt - 3.3) < 1e-5 and a.nsound % 2 == 0 and a.nsound >= 4
    assert a.dt / a.nsound <= a.dtsm * (1 + 1e-6)
    b = timestep.AdaptiveTimeStep(3.0, 500.0)
    b.start(2.0, 0.0)
    assert abs(b.dt - 1.5) < 1e-6
    c = timestep.AdaptiveTimeStep(3.0, 500.0)
    for _ in range(30):
        c.end_step(1e-3, 0.0)
    assert abs(c.dt - 6.0) < 1e-5       # 2 dtl
    d = timestep.AdaptiveTimeStep(3.0, 500.0)
    d.start(0.5, 0.2)                    # ks 0.2 * 3.3/3 > 0.09: the diffusion limit
    assert abs(d.dt - timestep.f(timestep.f(3.0 * d.ks_limit) / 0.2)) < 1e-6
    w = np.array([np.float32(0.25).view(np.uint32), np.float32(0.04).view(np.uint32)], np.uint32)
    assert timestep.stability_from_words(w) == (timestep.f(0.5), timestep.f(0.2))


def _adaptive_steps(step, read, zero, use, run, n):
    """n adaptive steps: step, read the stability words, clear them, new dt / nsound."""
    sid = run.rec.ids['stability']
    g = run.grid
    clock = timestep.AdaptiveTimeStep(run.cfg.dt, min(g.dx, g.dy))
    seq = []
    for _ in range(n):
        step()
        cfl, ks = timestep.stability_from_words(read(sid))
        zero(sid)
        clock.end_step(cfl, ks)
        run.set_time_step(clock.dt, clock.nsound)
        use(run.encode())
        seq.append((float(clock.dt), clock.nsound))
    return seq


@pytest.mark.gpu
def test_gpu_dry_adaptive_steps_equal_the_oracle():
    """Three adaptive steps of the dry step on the GPU and on the oracle: the same dt and
    substep sequence, and the same memory word for word after each."""
    run_g, run_c = _dry_run(), _dry_run()
    tape = run_g.tape(1)
    run_c.tape(1)
    init = run_g.initial_buffers()
    gpu = helpers.gpu_replayer(tape, init, hashes=False)
    cpu = helpers.cpu_run(tape, init, nsteps=0, hashes=False)
    z = np.zeros(2, np.uint32)
    seq_g = _adaptive_steps(lambda: gpu.encode_steps(1), lambda sid: gpu.read(2, gpu.base[sid]),
                            lambda sid: gpu.write_words(gpu.base[sid], z), gpu.use_step, run_g, 3)
    seq_c = _adaptive_steps(lambda: cpu.run(helpers.oracle().get), lambda sid: cpu.M[cpu.base[sid]:cpu.base[sid] + 2],
                            lambda sid: cpu.write_words(cpu.base[sid], z), cpu.use_step, run_c, 3)
    assert seq_g == seq_c
    assert len({n for _, n in seq_g}) >= 1 and seq_g[0][0] != run_g.cfg.dt
    assert np.array_equal(gpu.read(gpu.buffers_end), cpu.M[:gpu.buffers_end])
    gpu.close()
