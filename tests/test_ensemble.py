"""Batched ensembles of uneven members and the launch-shape autotuner."""
import numpy as np
import pytest

from tests import helpers
from thunderengine_web_b200 import scenario, timestep


def test_ensemble_members_are_seeded_and_in_range():
    a = scenario.ensemble(64, seed=7)
    b = scenario.ensemble(64, seed=7)
    assert [(m.nx, m.ny, m.nz, m.dt, m.nsound, m.us, m.qv_pbl) for m in a] == \
           [(m.nx, m.ny, m.nz, m.dt, m.nsound, m.us, m.qv_pbl) for m in b]
    assert all(64 <= m.nx <= 192 and 64 <= m.ny <= 192 and 40 <= m.nz <= 64 for m in a)
    assert all(m.dt in (3.0, 6.0) and m.dx == (500.0 if m.dt == 3.0 else 1000.0) for m in a)
    assert all(6 <= m.nsound <= 8 and 10.0 <= m.us <= 30.0 for m in a)
    assert all(1000.0 <= m.cape <= 4000.0 for m in a)
    # uneven: many distinct shapes and substep schedules
    assert len({(m.nx, m.ny, m.nz) for m in a}) > 40
    assert len({timestep.AcousticSchedule(m.nsound, timestep.f(m.dt)).total for m in a}) >= 2


def test_cape_of_the_moisture_cap():
    """CAPE grows with the boundary-layer moisture cap; the bisection hits its target."""
    c = [scenario.cape(q) for q in (0.012, 0.014, 0.016)]
    assert c[0] < c[1] < c[2]
    q = scenario.qv_pbl_for_cape(2500.0)
    assert abs(scenario.cape(q) - 2500.0) < 5.0


def _members(mode):
    cfgs = [scenario.tiny(24, 20, 12, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0),
            scenario.tiny(40, 16, 10, dx=1000.0, dz=500.0, dt=6.0, nsound=6, us=12.0),
            scenario.tiny(16, 32, 14, dx=500.0, dz=250.0, dt=3.0, nsound=7, us=18.0)]
    runs = [timestep.Run(c) for c in cfgs]
    reps = []
    for run in runs:
        tape = run.tape(1)
        reps.append((run, tape, run.initial_buffers(), helpers.gpu_replayer(tape, run.initial_buffers(), hashes=False,
                                                                           mode=mode)))
    return reps


@pytest.mark.gpu
@pytest.mark.parametrize('mode', [0, 1])
def test_ensemble_steps_equal_each_member_stepped_alone(mode):
    """Three members of different sizes, time steps and substep counts: two ensemble steps
    leave every member's memory equal, word for word, to two steps of that member alone."""
    from thunderengine_web_b200.replayer import Ensemble
    reps = _members(mode)
    ens = Ensemble([r for _, _, _, r in reps])
    ens.run(2)
    ens.sync()
    for run, tape, init, r in reps:
        alone = helpers.gpu_replayer(tape, init, hashes=False, mode=mode)
        alone.encode_steps(2)
        assert np.array_equal(r.read(r.buffers_end), alone.read(alone.buffers_end))
        alone.close()
    ens.close()
    for *_, r in reps:
        r.close()


@pytest.mark.gpu
def test_autotune_leaves_state_and_results_unchanged():
    """Tuning times the ops on the live memory and restores it; a step with the tuned
    shapes equals the oracle's step."""
    run = timestep.Run(scenario.tiny(37, 29, 13, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0))
    tape = run.tape(1)
    init = run.initial_buffers()
    r = helpers.gpu_replayer(tape, init, hashes=False)
    before = r.read(r.buffers_end)
    r.autotune(reps=2)
    assert np.array_equal(r.read(r.buffers_end), before)
    r.encode_steps(1)
    cpu = helpers.cpu_run(tape, init, nsteps=1, hashes=False)
    assert np.array_equal(r.read(r.buffers_end), cpu.M[:r.buffers_end])
    r.close()
