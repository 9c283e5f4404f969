"""Step encoder (thunderengine_web_b200.timestep) against the reference's recorded tape."""
import numpy as np
import pytest

from tests import helpers
from thunderengine_web_b200 import scenario, timestep


def test_acoustic_schedule_matches_reference_rule():
    # AcousticSchedule (timestep.js:74-86): nsound=6 -> 2+3+6, nsound=8 at dt=3 -> 3+4+8
    s6 = timestep.AcousticSchedule(6, 6.0)
    assert [c for c, _ in s6.loops] == [2, 3, 6] and s6.total == 11
    assert [d for _, d in s6.loops] == [1.0, 1.0, 1.0]
    s8 = timestep.AcousticSchedule(8, 3.0)
    assert [c for c, _ in s8.loops] == [3, 4, 8] and s8.total == 15
    assert abs(s8.loops[0][1] - 1.0 / 3.0) < 1e-15 and s8.loops[2][1] == 0.375


def test_weno_epsilon():
    # timestep.js:387-392
    assert timestep.weno_epsilon('th') == timestep.f(10 * timestep.f(1e-18))
    assert timestep.weno_epsilon('qv') == timestep.f(timestep.f(1e-2) * timestep.f(1e-18))


def _bound_per_kernel(cmds):
    out = {}
    bind = set()
    pipe = None
    for c in cmds:
        if c['op'] == 'pipe':
            pipe = c['name']
        elif c['op'] in ('buf', 'bytes', 'bufoff'):
            bind.add(c['index'])
        elif c['op'] == 'end':
            bind = set()
        elif c['op'] == 'dispatch':
            out.setdefault(pipe, []).append(set(bind))
    return out


def test_bindings_cover_the_reference_encoder():
    """Every parameter the reference encoder binds for a kernel is bound by ours too."""
    golden, _, _, _ = helpers.load_golden_scenario()
    km = helpers.kernels_meta()
    run = timestep.Run(scenario.tiny())
    mine = _bound_per_kernel(run.encode())
    ref = _bound_per_kernel(golden['steps'][0])
    common = [k for k in mine if k in ref]
    assert len(common) >= 35
    terrain_only = {20, 21, 22, 23, 24, 25, 26}
    for k in common:
        params = {p['index'] for p in km[k]['params']}
        need = set().union(*ref[k]) & params - terrain_only
        for b in mine[k]:
            assert need <= b, (k, sorted(need - b))


def test_step_structure_counts():
    cfg = scenario.tiny(16, 12, 10, nsound=8, dt=3.0)
    run = timestep.Run(cfg)
    cmds = run.encode()
    names = [c['name'] for c in cmds if c['op'] == 'pipe']
    assert names.count('acoustic_w_solve') == 15
    assert names.count('adv_flux_x_weno') == 2 and names.count('adv_flux_x') == 4
    assert names.count('adv_flux_x_weno_uv') == 2 and names.count('adv_flux_x_weno_w') == 1
    assert names.count('pdef_apply') == 1
    assert sum(1 for c in cmds if c['op'] == 'copy') == 6


def test_weisman_klemp_base_state():
    p = scenario.profiles(scenario.SMALL)
    th0, qv0, pi0, rho0 = p['th0'], p['qv0'], p['pi0'], p['rho0']
    assert np.all(np.diff(th0) > 0) and np.all(np.diff(pi0) < 0) and np.all(np.diff(rho0) < 0)
    assert qv0.max() <= np.float32(0.014) and qv0.min() > 0
    assert abs(float(th0[0]) - 300.0) < 2.0
    assert p['rf0'].shape == (scenario.SMALL.nz + 1,)


def test_initial_arena_is_periodic_and_bubble_centred():
    cfg = scenario.tiny(24, 20, 12)
    run = timestep.Run(cfg)
    arena = run.initial_arena()
    g = run.grid
    th = arena[run.fields['th'] // 4: run.fields['th'] // 4 + g.count].reshape(g.nz + 1, g.strideK, g.strideJ)
    h = scenario.HALO
    assert np.array_equal(th[:g.nz, :, :h], th[:g.nz, :, g.nx:g.nx + h])
    assert np.array_equal(th[:g.nz, :h, :], th[:g.nz, g.ny:g.ny + h, :])
    assert th.max() > 1.5      # 2 K bubble
