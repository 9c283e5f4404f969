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


def _dispatches(cmds, fields=None):
    """(kernel, grid, workgroup, {binding: setBytes payload}, {binding: arena field}) per
    dispatch of a command stream."""
    by_off = {v: k for k, v in (fields or {}).items()}
    out, pipe, byts, bufs = [], None, {}, {}
    for c in cmds:
        if c['op'] == 'pipe':
            pipe, byts, bufs = c['name'], {}, {}
        elif c['op'] == 'bytes':
            byts[c['index']] = c['data']
        elif c['op'] == 'buf':
            bufs[c['index']] = by_off.get(c['offset'])
        elif c['op'] == 'dispatch':
            out.append((pipe, list(c['grid']), list(c['tg']), dict(byts), dict(bufs)))
    return out


# ops of the recording that exist for its open lateral boundaries (and the periodic halo
# fills that replace them here), and the setBytes payloads that carry the open flags
OPEN_BC = ('bc_open_x', 'bc_open_y', 'radbc_ew', 'radbc_ns', 'openbc_uv_tendency', 'bc_periodic_x', 'bc_periodic_y')
OPEN_FLAGS = {'acoustic_uv': {8}, 'adv_assemble': {17}}


def _segment(ops, first, names):
    """The dispatches from `first` whose kernel is in `names`, in order, up to the next
    dispatch of `first`'s kernel (one acoustic substep / one advection call)."""
    out = []
    for o in ops[first:]:
        if out and o[0] == ops[first][0] and len(out) > 1:
            break
        if o[0] in OPEN_BC:
            continue
        if o[0] not in names:
            break
        out.append(o)
    return out


def test_substep_and_advection_commands_equal_the_recording():
    """The command stream of the first acoustic substep and of the stage-1 advection of
    u, v and w equals the reference's recorded single_cell step (120x120x40, dt 6 s,
    4 substeps, timestep.js:1997-2060 and 1629-1900): kernel order, dispatch grids,
    workgroup sizes and every setBytes payload, with the recording's open-boundary
    kernels and open flags set aside (this encoder writes periodic boundaries)."""
    golden, _, _, _ = helpers.load_golden_scenario('single_cell')
    rec = _dispatches(golden['steps'][0])
    run = timestep.Run(scenario.tiny(120, 120, 40, dx=1000.0, dz=500.0, dt=6.0, nsound=4))
    mine = _dispatches(run.encode())
    substep = ('acoustic_uv', 'acoustic_fpk', 'acoustic_w_solve', 'acoustic_pp', 'acoustic_accumulate')
    advect = ('adv_flux_x_stag', 'adv_flux_y_stag', 'adv_flux_z_stag', 'adv_assemble')

    def first(ops, name):
        return next(q for q, o in enumerate(ops) if o[0] == name)

    for names, start in ((substep, 'acoustic_uv'), (advect, 'adv_flux_x_stag')):
        a = [o for o in _segment(rec, first(rec, start), names)]
        b = [o for o in _segment(mine, first(mine, start), names)]
        if start == 'adv_flux_x_stag':   # u, v and w: three calls of four kernels
            a = [o for o in rec[first(rec, start):] if o[0] in names][:12]
            b = [o for o in mine[first(mine, start):] if o[0] in names][:12]
        assert [o[0] for o in a] == [o[0] for o in b] and len(a) >= 4
        for x, y in zip(a, b):
            assert x[1] == y[1] and x[2] == y[2], (x[0], x[1], y[1], x[2], y[2])
            skip = OPEN_FLAGS.get(x[0], set())
            assert {k: v for k, v in x[3].items() if k not in skip} == \
                   {k: v for k, v in y[3].items() if k not in skip}, x[0]


def test_aligned_rows_change_only_the_layout():
    """With the row pitch rounded up to 32 floats, one oracle step leaves every point of
    every non-scratch field equal, bit for bit, to the unpadded run's, and the padding
    columns of every field at 0.  (Scratch faces such as fx at i = -1 take stencil values
    from past the row's first halo point, which the two layouts hold differently; nothing
    reads those faces.)"""
    runs, mems = [], []
    for align in (False, True):
        run = timestep.Run(scenario.tiny(20, 16, 12, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0, align_rows=align))
        tape = run.tape(1)
        mems.append(helpers.cpu_run(tape, run.initial_buffers(), nsteps=1, hashes=False))
        runs.append(run)
    (ra, rb), (ma, mb) = runs, mems
    g, h = ra.grid, rb.grid
    assert h.strideJ == 32 and g.strideJ == 27
    ba, bb = ma.base[ra.rec.ids['arena']], mb.base[rb.rec.ids['arena']]
    for name in ra.fields:
        a = ma.M[ba + ra.fields[name] // 4:ba + ra.fields[name] // 4 + g.count].reshape(g.nz + 1, g.strideK, g.strideJ)
        b = mb.M[bb + rb.fields[name] // 4:bb + rb.fields[name] // 4 + h.count].reshape(h.nz + 1, h.strideK, h.strideJ)
        if name not in helpers.SCRATCH:
            assert np.array_equal(a, b[:, :, :g.strideJ]), name
        assert not b[:, :, g.strideJ:].any(), name
