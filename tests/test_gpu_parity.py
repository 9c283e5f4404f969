"""CUDA path (through the C-ABI) against the CPU oracle and the golden recording."""
import ctypes

import numpy as np
import pytest

from tests import helpers
from thunderengine_web_b200 import scenario, timestep

pytestmark = pytest.mark.gpu


def _compare(run, tape, init, nsteps, mode=0, hashes=True):
    cpu = helpers.cpu_run(tape, init, nsteps=nsteps, hashes=hashes)
    gpu = helpers.gpu_replayer(tape, init, hashes=hashes, mode=mode)
    for _ in range(nsteps):
        gpu.encode_steps(1, with_hashes=hashes)
    mem = gpu.read(gpu.buffers_end)
    return cpu, gpu, mem


def test_tiny_step_bit_exact_every_dispatch():
    run = timestep.Run(scenario.tiny(16, 12, 10))
    tape = run.tape(1)
    init = run.initial_buffers()
    cpu, gpu, mem = _compare(run, tape, init, nsteps=2)
    assert gpu.hash_count == cpu.hash_count
    h = gpu.read_hashes()
    bad = np.nonzero(h != cpu.hashes[:gpu.hash_count])[0]
    assert bad.size == 0, [gpu.op_name(0)] + list(bad[:5])
    assert np.array_equal(mem, cpu.M[:gpu.buffers_end])


def test_small_config_step_bit_exact():
    cfg = scenario.SMALL   # 64x64x40, dt 6 s, nsound 6
    run = timestep.Run(cfg)
    tape = run.tape(1)
    init = run.initial_buffers()
    cpu, gpu, mem = _compare(run, tape, init, nsteps=1, hashes=False)
    assert np.array_equal(mem, cpu.M[:gpu.buffers_end])


def test_nsound8_grid_not_multiple_of_block():
    run = timestep.Run(scenario.tiny(37, 29, 13, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0))
    tape = run.tape(1)
    init = run.initial_buffers()
    cpu, gpu, mem = _compare(run, tape, init, nsteps=1)
    assert np.array_equal(gpu.read_hashes(), cpu.hashes[:gpu.hash_count])
    assert np.array_equal(mem, cpu.M[:gpu.buffers_end])


def test_subnormal_inputs_flush_like_the_oracle():
    """Perturbations scaled to ~1e-36 drive WENO smoothness terms below FLT_MIN."""
    run = timestep.Run(scenario.tiny(16, 12, 10))
    tape = run.tape(1)
    init = run.initial_buffers()
    arena = np.frombuffer(init[run.rec.ids['arena']], dtype=np.float32).copy()
    g = run.grid
    for name in ('th', 'th_a'):
        o = run.fields[name] // 4
        arena[o:o + g.count] *= np.float32(1e-36)
    o = run.fields['w'] // 4
    arena[o:o + g.count] = np.float32(3e-39)          # subnormal input
    init[run.rec.ids['arena']] = arena.tobytes()
    cpu, gpu, mem = _compare(run, tape, init, nsteps=1)
    assert np.array_equal(gpu.read_hashes(), cpu.hashes[:gpu.hash_count])
    assert np.array_equal(mem, cpu.M[:gpu.buffers_end])


def test_use_step_rewrites_changed_parameters():
    run = timestep.Run(scenario.tiny(16, 12, 10))
    tape = run.tape(1)
    init = run.initial_buffers()
    gpu = helpers.gpu_replayer(tape, init, hashes=False)
    gpu.encode_steps(1)
    run.dt = timestep.f(5.0)                       # new dt: same structure, new bytes
    run.schedule = timestep.AcousticSchedule(6, run.dt)
    cmds = run.encode()
    gpu.use_step(cmds)
    gpu.encode_steps(1)
    mem = gpu.read(gpu.buffers_end)
    cpu = helpers.cpu_run(tape, init, nsteps=1, hashes=False)
    cpu.use_step(cmds)
    cpu.run(helpers.oracle().get)
    assert np.array_equal(mem, cpu.M[:gpu.buffers_end])


def test_unknown_kernel_is_an_error_at_plan_or_run():
    run = timestep.Run(scenario.tiny(8, 8, 6))
    tape = run.tape(1)
    tape['steps'][0] = [{'op': 'pipe', 'name': 'no_such_kernel'},
                        {'op': 'dispatch', 'kind': 'threads', 'grid': [1, 1, 1], 'tg': [1, 1, 1]}]
    from thunderengine_web_b200.replayer import Replayer
    r = Replayer(tape, helpers.kernels_meta())
    r.plan(False)
    with pytest.raises(RuntimeError, match='no kernel'):
        r.build()
    r2 = Replayer(tape, dict(helpers.kernels_meta(), no_such_kernel={'params': [], 'scratch': 0}),
                  defer_missing=True)
    r2.plan(False)
    r2.build()
    with pytest.raises(RuntimeError, match='no CUDA kernel'):
        r2.encode_steps(1, with_hashes=True)


# Recorded scenarios and whether the oracle reproduces the recording itself.  On the
# horizontally stretched grid the grid scale (dx dy dz)^(1/3) of turb_km_kh.wgsl takes many
# values, and at some of them the recording's pow builtin (whose precision WGSL leaves to
# the implementation) is not the correctly rounded power; from that dispatch on the
# recording is not reproducible bit for bit, so there the GPU is checked against the
# oracle dispatch by dispatch only.
GOLDEN_SCENARIOS = {'single_cell': True, 'squall_line': True, 'supercell_stretched': False}


@pytest.mark.parametrize('scen', list(GOLDEN_SCENARIOS))
def test_golden_in_scope_dispatches(scen):
    """A recorded step 1, dispatch by dispatch: every dispatch runs on the GPU from the
    CPU's memory, its region hashes equal to the oracle's (the reference's own kernel for
    the Morrison column, with the WGSL builtins in binary64); where the oracle reproduces
    the recording, region hashes and buffer FNVs are also compared with the recording
    (scratch tend/fpk hashes exempt, as the reference documents)."""
    ref = helpers.reference()
    if ref is None:
        pytest.skip('oracle/_ref not built')
    from oracle.player import CpuPlayer, fnv1a
    tape, init, want, step1 = helpers.load_golden_scenario(scen)
    km = helpers.kernels_meta()
    cpu = CpuPlayer(tape, km)
    cpu.plan(True)
    for i, b in init.items():
        cpu.upload(i, b)
    from thunderengine_web_b200 import replayer as rp
    import ctypes
    # which ops the GPU library implements
    lib = rp.load_library()
    n = lib.te_kernel_table_json(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib.te_kernel_table_json(buf, n + 1)
    import json
    ours = set(json.loads(buf.value.decode()))
    ref64 = helpers.reference64()

    def cpu_kernel(name):
        return ref64.get(name) if name == 'morr_column' else helpers.oracle().get(name)

    # CPU replay; before every in-scope dispatch, hand the GPU the regions written since
    ngpu = 0
    gpu_hashes = {}
    from thunderengine_web_b200.replayer import Replayer
    r = Replayer(tape, km)
    r.plan(True)
    r.build()
    assert r.mem_words == cpu.mem_words and r.hash_count == want.size
    dirty = [(0, cpu.buffers_end)]
    for oi, o in enumerate(cpu.ops):
        if o.kind == 'k' and o.name in ours:
            for off, ln in dirty:
                r.write_words(off, cpu.M[off:off + ln])
            dirty = []
            r.clear_hashes()
            r.run_ops(oi, oi, with_hashes=True)
            h = r.read_hashes()
            for slot, off, ln in o.hashes:
                gpu_hashes[slot] = int(h[slot])
            ngpu += 1
            # the CPU continues with the oracle so the two memories stay identical
            cpu.run(cpu_kernel, with_hashes=True, ops=[o])
            for slot, off, ln in o.hashes:
                assert gpu_hashes[slot] == int(cpu.hashes[slot]), (oi, o.name)
        else:
            cpu.run(ref.get, with_hashes=True, ops=[o])
            if o.kind == 'copy':
                dirty.append((o.dst, o.n))
            else:
                dirty.extend((off, ln) for _, off, ln in o.hashes if off is not None and ln)
    # every dispatch, the Morrison microphysics column (morr_column) included
    assert ngpu == sum(1 for o in cpu.ops if o.kind == 'k')
    if not GOLDEN_SCENARIOS[scen]:
        return
    fields = {v // 4 + cpu.base[2]: k for k, v in tape['fields'].items()}
    slot_field = {s: fields.get(off) for o in cpu.ops if o.kind == 'k' for s, off, _ in o.hashes}
    bad = [s for s in gpu_hashes if gpu_hashes[s] != int(want[s])]
    assert {slot_field[s] for s in bad} <= {'tend', 'fpk'}
    for b in tape['buffers']:
        assert fnv1a(cpu.buffer_words(b['id'])) == step1[b['id']], b['label']



def test_branches_the_recording_does_not_take():
    """Kernels of the recorded single_cell step, each at its first dispatch, with the
    parameter structs of the branches the recording does not take (helpers.UNTAKEN_BRANCHES),
    set through use_step (the reference's useStep rewrites changed setBytes payloads): the
    GPU's written regions equal the oracle's."""
    import base64
    from oracle.player import CpuPlayer
    from thunderengine_web_b200.replayer import Replayer
    if helpers.reference() is None:
        pytest.skip('oracle/_ref not built')
    tape, init, want, step1 = helpers.load_golden_scenario()
    km = helpers.kernels_meta()
    cpu = CpuPlayer(tape, km)
    cpu.plan(False)
    for i, b in init.items():
        cpu.upload(i, b)
    r = Replayer(tape, km)
    r.plan(False)
    r.build()
    cmds0 = tape['steps'][0]
    todo = dict(helpers.UNTAKEN_BRANCHES)
    checked = 0
    for oi, o in enumerate(cpu.ops):
        if o.kind == 'copy':
            cpu.M[o.dst:o.dst + o.n] = cpu.M[o.src:o.src + o.n]
            continue
        cases = todo.pop(o.name, [])
        gd = o.bind[0] if cases else 0
        for changes in cases:
            cmds = list(cmds0)
            E = cpu.M.copy()
            helpers.fill_for_branches(o.name, o.bind, E, int(E[gd + 3]) * int(E[gd + 4]))
            for n, words in changes.items():
                if isinstance(n, tuple):   # buffer words, handed over with the rest of memory
                    E[o.bind[n[1]] + n[2]:o.bind[n[1]] + n[2] + len(words)] = words
                    continue
                ci = max(c for c in range(o.index) if cmds0[c]['op'] == 'bytes' and cmds0[c]['index'] == n)
                raw = bytearray(base64.b64decode(cmds0[ci]['data']))
                raw[:4 * len(words)] = np.asarray(words, dtype=np.uint32).tobytes()
                cmds[ci] = dict(cmds0[ci], data=base64.b64encode(bytes(raw)).decode())
                E[o.bind[n]:o.bind[n] + len(words)] = words
            r.use_step(cmds)
            r.write_words(0, E[:cpu.buffers_end])
            r.run_ops(oi, oi)
            helpers.oracle().get(o.name)(E.ctypes.data_as(ctypes.c_void_p), o.arg.ctypes.data_as(ctypes.c_void_p))
            for prm in km[o.name]['params']:
                if prm['write'] and prm['index'] in o.bind:
                    off = o.bind[prm['index']]
                    ln = cpu.region_len(off)
                    assert np.array_equal(r.read(ln, off), E[off:off + ln]), (o.name, changes, prm['name'])
            checked += 1
        helpers.mixed(o.name)(cpu.M.ctypes.data_as(ctypes.c_void_p), o.arg.ctypes.data_as(ctypes.c_void_p))
        if not todo:
            break
    assert checked == sum(len(v) for v in helpers.UNTAKEN_BRANCHES.values())


STEP_SCRATCH = set(helpers.SCRATCH)


def _fused_vs_oracle(cfg, nsteps):
    from thunderengine_web_b200.replayer import TE_MODE_FUSED
    run = timestep.Run(cfg)
    tape = run.tape(1)
    init = run.initial_buffers()
    cpu = helpers.cpu_run(tape, init, nsteps=nsteps, hashes=False)
    gpu = helpers.gpu_replayer(tape, init, hashes=False, mode=TE_MODE_FUSED)
    segs = gpu.fused_segments()
    assert sum(1 for s in segs if s[0] == 1) == timestep.AcousticSchedule(cfg.nsound, cfg.dt).total
    gpu.encode_steps(nsteps)
    mem = gpu.read(gpu.buffers_end)
    base = gpu.base[run.rec.ids['arena']]
    bad = []
    for name in run.fields:
        a = helpers.field_view(mem, run, base, name).view(np.uint32)
        b = helpers.field_view(cpu.M, run, base, name).view(np.uint32)
        if not np.array_equal(a, b):
            bad.append(name)
    assert not [b for b in bad if b not in STEP_SCRATCH], bad
    # the non-arena buffers (profiles, metric) are untouched by the step
    assert np.array_equal(mem[:base], cpu.M[:base])


def test_fused_mode_matches_oracle_tiny():
    _fused_vs_oracle(scenario.tiny(16, 12, 10), nsteps=3)


def test_fused_mode_matches_oracle_small_config():
    _fused_vs_oracle(scenario.SMALL, nsteps=1)


def test_fused_mode_odd_sizes_nsound8():
    _fused_vs_oracle(scenario.tiny(37, 29, 13, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0), nsteps=2)


@pytest.mark.parametrize('dims', [(37, 29, 13), (64, 40, 24)])
def test_aligned_rows_exact_and_fused_vs_oracle(dims):
    """Rows padded to a multiple of 32 floats (the reference's alignRows layout: every row
    starts on a 128-byte boundary): the per-dispatch step equals the oracle word for word,
    the fused step on every non-scratch field, and the padding columns stay untouched."""
    nx, ny, nz = dims
    cfg = scenario.tiny(nx, ny, nz, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0, align_rows=True)
    run = timestep.Run(cfg)
    assert run.grid.strideJ % 32 == 0 and run.grid.strideJ > nx + 7
    tape = run.tape(1)
    init = run.initial_buffers()
    cpu, gpu, mem = _compare(run, tape, init, nsteps=2, hashes=False)
    assert np.array_equal(mem, cpu.M[:gpu.buffers_end])
    gpu.close()
    _fused_vs_oracle(cfg, nsteps=2)


def test_aliased_bindings_keep_program_order():
    """A tape may bind one field to several parameters of a dispatch.  Here
    stage_state_reset reads v's source from the u it has just written (va := u), so a
    thread that loaded every input before storing would read the old u; the player must
    run the dispatch with the ordering the reference kernel has (u first, then v = u)."""
    run = timestep.Run(scenario.tiny(16, 12, 10))
    tape = run.tape(1)
    arena = run.rec.ids['arena']
    cmds = tape['steps'][0]
    pipe, changed = None, 0
    for c in cmds:
        if c['op'] == 'pipe':
            pipe = c['name']
        elif c['op'] == 'buf' and pipe == 'stage_state_reset' and c['index'] == 2 and c['buf'] == arena:
            c['offset'] = run.fields['u']
            changed += 1
    assert changed >= 1
    init = run.initial_buffers()
    cpu, gpu, mem = _compare(run, tape, init, nsteps=1)
    assert np.array_equal(gpu.read_hashes(), cpu.hashes[:gpu.hash_count])
    assert np.array_equal(mem, cpu.M[:gpu.buffers_end])


def test_fused_plan_covers_the_step():
    """The fused planner recognises every acoustic substep, the advection of every variable
    (the stage-3 scalar WENO one storing the fluxes pdef_dum and pdef_apply read) and the
    halo-fill runs; a structural change that made it fall back to per-dispatch kernels
    shows here."""
    from thunderengine_web_b200.replayer import TE_MODE_FUSED
    run = timestep.Run(scenario.tiny(37, 29, 13, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0))
    tape = run.tape(1)
    gpu = helpers.gpu_replayer(tape, run.initial_buffers(), hashes=False, mode=TE_MODE_FUSED)
    segs = gpu.fused_segments()
    kinds = [s[0] for s in segs]
    assert kinds.count(1) == sum(n for n, _ in run.schedule.loops)   # every acoustic substep (15)
    assert kinds.count(3) == 15
    assert kinds.count(2) >= 10
    exact_ops = sum(s[2] - s[1] + 1 for s in segs if s[0] == 0)
    assert exact_ops < gpu.num_ops // 3


# ---------------------------------------------------------------- the benchmarked configuration

def _nonscratch_mismatches(run, mem_a, mem_b, base):
    bad = []
    for name in run.fields:
        if name in STEP_SCRATCH:
            continue
        a = helpers.field_view(mem_a, run, base, name).view(np.uint32)
        b = helpers.field_view(mem_b, run, base, name).view(np.uint32)
        if not np.array_equal(a, b):
            bad.append((name, int(np.count_nonzero(a != b))))
    return bad


def test_headline_config_one_step_exact_and_fused_vs_oracle():
    """256x256x80, dt 3 s, nsound 8 (15 acoustic substeps, 5 passes of the fused column
    kernel, every epilogue slot up to level 80): one large step in exact mode equals the
    oracle in every memory word, and in fused mode in every non-scratch field."""
    from thunderengine_web_b200.replayer import TE_MODE_FUSED
    run = timestep.Run(scenario.AT_SCALE)
    tape = run.tape(1)
    init = run.initial_buffers()
    cpu = helpers.cpu_run(tape, init, nsteps=1, hashes=False)
    gpu = helpers.gpu_replayer(tape, init, hashes=False)
    gpu.encode_steps(1)
    mem = gpu.read(gpu.buffers_end)
    base = gpu.base[run.rec.ids['arena']]
    diff = np.nonzero(mem != cpu.M[:gpu.buffers_end])[0]
    assert diff.size == 0, 'exact mode: %d words differ, first at %d' % (diff.size, diff[0])
    gpu.close()
    del mem
    fz = helpers.gpu_replayer(tape, init, hashes=False, mode=TE_MODE_FUSED)
    fz.encode_steps(1)
    mem = fz.read(fz.buffers_end)
    assert not _nonscratch_mismatches(run, mem, cpu.M, base)
    assert np.array_equal(mem[:base], cpu.M[:base])
    fz.close()


@pytest.mark.parametrize('nz', [80, 100])
def test_fused_tall_columns_vs_oracle(nz):
    """Narrow grids with the benchmark's depth and deeper: the fused column kernel's
    epilogue slots 3-5 (levels 51..101) and 5-7 passes of 16 levels, three steps."""
    _fused_vs_oracle(scenario.tiny(24, 20, nz, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0), nsteps=3)


def test_headline_config_fused_equals_exact_over_20_steps():
    """20 large steps at 256x256x80 in fused and in exact mode on the GPU: every
    non-scratch field bit-identical."""
    from thunderengine_web_b200.replayer import TE_MODE_FUSED
    run = timestep.Run(scenario.AT_SCALE)
    tape = run.tape(1)
    init = run.initial_buffers()
    ex = helpers.gpu_replayer(tape, init, hashes=False)
    ex.encode_steps(20)
    mem_ex = ex.read(ex.buffers_end)
    base = ex.base[run.rec.ids['arena']]
    ex.close()
    fz = helpers.gpu_replayer(tape, init, hashes=False, mode=TE_MODE_FUSED)
    fz.encode_steps(20)
    mem_fz = fz.read(fz.buffers_end)
    fz.close()
    assert not _nonscratch_mismatches(run, mem_fz, mem_ex, base)
    # the state moved: the comparison is not of two untouched arenas
    th0 = helpers.field_view(np.frombuffer(init[run.rec.ids['arena']], dtype=np.uint32), run, 0, 'w')
    assert not np.array_equal(helpers.field_view(mem_ex, run, base, 'w').view(np.uint32), th0)


def test_large_domain_step_fused_equals_exact():
    """1024x1024x100 (dx 250 m, dt 1.5 s, nsound 8, three-bubble line): ~21 GB of arena,
    word offsets past 2^32.  One step in fused and in exact mode: every non-scratch field
    bit-identical, finite, and the state moved."""
    import psutil
    from thunderengine_web_b200.replayer import Replayer, TE_MODE_FUSED
    if psutil.virtual_memory().available < 64 << 30:
        pytest.skip('needs 64 GB of host memory for the initial arena')
    run = timestep.Run(scenario.LARGE)
    tape = run.tape(1)
    arena = run.initial_arena()
    aid = run.rec.ids['arena']
    reps = []
    for mode in (0, TE_MODE_FUSED):
        r = Replayer(tape, None)
        r.plan(False)
        r.build()
        assert r.mem_words > 1 << 32
        for b in tape['buffers']:
            if b['id'] != aid:
                r.upload(b['id'], run.buffer_bytes(b['label']))
        r.write_words(r.base[aid], arena)
        r.set_mode(mode)
        r.encode_steps(1)
        r.sync()
        reps.append(r)
    g = run.grid
    base = reps[0].base[aid]
    for name in run.fields:
        if name in STEP_SCRATCH:
            continue
        off = base + run.fields[name] // 4
        a = reps[0].read(g.count, off)
        b = reps[1].read(g.count, off)
        assert np.array_equal(a, b), name
        assert np.isfinite(a.view(np.float32)).all(), name
    w = reps[0].read(g.count, base + run.fields['w'] // 4).view(np.float32)
    assert np.abs(w).max() > 0
    for r in reps:
        r.close()


def test_fast_power_route_equals_two_float_power_everywhere():
    """update_rho_prs raises the Exner function to cp/rd by a binary64 route that falls
    back to the reference's two-float power near rounding boundaries.  On every
    non-negative binary32 pattern (finite, infinite and NaN included) both routes give the
    same bits."""
    from thunderengine_web_b200 import replayer
    lib = replayer.load_library()
    cpdrd = float(np.float32(1005.7) / np.float32(287.04))
    bad = ctypes.c_uint64(0)
    first = ctypes.c_uint32(0)
    assert lib.te_check_pow(cpdrd, 0, 0x80000000, ctypes.byref(bad), ctypes.byref(first)) == 0
    assert bad.value == 0, 'first differing pattern 0x%08x' % first.value


@pytest.mark.parametrize('scen', [k for k, v in GOLDEN_SCENARIOS.items() if v])
def test_recorded_step_plays_whole_on_the_gpu(scen):
    """The reference's recorded step 1 (full physics: turbulence, Morrison microphysics,
    open boundaries, mass conservation) played as one te_run on the GPU, every dispatch on
    the device: every buffer's FNV-1a equals the recording's, and every region hash but the
    scratch tendencies the reference itself exempts (tend, fpk); then the tape's display
    diagnostic (radar reflectivity) equals the reference's kernels on the CPU."""
    from oracle.player import CpuPlayer, fnv1a
    tape, init, want, step1 = helpers.load_golden_scenario(scen)
    km = helpers.kernels_meta()
    from thunderengine_web_b200.replayer import Replayer
    gpu = Replayer(tape, km)
    gpu.plan(True)
    gpu.build()
    for i, b in init.items():
        gpu.upload(i, b)
    gpu.encode_steps(1, with_hashes=True)
    got = gpu.read_hashes()
    mem = gpu.read(gpu.buffers_end)
    cpu = CpuPlayer(tape, km)
    cpu.plan(True)
    fields = {v // 4 + cpu.base[2]: k for k, v in tape['fields'].items()}
    slot_field = {s: fields.get(off) for o in cpu.ops if o.kind == 'k' for s, off, _ in o.hashes}
    bad = np.nonzero(got[:want.size] != want)[0]
    assert {slot_field[int(s)] for s in bad} <= {'tend', 'fpk'}
    for b in tape['buffers']:
        off = gpu.base[b['id']]
        assert fnv1a(mem[off:off + b['length'] // 4]) == step1[b['id']], b['label']
    # the display diagnostic after the step (encodeDiag: morr_prep, morr_refl10cm) equals
    # the reference's kernels run on the CPU from the same memory
    gpu.encode_diag()
    dmem = gpu.read(gpu.buffers_end)
    gpu.close()
    cpu.M[:gpu.buffers_end] = mem
    ref64 = helpers.reference64()
    if ref64 is None:
        pytest.skip('oracle/_ref not built (needs the reference checkout)')
    cpu.run(lambda n: ref64.get(n) if n == 'morr_refl10cm' else helpers.oracle().get(n), ops=cpu.diag_ops)
    assert np.count_nonzero(dmem != mem) > 0
    assert np.array_equal(dmem, cpu.M[:gpu.buffers_end])


def test_recorded_step_in_fused_mode_equals_exact():
    """The single_cell recording (open lateral boundaries, full physics) in fused mode: the
    planner fuses the advection of every variable there (with adv_assemble's open-edge
    branches) and runs the rest per dispatch; after one step every field but the step
    scratch equals the exact-mode step, word for word."""
    from thunderengine_web_b200.replayer import Replayer, TE_MODE_FUSED
    tape, init, _, _ = helpers.load_golden_scenario('single_cell')
    km = helpers.kernels_meta()
    mems = []
    for mode in (0, TE_MODE_FUSED):
        r = Replayer(tape, km)
        r.plan(False)
        r.build()
        for i, b in init.items():
            r.upload(i, b)
        r.set_mode(mode)
        if mode:
            segs = r.fused_segments()
            assert sum(1 for s in segs if s[0] == 3) >= 10   # the advection phases are fused
        r.encode_steps(1)
        mems.append(r.read(r.buffers_end))
        base = r.base[2]
        r.close()
    for name, off in tape['fields'].items():
        if name in STEP_SCRATCH:
            continue
        n = (tape['nx'] + 7) * (tape['ny'] + 7) * (tape['nz'] + 1)
        a = mems[0][base + off // 4:base + off // 4 + n]
        b = mems[1][base + off // 4:base + off // 4 + n]
        assert np.array_equal(a, b), name
