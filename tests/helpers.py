"""Shared test helpers: oracle / reference kernel sets, CPU replays, GPU replays."""
import ctypes
import json
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, 'tests', 'golden')
ORACLE_SO = os.path.join(ROOT, 'oracle', 'liboracle.so')
REF_SO = os.path.join(ROOT, 'oracle', '_ref', 'libteref.so')
REF64_SO = os.path.join(ROOT, 'oracle', '_ref', 'libteref64.so')

# Scratch fields of a step (timestep.js:334-337 Fields.scratchFields): their contents
# between dispatches are not part of the step's result.
SCRATCH = ['rru', 'rrv', 'rrw', 'fx', 'fy', 'fz', 'tend', 'divx', 'qk', 'pk1', 'pk2', 'mm', 'fpk', 'cA', 'cB',
           'sadv']

_ORACLE = None
_REF = None
_REF64 = None


def oracle():
    """The hand-written C oracle (built by oracle/Makefile), FTZ/DAZ enabled."""
    global _ORACLE
    if _ORACLE is None:
        from oracle.player import KernelSet
        if not os.path.exists(ORACLE_SO):
            subprocess.check_call(['make', '-C', os.path.join(ROOT, 'oracle')])
        _ORACLE = KernelSet(ORACLE_SO, 'teor_')
        _ORACLE.lib.te_set_ftz(1)
    return _ORACLE


def reference():
    """The reference's own kernels translated to C++ (oracle/_ref), or None."""
    global _REF
    if _REF is None:
        if not os.path.exists(REF_SO):
            return None
        from oracle.player import KernelSet
        _REF = KernelSet(REF_SO, 'teref_')
        oracle()   # FTZ/DAZ on the shared OpenMP team
    return _REF


def kernels_meta():
    with open(os.path.join(GOLDEN, 'kernels.json')) as fh:
        return json.load(fh)


def reference64():
    """The reference's kernels that call WGSL exp/log/pow/log2/atan2, with those evaluated in binary64
    like the CUDA kernels (oracle/_ref/libteref64.so), or None."""
    global _REF64
    if _REF64 is None:
        if not os.path.exists(REF64_SO):
            return None
        oracle()
        from oracle.player import KernelSet
        _REF64 = KernelSet(REF64_SO, 'teref_')
    return _REF64


def mixed(name):
    """Oracle kernel where one exists, else the translated reference kernel."""
    o = oracle()
    if o.has(name):
        return o.get(name)
    r = reference()
    if r is None:
        raise RuntimeError('kernel %s needs oracle/_ref' % name)
    return r.get(name)


def cpu_run(tape, init, nsteps=1, hashes=True, kernels=None):
    """Replay a tape on the CPU oracle; returns the player (memory in .M)."""
    from oracle.player import CpuPlayer
    p = CpuPlayer(tape, kernels_meta())
    p.plan(hashes)
    for i, b in init.items():
        p.upload(i, b)
    kern = kernels or oracle().get
    for _ in range(nsteps):
        p.run(kern, with_hashes=hashes)
    return p


def gpu_replayer(tape, init, hashes=True, kernels_json=True, mode=0):
    from thunderengine_web_b200.replayer import Replayer
    r = Replayer(tape, kernels_meta() if kernels_json else None)
    r.plan(hashes)
    r.build()
    for i, b in init.items():
        r.upload(i, b)
    if mode:
        r.set_mode(mode)
    return r


def field_view(mem, run_or_tape, base, name):
    """(k, j, i) float32 view of an arena field from a memory word array."""
    if hasattr(run_or_tape, 'fields'):
        fields, g = run_or_tape.fields, run_or_tape.grid
        sJ, sK, nz, count = g.strideJ, g.strideK, g.nz, g.count
    else:
        t = run_or_tape
        fields = t['fields']
        sJ, sK, nz = t['nx'] + 7, t['ny'] + 7, t['nz']
        count = sJ * sK * (nz + 1)
    off = base + fields[name] // 4
    return mem[off:off + count].view(np.float32).reshape(nz + 1, sK, sJ)


def load_golden_scenario(name='single_cell'):
    import gzip
    d = os.path.join(GOLDEN, name)
    with open(os.path.join(d, 'tape.json')) as fh:
        tape = json.load(fh)
    init = {}
    for b in tape['buffers']:
        p = os.path.join(d, 'state', '%d.bin.gz' % b['id'])
        if os.path.exists(p):
            with gzip.open(p, 'rb') as fh:
                init[b['id']] = fh.read()
    hashes = np.fromfile(os.path.join(d, 'hashes.ref.bin'), dtype=np.uint32)
    with open(os.path.join(d, 'step1.json')) as fh:
        step1 = {int(k): v for k, v in json.load(fh).items()}
    return tape, init, hashes, step1


def f32_word(x):
    return int(np.float32(x).view(np.uint32))


# Branches the recorded single_cell step does not take: per kernel, cases of
# {binding: words written over the start of that binding's parameter struct}; a key
# ('at', binding, offset) writes buffer words at that offset of a pointer binding instead.
_W = f32_word
UNTAKEN_BRANCHES = {
    'turb_scalar_vert_implicit': [
        {15: [uf], 16: [ez], 18: [bt], 17: [_W(0.37), _W(301.5), _W(290.25), _W(ww)]}
        for uf, ez, bt, ww in [(1, 0, 1, 0.0), (0, 0, 2, 0.0), (1, 1, 1, 0.0), (0, 1, 2, 0.0),
                               (0, 1, 1, 1.0), (0, 1, 1, 2.0), (0, 0, 2, 1.0), (0, 0, 1, 2.0)]],
    'rayleigh_damping': [{16: [1], 17: [0]}, {16: [0], 17: [1]}, {16: [1], 17: [1]}],
    'mp_pdefq': [{3: [_W(1e-5)]}, {3: [_W(-1.0)]}],
    'turb_km_kh': [{11: [_W(5.0)]}, {12: [_W(0.001)]}],
    'turb_nm': [{16: [0]}, {18: [1]}, {16: [0], 18: [1]}],
    'turb_sfcstress': [{5: [m], 10: [top], 8: [_W(1.5), _W(-0.5)]}
                       for m, top in [(0, 1), (1, 0), (2, 0), (3, 1), (4, 0), (4, 1)]],
    'turb_dissipative_heating': [{11: [moist, 1, _W(0.1), _W(500.0), zf]}
                                 for moist, zf in [(1, 0), (1, 1), (0, 0), (0, 1)]] + [{11: [0]}],
    'turb_u_tendency': [{17: [1]}, {16: [0, 0]}, {16: [0, 1], 17: [1]}],
    'turb_v_tendency': [{17: [1]}, {16: [0, 0]}, {16: [1, 0], 17: [1]}],
    'turb_w_tendency': [{15: [1]}, {14: [0, 0]}, {14: [0, 1], 15: [1]}],
    'tke_transport': [{15: [1]}, {14: [0, 0]}, {14: [1, 0], 15: [1]}],
    'mass_reference_init': [{('at', 2, 2): [_W(1.0)]}],
    # the recorded total mass is 2.75e5: these references make r = 0.45 and -0.27
    'mass_correction_apply': [{1: [0]}, {('at', 4, 0): [_W(4.0e5)]}, {('at', 4, 0): [_W(2.0e5)], 1: [0]}],
}
# (binding, planes of one level each) filled with seeded positive values before those
# cases, so that the branches read surface data that is not all zero
BRANCH_FILLS = {'turb_scalar_vert_implicit': (14, 1), 'turb_sfcstress': (1, 17),
                'turb_dissipative_heating': (12, 17)}


def fill_for_branches(name, bind, mem, plane):
    """Seeded surface data for the UNTAKEN_BRANCHES cases of `name` (in place)."""
    if name not in BRANCH_FILLS:
        return
    idx, planes = BRANCH_FILLS[name]
    vals = np.random.default_rng(7).uniform(0.05, 2.0, planes * plane).astype(np.float32)
    mem[bind[idx]:bind[idx] + planes * plane] = vals.view(np.uint32)
