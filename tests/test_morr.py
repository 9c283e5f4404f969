"""Morrison microphysics column (morr_column) and its radar reflectivity diagnostic
(morr_refl10cm): the library's restatements (thunderengine-web_b200/csrc/te_morr.cuh,
te_refl.cuh) against the reference's own kernels.

The checker is the reference's WGSL translated to C++ (oracle/_ref/libteref64.so, the
variant that evaluates the WGSL exp/log/pow/log2/atan2 builtins in binary64 like the CUDA
kernels).
The CPU test compiles te_morr.cuh for the host (tests/native/morr_host.cpp) and compares
every memory word after one dispatch; the GPU test runs the CUDA kernel through the C-ABI.
The states: the single_cell recording's memory at its morr_column dispatch (which at step 1
holds no condensate: the recorded dispatch itself is checked in the golden GPU test) with
seeded random hydrometeor mass and number mixing ratios and scaled vapour (both
temperature branches, all five sedimenting species, the saturation adjustment), and a
strongly supersaturated variant with the radiation radii (dorad) and the drizzle fall
speed switched on; together they execute 97 % of the lines of te_morr.cuh (gcov of the
host build), the rest being branches no caller reaches (the gamma function below 1,
Hallett-Mossop outside its temperature window).  The reflectivity case is the single_cell
recording's diagnostic dispatch over seeded random rain, snow and graupel."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

from tests import helpers

ROOT = helpers.ROOT
HOST_SRC = os.path.join(ROOT, 'tests', 'native', 'morr_host.cpp')
_HOST = None


def host_kernels():
    """The library's morr column built for the host, as an oracle-style KernelSet."""
    global _HOST
    if _HOST is None:
        from oracle.player import KernelSet
        helpers.oracle()  # liboracle.so built and FTZ/DAZ on
        out = os.path.join(tempfile.mkdtemp(prefix='te_morr_'), 'libmorrhost.so')
        odir = os.path.join(ROOT, 'oracle')
        subprocess.check_call(['g++', '-std=c++17', '-O2', '-fopenmp', '-fPIC', '-shared', '-ffp-contract=off', '-fno-fast-math',
                               '-fwrapv', '-march=x86-64-v2', '-mfma', '-o', out, HOST_SRC, '-L' + odir, '-loracle',
                               '-Wl,-rpath,' + odir])
        _HOST = KernelSet(out, 'temh_')
    return _HOST


def morr_case(variant, seed=1):
    """(player, op, memory) at the single_cell morr_column dispatch: the recorded initial
    memory with morr_prep applied (T = (th0 + th)(pi0 + pi')), then `variant`."""
    from oracle.player import CpuPlayer
    tape, init, _, _ = helpers.load_golden_scenario('single_cell')
    cpu = CpuPlayer(tape, helpers.kernels_meta())
    cpu.plan(False)
    for i, b in init.items():
        cpu.upload(i, b)
    ks = [k for k, o in enumerate(cpu.ops) if o.kind == 'k' and o.name == 'morr_column']
    op = cpu.ops[ks[0]]
    prep = cpu.ops[ks[0] - 1]
    assert prep.name == 'morr_prep'
    cpu.run(helpers.oracle().get, ops=[prep])
    M = cpu.M
    if variant != 'recorded':
        rng = np.random.default_rng(seed)
        nx, ny, nz = tape['nx'], tape['ny'], tape['nz']
        n = (nx + 7) * (ny + 7) * nz
        for b, lo, hi in [(3, 1e-7, 3e-3), (4, 1e-8, 5e-3), (5, 1e-8, 2e-3), (6, 1e-8, 3e-3), (7, 1e-8, 4e-3)]:
            v = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.float32)
            v[rng.random(n) < 0.3] = 0
            M[op.bind[b]:op.bind[b] + n] = v.view(np.uint32)
        for b, lo, hi in [(8, 1e2, 1e6), (9, 1e2, 1e6), (10, 1e2, 1e6), (11, 1e1, 1e5)]:
            v = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.float32)
            M[op.bind[b]:op.bind[b] + n] = v.view(np.uint32)
        lo, hi = (0.8, 1.3) if variant == 'random' else (1.0, 2.0)
        off = op.bind[2]
        qv = M[off:off + n].view(np.float32) * rng.uniform(lo, hi, n).astype(np.float32)
        M[off:off + n] = qv.view(np.uint32)
        if variant == 'supersaturated':
            M[op.bind[19]] = 1                                      # dorad
            M[op.bind[0] + 68] = np.float32(1.0).view(np.uint32)    # drizzleVt
    return cpu, op, M.copy()


def reference_after(cpu, op, M):
    ref64 = helpers.reference64()
    cpu.M = M.copy()
    cpu.run(ref64.get, ops=[op])
    return cpu.M


@pytest.mark.parametrize('variant,seed', [('random', 1), ('supersaturated', 3)])
def test_host_build_of_the_library_column_equals_reference(variant, seed):
    if helpers.reference64() is None:
        pytest.skip('oracle/_ref not built (needs the reference checkout)')
    cpu, op, M0 = morr_case(variant, seed)
    want = reference_after(cpu, op, M0)
    cpu.M = M0.copy()
    cpu.run(host_kernels().get, ops=[op])
    end = cpu.buffers_end
    changed = int(np.count_nonzero(want[:end] != M0[:end]))
    assert changed > 1_000_000  # the column did work
    bad = np.nonzero(cpu.M[:end] != want[:end])[0]
    assert bad.size == 0, 'first differing word %d of %d changed' % (bad[0], changed)


@pytest.mark.gpu
@pytest.mark.parametrize('variant,seed', [('random', 1), ('supersaturated', 3)])
def test_gpu_column_equals_reference(variant, seed):
    if helpers.reference64() is None:
        pytest.skip('oracle/_ref not built (needs the reference checkout)')
    cpu, op, M0 = morr_case(variant, seed)
    want = reference_after(cpu, op, M0)
    tape, _, _, _ = helpers.load_golden_scenario('single_cell')
    from thunderengine_web_b200.replayer import Replayer
    r = Replayer(tape, helpers.kernels_meta())
    r.plan(False)
    r.build()
    assert r.mem_words == cpu.mem_words
    r.write_words(0, M0[:r.buffers_end])
    for w in (op.bind[19], op.bind[0] + 68):   # dorad, drizzleVt (parameter words)
        r.write_words(w, M0[w:w + 1])
    oi = [k for k, o in enumerate(cpu.ops) if o is op][0]
    r.run_ops(oi, oi)
    got = r.read(r.buffers_end)
    r.close()
    bad = np.nonzero(got != want[:r.buffers_end])[0]
    assert bad.size == 0, 'first differing word %d' % bad[0]


def refl_case(seed=1):
    """(player, op, memory) at the single_cell recording's morr_refl10cm dispatch (its
    display diagnostic): the recorded memory with the diagnostic's morr_prep applied (T),
    then seeded random rain, snow and graupel mass and number mixing ratios (30 % of the
    masses zero).  The temperature profile puts the 0 C level inside the column, so most
    columns find a melting layer and integrate the melting snow and graupel over the bins."""
    from oracle.player import CpuPlayer
    tape, init, _, _ = helpers.load_golden_scenario('single_cell')
    cpu = CpuPlayer(tape, helpers.kernels_meta())
    cpu.plan(False)
    for i, b in init.items():
        cpu.upload(i, b)
    ks = [k for k, o in enumerate(cpu.diag_ops) if o.kind == 'k' and o.name == 'morr_refl10cm']
    op = cpu.diag_ops[ks[0]]
    prep = cpu.diag_ops[ks[0] - 1]
    assert prep.name == 'morr_prep'
    cpu.run(helpers.oracle().get, ops=[prep])
    M = cpu.M
    rng = np.random.default_rng(seed)
    nx, ny, nz = tape['nx'], tape['ny'], tape['nz']
    n = (nx + 7) * (ny + 7) * nz
    for b, lo, hi in [(6, 1e-7, 3e-3), (7, 1e-8, 5e-3), (8, 1e-8, 4e-3)]:
        v = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.float32)
        v[rng.random(n) < 0.3] = 0
        M[op.bind[b]:op.bind[b] + n] = v.view(np.uint32)
    for b, lo, hi in [(9, 1e2, 1e6), (10, 1e2, 1e6), (11, 1e1, 1e5)]:
        v = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.float32)
        M[op.bind[b]:op.bind[b] + n] = v.view(np.uint32)
    return cpu, tape, op, M.copy()


def test_host_build_of_the_library_reflectivity_equals_reference():
    if helpers.reference64() is None:
        pytest.skip('oracle/_ref not built (needs the reference checkout)')
    cpu, tape, op, M0 = refl_case()
    want = reference_after(cpu, op, M0)
    cpu.M = M0.copy()
    cpu.run(host_kernels().get, ops=[op])
    end = cpu.buffers_end
    nx, ny, nz = tape['nx'], tape['ny'], tape['nz']
    changed = int(np.count_nonzero(want[:end] != M0[:end]))
    assert changed == nx * ny * nz  # every dbz word of the interior
    dbz = want[op.bind[13]:op.bind[13] + (nx + 7) * (ny + 7) * nz].view(np.float32)
    dbz = dbz.reshape(nz, ny + 7, nx + 7)[:, 3:3 + ny, 3:3 + nx]
    assert np.isfinite(dbz).all() and dbz.max() > 40.0
    bad = np.nonzero(cpu.M[:end] != want[:end])[0]
    assert bad.size == 0, 'first differing word %d of %d changed' % (bad[0], changed)


@pytest.mark.gpu
def test_gpu_reflectivity_equals_reference():
    if helpers.reference64() is None:
        pytest.skip('oracle/_ref not built (needs the reference checkout)')
    cpu, tape, op, M0 = refl_case()
    want = reference_after(cpu, op, M0)
    from thunderengine_web_b200.replayer import Replayer
    r = Replayer(tape, helpers.kernels_meta())
    r.plan(False)
    r.build()
    assert r.mem_words == cpu.mem_words
    r.write_words(0, M0[:r.buffers_end])
    r.encode_diag()   # morr_prep (T from th, pi') then the reflectivity columns
    got = r.read(r.buffers_end)
    r.close()
    assert np.count_nonzero(got != M0[:r.buffers_end]) > 0
    bad = np.nonzero(got != want[:r.buffers_end])[0]
    assert bad.size == 0, 'first differing word %d' % bad[0]
