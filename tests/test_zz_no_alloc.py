"""te_w_solve_static_scratch: the column solve for callers that cannot allocate.

Some callers of this library cannot allocate device memory at the point where they run
the solve: their device memory belongs to another allocator, or the host application
forbids allocation once it is running.  te_w_solve_static_scratch takes only the
caller's input and output fields and keeps the Thomas coefficients in a fixed array
inside the library.  These tests check it against the tape kernel acoustic_w_solve run
by the player (the existing entry point), on two calls in a row that share the array.

This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from tests import helpers

IN_FIELDS = ('pk1', 'pk2', 'qk', 'mm', 'fpk', 'wten', 'pp3d')


def _lib():
    from thunderengine_web_b200 import replayer
    return replayer.load_library()


def test_oversize_grid_is_rejected_before_any_device_work():
    from thunderengine_web_b200.replayer import TeWSolveFields
    lib = _lib()
    f = TeWSolveFields(*([1] * 8))          # never dereferenced: the size check comes first
    err = ctypes.create_string_buffer(256)
    rc = lib.te_w_solve_static_scratch(ctypes.byref(f), 1024, 1024, 100, 1.0, 0.6, 0.4, None, err, 256)
    assert rc == -5                          # TE_ERANGE
    assert b'scratch' in err.value and b'8388608' in err.value
    rc = lib.te_w_solve_static_scratch(ctypes.byref(f), 16, 16, 2, 1.0, 0.6, 0.4, None, err, 256)
    assert rc == -1                          # TE_EINVAL: nz < 3
    rc = lib.te_w_solve_static_scratch(ctypes.byref(f), 1, 300000, 3, 1.0, 0.6, 0.4, None, err, 256)
    assert rc == -5 and b'262140' in err.value   # more rows than one launch covers


# 37x29x13: odd sizes; 33x5x3: the shallowest column (no middle forward level, the top
# level reads the coefficients of level 1) on a row count that is not a multiple of the
# launch's 4 rows per block
@pytest.mark.gpu
@pytest.mark.parametrize('nx,ny,nz', [(37, 29, 13), (33, 5, 3)])
def test_static_scratch_solve_matches_the_tape_kernel_twice(nx, ny, nz):
    import torch
    from thunderengine_web_b200 import scenario, timestep
    from thunderengine_web_b200.replayer import TeWSolveFields
    run = timestep.Run(scenario.tiny(nx, ny, nz, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0))
    tape = run.tape(1)
    r = helpers.gpu_replayer(tape, run.initial_buffers(), hashes=False)
    solves = [q for q in range(r.num_ops) if r.op_name(q) == 'acoustic_w_solve'][:2]
    assert len(solves) == 2
    g = run.grid
    base = r.base[run.rec.ids['arena']]
    off = {n: base + run.fields[n] // 4 for n in run.fields}
    # both solves are substeps of the first RK stage: same acoustic parameters
    dts = float(np.float32(run.schedule.loops[0][1]))
    alph, beta = run.acoustic['alph'], run.acoustic['beta']

    # the existing entry point: the player runs the tape kernel; keep the memory before
    # each solve and w after it
    before, want, prev = [], [], 0
    for q in solves:
        if q > prev:
            r.run_ops(prev, q - 1)
        before.append(r.read(r.buffers_end))
        r.run_ops(q, q)
        want.append(r.read(g.count, off['w']))
        prev = q + 1

    lib = _lib()
    ptr = {n: r.device_ptr(off[n]) for n in IN_FIELDS + ('w',)}
    f = TeWSolveFields(*[ptr[n] for n in IN_FIELDS + ('w',)])
    err = ctypes.create_string_buffer(256)
    for call in range(2):
        r.write_words(0, before[call])       # the inputs of this solve, w before it
        r.sync()
        rc = lib.te_w_solve_static_scratch(ctypes.byref(f), g.nx, g.ny, g.nz, dts, alph, beta, None, err, 256)
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()
        got = r.read(g.count, off['w'])
        # bit-exact, as every parity test of this library
        bad = np.nonzero(got != want[call])[0]
        assert bad.size == 0, 'call %d: %d words of w differ (first at %d)' % (call, bad.size, bad[0])
        # nothing else in the player's memory changed, cA and cB included
        mem = r.read(r.buffers_end)
        mem[off['w']:off['w'] + g.count] = before[call][off['w']:off['w'] + g.count]
        assert np.array_equal(mem, before[call])
