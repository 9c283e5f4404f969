"""The adjoint configuration at full size: 128x128x64, a 60-step window of the
dynamics-core step with checkpoints every 10 steps, J = sum of w^2 dx dy dz at the end,
gradient with respect to th', u, v at the start.  Test infrastructure (not collected by
pytest); two parts, so that the binary64 work runs on any host:

    python -m tests.adjoint_config3 gpu   --out DIR   # on a B200: binary32 gradient + timing
    python -m tests.adjoint_config3 check --out DIR   # on the host: binary64 checks of it

(`profile --steps N` runs one backward of an N-step window inside a profiler range, for an
ncu launch list.)

`gpu` writes DIR/grad32.npy (the concatenated th', u, v gradient), DIR/gpu.json (J, the
timing of the plain window, the forward with checkpoints and the backward, device memory).
`check` computes the binary64 adjoint of the same window (oracle/libadjoint64.so over
the binary64 twin, checkpoints every 10), the binary64 adjoint around the binary32
trajectory (the one the GPU follows), binary64 central differences of J along 16 seeded
unit directions (eps = 1e-3, and 1e-5 on the first 4), and writes DIR/check.json.

Physics as the 256x256x80 workload (dx = 500 m, dz = 250 m, dt = 3 s, nsound 8,
Us = 25 m/s); the window starts after one regular large step of the synthetic supercell
state, computed identically on both sides (the GPU's exact step equals the oracle's).
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

NX, NY, NZ, STEPS, EVERY = 128, 128, 64, 60, 10


def make_run():
    from thunderengine_web_b200 import scenario, timestep
    cfg = scenario.tiny(NX, NY, NZ, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0)
    return timestep.Run(cfg, core=True)


def part_gpu(out):
    from tests import helpers
    from thunderengine_web_b200.adjoint import CoreWindow
    run = make_run()
    tape = run.tape(1)
    r = helpers.gpu_replayer(tape, run.initial_buffers(), hashes=False)
    r.encode_steps(1)
    r.sync()
    init = {b['id']: r.read(b['length'] // 4, r.base[b['id']]).tobytes() for b in tape['buffers']}
    r.close()
    g = run.grid
    win = CoreWindow(run, init, STEPS, checkpoint_every=EVERY)
    arena = np.frombuffer(init[run.rec.ids['arena']], dtype=np.float32)
    ctl = [arena[run.fields[n] // 4:run.fields[n] // 4 + g.count].reshape(g.nz + 1, g.strideK, g.strideJ)
           [:g.nz, 3:3 + g.ny, 3:3 + g.nx] for n in ('th', 'u', 'v')]
    # the plain window (graph replay of the step), for the cost ratio
    win.r.upload(run.rec.ids['arena'], arena.tobytes())
    win.r.encode_steps(2)
    win.r.sync()
    t0 = time.perf_counter()
    win.r.encode_steps(STEPS)
    win.r.sync()
    t_plain = time.perf_counter() - t0
    win.forward(*ctl)  # warm-up: builds the tables
    win.load(*ctl)
    win.r.sync()
    t0 = time.perf_counter()
    win.run_forward()
    win.r.sync()
    t_fwd = time.perf_counter() - t0
    w = win.read_w()
    dV = g.dx * g.dy * g.dz
    gw = 2.0 * w.astype(np.float64) * dV
    win.backward(gw)  # the first backward captures the block graphs
    t0 = time.perf_counter()
    grads = win.backward(gw)
    win.r.sync()
    t_bwd = time.perf_counter() - t0
    w = win.forward(*ctl)
    J = float((w.astype(np.float64) ** 2).sum()) * dV
    os.makedirs(out, exist_ok=True)
    np.save(os.path.join(out, 'grad32.npy'), np.concatenate([x.ravel() for x in grads]))
    pts = g.nx * g.ny * g.nz
    res = {'grid': [NX, NY, NZ], 'steps': STEPS, 'checkpoint_every': EVERY, 'J': J,
           'plain_window_s': t_plain, 'forward_with_checkpoints_s': t_fwd, 'backward_s': t_bwd,
           'backward_over_plain': t_bwd / t_plain, 'forward_grid_pt_steps_per_s': pts * STEPS / t_plain,
           'adjoint_grid_pt_steps_per_s': pts * STEPS / t_bwd, 'device_bytes': win.r.adjoint_memory()}
    with open(os.path.join(out, 'gpu.json'), 'w') as fh:
        json.dump(res, fh, indent=1)
    print(json.dumps(res))


def part_check(out, ndir=16):
    from tests import helpers
    from oracle.adjoint import Control, CpuAdjoint64, cost_w2, seed_w2
    from oracle.player import CpuPlayer64
    run = make_run()
    tape = run.tape(1)
    cpu = helpers.cpu_run(tape, run.initial_buffers(), nsteps=1, hashes=False)
    init = {b['id']: cpu.buffer_words(b['id']).tobytes() for b in tape['buffers']}
    del cpu
    ctape = run.tape(1, core=True)
    km = helpers.kernels_meta()
    t0 = time.perf_counter()
    A = CpuAdjoint64(ctape, km, init)
    base = A.p.base[run.rec.ids['arena']]
    A.forward(STEPS, EVERY)
    J64 = cost_w2(run, A.D, base)
    L = A.backward(seed_w2(run, A.D, base, A.D.size))
    ctl = Control(run, base)
    g64 = ctl.gradient(L)
    t_adj = time.perf_counter() - t0
    del A, L
    # the binary64 adjoint around the binary32 trajectory (the GPU's, bit for bit)
    A = CpuAdjoint64(ctape, km, init, linearize='f32', kernels32=helpers.oracle().get)
    A.forward(STEPS, EVERY)
    g64on32 = ctl.gradient(A.backward(seed_w2(run, A.D, base, A.D.size)))
    del A
    g32 = np.load(os.path.join(out, 'grad32.npy')).astype(np.float64)
    with open(os.path.join(out, 'gpu.json')) as fh:
        gpu = json.load(fh)
    n = NX * NY * NZ
    def rel(a, b):
        return {f: float(np.linalg.norm(a[q * n:(q + 1) * n] - b[q * n:(q + 1) * n]) /
                         np.linalg.norm(b[q * n:(q + 1) * n])) for q, f in enumerate(('th', 'u', 'v'))}
    field_err = rel(g32, g64on32)
    traj_err = rel(g64on32, g64)

    def J_of(d, eps):
        p = CpuPlayer64(ctape, km)
        p.plan()
        for i, b in init.items():
            p.upload(i, b)
        p.values_from_words()
        ctl.add(p.D, d, eps)
        p.run64(STEPS)
        return cost_w2(run, p.D, base)

    rng = np.random.default_rng(2024)
    dirs = []
    t0 = time.perf_counter()
    for q in range(ndir):
        d = rng.standard_normal(ctl.size)
        d /= np.linalg.norm(d)
        row = {'adjoint32': float(g32 @ d), 'adjoint64': float(g64 @ d), 'adjoint64_on_f32': float(g64on32 @ d)}
        for eps in ((1e-3, 1e-5) if q < 4 else (1e-3,)):
            fd = (J_of(d, eps) - J_of(d, -eps)) / (2 * eps)
            row['fd_%g' % eps] = fd
            row['rel32_%g' % eps] = abs(row['adjoint32'] - fd) / abs(fd)
            row['rel64_%g' % eps] = abs(row['adjoint64'] - fd) / abs(fd)
        dirs.append(row)
        print(json.dumps(row), flush=True)
    res = {'grid': [NX, NY, NZ], 'steps': STEPS, 'checkpoint_every': EVERY, 'J32': gpu['J'], 'J64': J64,
           'grad32_vs_grad64_same_trajectory_rel_2norm': field_err,
           'grad64_f32_trajectory_vs_f64_trajectory_rel_2norm': traj_err, 'directions': dirs,
           'max_rel32_eps1e-3': max(r['rel32_0.001'] for r in dirs),
           'max_rel64_eps1e-3': max(r['rel64_0.001'] for r in dirs),
           'max_rel32_eps1e-5': max(r['rel32_1e-05'] for r in dirs if 'rel32_1e-05' in r),
           'max_rel64_eps1e-5': max(r['rel64_1e-05'] for r in dirs if 'rel64_1e-05' in r),
           'cpu_adjoint_s': t_adj, 'fd_s': time.perf_counter() - t0}
    with open(os.path.join(out, 'check.json'), 'w') as fh:
        json.dump(res, fh, indent=1)
    print(json.dumps({k: v for k, v in res.items() if k != 'directions'}))


def part_profile(steps):
    """A `steps`-step window with one checkpoint: forward and backward once, then a second
    backward between cudaProfilerStart/Stop, so that `ncu --profile-from-start off` lists
    exactly the launches of one backward (the logged replay, the undo copies and the
    reverse walk)."""
    import torch
    from tests import helpers
    from thunderengine_web_b200.adjoint import CoreWindow
    run = make_run()
    tape = run.tape(1)
    r = helpers.gpu_replayer(tape, run.initial_buffers(), hashes=False)
    r.encode_steps(1)
    r.sync()
    init = {b['id']: r.read(b['length'] // 4, r.base[b['id']]).tobytes() for b in tape['buffers']}
    r.close()
    g = run.grid
    win = CoreWindow(run, init, steps, checkpoint_every=steps)
    arena = np.frombuffer(init[run.rec.ids['arena']], dtype=np.float32)
    ctl = [arena[run.fields[n] // 4:run.fields[n] // 4 + g.count].reshape(g.nz + 1, g.strideK, g.strideJ)
           [:g.nz, 3:3 + g.ny, 3:3 + g.nx] for n in ('th', 'u', 'v')]
    win.forward(*ctl)
    gw = 2.0 * win.read_w().astype(np.float64)
    win.backward(gw)
    win.r.sync()
    t0 = time.perf_counter()
    win.backward(gw)
    win.r.sync()
    print(json.dumps({'steps': steps, 'backward_s': time.perf_counter() - t0}))
    torch.cuda.profiler.start()
    win.backward(gw)
    win.r.sync()
    torch.cuda.profiler.stop()
    win.close()


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('part', choices=['gpu', 'check', 'profile'])
    ap.add_argument('--out', default='adjoint_config3_out')
    ap.add_argument('--directions', type=int, default=16)
    ap.add_argument('--steps', type=int, default=2, help='window of the profile part')
    a = ap.parse_args()
    if a.part == 'gpu':
        part_gpu(a.out)
    elif a.part == 'profile':
        part_profile(a.steps)
    else:
        part_check(a.out, a.directions)
