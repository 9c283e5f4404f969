"""Benchmark: CM1 large-step dynamics (WENO5 advection + acoustic substeps) on B200.

One "step" is one large time step (3 RK stages, 15 acoustic substeps at nsound=8) of the
256x256x80 synthetic Weisman-Klemp supercell workload, played as the reference's command
tape through the C-ABI player.  Metric: grid-pt-steps/s = nx*ny*nz*steps / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--mode fused|exact]

Multi-GPU (torchrun, one process per GPU): each rank advances its own independent
replica (ensemble member); no collective on the data path ("replicas only"), the
timed region is bracketed by barriers and the max over ranks is reported.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'grid-pt-steps/s'


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--mode', default='fused', choices=['fused', 'exact'])
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-roofline', action='store_true', help='skip the per-kernel timing pass')
    ap.add_argument('--no-fp64', action='store_true', help='skip the error statement against the binary64 oracle')
    ap.add_argument('--no-adjoint', action='store_true', help='skip the adjoint window (128x128x64, 60 steps)')
    ap.add_argument('--no-ensemble', action='store_true', help='skip the 64-member uneven ensemble')
    ap.add_argument('--ensemble-members', type=int, default=64)
    ap.add_argument('--workload', default='at_scale', choices=['at_scale', 'medium', 'small'],
                    help='at_scale = 256x256x80 (the benchmark); medium = 160x160x80 with the same '
                         'physics, for profiler captures; small = 64x64x40')
    return ap.parse_args()


# ---------------------------------------------------------------- distributed

def dist_init(n):
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import torch
        import torch.distributed as dist
        backend = 'nccl' if torch.cuda.is_available() else 'gloo'
        if backend == 'nccl':
            torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64,
                     device='cuda' if dist.get_backend() == 'nccl' else 'cpu')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------- clocks

class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed region: NVML
    polled every 5 ms from a thread (read-only queries), or nvidia-smi at 50 ms when
    NVML is unavailable."""
    NAMES = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')

    def __init__(self, device):
        self.device = device
        self.samples = []          # (sm_mhz, max_mhz, set of reason names)
        self.stop_flag = threading.Event()
        self.t = None
        self.nvml = None
        self.proc = None

    def _handle(self, nv):
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.device)
            bus = '%08x:%02x:%02x.0' % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.device)

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            bits = {'hw_slowdown': nv.nvmlClocksEventReasonHwSlowdown,
                    'hw_thermal_slowdown': nv.nvmlClocksEventReasonHwThermalSlowdown,
                    'sw_thermal_slowdown': nv.nvmlClocksEventReasonSwThermalSlowdown,
                    'sw_power_cap': nv.nvmlClocksEventReasonSwPowerCap}
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)

            def poll():
                while not self.stop_flag.is_set():
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((float(sm), float(mx), {n for n, b in bits.items() if r & b}))
                    time.sleep(0.005)
            self.nvml = nv
            self.t = threading.Thread(target=poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.device), '--query-gpu=clocks.sm,clocks.max.sm,'
                                          'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
                                          'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap',
                                          '--format=csv,noheader,nounits', '-lms', '50'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)

            def read():
                for line in self.proc.stdout:
                    parts = [p.strip() for p in line.split(',')]
                    try:
                        self.samples.append((float(parts[0]), float(parts[1]),
                                             {n for n, v in zip(self.NAMES, parts[2:6]) if v.lower() == 'active'}))
                    except (ValueError, IndexError):
                        pass
            self.t = threading.Thread(target=read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def wait_first(self, timeout=5.0):
        """Block until the sampler has its first sample, so the timed region is covered."""
        t0 = time.time()
        while not self.samples and time.time() - t0 < timeout and (self.t is not None):
            time.sleep(0.002)

    def stop(self):
        self.stop_flag.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.t is not None:
            self.t.join(timeout=2)
        if not self.samples:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['no clock samples'], 'samples': 0}
        reasons = set()
        for _, _, r in self.samples:
            reasons |= r
        return {'sm_mhz': statistics.median(x[0] for x in self.samples), 'sm_max_mhz': self.samples[-1][1],
                'reasons': sorted(reasons), 'samples': len(self.samples),
                'source': 'NVML, 5 ms polling' if self.nvml else 'nvidia-smi, 50 ms polling'}


# ------------------------------------------------------------------ workload

def workload(cfg_name='at_scale'):
    from thunderengine_web_b200 import scenario, timestep
    if cfg_name == 'medium':
        cfg = scenario.Config('cm1-dyn-160x160x80', 160, 160, 80, 500.0, 250.0, 3.0, 8, 25.0, 1)
    else:
        cfg = scenario.AT_SCALE if cfg_name == 'at_scale' else scenario.SMALL
    run = timestep.Run(cfg)
    return cfg, run


def peaks():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d['hbm_gbs']), 'measured'
    return 6650.0, 'fallback'


def cpu_baseline_sample(budget_s=10.0):
    """Time the reference's kernels (oracle/_ref, else the oracle port) on the host cores:
    large steps of the benchmark configuration itself (256x256x80), as many as fit in
    about ``budget_s`` seconds after one warm-up step."""
    from tests import helpers
    from thunderengine_web_b200 import scenario, timestep
    ref = helpers.reference()
    kind = 'reference' if ref is not None else 'port'
    kern = (ref or helpers.oracle()).get
    helpers.oracle()   # FTZ on the OpenMP team
    cfg = scenario.AT_SCALE
    run = timestep.Run(cfg)
    tape = run.tape(1)
    init = run.initial_buffers()
    from oracle.player import CpuPlayer
    p = CpuPlayer(tape, helpers.kernels_meta())
    p.plan(False)
    for i, b in init.items():
        p.upload(i, b)
    t0 = time.perf_counter()
    p.run(kern)                      # warm-up step
    t_one = time.perf_counter() - t0
    after_one = p.M.copy()           # the state after one step: the parity check of the GPU step
    nsteps = max(1, min(20, int(budget_s / max(t_one, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(nsteps):
        p.run(kern)
    dt = time.perf_counter() - t0
    pts = cfg.nx * cfg.ny * cfg.nz
    return {'value': pts * nsteps / dt, 'unit': METRIC, 'cores': os.cpu_count(), 'kind': kind,
            'sample': '%d large step(s) of the 256x256x80 workload after one warm-up step, %s kernels, '
                      'OpenMP over the dispatch grid on all host cores' % (
                          nsteps, "the reference's WGSL translated to C++" if kind == 'reference' else 'oracle'),
            'seconds': dt, '_after_one_step': after_one}


def parity_vs_cpu(r, run, init, cpu_mem, kind):
    """One large step of the benchmarked workload on the GPU (the mode being measured)
    against the same step on the host (the reference kernels, or the oracle): every
    non-scratch arena field compared word for word."""
    from thunderengine_web_b200.timestep import SCRATCH_FIELDS
    for i, b in init.items():
        r.upload(i, b)
    r.encode_steps(1)
    r.sync()
    g = run.grid
    aid = run.rec.ids['arena']
    base = r.base[aid]
    names = [n for n in run.fields if n not in SCRATCH_FIELDS]
    bad = [n for n in names if not np.array_equal(r.read(g.count, base + run.fields[n] // 4),
                                                  cpu_mem[base + run.fields[n] // 4:base + run.fields[n] // 4 + g.count])]
    return {'against': "the reference's kernels on the host (oracle/_ref)" if kind == 'reference' else 'the oracle',
            'steps': 1, 'fields_compared': len(names), 'fields_differing': bad, 'bit_exact': not bad}


PROGNOSTIC = ('th', 'qv', 'u', 'v', 'w', 'pp3d')


def interior(a, g):
    return a.reshape(g.nz + 1, g.strideK, g.strideJ)[:g.nz, 3:3 + g.ny, 3:3 + g.nx]


def fp64_error(r, run, init, checkpoints=(1, 20)):
    """Error of the binary32 step against the binary64 twin of the oracle
    (oracle/liboracle64.so: the same kernels evaluated in binary64) after each number of
    large steps in ``checkpoints``, from the same initial state: per prognostic field the
    largest absolute error over the interior points and that divided by the largest
    |value| of the binary64 field (normwise relative error).  The binary32 states are
    the GPU's (this library, the mode being measured)."""
    from tests import helpers
    from oracle.player import CpuPlayer64
    g = run.grid
    aid = run.rec.ids['arena']
    p = CpuPlayer64(run.tape(1), helpers.kernels_meta())
    p.plan()
    for i, b in init.items():
        p.upload(i, b)
    p.values_from_words()
    for i, b in init.items():
        r.upload(i, b)
    base = r.base[aid]
    assert base == p.base[aid]
    out, done, t0 = {}, 0, time.perf_counter()
    for n in checkpoints:
        r.encode_steps(n - done)
        r.sync()
        p.run64(n - done)
        done = n
        per = {}
        for f in PROGNOSTIC:
            o = base + run.fields[f] // 4
            a = interior(r.read(g.count, o).view(np.float32), g).astype(np.float64)
            b = interior(p.field64(o, g.count), g)
            err = float(np.abs(a - b).max())
            scale = float(np.abs(b).max())
            per[f] = {'max_abs': err, 'max_rel': err / scale if scale > 0 else None}
        out['after_%d_steps' % n] = per
    out['reference'] = ('the binary64 twin of the oracle (same kernels, same order, binary64 arithmetic, '
                        'binary32 constants), from the same initial state')
    out['max_rel_definition'] = 'max |f32 - f64| / max |f64| over the interior points of the field'
    out['seconds'] = time.perf_counter() - t0
    return out


def adjoint_leg(dev, nx=128, ny=128, nz=64, steps=60, every=10):
    """The adjoint configuration: a window of `steps` dynamics-core steps at nx x ny x nz
    (physics of the 256x256x80 workload) with checkpoints every `every` steps, cost
    J = sum of w^2 dx dy dz at the end.  Times, with CUDA events on the window's stream:
    the plain window (graph replay of the step), the forward with checkpoints and the
    backward (replay of each block with the undo log + the reverse walk)."""
    import torch
    from thunderengine_web_b200 import scenario, timestep
    from thunderengine_web_b200.adjoint import CoreWindow
    from thunderengine_web_b200.replayer import Replayer
    cfg = scenario.tiny(nx, ny, nz, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0)
    run = timestep.Run(cfg, core=True)
    tape = run.tape(1)
    r = Replayer(tape, None, device=dev)
    r.plan(False)
    r.build()
    for i, b in run.initial_buffers().items():
        r.upload(i, b)
    r.encode_steps(1)  # the window starts after one regular step
    r.sync()
    init = {b['id']: r.read(b['length'] // 4, r.base[b['id']]).tobytes() for b in tape['buffers']}
    r.close()
    win = CoreWindow(run, init, steps, checkpoint_every=every, device=dev)
    stream = torch.cuda.Stream(device=dev)
    win.r.set_stream(stream.cuda_stream)
    g = run.grid
    arena = np.frombuffer(init[run.rec.ids['arena']], dtype=np.float32)
    ctl = [arena[run.fields[n] // 4:run.fields[n] // 4 + g.count].reshape(g.nz + 1, g.strideK, g.strideJ)
           [:g.nz, 3:3 + g.ny, 3:3 + g.nx] for n in ('th', 'u', 'v')]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        torch.cuda.synchronize()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3, out

    win.r.encode_steps(2)
    t_plain, _ = timed(lambda: win.r.encode_steps(steps))
    w = win.forward(*ctl)
    dV = g.dx * g.dy * g.dz
    gw = 2.0 * w.astype(np.float64) * dV
    win.backward(gw)  # captures the block graphs
    win.load(*ctl)
    t_fwd, _ = timed(win.run_forward)
    w = win.read_w()
    lw = np.zeros((g.nz + 1, g.strideK, g.strideJ), dtype=np.float32)
    lw[1:g.nz, 3:3 + g.ny, 3:3 + g.nx] = 2.0 * w.astype(np.float64) * dV
    win.r.adjoint_zero()
    win.r.adjoint_write_words(win.base + run.fields['w'] // 4, lw.ravel())
    t_bwd, _ = timed(lambda: win.r.adjoint_backward())
    pts = g.nx * g.ny * g.nz
    out = {'grid': [nx, ny, nz], 'window_steps': steps, 'checkpoint_every': every, 'cost': 'sum of w^2 dx dy dz at the end',
           'control': "th', u, v at the start", 'dtype': 'f32',
           'value': pts * steps / t_bwd, 'unit': 'grid-pt-steps/s (adjoint: backward with recompute)',
           'forward_value': pts * steps / t_plain, 'backward_s': t_bwd, 'plain_window_s': t_plain,
           'forward_with_checkpoints_s': t_fwd, 'backward_over_forward': t_bwd / t_plain,
           'device_bytes': win.r.adjoint_memory(),
           'timing': 'CUDA events on the window stream; forward = graph replay of the dynamics-core step'}
    win.close()
    return out


def ensemble_leg(dev, n=64, steps=50, warmup=2):
    """The batched-ensemble configuration: `n` members of uneven grids from 64x64x40 to
    192x192x64 (seeded sizes, CAPE, shear, dt 3/6 s, nsound 6..8), fused mode, block
    shapes autotuned per member.  member-steps/s of one ensemble graph launch per large
    step against looping the plain step member by member on one stream."""
    import torch
    from thunderengine_web_b200 import scenario, timestep
    from thunderengine_web_b200.replayer import Ensemble, Replayer, TE_MODE_FUSED
    cfgs = scenario.ensemble(n, seed=7, steps=steps)
    stream = torch.cuda.Stream(device=dev)
    reps, tuned, pts = [], 0, 0
    for cfg in cfgs:
        run = timestep.Run(cfg)
        r = Replayer(run.tape(1), None, device=dev)
        r.plan(False)
        r.build()
        for i, b in run.initial_buffers().items():
            r.upload(i, b)
        r.set_mode(TE_MODE_FUSED)
        tuned += r.autotune(reps=2)
        r.set_stream(stream.cuda_stream)
        reps.append(r)
        pts += cfg.nx * cfg.ny * cfg.nz
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # looping the plain step: every member's step graph, one member after another
    for _ in range(warmup):
        for r in reps:
            r.encode_steps(1)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        for r in reps:
            r.encode_steps(1)
    e1.record(stream)
    torch.cuda.synchronize()
    t_loop = e0.elapsed_time(e1) / 1e3
    ens = Ensemble(reps)
    es = torch.cuda.ExternalStream(ens.stream(), device=dev)
    ens.run(warmup)
    ens.sync()
    e0.record(es)
    ens.run(steps)
    e1.record(es)
    torch.cuda.synchronize()
    t_ens = e0.elapsed_time(e1) / 1e3
    ens.close()
    mem = sum(r.mem_words for r in reps) * 4
    for r in reps:
        r.close()
    return {'members': n, 'steps': steps, 'value': n * steps / t_ens, 'unit': 'member-steps/s',
            'loop_value': n * steps / t_loop, 'speedup_vs_loop': t_loop / t_ens,
            'grid_pt_steps_per_s': pts * steps / t_ens, 'grid_points_total': pts,
            'substeps_per_step': sorted({timestep.AcousticSchedule(c.nsound, timestep.f(c.dt)).total for c in cfgs}),
            'autotuned_ops': tuned, 'device_bytes': mem, 'mode': 'fused',
            'how': 'one graph launch per large step (every member a child graph, no edges between members) vs '
                   'each member\'s step graph launched in turn on one stream; CUDA events'}


# ---------------------------------------------------------------- our arm

def run_ours(a, rank, world, local):
    import torch
    from thunderengine_web_b200.replayer import Replayer, TE_MODE_EXACT, TE_MODE_FUSED
    dev = local if torch.cuda.device_count() > local else 0
    torch.cuda.set_device(dev)
    cfg, run = workload(a.workload)
    tape = run.tape(1)
    run.tape_cmds = tape['steps'][0]
    init = run.initial_buffers()
    r = Replayer(tape, None, device=dev)
    r.plan(False)
    r.build()
    for i, b in init.items():
        r.upload(i, b)
    # a dedicated (non-default) stream shared by the library and torch's events
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    r.set_stream(stream.cuda_stream)
    mode = TE_MODE_FUSED if a.mode == 'fused' else TE_MODE_EXACT
    r.set_mode(mode)
    pts = cfg.nx * cfg.ny * cfg.nz
    for _ in range(max(a.warmup, 3)):
        r.encode_steps(1)
    torch.cuda.synchronize()
    sampler = ClockSampler(dev)
    sampler.start()
    sampler.wait_first()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    r.encode_steps(a.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ms, world)
    value = pts * a.steps * world / (ms / 1e3)

    # per-kernel timing for the roofline: each distinct op of the step alone, events on
    # the launch stream; achieved = algorithmic bytes per launch / launch time
    roof = None if a.no_roofline else kernel_roofline(r, run, stream, mode)

    # end to end through the public API with host buffers: every step uploads the state
    # fields from pinned memory, plays the step, reads the prognostic fields back
    e2e = None if a.no_e2e else end_to_end(r, run, init, cfg, a, world, mode, dev)
    cpu = None
    parity = None
    f64err = None
    adjoint = None if (a.no_adjoint or rank != 0) else adjoint_leg(dev)
    ens = None if (a.no_ensemble or rank != 0) else ensemble_leg(dev, a.ensemble_members)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline_sample()
        parity = parity_vs_cpu(r, run, init, cpu.pop('_after_one_step'), cpu['kind'])
        f64err = None if a.no_fp64 else fp64_error(r, run, init)
    ops = r.num_ops
    if roof is not None:
        launches = roof.pop('_launches_per_step')
    elif mode == TE_MODE_FUSED:
        launches = sum(sg[3] for sg in r.fused_segments())
    else:
        launches = r.num_dispatches
    out = {
        'metric': METRIC, 'value': value, 'unit': METRIC, 'n_gpus': world, 'steps': a.steps, 'warmup': a.warmup,
        'ms_per_step': ms / a.steps, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f32', 'data': 'synthetic (Weisman-Klemp sounding, 2 K bubble, seeded noise)',
        'config': dict(cfg.as_dict(), grid_points=pts, mode=a.mode, parallelism='replicas x%d' % world,
                       tape_ops_per_step=ops,
                       l2='inputs larger than L2: %.2f GB arena per replica' % (run.arena_bytes / 1e9)),
        'roofline': roof, 'cpu_baseline': cpu, 'e2e': e2e, 'gpu_launches': launches * a.steps, 'clocks': clocks,
        'parity': parity, 'fp64_error': f64err, 'adjoint': adjoint, 'ensemble': ens,
    }
    if rank == 0:
        print(json.dumps(out))
    r.close()


def kernel_roofline(r, run, stream, mode):
    """Per-kernel device time of one step, measured with CUDA events on the launch stream:
    each exact dispatch kind and each fused kernel is re-launched alone `reps` times.
    The dominant kernel (time x launches per step) gets the roofline figures."""
    import torch
    peak, src = peaks()
    km = kernel_meta(r.lib)
    disp = tape_dispatches(run, run.tape_cmds)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 5

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    stats = {}   # name -> [ms per launch, launches per step, algorithmic bytes per launch]
    g = run.grid
    if mode == 1:
        segs = r.fused_segments()
        exact_ops = [i for (kind, a, b, _) in segs if kind == 0 for i in range(a, b + 1)]
        acu = [q for q, sg in enumerate(segs) if sg[0] == 1]
        halo = [q for q, sg in enumerate(segs) if sg[0] == 2]
        if acu:
            q = acu[-1]
            pts_whole = g.count
            pts = g.nx * g.ny * g.nz
            stats['acoustic_uv_accumulate (fused)'] = [timed(lambda: r.run_segment(q, 0)), len(acu), 12 * 4 * pts_whole]
            # the timed launch is a stage-3 substep: reads u, v, w, piadv, ppten, ppterm, pk1,
            # pk2, qk, mm, wten, pp3d, rrw; writes w, pp3d, ppd, rrw and ppx (stages 1-2: no ppx)
            stats['acoustic_column (fused fpk+w_solve+pp+accumulate)'] = [timed(lambda: r.run_segment(q, 1)), len(acu),
                                                                          18 * 4 * pts]
            stats['halo_periodic x4 (fused)'] = [timed(lambda: r.run_segment(q, 2)), len(acu),
                                                 4 * 2 * 4 * 7 * (g.strideK + g.nx) * (g.nz + 1)]
        if halo:
            q = halo[0]
            nf = segs[q][2] - segs[q][1] + 1
            stats['halo_periodic (fused)'] = [timed(lambda: r.run_segment(q, -1)), len(halo),
                                              (nf // 2) * 2 * 4 * 7 * (g.strideK + g.nx) * (g.nz + 1)]
        # fused advection: one kernel per variable and stage, grouped by flux kind; bytes =
        # the distinct arena fields its ops bind, except the fx/fy/fz fluxes it never
        # touches, x 4 B x interior points
        for q, sg in enumerate(segs):
            if sg[0] != 3:
                continue
            name = 'advect %s (fused flux+assemble%s)' % (r.op_name(sg[1]).replace('adv_flux_x', '').strip('_') or 'lin',
                                                          '+rk' if sg[2] - sg[1] > 3 else '')
            fields = set()
            for i in range(sg[1], sg[2] + 1):
                fields |= {f for f in disp[i]['fields'].values() if f is not None}
            byts = len(fields - {'fx', 'fy', 'fz'}) * 4 * g.nx * g.ny * g.nz
            ms = timed(lambda: r.run_segment(q, -1))
            if name in stats:
                o = stats[name]
                stats[name] = [(o[0] * o[1] + ms) / (o[1] + 1), o[1] + 1, (o[2] * o[1] + byts) / (o[1] + 1)]
            else:
                stats[name] = [ms, 1, byts]
    else:
        exact_ops = list(range(r.num_ops))
    seen = {}
    for i in exact_ops:
        n = r.op_name(i)
        if n != 'copy':
            seen.setdefault(n, []).append(i)
    for n, idx in seen.items():
        i = idx[0]
        stats[n] = [timed(lambda: r.run_ops(i, i)), len(idx), dispatch_bytes(disp[i], km, g.nz)]
    tot = sum(v[0] * v[1] for v in stats.values())
    top = max(stats, key=lambda n: stats[n][0] * stats[n][1])
    ms, _, byts = stats[top]
    achieved = byts / (ms / 1e3) / 1e9
    shares = sorted(((n, v[0] * v[1] / tot) for n, v in stats.items()), key=lambda x: -x[1])
    launches = sum(v[1] for v in stats.values())
    if mode == 1:
        launches = sum(sg[3] for sg in r.fused_segments())
    dram = NCU_DRAM_BYTES_PER_POINT.get(top)
    return {'kernel': top, 'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
            'frac': achieved / peak, 'peak_source': ('measured (MEASURED_PEAKS.json hbm_gbs)' if src == 'measured'
                                                     else 'fallback 6650 GB/s'),
            'algorithmic_bytes_per_launch': byts, 'launch_ms': ms,
            'traffic': dram * g.nx * g.ny * g.nz if dram else None,
            'traffic_source': ('ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch on the 256x256x80 '
                               'workload, per interior point, times this run\'s interior points' if dram else None),
            'share_of_step': shares[0][1], 'sum_of_kernel_ms_per_step': tot,
            'top_kernels': [[n, round(sv, 4), round(stats[n][0], 4), stats[n][1],
                             round(stats[n][2] / (stats[n][0] / 1e3) / 1e9, 1)] for n, sv in shares[:10]],
            'top_kernels_columns': ['kernel', 'share', 'ms_per_launch', 'launches_per_step', 'achieved_GBps'],
            '_launches_per_step': launches}


# DRAM bytes per interior point of one launch of the dominant kernels: one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum, a one-pass metric set) of the kernel on
# the 256x256x80 workload, divided by its interior points; traffic grows with the points
# a launch processes.  Writes still held in L2 when the launch ends are not counted.
NCU_DRAM_BYTES_PER_POINT = {
    'acoustic_column (fused fpk+w_solve+pp+accumulate)': (286.53e6 + 84.02e6) / (256 * 256 * 80),
}


# Fields a kernel both reads and writes at the same points (binding indices), counted
# twice in the algorithmic bytes; every other bound arena field counts once.
RMW = {
    'acoustic_uv': (6, 7), 'acoustic_w_solve': (9,), 'acoustic_pp': (7,), 'acoustic_accumulate': (5, 6, 7),
    'pdef_apply': (16,), 'buoyancy_apply': (4,), 'apply_thterm': (3,), 'velocity_to_massflux': (3, 4, 5),
    'diabatic_unapply': (2, 3, 4, 5, 6, 7, 8, 9), 'diabatic_rates': (6, 7, 8, 9), 'ppx_finish': (2,),
    'bc_periodic_x': (1,), 'bc_periodic_y': (1,),
}


def tape_dispatches(run, cmds):
    """Per op of a step (dispatches and copies, in op order): kernel name, grid and the
    arena field bound at each binding index."""
    by_off = {off: n for n, off in run.fields.items()}
    arena_id = run.rec.ids['arena']
    out, bind, pipe = [], {}, None
    for c in cmds:
        op = c['op']
        if op == 'pipe':
            pipe = c['name']
        elif op == 'buf':
            bind[c['index']] = by_off.get(c['offset']) if c['buf'] == arena_id else None
        elif op == 'bytes':
            bind[c['index']] = None
        elif op == 'end':
            bind = {}
        elif op == 'copy':
            out.append({'name': 'copy', 'grid': [c['size'] // 4, 1, 1], 'fields': {}})
        elif op == 'dispatch':
            out.append({'name': pipe, 'grid': c['grid'], 'fields': dict(bind)})
    return out


# Kernels launched once per column (kernels.json "rank": 2): a dispatched thread covers nz levels.
COLUMN_KERNELS = {'acoustic_w_solve'}


def kernel_meta(lib):
    """The library's own kernel table (kernels.json-shaped: parameter index, kind, write)."""
    import ctypes
    n = lib.te_kernel_table_json(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib.te_kernel_table_json(buf, n + 1)
    table = json.loads(buf.value.decode())
    for name, k in table.items():
        k['rank'] = 2 if name in COLUMN_KERNELS else 3
    return table


def dispatch_bytes(d, km, nz):
    """Algorithmic bytes of one dispatch: (distinct arena fields bound to its pointer
    parameters, read-modify-write fields twice) x 4 B x points of its range; a column
    kernel (rank 2, e.g. acoustic_w_solve) covers nz levels per dispatched column."""
    params = {p['index']: p for p in km[d['name']]['params']}
    fields = {}
    for idx, f in d['fields'].items():
        p = params.get(idx)
        if f is None or p is None or p['kind'] != 'ptr':
            continue
        w = 2 if idx in RMW.get(d['name'], ()) else 1
        fields[f] = max(fields.get(f, 0), w)
    pts = d['grid'][0] * d['grid'][1] * d['grid'][2]
    if km[d['name']].get('rank') == 2:
        pts *= nz
    return sum(fields.values()) * 4 * pts


def step_inputs(rep, run, init, state):
    """The arena fields one step reads before it writes them (its inputs), found with this
    library's own kernels: each non-scratch field in turn is filled with seeded garbage
    before one step from the initial state; a field whose garbage leaves every
    non-scratch field after the step bit-identical is fully rewritten before any read.
    Returns (inputs, the non-scratch fields after one step from the initial state)."""
    g = run.grid
    aid = run.rec.ids['arena']
    base = rep.base[aid]
    rng = np.random.default_rng(11)

    def one_step(poison=None):
        for i, buf in init.items():
            rep.upload(i, buf)
        if poison is not None:
            junk = rng.uniform(-3.0, 3.0, g.count).astype(np.float32).view(np.uint32)
            rep.write_words(base + run.fields[poison] // 4, junk)
        rep.encode_steps(1)
        rep.sync()
        return {n: rep.read(g.count, base + run.fields[n] // 4) for n in state}

    want = one_step()
    inputs = [n for n in state if any(not np.array_equal(v, want[m]) for m, v in one_step(n).items())]
    return inputs, want


def end_to_end(r, run, init, cfg, a, world, mode, dev):
    """The same metric through the public API with host buffers.  Every step uploads the
    step's inputs (the arena fields it reads before writing, step_inputs) from pinned host
    memory, plays the step and reads th, qv, u, v, w, pp3d back into pinned memory.  Two
    replicas (the context of the timed run and a second one on its own stream) take the
    steps in turn, so one replica's copies overlap the other's step (te_write_words_async /
    te_read_async); the serial figure (one context, blocking copies) is reported beside it.
    The fields read back after the timed steps are checked bit for bit against a step whose
    every non-scratch field was uploaded."""
    import torch
    from thunderengine_web_b200.replayer import Replayer
    from thunderengine_web_b200.timestep import SCRATCH_FIELDS
    g = run.grid
    aid = run.rec.ids['arena']
    arena0 = np.frombuffer(init[aid], dtype=np.uint32)
    nonscratch = [n for n in run.fields if n not in SCRATCH_FIELDS]
    outs = ['th', 'qv', 'u', 'v', 'w', 'pp3d']
    lib = r.lib
    r2 = Replayer(run.tape(1), None, device=dev)
    r2.plan(False)
    r2.build()
    r2.set_mode(mode)
    state, want = step_inputs(r2, run, init, nonscratch)
    for i, buf in init.items():
        r2.upload(i, buf)
    pin_in = torch.empty((len(state), g.count), dtype=torch.int32).pin_memory()
    for q, n in enumerate(state):
        o = run.fields[n] // 4
        pin_in[q].numpy()[:] = arena0[o:o + g.count].view(np.int32)
    s2 = torch.cuda.Stream(device=dev)
    r2.set_stream(s2.cuda_stream)
    reps = [(r, torch.empty((len(outs), g.count), dtype=torch.int32).pin_memory()),
            (r2, torch.empty((len(outs), g.count), dtype=torch.int32).pin_memory())]

    def step_async(rep, pout):
        base = rep.base[aid]
        for q, n in enumerate(state):
            rep._check(lib.te_write_words_async(rep.h, base + run.fields[n] // 4, pin_in[q].data_ptr(), g.count * 4))
        rep.encode_steps(1)
        for q, n in enumerate(outs):
            rep._check(lib.te_read_async(rep.h, base + run.fields[n] // 4, g.count, pout[q].data_ptr()))

    def step_serial(rep, pout):
        base = rep.base[aid]
        for q, n in enumerate(state):
            rep._check(lib.te_write_words(rep.h, base + run.fields[n] // 4, pin_in[q].data_ptr(), g.count * 4))
        rep.encode_steps(1)
        for q, n in enumerate(outs):
            rep._check(lib.te_read(rep.h, base + run.fields[n] // 4, g.count, pout[q].data_ptr()))

    pts = cfg.nx * cfg.ny * cfg.nz
    steps = max(2, min(a.steps, 6))

    def timed(fn, nsteps):
        for s in range(4):
            fn(*reps[s % 2])
        r.sync()
        r2.sync()
        barrier(world)
        t0 = time.perf_counter()
        for s in range(nsteps):
            fn(*reps[s % 2])
        r.sync()
        r2.sync()
        return max_over_ranks(time.perf_counter() - t0, world)

    dt = timed(step_async, steps)
    verified = all(np.array_equal(pout[q].numpy().view(np.uint32), want[n]) for _, pout in reps for q, n in enumerate(outs))
    dt_serial = timed(step_serial, steps)
    verified = verified and all(np.array_equal(pout[q].numpy().view(np.uint32), want[n])
                                for _, pout in reps for q, n in enumerate(outs))
    barrier(world)
    r2.close()
    if not verified:
        raise RuntimeError('end-to-end steps did not reproduce the full-upload step')
    return {'value': pts * steps * world / dt, 'unit': METRIC, 'h2d_bytes_per_step': len(state) * g.count * 4,
            'd2h_bytes_per_step': len(outs) * g.count * 4, 'steps': steps,
            'serial_value': pts * steps * world / dt_serial,
            'inputs': state, 'verified': True,
            'path': 'per step: Replayer write_words_async of each input field of the step (pinned host) -> '
                    'encode_steps(1) -> read_async x6 (pinned host); two replicas alternate steps so copies overlap '
                    'the other replica\'s step; serial_value: one context at a time with blocking copies; the read-back '
                    'fields equal those of a step with every non-scratch field uploaded'}


# -------------------------------------------------------- reference arm (CPU)

def run_reference(a, rank, world):
    """The reference's own kernels (its WGSL translated to C++, oracle/_ref) on the host
    cores, same metric; rank 0 only."""
    if rank != 0:
        return
    from tests import helpers
    from thunderengine_web_b200 import scenario, timestep
    from oracle.player import CpuPlayer
    ref = helpers.reference()
    kind = 'reference' if ref is not None else 'port'
    kern = (ref or helpers.oracle()).get
    helpers.oracle()
    cfg = scenario.AT_SCALE
    run = timestep.Run(cfg)
    tape = run.tape(1)
    init = run.initial_buffers()
    p = CpuPlayer(tape, helpers.kernels_meta())
    p.plan(False)
    for i, b in init.items():
        p.upload(i, b)
    for _ in range(a.warmup):
        p.run(kern)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        p.run(kern)
    dt = time.perf_counter() - t0
    pts = cfg.nx * cfg.ny * cfg.nz
    v = pts * a.steps / dt
    big = cfg
    out = {'metric': METRIC, 'value': v, 'unit': METRIC, 'n_gpus': world, 'steps': a.steps, 'warmup': a.warmup,
           'ms_per_step': dt / a.steps * 1e3, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
           'dtype': 'f32', 'data': 'synthetic (Weisman-Klemp sounding, 2 K bubble, seeded noise)', 'impl': 'reference',
           'config': dict(big.as_dict(), grid_points=pts, mode=a.mode, parallelism='replicas x%d' % world,
                          tape_ops_per_step=sum(1 for c in tape['steps'][0] if c['op'] in ('dispatch', 'copy')),
                          l2='inputs larger than L2: %.2f GB arena per replica' % (run.arena_bytes / 1e9)),
           'cpu_baseline': {'value': v, 'unit': METRIC, 'cores': os.cpu_count(), 'kind': kind,
                            'sample': 'each step = one large step of the 256x256x80 workload on all host cores'},
           'e2e': {'value': v, 'unit': METRIC, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(out))


def main():
    a = parse()
    rank, world, local = dist_init(a.gpus)
    try:
        if a.impl == 'reference':
            run_reference(a, rank, world)
        else:
            run_ours(a, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == '__main__':
    main()
