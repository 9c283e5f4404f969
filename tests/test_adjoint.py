"""Discrete adjoint of the dynamics-core step.

CPU: the binary64 adjoint (the library's adjoint operators in binary64 over the binary64
twin of the oracle) against binary64 central differences of the twin's forward step.
GPU: the library's binary32 adjoint through the C-ABI against the binary64 adjoint and
against central differences, the memory it leaves, and its independence of the
checkpoint interval.  Cost J = sum of w^2 dx dy dz over the interior faces at the end
of the window; control = th', u, v at its start.
"""
import numpy as np
import pytest

from tests import helpers
from thunderengine_web_b200 import scenario, timestep


def _window_start(nx, ny, nz, regular_steps=1):
    """A Run (core=True) and the memory after `regular_steps` regular large steps of the
    synthetic supercell state: the window starts from a state whose thermodynamic
    coefficients are those of a real step."""
    cfg = scenario.tiny(nx, ny, nz, dx=500.0, dz=250.0, dt=3.0, nsound=8, us=25.0)
    run = timestep.Run(cfg, core=True)
    tape = run.tape(1)
    cpu = helpers.cpu_run(tape, run.initial_buffers(), nsteps=regular_steps, hashes=False)
    init = {b['id']: cpu.buffer_words(b['id']).tobytes() for b in tape['buffers']}
    return run, init


def _fd(run, init, ctl, d, eps, nsteps):
    from oracle.adjoint import cost_w2
    from oracle.player import CpuPlayer64
    vals = []
    for e in (eps, -eps):
        p = CpuPlayer64(run.tape(1, core=True), helpers.kernels_meta())
        p.plan()
        for i, b in init.items():
            p.upload(i, b)
        p.values_from_words()
        ctl.add(p.D, d, e)
        p.run64(nsteps)
        vals.append(cost_w2(run, p.D, p.base[run.rec.ids['arena']]))
    return (vals[0] - vals[1]) / (2 * eps)


def _cpu_gradient(run, init, nsteps, linearize='f64'):
    from oracle.adjoint import Control, CpuAdjoint64, cost_w2, seed_w2
    A = CpuAdjoint64(run.tape(1, core=True), helpers.kernels_meta(), init, linearize=linearize,
                     kernels32=helpers.oracle().get)
    base = A.p.base[run.rec.ids['arena']]
    A.forward(nsteps)
    J = cost_w2(run, A.D, base)  # before backward, which returns memory to the start state
    L = A.backward(seed_w2(run, A.D, base, A.D.size))
    ctl = Control(run, base)
    return ctl, ctl.gradient(L), J


def test_every_core_kernel_has_an_adjoint_operator():
    from oracle.adjoint import adjoint_lib
    run = timestep.Run(scenario.tiny(16, 12, 10), core=True)
    names = {c['name'] for c in run.tape(1, core=True)['steps'][0] if c['op'] == 'pipe'}
    assert len(names) == 37
    lib = adjoint_lib()
    assert all(lib.teadj_has(n.encode()) for n in names)
    # the regular step has kernels the core step leaves out (no adjoint operator)
    full = {c['name'] for c in run.tape(1)['steps'][0] if c['op'] == 'pipe'}
    assert not lib.teadj_has(b'pressure_tendency') and 'pressure_tendency' in full - names


def test_control_map_and_its_adjoint():
    """<gradient(L), x> = <L, add(x)>: the fold of the halos is the fill's adjoint."""
    from oracle.adjoint import Control
    run, init = _window_start(16, 12, 10, regular_steps=0)
    g = run.grid
    ctl = Control(run, 0)
    rng = np.random.default_rng(3)
    size = max(run.fields.values()) // 4 + g.count + 64
    x = rng.standard_normal(ctl.size)
    L = rng.standard_normal(size)
    mem = np.zeros(size)
    ctl.add(mem, x)
    assert abs(ctl.gradient(L) @ x - L @ mem) <= 1e-9 * abs(L @ mem)


def test_binary64_adjoint_matches_central_differences():
    """Two core steps on a 16x12x10 grid (nsound 8): the directional derivative of J from
    the binary64 adjoint equals binary64 central differences along seeded unit
    directions (eps = 1e-5: small enough that the WENO weights stay in their linear
    range, large enough for binary64 rounding)."""
    run, init = _window_start(16, 12, 10)
    ctl, grad, J = _cpu_gradient(run, init, 2)
    assert J > 0 and np.isfinite(grad).all()
    rng = np.random.default_rng(5)
    for _ in range(3):
        d = rng.standard_normal(ctl.size)
        d /= np.linalg.norm(d)
        fd = _fd(run, init, ctl, d, 1e-5, 2)
        ad = float(grad @ d)
        assert abs(fd - ad) <= 1e-5 * abs(fd), (fd, ad)


# ------------------------------------------------------------------ GPU

def _gpu_window(run, init, nsteps, every):
    from thunderengine_web_b200.adjoint import CoreWindow
    return CoreWindow(run, init, nsteps, checkpoint_every=every)


def _controls(run, init):
    g = run.grid
    arena = np.frombuffer(init[run.rec.ids['arena']], dtype=np.float32)
    out = []
    for name in ('th', 'u', 'v'):
        off = run.fields[name] // 4
        out.append(arena[off:off + g.count].reshape(g.nz + 1, g.strideK, g.strideJ)[:g.nz, 3:3 + g.ny, 3:3 + g.nx].copy())
    return out


@pytest.mark.gpu
def test_gpu_adjoint_matches_binary64_adjoint_and_differences():
    """24x20x16, 4 core steps, checkpoints every 2: the GPU's binary32 gradient against the
    binary64 adjoint around the same (binary32) trajectory (relative 2-norm error per
    control field), and its directional derivatives against binary64 central differences
    of the binary64 step along seeded directions (the two trajectories differ by rounding,
    which the WENO weights' derivatives amplify where stencil values are nearly equal)."""
    run, init = _window_start(24, 20, 16)
    g = run.grid
    # the binary64 adjoint around the binary32 trajectory, which the GPU follows bit for bit
    ctl, grad64, J = _cpu_gradient(run, init, 4, linearize='f32')
    win = _gpu_window(run, init, 4, 2)
    th, u, v = _controls(run, init)
    w = win.forward(th, u, v)
    dV = g.dx * g.dy * g.dz
    J32 = float((w.astype(np.float64) ** 2).sum()) * dV
    assert abs(J32 - J) <= 1e-4 * J
    gth, gu, gv = win.backward(2.0 * w.astype(np.float64) * dV)
    grad32 = np.concatenate([gth.ravel(), gu.ravel(), gv.ravel()]).astype(np.float64)
    n = g.nz * g.ny * g.nx
    errs = [float(np.linalg.norm(grad32[q * n:(q + 1) * n] - grad64[q * n:(q + 1) * n]) /
                  np.linalg.norm(grad64[q * n:(q + 1) * n])) for q in range(3)]
    assert max(errs) <= 1e-5, errs
    # against central differences of the binary64 step: the binary32 and binary64
    # trajectories part by rounding, and the WENO weights' derivatives amplify that where
    # stencil values are nearly equal, so the gradients of the two models differ by
    # ~1e-3..1e-2 per field (the binary64 adjoint itself meets its own differences to
    # ~1e-7: test_binary64_adjoint_matches_central_differences)
    rng = np.random.default_rng(9)
    rel = []
    for _ in range(2):
        d = rng.standard_normal(ctl.size)
        d /= np.linalg.norm(d)
        fd = _fd(run, init, ctl, d, 1e-5, 4)
        rel.append(abs(float(grad32 @ d) - fd) / abs(fd))
    assert max(rel) <= 0.1, (errs, rel)
    print('gradient error against the binary64 adjoint per field', errs, 'directional vs binary64 FD', rel)
    win.close()


@pytest.mark.gpu
def test_gpu_adjoint_leaves_the_start_state_and_ignores_the_checkpoint_interval():
    """After backward the memory is the window's start state, bit for bit; the forward's
    end state equals plain steps of the same tape; the gradient does not depend on the
    checkpoint interval (up to the order of the binary32 atomic sums)."""
    run, init = _window_start(24, 20, 16)
    g = run.grid
    th, u, v = _controls(run, init)
    grads = []
    for every in (1, 3):
        win = _gpu_window(run, init, 5, every)
        w = win.forward(th, u, v)
        end = win.r.read(win.r.buffers_end)
        plain = helpers.gpu_replayer(run.tape(1, core=True), init, hashes=False)
        plain.encode_steps(5)
        assert np.array_equal(plain.read(plain.buffers_end), end)
        plain.close()
        grads.append(win.backward(2.0 * w.astype(np.float64)))
        # memory is back at the start state
        start = win.r.read(win.r.buffers_end)
        ref = helpers.gpu_replayer(run.tape(1, core=True), init, hashes=False)
        assert np.array_equal(start, ref.read(ref.buffers_end))
        ref.close()
        win.close()
    for a, b in zip(grads[0], grads[1]):
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b)


@pytest.mark.gpu
def test_autograd_function_gives_the_window_gradient():
    """core_window_function(): torch.autograd over the window returns, for J = sum w^2,
    the gradients CoreWindow.backward gives for dJ/dw = 2 w."""
    import torch
    from thunderengine_web_b200.adjoint import core_window_function
    run, init = _window_start(24, 20, 16)
    th, u, v = _controls(run, init)
    win = _gpu_window(run, init, 3, 2)
    Window = core_window_function()
    xs = [torch.tensor(x, device='cuda', requires_grad=True) for x in (th, u, v)]
    w = Window.apply(*xs, win)
    (w.double() ** 2).sum().backward()
    want = win.backward(2.0 * w.detach().cpu().numpy().astype(np.float64))
    for x, ref in zip(xs, want):
        assert x.grad is not None
        np.testing.assert_allclose(x.grad.cpu().numpy(), ref, rtol=1e-5, atol=1e-6 * np.abs(ref).max())
    win.close()
