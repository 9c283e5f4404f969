"""Forward/backward pair of a window of dynamics-core steps on the GPU (the discrete
adjoint; no counterpart in the reference).

The dynamics-core step (``timestep.Run(cfg, core=True).tape(1, core=True)``) is the
large step of the reference's ``TimeStep.encode`` (web/core/timestep.js:797-2201)
restricted to the WENO / upwind advection of th', u, v, w, the acoustic substeps and the
buoyancy coupling, with the thermodynamic coefficients (thv, ppterm, piadv, thterm, qk,
pk1, pk2, mm, ppten) held at their values when the window starts.  ``CoreWindow``
plays ``nsteps`` of it from a start state with the library's C-ABI
(``te_adjoint_forward``: checkpoints every ``checkpoint_every`` steps) and returns the
vertical velocity at the end; its ``backward`` turns d(cost)/d(w at the end) into
d(cost)/d(th', u, v at the start) with ``te_adjoint_backward``.  ``CoreWindowFunction``
wraps the pair as a ``torch.autograd.Function``.

Control and output layout: interior arrays indexed [k, j, i] - th', u, v of shape
(nz, ny, nx) (u at the west face of cell i, v at the south face of cell j), w of shape
(nz - 1, ny, nx) (faces k = 1..nz-1).  A control value sets both the current and the
start-of-step copy of the field (th/th_a, ...), halos filled periodically.
"""
import numpy as np

from .replayer import Replayer

FIELDS = ('th', 'u', 'v')


def _fill_halo(f, nx, ny):
    """Periodic halo images of the interior of a (levels, ny+7, nx+7) array."""
    for i in list(range(-3, 0)) + list(range(nx, nx + 4)):
        f[:, 3:3 + ny, i + 3] = f[:, 3:3 + ny, (i % nx) + 3]
    for j in list(range(-3, 0)) + list(range(ny, ny + 4)):
        f[:, j + 3, :] = f[:, (j % ny) + 3, :]


def _fold_halo(f, nx, ny):
    """Adjoint of _fill_halo: halo values added onto their interior images (in place)."""
    for j in list(range(ny, ny + 4))[::-1] + list(range(-3, 0))[::-1]:
        f[:, (j % ny) + 3, :] += f[:, j + 3, :]
        f[:, j + 3, :] = 0.0
    for i in list(range(nx, nx + 4))[::-1] + list(range(-3, 0))[::-1]:
        f[:, 3:3 + ny, (i % nx) + 3] += f[:, 3:3 + ny, i + 3]
        f[:, 3:3 + ny, i + 3] = 0.0


class CoreWindow:
    """``nsteps`` dynamics-core steps of ``run`` (a ``timestep.Run`` made with core=True)
    from the start state ``init`` (buffer id -> bytes: the memory the window starts from,
    whose thermodynamic coefficients it keeps)."""

    def __init__(self, run, init, nsteps, checkpoint_every=10, device=0):
        if not run.core:
            raise ValueError('CoreWindow needs a timestep.Run made with core=True')
        self.run = run
        self.nsteps = int(nsteps)
        self.every = int(checkpoint_every)
        self.r = Replayer(run.tape(1, core=True), None, device=device)
        self.r.plan(False)
        self.r.build()
        self.init = dict(init)
        self.aid = run.rec.ids['arena']
        self.base = self.r.base[self.aid]
        g = run.grid
        self.g = g
        self.arena0 = np.frombuffer(self.init[self.aid], dtype=np.float32).copy()

    def close(self):
        self.r.close()

    def _field(self, arena, name):
        g = self.g
        off = self.run.fields[name] // 4
        return arena[off:off + g.count].reshape(g.nz + 1, g.strideK, g.strideJ)

    def forward(self, th, u, v):
        """Sets the start state from the controls (numpy or torch, shape (nz, ny, nx)),
        runs the window keeping checkpoints and returns w at the end, shape
        (nz - 1, ny, nx), float32 numpy."""
        self.load(th, u, v)
        self.run_forward()
        return self.read_w()

    def load(self, th, u, v):
        """Uploads the start state with the controls th', u, v (no steps run)."""
        g = self.g
        arena = self.arena0.copy()
        for name, x in zip(FIELDS, (th, u, v)):
            x = x.detach().cpu().numpy() if hasattr(x, 'detach') else np.asarray(x)
            for f in (name, name + '_a'):
                a = self._field(arena, f)
                a[:g.nz, 3:3 + g.ny, 3:3 + g.nx] = x.astype(np.float32)
                _fill_halo(a, g.nx, g.ny)
        for i, b in self.init.items():
            if i != self.aid:
                self.r.upload(i, b)
        self.r.upload(self.aid, arena.tobytes())

    def run_forward(self):
        """The window from the loaded start state, keeping checkpoints (device work only)."""
        self.r.adjoint_forward(self.nsteps, self.every)

    def read_w(self):
        """w at the end of the window, shape (nz - 1, ny, nx)."""
        g = self.g
        w = self.r.read(g.count, self.base + self.run.fields['w'] // 4).view(np.float32)
        return w.reshape(g.nz + 1, g.strideK, g.strideJ)[1:g.nz, 3:3 + g.ny, 3:3 + g.nx].copy()

    def backward(self, grad_w):
        """d(cost)/d(w at the end), shape (nz - 1, ny, nx) -> the gradients with respect to
        the th', u, v controls (float32 numpy, shape (nz, ny, nx) each).  Memory returns to
        the start state."""
        g = self.g
        gw = grad_w.detach().cpu().numpy() if hasattr(grad_w, 'detach') else np.asarray(grad_w)
        lw = np.zeros((g.nz + 1, g.strideK, g.strideJ), dtype=np.float32)
        lw[1:g.nz, 3:3 + g.ny, 3:3 + g.nx] = gw
        self.r.adjoint_zero()
        self.r.adjoint_write_words(self.base + self.run.fields['w'] // 4, lw.ravel())
        self.r.adjoint_backward()
        out = []
        for name in FIELDS:
            tot = np.zeros((g.nz + 1, g.strideK, g.strideJ), dtype=np.float64)
            for f in (name, name + '_a'):
                tot += self.r.adjoint_read(g.count, self.base + self.run.fields[f] // 4).reshape(tot.shape)
            _fold_halo(tot, g.nx, g.ny)
            out.append(tot[:g.nz, 3:3 + g.ny, 3:3 + g.nx].astype(np.float32))
        return tuple(out)


def core_window_function():
    """``torch.autograd.Function`` over a CoreWindow: apply(th, u, v, window) -> w."""
    import torch

    class CoreWindowFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, th, u, v, window):
            ctx.window = window
            ctx.device = th.device
            return torch.from_numpy(window.forward(th, u, v)).to(th.device)

        @staticmethod
        def backward(ctx, grad_w):
            gth, gu, gv = ctx.window.backward(grad_w)
            dev = ctx.device
            return torch.from_numpy(gth).to(dev), torch.from_numpy(gu).to(dev), torch.from_numpy(gv).to(dev), None

    return CoreWindowFunction
