"""Binary64 CPU adjoint and finite differences of the dynamics-core step (TEST
INFRASTRUCTURE ONLY: tests/ and bench.py's adjoint check use it).

* ``CpuAdjoint64`` runs the step forward on the binary64 twin of the oracle
  (``CpuPlayer64``) and backward with the library's adjoint operators instantiated in
  binary64 (``oracle/libadjoint64.so``), by the same scheme as the GPU: per step, replay
  op by op saving each op's written regions, then walk the ops in reverse restoring
  them and applying each op's adjoint.
* ``Control`` maps the control vector (interior th', u, v at the window's start) into
  the arena (both the current and the start-of-step copy of each, halos filled
  periodically) and folds adjoints back (the adjoint of that map).
* ``cost_w2`` is the cost J = sum over interior w faces of w^2 dx dy dz at the final
  time, and ``seed_w2`` its gradient with respect to memory.
"""
import ctypes
import os

import numpy as np

from oracle.player import CpuPlayer64

HERE = os.path.dirname(os.path.abspath(__file__))
ADJ_SO = os.path.join(HERE, 'libadjoint64.so')

_LIB = None


def adjoint_lib():
    global _LIB
    if _LIB is None:
        lib = ctypes.CDLL(ADJ_SO)
        lib.teadj_run.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_uint64, ctypes.c_int]
        lib.teadj_run.restype = ctypes.c_int
        lib.teadj_has.argtypes = [ctypes.c_char_p]
        lib.teadj_has.restype = ctypes.c_int
        _LIB = lib
    return _LIB


class CpuAdjoint64:
    """``linearize='f64'``: the forward and the states the adjoint operators see are the
    binary64 twin's.  ``linearize='f32'``: they are the binary32 oracle's (the trajectory
    the GPU follows bit for bit), widened to binary64 for the adjoint operators - the
    binary64 adjoint around the GPU's own trajectory."""

    def __init__(self, tape, kernels_meta, init, linearize='f64', kernels32=None):
        self.km = kernels_meta
        self.f32 = linearize == 'f32'
        self.k32 = kernels32
        self.p = CpuPlayer64(tape, kernels_meta)
        self.p.plan()
        for i, b in init.items():
            self.p.upload(i, b)
        self.p.values_from_words()
        self.lib = adjoint_lib()
        self.info = []
        for o in self.p.ops:
            if o.kind == 'copy':
                self.info.append((0, 0, [(o.dst, o.n)]))
                continue
            if not self.lib.teadj_has(o.name.encode()):
                raise RuntimeError('no adjoint operator for ' + o.name)
            params = self.km[o.name]['params']
            mask = 0
            regions = []
            for prm in params:
                if prm['kind'] == 'ptr':
                    mask |= 1 << prm['index']
                    if prm['write'] and prm['index'] in o.bind:
                        off = o.bind[prm['index']]
                        regions.append((off, self.p.region_len(off)))
            self.info.append((mask, 1 if o.name.startswith('acoustic_') else 0, regions))
        self.states = []

    @property
    def D(self):
        return self.p.D

    def _step(self):
        """One forward step of the chosen trajectory (D mirrors M in binary32 mode)."""
        if self.f32:
            p = self.p
            mp = p.M.ctypes.data_as(ctypes.c_void_p)
            for o in p.ops:
                if o.kind == 'copy':
                    p.M[o.dst:o.dst + o.n] = p.M[o.src:o.src + o.n]
                else:
                    self.k32(o.name)(mp, o.arg.ctypes.data_as(ctypes.c_void_p))
            p.D[:] = p.M.view(np.float32)
        else:
            self.p.run64(1)

    def _state(self):
        return (self.p.M.copy(), self.p.D.copy()) if self.f32 else self.p.D.copy()

    def _set_state(self, st):
        if self.f32:
            self.p.M[:] = st[0]
            self.p.D[:] = st[1]
        else:
            self.p.D[:] = st

    def forward(self, nsteps, checkpoint_every=None):
        """Runs nsteps steps from the current state, keeping the start state of every
        `checkpoint_every`-th step (every step by default)."""
        self.every = checkpoint_every or 1
        self.nsteps = nsteps
        self.ckpt = {}
        for s in range(nsteps):
            if s % self.every == 0:
                self.ckpt[s] = self._state()
            self._step()

    def _step_starts(self, b):
        """Start states of the steps of block b, replayed from its checkpoint."""
        s0, s1 = b * self.every, min((b + 1) * self.every, self.nsteps)
        self._set_state(self.ckpt[s0])
        out = []
        for s in range(s0, s1):
            out.append(self._state())
            if s + 1 < s1:
                self._step()
        return out

    def backward(self, L):
        """L: adjoint of the final state (float64, memory layout); returns the adjoint of
        the state before the first step of the last forward()."""
        p = self.p
        mp = p.M.ctypes.data_as(ctypes.c_void_p)
        dp = p.D.ctypes.data_as(ctypes.c_void_p)
        L = np.ascontiguousarray(L, dtype=np.float64)
        lp = L.ctypes.data_as(ctypes.c_void_p)
        nb = (self.nsteps + self.every - 1) // self.every
        for b in range(nb - 1, -1, -1):
            starts = self._step_starts(b)
            for start in starts[::-1]:
                p.lib64.te64_bind(dp)
                self._reverse_step(start, L, mp, dp, lp)
        return L

    def _reverse_step(self, start, L, mp, dp, lp):
        p = self.p
        self._set_state(start)
        log = []
        for o, (mask, acu, regions) in zip(p.ops, self.info):
            log.append([(p.D[off:off + n].copy(), p.M[off:off + n].copy() if self.f32 else None)
                        for off, n in regions])
            if o.kind == 'copy':
                p.D[o.dst:o.dst + o.n] = p.D[o.src:o.src + o.n]
                p.M[o.dst:o.dst + o.n] = p.M[o.src:o.src + o.n]
            elif self.f32:
                self.k32(o.name)(mp, o.arg.ctypes.data_as(ctypes.c_void_p))
                for off, n in regions:
                    p.D[off:off + n] = p.M[off:off + n].view(np.float32)
            else:
                p.kernel(o.name)(mp, o.arg.ctypes.data_as(ctypes.c_void_p))
        for oi in range(len(p.ops) - 1, -1, -1):
            o = p.ops[oi]
            mask, acu, regions = self.info[oi]
            for (off, n), (saved, saved32) in zip(regions, log[oi]):
                p.D[off:off + n] = saved
                if saved32 is not None:
                    p.M[off:off + n] = saved32
            if o.kind == 'copy':
                x = L[o.dst:o.dst + o.n].copy()
                L[o.dst:o.dst + o.n] = 0.0
                L[o.src:o.src + o.n] += x
            else:
                rc = self.lib.teadj_run(o.name.encode(), mp, dp, lp, o.arg.ctypes.data_as(ctypes.c_void_p),
                                        ctypes.c_uint64(mask), acu)
                if rc != 0:
                    raise RuntimeError('adjoint failed for ' + o.name)


class Control:
    """Interior th', u, v at the window's start <-> the arena of a Run."""
    FIELDS = ('th', 'u', 'v')

    def __init__(self, run, base):
        self.run = run
        self.base = base
        g = run.grid
        self.shape = (g.nz, g.ny, g.nx)
        self.size = 3 * g.nz * g.ny * g.nx

    def view(self, mem, name):
        g = self.run.grid
        off = self.base + self.run.fields[name] // 4
        return mem[off:off + g.count].reshape(g.nz + 1, g.strideK, g.strideJ)

    @staticmethod
    def _fill_halo(f, g):
        """Periodic halo images of the interior (the bc_periodic_x then _y pair)."""
        nx, ny = g.nx, g.ny
        for i in list(range(-3, 0)) + list(range(nx, nx + 4)):
            f[:, 3:3 + ny, i + 3] = f[:, 3:3 + ny, (i % nx) + 3]
        for j in list(range(-3, 0)) + list(range(ny, ny + 4)):
            f[:, j + 3, :] = f[:, (j % ny) + 3, :]

    @staticmethod
    def _fold_halo(f, g):
        """Adjoint of _fill_halo: halo adjoints added to their interior images."""
        nx, ny = g.nx, g.ny
        f = f.copy()
        for j in list(range(ny, ny + 4))[::-1] + list(range(-3, 0))[::-1]:
            f[:, (j % ny) + 3, :] += f[:, j + 3, :]
            f[:, j + 3, :] = 0.0
        for i in list(range(nx, nx + 4))[::-1] + list(range(-3, 0))[::-1]:
            f[:, 3:3 + ny, (i % nx) + 3] += f[:, 3:3 + ny, i + 3]
            f[:, 3:3 + ny, i + 3] = 0.0
        return f

    def add(self, mem, x, eps=1.0):
        """mem (float array, memory layout) += eps * x in both copies of th', u, v."""
        g = self.run.grid
        nz, ny, nx = self.shape
        parts = np.split(np.asarray(x, dtype=np.float64), 3)
        for name, part in zip(self.FIELDS, parts):
            d = np.zeros((g.nz + 1, g.strideK, g.strideJ))
            d[:nz, 3:3 + ny, 3:3 + nx] = part.reshape(self.shape) * eps
            self._fill_halo(d, g)
            for f in (name, name + '_a'):
                v = self.view(mem, f)
                v += d.astype(v.dtype)

    def gradient(self, L):
        """Adjoint of add(): the gradient with respect to the control vector."""
        g = self.run.grid
        nz, ny, nx = self.shape
        out = []
        for name in self.FIELDS:
            tot = np.zeros((g.nz + 1, g.strideK, g.strideJ))
            for f in (name, name + '_a'):
                tot += self.view(L, f).astype(np.float64)
            tot = self._fold_halo(tot, g)
            out.append(tot[:nz, 3:3 + ny, 3:3 + nx].ravel())
        return np.concatenate(out)


def cost_w2(run, mem, base):
    """J = sum over interior faces k = 1..nz-1 of w^2 dx dy dz."""
    g = run.grid
    off = base + run.fields['w'] // 4
    w = mem[off:off + g.count].reshape(g.nz + 1, g.strideK, g.strideJ)[1:g.nz, 3:3 + g.ny, 3:3 + g.nx]
    w = w.astype(np.float64)
    return float((w * w).sum()) * g.dx * g.dy * g.dz


def seed_w2(run, mem, base, size):
    """dJ/d(memory) at the final state (float64, memory layout of `size` words)."""
    g = run.grid
    L = np.zeros(size, dtype=np.float64)
    off = base + run.fields['w'] // 4
    w = mem[off:off + g.count].reshape(g.nz + 1, g.strideK, g.strideJ).astype(np.float64)
    lw = L[off:off + g.count].reshape(g.nz + 1, g.strideK, g.strideJ)
    lw[1:g.nz, 3:3 + g.ny, 3:3 + g.nx] = 2.0 * w[1:g.nz, 3:3 + g.ny, 3:3 + g.nx] * g.dx * g.dy * g.dz
    return L
