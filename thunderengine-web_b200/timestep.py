"""Step encoder: the command tape of one CM1 large step (dynamics hot path).

Host-side restatement of ``TimeStep.encode`` (web/core/timestep.js:797-2201) for the
configuration this project accelerates: moist scalars [th, qv], momentum [u, v, w],
WENO on the last RK stage for scalars and momentum, periodic lateral boundaries, no
turbulence / Rayleigh / microphysics / radiation / terrain, pressure tendency on.
The tape format is the reference recorder's (web/core/gpu.js:48-96): a list of
``pipe | buf | bufoff | bytes | dispatch | end | copy`` commands with buffers numbered
by first use, so the same tape plays on the reference player (web/replay.js) and on
this project's CUDA player.

Parameter structs are packed as ``pack()`` does (timestep.js:22-36): ``GridDims``
(timestep.js:88-90), ``AcousticParamsGPU`` (timestep.js:46-52), and the acoustic
substep schedule is ``AcousticSchedule`` (timestep.js:54-86).
"""
import base64
import math
import struct

import numpy as np

from . import scenario as sc

F = np.float32
H = sc.HALO
TG3 = [32, 4, 1]
TGC = [32, 1, 1]


def f(x):
    return float(np.float32(x))


def pack(fmt, vals):
    out = b''
    for c, v in zip(fmt, vals):
        if c == 'f':
            out += struct.pack('<f', float(np.float32(v)))
        elif c == 'i':
            out += struct.pack('<i', int(v))
        elif c == 'u':
            out += struct.pack('<I', int(v) & 0xFFFFFFFF)
        else:
            out += struct.pack('<d', float(v))
    return out


def F1(v):
    return pack('f', [v])


def I1(v):
    return pack('i', [v])


def I2(v):
    return pack('ii', v)


def round_half_away(x):
    return math.copysign(math.floor(abs(x) + 0.5), x)


class AcousticSchedule:
    """Substep loops per RK stage (timestep.js:74-86)."""

    def __init__(self, n, dt):
        self.nsound = n
        self.dt = dt
        n1 = max(int(round_half_away(n / 3.0)), 1)
        d1 = dt / (n1 * 3.0)
        if d1 > dt / n:
            n1 += 1
            d1 = dt / (n1 * 3.0)
        self.loops = [(n1, d1), (n // 2, dt / n), (n, dt / n)]

    @property
    def total(self):
        return sum(c for c, _ in self.loops)


class AdaptiveTimeStep:
    """The adaptive time step of the reference's driver (web/core/adaptive.js, CM1
    getnewdt misclibs.F:543-742 and dtsmall :750-847): after each large step the host
    reads cflmax and ksmax from the 8-byte stability buffer (stability_max), picks the next
    dt (limited to a 10 % increase, CFL 1, the diffusion limit and 2 dtl) and its acoustic
    substep count.  Arithmetic as the reference: binary32 where it rounds with fround,
    binary64 elsewhere.  Output clocks (tape, stat, ...) are not modelled: every clock
    frequency is absent, which is the reference's behaviour for a run without output."""
    MAX_NSOUND = 192

    def __init__(self, dtl, min_horizontal_spacing, two_dimensional=False, min_vertical_spacing=None,
                 ks_check=True):
        self.dtl = f(dtl)
        self.ks_check = ks_check
        self.dtsm = self.small_step(min_horizontal_spacing, min_vertical_spacing, two_dimensional)
        self.ks_limit = f(0.18) if two_dimensional else f(f(0.18) / f(2.0))
        self.dbldt = float(self.dtl)
        self.dt = self.dtl
        self.dtlast = self.dt
        self.nsound = 0
        self.cflmax = 0.0
        self.ksmax = 0.0

    @staticmethod
    def small_step(dh, dv=None, two_d=False):
        """AcousticSchedule.smallStep (config.js:239-243)."""
        if dv is None:
            return f(f(f(0.60) * f(dh)) / f(360.0))
        m = f(min(dh, dv))
        return f(f((f(0.60) if two_d else f(0.50)) * m) / f(360.0))

    def start(self, cflmax, ksmax):
        self.getnewdt(cflmax, ksmax)

    def end_step(self, cflmax, ksmax):
        self.getnewdt(cflmax, ksmax)

    def getnewdt(self, c_in, k_in):
        cfl_limit, max_change = f(1.00), f(0.10)
        self.dtlast = self.dt
        cfl = f(max(c_in, f(1.0e-10)))
        ks = f(k_in)
        if cfl > cfl_limit:
            self.dbldt = self.dbldt * f(cfl_limit / cfl)
        else:
            self.dbldt = self.dbldt * min(f(f(1.0) + max_change), f(cfl_limit / cfl))
        if self.ks_check and (ks * self.dbldt / self.dt) > self.ks_limit:
            self.dbldt = min(self.dbldt, f(f(self.dt * self.ks_limit) / max(f(1.0e-10), ks)))
        self.dbldt = min(self.dbldt, f(f(2.0) * self.dtl))
        self.dt = f(self.dbldt)
        self.dtsmall()
        tem = f(self.dt / self.dtlast)
        self.cflmax = f(cfl * tem)
        self.ksmax = f(ks * tem)

    def dtsmall(self):
        x = self.dbldt / self.dtsm
        n = max(int(math.copysign(1, x) * round_half_away(abs(x))), 4)
        if n % 2 != 0:
            n += 1
        if self.dbldt / f(n) > self.dtsm:
            n += 2
        if n > self.MAX_NSOUND:
            n = self.MAX_NSOUND
            self.dbldt = f(f(n) * self.dtsm)
            self.dt = f(self.dbldt)
        self.nsound = n


def stability_from_words(words, two_dimensional=False):
    """cflmax, ksmax from the 2 words of the stability buffer (adaptive.js:104-110): the
    kernel reduces squares, the square root is taken here."""
    fl = np.asarray(words, dtype=np.uint32).view(np.float32)
    cfl = f(math.sqrt(float(fl[0])))
    ks = float(fl[1]) if two_dimensional else f(math.sqrt(float(fl[1])))
    return cfl, ks


def weno_epsilon(name):
    """timestep.js:387-392"""
    eps = f(1.0e-18)
    if name in ('th', 'tke'):
        return f(10 * eps)
    if name in ('nci', 'ncs', 'ncr', 'ncg'):
        return f(1.0e6 * eps)
    return f(f(1.0e-2) * eps)


class Recorder:
    """Command list with buffers numbered by first use (web/core/gpu.js:48-57)."""

    def __init__(self):
        self.ids = {}
        self.buffers = []
        self.commands = []

    def id(self, name):
        if name not in self.ids:
            self.ids[name] = len(self.buffers)
            self.buffers.append(name)
        return self.ids[name]


STATE_FIELDS_MOIST = ['th', 'qv', 'u', 'v', 'w', 'th_a', 'qv_a', 'u_a', 'v_a', 'w_a',
                      'ppterm', 'piadv', 'thv', 'pp3d', 'ppi', 'ppd', 'ppx', 'uten', 'vten', 'wten', 'ppten',
                      'buoy', 'prs', 'rho', 'thterm', 'div3d', 'qpten', 'qtten', 'qvten', 'qcten', 'qvten_t',
                      'qc', 'qzero']
# the dry step's state (Fields.stateFields, timestep.js:324-332, with scalars = [th])
STATE_FIELDS_DRY = ['th', 'u', 'v', 'w', 'th_a', 'u_a', 'v_a', 'w_a',
                    'ppterm', 'piadv', 'thv', 'pp3d', 'ppi', 'ppd', 'ppx', 'uten', 'vten', 'wten', 'ppten',
                    'buoy', 'prs', 'rho']
SCRATCH_FIELDS = ['rru', 'rrv', 'rrw', 'fx', 'fy', 'fz', 'tend', 'divx', 'qk', 'pk1', 'pk2', 'mm', 'fpk', 'cA',
                  'cB', 'sadv']


# Sink fields of the dynamics-core step: update_diagnostics_moist writes its thv, ppterm,
# piadv and thterm here, so those coefficients keep their window-start values.
CORE_SINKS = ['xthv', 'xppterm', 'xpiadv', 'xthterm']


class Run:
    """A synthetic run: grid, profiles, arena and the encoder state (driver.buildRun).

    ``arena_fields`` are sorted by name, as the reference scenario builder does
    (scenario.js:110-119).  ``qc`` is kept (zero) because the diabatic glue kernels of
    a moist step bind it (timestep.js:1473-1479).
    """

    def __init__(self, cfg, weno_momentum=True, core=False, moist=True, adaptive=False):
        self.cfg = cfg
        self.core = core
        self.moist = moist
        self.adaptive = adaptive
        if core and not moist:
            raise ValueError('the dynamics-core step is defined on the moist step')
        self.grid = sc.Grid(cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.dy, cfg.dz,
                            align_rows=getattr(cfg, 'align_rows', False))
        self.prof = sc.profiles(cfg, dry=not moist)
        self.dt = f(cfg.dt)
        self.schedule = AcousticSchedule(cfg.nsound, self.dt)
        self.weno_scalars = True
        self.weno_momentum = weno_momentum
        state = STATE_FIELDS_MOIST if moist else STATE_FIELDS_DRY
        names = sorted(set(state + SCRATCH_FIELDS + (CORE_SINKS if core else [])), key=lambda s: s.encode())
        g = self.grid
        self.fields = {n: i * g.field_stride for i, n in enumerate(names)}
        self.arena_bytes = g.field_stride * len(names)
        vg = self.prof['vg']
        self.host = {
            'hmetric': g.metric_values(),
            'c1': vg.c1, 'c2': vg.c2, 'mh': vg.mh, 'mf': vg.mf,
            'rho0': self.prof['rho0'], 'rr0': self.prof['rr0'], 'rf0': self.prof['rf0'],
            'th0': self.prof['th0'], 'pi0': self.prof['pi0'], 'rth0': self.prof['rth0'],
            'qv0': self.prof['qv0'], 'qc0': self.prof['qc0'], 'qi0': self.prof['qi0'],
        }
        if adaptive:
            self.host['stability'] = np.zeros(2, F)   # cflmax^2, ksmax bits (timestep.js:706-709)
        self.rec = Recorder()
        self.acoustic = dict(dts=f(0.1), alph=f(0.6), beta=f(1.0 - f(0.6)), kdiv=f(0.1), smeps=f(0.0))

    # ---- initial state
    def initial_arena(self):
        arena = np.zeros(self.arena_bytes // 4, dtype=F)
        sc.fill_arena(self.cfg, self.grid, self.prof, arena, self.fields)
        return arena

    def buffer_bytes(self, name, arena=None):
        if name == 'arena':
            return (arena if arena is not None else self.initial_arena()).tobytes()
        return np.asarray(self.host[name], dtype=F).tobytes()

    def buffer_length(self, name):
        if name == 'arena':
            return self.arena_bytes
        return np.asarray(self.host[name], dtype=F).nbytes

    # ---- encoding (timestep.js:797-2201, hot-path subset)
    def dims_bytes(self):
        g = self.grid
        return pack('iiiiifff', [g.nx, g.ny, g.nz, g.strideJ, g.strideK, f(1.0 / g.dx), f(1.0 / g.dy),
                                 f(1.0 / g.dz)])

    def acoustic_bytes(self):
        a = self.acoustic
        return pack('fffff', [a['dts'], a['alph'], a['beta'], a['kdiv'], a['smeps']])

    def encode(self, core=False):
        """Commands of one large step.

        ``core=True`` encodes the dynamics-core step that the discrete adjoint
        differentiates: the same kernels and order, with the thermodynamic fields held at
        their values when the window starts - no pressure_tendency (ppten fixed),
        update_diagnostics_moist writing thv, ppterm, piadv and thterm to sink fields
        (only its buoyancy is live), so acoustic_prepare forms each stage's implicit
        coefficients from fixed fields and that stage's dts - and without the moisture
        and diabatic kernels (qv advection and its pdef correction, diabatic_*,
        update_rho_prs).  The state it advances is th', u, v, w, pi' (pp3d, ppi, ppx).
        Needs a Run made with core=True.
        """
        if core and not self.core:
            raise ValueError('the dynamics-core step needs Run(..., core=True) (its sink fields)')
        cmds = []
        rec = self.rec
        g = self.grid
        dims = self.dims_bytes()

        def buf(name, index, offset=0):
            cmds.append({'op': 'buf', 'index': index, 'buf': rec.id(name), 'offset': offset})

        def fld(name, index):
            buf('arena', index, self.fields[name])

        def by(data, index):
            cmds.append({'op': 'bytes', 'index': index, 'data': base64.b64encode(data).decode()})

        def enc(kernel, gs, tg, acoustic, bind):
            cmds.append({'op': 'pipe', 'name': kernel})
            by(dims, 0)
            buf('hmetric', 30)
            if acoustic:
                by(self.acoustic_bytes(), 1)
            bind()
            cmds.append({'op': 'dispatch', 'kind': 'threads', 'grid': list(gs), 'tg': list(tg)})

        nx, ny, nz = g.nx, g.ny, g.nz
        full = [nx, ny, nz]
        fullU = [nx + 1, ny, nz]
        fullV = [nx, ny + 1, nz]
        fullW = [nx, ny, nz + 1]
        stag = [nx + 1, ny + 1, nz]
        cols = [nx, ny, 1]
        whole = [g.strideJ, g.strideK, nz + 1]
        open_ = I2([0, 0])
        fcor_axi = F1(0.0)
        dt = self.dt

        def halo_fill(name):
            enc('bc_periodic_x', [H + 1, ny + 1 + 2 * H, nz + 1], [H + 1, 8, 1], False, lambda: fld(name, 1))
            enc('bc_periodic_y', [H + 1, nx + 1 + 2 * H, nz + 1], [H + 1, 8, 1], False, lambda: fld(name, 1))

        def compute_div():
            def b():
                for i, n in enumerate(['rru', 'rrv', 'rrw']):
                    fld(n, i + 1)
                buf('mh', 4)
                fld('divx', 5)
            enc('div_massflux', whole, TG3, False, b)

        # pressure tendency (timestep.js:1507-1531)
        moist = self.moist

        def pt():
            for i, n in enumerate(['th_a', 'qv_a' if moist else 'th_a', 'rho', 'ppi']):
                fld(n, i + 1)
            fld('ppten', 5)
            fld('qpten' if moist else 'ppten', 6)
            buf('th0', 7)
            buf('pi0', 8)
            by(F1(dt), 9)
            by(I1(0), 10)
            fld('ppten', 11)
            by(I1(0), 12)
            fld('qvten_t' if moist else 'ppten', 13)
            by(I1(1 if moist else 0), 14)
        if not core:
            enc('pressure_tendency', full, TG3, False, pt)

        for nrk in range(3):
            dttmp_v = f(dt / (3 - nrk))
            dttmp = F1(dttmp_v)

            def diag():
                fld('th', 1)
                fld('pp3d', 2)
                for i, n in enumerate(['th0', 'pi0', 'qv0', 'qc0', 'qi0', 'rth0']):
                    buf(n, i + 3)
                for i, n in enumerate(['qv', 'qc', 'qr', 'qi', 'qs', 'qg']):
                    fld('qv' if n == 'qv' else 'qzero', i + 9)
                outs = CORE_SINKS + ['buoy'] if core else ['thv', 'ppterm', 'piadv', 'thterm', 'buoy']
                for i, n in enumerate(outs):
                    fld(n, i + 15)
            def diag_dry():
                fld('th', 1)
                fld('pp3d', 2)
                buf('th0', 3)
                buf('pi0', 4)
                for i, n in enumerate(['thv', 'ppterm', 'piadv']):
                    fld(n, i + 5)
                buf('rth0', 8)
                fld('buoy', 9)
            if moist:
                enc('update_diagnostics_moist', whole, TG3, False, diag)
            else:
                enc('update_diagnostics', whole, TG3, False, diag_dry)

            def rst():
                for i, n in enumerate(['uten', 'vten', 'wten']):
                    fld(n, i + 1)
            enc('stage_tendency_reset', whole, TG3, False, rst)

            def advect(s, stagger=1, dest='tend', accumulate=False, state=None):
                target = state or s
                if stagger == 1:
                    is_theta = target == 'th'
                    if self.weno_scalars and nrk == 2:
                        weps = F1(weno_epsilon(target))
                        pdef = I1(0 if is_theta else 1)
                        pdw = I1(0 if (is_theta or target == 'qv') else 1)

                        def bx():
                            fld(s, 1); fld('rru', 2); by(weps, 3); by(pdef, 4); fld('fx', 5)
                        enc('adv_flux_x_weno', fullU, TG3, False, bx)

                        def byy():
                            fld(s, 1); fld('rrv', 2); by(weps, 3); by(pdef, 4); fld('fy', 5)
                        enc('adv_flux_y_weno', fullV, TG3, False, byy)

                        def bz():
                            fld(s, 1); fld('rrw', 2); buf('c1', 3); buf('c2', 4); by(weps, 5); by(pdef, 6)
                            by(pdw, 7); fld('fz', 8)
                        enc('adv_flux_z_weno', fullW, TG3, False, bz)
                    else:
                        enc('adv_flux_x', fullU, TG3, False, lambda: (fld(s, 1), fld('rru', 2), fld('fx', 3)))
                        enc('adv_flux_y', fullV, TG3, False, lambda: (fld(s, 1), fld('rrv', 2), fld('fy', 3)))
                        enc('adv_flux_z', fullW, TG3, False,
                            lambda: (fld(s, 1), fld('rrw', 2), buf('c1', 3), buf('c2', 4), fld('fz', 5)))
                else:
                    st = I1(stagger)
                    stag_lo = [nx + 2, ny + 2, nz]
                    weno_w = stagger == 4 and s == 'w' and self.weno_momentum and nrk == 2
                    weno_uv = stagger in (2, 3) and self.weno_momentum and nrk == 2
                    if weno_uv:
                        weps = F1(f(100.0 * 1.0e-18))
                        for kernel, flux, rr in (('adv_flux_x_weno_uv', 'fx', 'rru'), ('adv_flux_y_weno_uv', 'fy', 'rrv')):
                            enc(kernel, stag_lo, TG3, False,
                                lambda flux=flux, rr=rr: (by(st, 1), fld(s, 2), fld(rr, 3), by(weps, 4), fld(flux, 5)))
                        enc('adv_flux_z_weno_uv', [nx + 1, ny + 1, nz + 1], TG3, False,
                            lambda: (by(st, 1), fld(s, 2), fld('rrw', 3), buf('c1', 4), buf('c2', 5), by(weps, 6),
                                     fld('fz', 7)))
                    elif weno_w:
                        weps = F1(f(100.0 * 1.0e-18))
                        for kernel, flux, rr in (('adv_flux_x_weno_w', 'fx', 'rru'), ('adv_flux_y_weno_w', 'fy', 'rrv')):
                            enc(kernel, stag_lo, TG3, False,
                                lambda flux=flux, rr=rr: (fld(s, 1), fld(rr, 2), buf('c2', 3), by(weps, 4), fld(flux, 5)))
                        enc('adv_flux_z_weno_w', [nx + 1, ny + 1, nz + 1], TG3, False,
                            lambda: (fld(s, 1), fld('rrw', 2), by(weps, 3), fld('fz', 4)))
                    else:
                        for kernel, flux, gs in (('adv_flux_x_stag', 'fx', stag_lo), ('adv_flux_y_stag', 'fy', stag_lo),
                                                 ('adv_flux_z_stag', 'fz', [nx + 1, ny + 1, nz + 1])):
                            def b(flux=flux):
                                by(st, 1)
                                fld(s, 2)
                                for i, n in enumerate(['rru', 'rrv', 'rrw']):
                                    fld(n, i + 3)
                                buf('c1', 6)
                                buf('c2', 7)
                                fld(flux, 8)
                            enc(kernel, gs, TG3, False, b)
                st = I1(stagger)
                acc = I1(1 if accumulate else 0)
                asm = [nx + (1 if stagger == 2 else 0), ny + (1 if stagger == 3 else 0), nz]

                def ba():
                    by(st, 1)
                    fld(s, 2)
                    for i, n in enumerate(['fx', 'fy', 'fz', 'divx']):
                        fld(n, i + 3)
                    buf('rho0', 7); buf('rf0', 8); buf('mh', 9); buf('mf', 10)
                    fld(dest, 11)
                    by(acc, 12)
                    fld('rru', 13); fld('rrv', 14)
                    buf('c1', 15); buf('c2', 16)
                    by(open_, 17)
                    buf('rr0', 18)
                    fld('tend', 19)
                    by(fcor_axi, 27)
                enc('adv_assemble', asm, TG3, False, ba)
                if accumulate:
                    return
                if stagger == 1 and nrk == 2 and target != 'th':
                    s0 = target + '_a'
                    for dd, names in enumerate((('fx', 'rru', 'pk1'), ('fy', 'rrv', 'pk2'), ('fz', 'rrw', 'fpk'))):
                        def bp(dd=dd, names=names):
                            by(I1(dd), 1); fld(s, 2); fld(s0, 3); fld(names[0], 4); fld(names[1], 5)
                            buf('rho0', 6); buf('mh', 7); by(dttmp, 8); by(open_, 9); fld(names[2], 10)
                        enc('pdef_dum', asm, TG3, False, bp)
                    halo_fill('pk1')
                    halo_fill('pk2')

                    def bq():
                        for i, n in enumerate([s, s0, 'fx', 'fy', 'fz', 'rru', 'rrv', 'rrw', 'pk1', 'pk2', 'fpk']):
                            fld(n, i + 1)
                        buf('rho0', 12); buf('mh', 13); by(dttmp, 14); by(open_, 15); fld('tend', 16)
                    enc('pdef_apply', asm, TG3, False, bq)
                if target == 'th' and moist:
                    enc('apply_thterm', full, TG3, False,
                        lambda: (fld('div3d', 1), fld('thterm', 2), fld('tend', 3)))
                enc('rk_update', asm, TG3, False,
                    lambda: (by(I1(stagger), 1), fld(target + '_a', 2), fld('tend', 3), fld(target, 4), by(dttmp, 5)))
                halo_fill(target)

            # 1. mass fluxes (timestep.js:1902-1912)
            def mfs():
                for i, n in enumerate(['u', 'v', 'w']):
                    fld(n, i + 1)
                buf('rho0', 4)
                buf('rf0', 5)
                for i, n in enumerate(['rru', 'rrv', 'rrw']):
                    fld(n, i + 6)
            enc('massflux_from_state', whole, TG3, False, mfs)
            compute_div()
            # 2. momentum advection (timestep.js:1914-1925)
            for n, s in enumerate(['u', 'v', 'w']):
                advect(s, stagger=n + 2, dest=['uten', 'vten', 'wten'][n], accumulate=True)
            # buoyancy (timestep.js:1945-1952)
            enc('buoyancy_apply', [nx, ny, max(nz - 1, 1)], TG3, False,
                lambda: (fld('buoy', 1), buf('c1', 2), buf('c2', 3), fld('wten', 4)))

            # 3. acoustic substeps (timestep.js:1967-2091)
            def ssr():
                for i, n in enumerate(['u_a', 'v_a', 'w_a', 'ppi']):
                    fld(n, i + 1)
                for i, n in enumerate(['u', 'v', 'w', 'pp3d', 'ppd']):
                    fld(n, i + 5)
                fld('ppx', 10)
            enc('stage_state_reset', whole, TG3, False, ssr)
            nloop, dts = self.schedule.loops[nrk]
            self.acoustic['dts'] = f(dts)

            def prep():
                for i, n in enumerate(['ppterm', 'piadv', 'thv']):
                    fld(n, i + 2)
                buf('rr0', 5); buf('rf0', 6); buf('mh', 7); buf('mf', 8); buf('c1', 9); buf('c2', 10)
                for i, n in enumerate(['qk', 'pk1', 'pk2', 'mm']):
                    fld(n, i + 11)
            enc('acoustic_prepare', full, TG3, True, prep)

            def beg():
                fld('w', 2)
                for i, n in enumerate(['rru', 'rrv', 'rrw']):
                    fld(n, i + 3)
            enc('acoustic_begin', whole, TG3, True, beg)
            for n in range(nloop):
                def uv():
                    for i, nm in enumerate(['ppd', 'thv', 'uten', 'vten', 'u', 'v']):
                        fld(nm, i + 2)
                    by(open_, 8)
                enc('acoustic_uv', stag, TG3, True, uv)
                save_x = I1(1 if nrk == 2 else 0)

                def fpk():
                    for i, nm in enumerate(['u', 'v', 'w', 'piadv', 'ppten', 'ppterm', 'pk1', 'pk2', 'qk', 'fpk']):
                        fld(nm, i + 2)
                    buf('rho0', 15); buf('rr0', 16); buf('rf0', 17)
                enc('acoustic_fpk', full, TG3, True, fpk)

                def ws():
                    for i, nm in enumerate(['pk1', 'pk2', 'qk', 'mm', 'fpk', 'wten', 'pp3d', 'w', 'cA', 'cB']):
                        fld(nm, i + 2)
                enc('acoustic_w_solve', cols, TGC, True, ws)

                def pp():
                    for i, nm in enumerate(['w', 'pk1', 'pk2', 'qk', 'fpk', 'pp3d', 'ppd']):
                        fld(nm, i + 2)
                    fld('ppx', 9)
                    by(save_x, 10)
                enc('acoustic_pp', full, TG3, True, pp)
                halo_fill('ppd')
                tavg = F1(f(1.0 / nloop if n == nloop - 1 else 0.0))

                def accu():
                    for i, nm in enumerate(['u', 'v', 'w', 'rru', 'rrv', 'rrw']):
                        fld(nm, i + 2)
                    by(tavg, 8)
                enc('acoustic_accumulate', whole, TG3, True, accu)
                halo_fill('u')
                halo_fill('v')
                halo_fill('w')
            halo_fill('pp3d')
            if moist:
                enc('divergence3d', full, TG3, False,
                    lambda: ([fld(n, i + 1) for i, n in enumerate(['rru', 'rrv', 'rrw'])], buf('mh', 4), fld('div3d', 5)))
            # 4. averaged velocities -> mass fluxes (timestep.js:2102-2113)
            enc('velocity_to_massflux', whole, TG3, False,
                lambda: (buf('rho0', 1), buf('rf0', 2), [fld(n, i + 3) for i, n in enumerate(['rru', 'rrv', 'rrw'])]))
            compute_div()
            # 5. scalar advection (timestep.js:2115-2127)
            enc('build_sadv', whole, TG3, False, lambda: (buf('th0', 1), fld('th', 2), fld('sadv', 3)))
            advect('sadv', state='th')
            if core:
                continue
            if moist:
                advect('qv')
            if nrk == 2 and not moist:
                enc('update_rho_prs', full, TG3, False,
                    lambda: (by(I1(0), 1), fld('th', 2), fld('pp3d', 3), buf('th0', 4), buf('pi0', 5), fld('th', 6),
                             fld('prs', 7), fld('rho', 8)))
            elif nrk == 2:
                dtb = F1(dt)
                enc('diabatic_unapply', full, TG3, False,
                    lambda: (by(dtb, 1), [fld(n, i + 2) for i, n in
                                          enumerate(['pp3d', 'th', 'qv', 'qc', 'qpten', 'qtten', 'qvten', 'qcten'])]))
                enc('update_rho_prs', full, TG3, False,
                    lambda: (by(I1(1), 1), fld('th', 2), fld('pp3d', 3), buf('th0', 4), buf('pi0', 5), fld('qv', 6),
                             fld('prs', 7), fld('rho', 8)))
        dtb = F1(dt)
        if not core and moist:
            enc('diabatic_rates', full, TG3, False,
                lambda: (by(dtb, 1), [fld(n, i + 2) for i, n in
                                      enumerate(['pp3d', 'th', 'qv', 'qc', 'qpten', 'qtten', 'qvten', 'qcten'])]))
        enc('ppx_finish', full, TG3, False, lambda: (fld('pp3d', 1), fld('ppx', 2)))
        halo_fill('ppx')
        if self.adaptive:
            # the stability reduction for the adaptive time step (timestep.js:742-762, 2193)
            d = f(dt)
            sp = pack('fffffii', [f(f(F(0.5) * d) * f(1.0 / g.dx)), f(f(F(0.5) * d) * f(1.0 / g.dy)),
                                  f(f(F(0.5) * d) * f(1.0 / g.dz)), f(f(d * f(1.0 / g.dx)) * f(1.0 / g.dx)),
                                  f(f(d * f(1.0 / g.dy)) * f(1.0 / g.dy)), 0, 0])

            def stab():
                by(sp, 1)
                for i, n in enumerate(['u', 'v', 'w']):
                    fld(n, i + 2)
                buf('mh', 5)
                for i in range(3):
                    fld('u', 6 + i)
                buf('stability', 9)
            enc('stability_max', full, TG3, False, stab)
        cmds.append({'op': 'end'})
        # state swap (timestep.js:766-774)
        nbytes = g.count * 4
        aid = rec.id('arena')
        swaps = [('th', 'th_a'), ('qv', 'qv_a'), ('u', 'u_a'), ('v', 'v_a'), ('w', 'w_a'), ('pp3d', 'ppi')]
        for src, dst in [sw for sw in swaps if not ((core or not moist) and sw[0] == 'qv')]:
            cmds.append({'op': 'copy', 'src': aid, 'srcOffset': self.fields[src], 'dst': aid,
                         'dstOffset': self.fields[dst], 'size': nbytes})
        return cmds

    def set_time_step(self, dt, nsound):
        """TimeStep.setTimeStep (timestep.js:711-716): the next encode() uses dt, nsound."""
        self.dt = f(dt)
        self.schedule = AcousticSchedule(int(nsound), self.dt)

    def tape(self, nsteps=1, core=False):
        """Tape in the reference format (driver.js:62-74); ``core`` selects the
        dynamics-core step (see encode)."""
        steps = [self.encode(core=core) for _ in range(max(1, nsteps))]
        g = self.grid
        buffers = [{'id': i, 'length': self.buffer_length(n), 'label': n, 'arena': n == 'arena'}
                   for i, n in enumerate(self.rec.buffers)]
        return {'nx': g.nx, 'ny': g.ny, 'nz': g.nz, 'dt': self.dt, 'halo': H, 'warmSteps': 0,
                'constants': {'terrain': False, 'axisymmetric': False, 'warmOnly': False, 'thermoDefault': True,
                              'testcase': 0},
                'buffers': buffers, 'fields': dict(self.fields), 'fieldStride': g.field_stride,
                'steps': steps, 'diag': []}

    def initial_buffers(self):
        """Initial contents per buffer id (the ``state/<id>.bin`` of a recording)."""
        arena = self.initial_arena()
        return {i: self.buffer_bytes(n, arena) for i, n in enumerate(self.rec.buffers)}
