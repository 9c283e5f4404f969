"""``Replayer``: host-side mirror of the reference's tape player over the CUDA C-ABI.

The reference player (web/replay.js:36-396) is a JavaScript class driving WebGPU.  This
class has the same methods and fields, with the same argument meaning, but plays the
tape on a B200 through ``libthunderstep.so`` (include/thunderstep.h):

=========================================  ==========================================
reference (web/replay.js)                  here
=========================================  ==========================================
``new Replayer(device, tape, kernels, s)``  ``Replayer(tape, kernels=None, device=0)``
``plan(withHashes)`` + ``await build()``   ``plan(with_hashes)`` + ``build()``
``upload(id, u8)`` / ``uploadAsync``       ``upload(buf_id, data)``
``await useStep(cmds)``                    ``use_step(cmds)``
``encodeSteps(enc, n, withHashes, last)``  ``encode_steps(n, with_hashes, last_op)``
``encodeDiag(enc)``                        ``encode_diag()``
``await read(words, offWords)``            ``read(words, off_words)`` -> numpy uint32
``await readHashes()``                     ``read_hashes()`` -> numpy uint32
``base``, ``buffersEnd``, ``memWords``,     ``base``, ``buffers_end``, ``mem_words``,
``hashCount``                              ``hash_count``
=========================================  ==========================================

Errors raise ``RuntimeError`` with the library's message, where the reference throws
``Error`` (unknown kernel, bytes overflow, ...).  There is no CPU fallback: when the
library cannot be loaded or no CUDA device is present, construction fails.
"""
import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libthunderstep.so')

TE_FLAG_DEFER_MISSING = 1
TE_MODE_EXACT = 0
TE_MODE_FUSED = 1

_LIB = None


class TeInfo(ctypes.Structure):
    _fields_ = [('mem_words', ctypes.c_uint64), ('buffers_end', ctypes.c_uint64),
                ('scratch_base', ctypes.c_uint64), ('hash_count', ctypes.c_uint32),
                ('num_buffers', ctypes.c_uint32), ('num_ops', ctypes.c_uint32),
                ('num_dispatches', ctypes.c_uint32)]


class TeSegment(ctypes.Structure):
    _fields_ = [('kind', ctypes.c_int), ('first_op', ctypes.c_int), ('last_op', ctypes.c_int),
                ('kernels', ctypes.c_int)]


class TeConfig(ctypes.Structure):
    _fields_ = [('device', ctypes.c_int), ('flags', ctypes.c_int), ('reserved', ctypes.c_uint64 * 4)]


class TeWSolveFields(ctypes.Structure):
    """``te_wsolve_fields``: device pointers of one w-pi' column solve."""
    _fields_ = [(n, ctypes.c_void_p) for n in ('pk1', 'pk2', 'qk', 'mm', 'fpk', 'wten', 'pp3d', 'w')]


EXPORTS = {
    'te_create': ([ctypes.POINTER(TeConfig), ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    'te_plan': ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int],
                ctypes.c_int),
    'te_get_info': ([ctypes.c_void_p, ctypes.POINTER(TeInfo)], ctypes.c_int),
    'te_buffer_base': ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
    'te_upload': ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t], ctypes.c_int),
    'te_write_words': ([ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t], ctypes.c_int),
    'te_use_step': ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
    'te_run': ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    'te_run_ops': ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    'te_run_diag': ([ctypes.c_void_p], ctypes.c_int),
    'te_read': ([ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p], ctypes.c_int),
    'te_read_hashes': ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t], ctypes.c_int),
    'te_clear_hashes': ([ctypes.c_void_p], ctypes.c_int),
    'te_device_ptr': ([ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    'te_set_mode': ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    'te_op_name': ([ctypes.c_void_p, ctypes.c_int], ctypes.c_char_p),
    'te_sync': ([ctypes.c_void_p], ctypes.c_int),
    'te_destroy': ([ctypes.c_void_p], None),
    'te_last_error': ([ctypes.c_void_p], ctypes.c_char_p),
    'te_region_hash_host': ([ctypes.c_void_p, ctypes.c_uint64], ctypes.c_uint32),
    'te_check_pow': ([ctypes.c_float, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64),
                      ctypes.POINTER(ctypes.c_uint32)], ctypes.c_int),
    'te_set_stream': ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    'te_kernel_table_json': ([ctypes.c_char_p, ctypes.c_size_t], ctypes.c_size_t),
    'te_fused_segments': ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    'te_run_segment': ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    'te_write_words_async': ([ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t], ctypes.c_int),
    'te_read_async': ([ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p], ctypes.c_int),
    'te_adjoint_forward': ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    'te_adjoint_backward': ([ctypes.c_void_p], ctypes.c_int),
    'te_adjoint_write_words': ([ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t], ctypes.c_int),
    'te_adjoint_read': ([ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p], ctypes.c_int),
    'te_adjoint_zero': ([ctypes.c_void_p], ctypes.c_int),
    'te_adjoint_device_ptr': ([ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    'te_adjoint_memory': ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
    'te_autotune': ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    'te_ensemble_create': ([ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
                           ctypes.c_int),
    'te_ensemble_run': ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    'te_ensemble_stream': ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    'te_ensemble_sync': ([ctypes.c_void_p], ctypes.c_int),
    'te_ensemble_last_error': ([ctypes.c_void_p], ctypes.c_char_p),
    'te_ensemble_destroy': ([ctypes.c_void_p], None),
    'te_w_solve_static_scratch': ([ctypes.POINTER(TeWSolveFields), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_void_p,
                                   ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
}


def load_library(path=LIB_PATH):
    """Load ``libthunderstep.so`` (raises if it is missing: there is no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError('libthunderstep.so is not built (%s); run __graft_entry__.build()' % path)
    lib = ctypes.CDLL(path)
    for name, (args, res) in EXPORTS.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _LIB = lib
    return lib


def _json_bytes(x):
    if isinstance(x, (bytes, bytearray)):
        return bytes(x)
    if isinstance(x, str):
        return x.encode()
    return json.dumps(x, separators=(',', ':')).encode()


class Replayer:
    """Plays a ThunderEngine command tape on one B200 (see the module docstring)."""

    def __init__(self, tape, kernels=None, device=0, defer_missing=False):
        self.lib = load_library()
        self.tape = tape
        self.kernels = kernels
        self.device = device
        cfg = TeConfig(device=device, flags=TE_FLAG_DEFER_MISSING if defer_missing else 0)
        h = ctypes.c_void_p()
        rc = self.lib.te_create(ctypes.byref(cfg), ctypes.byref(h))
        self.h = h
        if rc != 0:
            msg = self.lib.te_last_error(h).decode() if h else 'te_create failed'
            self.lib.te_destroy(h)
            self.h = None
            raise RuntimeError(msg)
        self.base = []
        self.buffers_end = self.mem_words = self.hash_count = 0
        self._with_hashes = False

    # ---- helpers
    def _check(self, rc):
        if rc != 0:
            raise RuntimeError('thunderstep error %d: %s' % (rc, self.lib.te_last_error(self.h).decode()))

    def close(self):
        if getattr(self, 'h', None):
            self.lib.te_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- Replayer API
    def plan(self, with_hashes=False):
        """Record the layout request; memory is laid out and allocated by ``build``."""
        self._with_hashes = bool(with_hashes)

    def build(self):
        tj = _json_bytes(self.tape)
        kj = _json_bytes(self.kernels) if self.kernels is not None else None
        self._check(self.lib.te_plan(self.h, tj, len(tj), kj, len(kj) if kj else 0, 1 if self._with_hashes else 0))
        info = TeInfo()
        self._check(self.lib.te_get_info(self.h, ctypes.byref(info)))
        self.mem_words = info.mem_words
        self.buffers_end = info.buffers_end
        self.hash_count = info.hash_count
        self.num_ops = info.num_ops
        self.num_dispatches = info.num_dispatches
        self.base = []
        for i in range(info.num_buffers):
            o = ctypes.c_uint64()
            self._check(self.lib.te_buffer_base(self.h, i, ctypes.byref(o)))
            self.base.append(o.value)

    def upload(self, buf_id, data):
        b = np.ascontiguousarray(np.frombuffer(bytes(data), dtype=np.uint8) if isinstance(data, (bytes, bytearray))
                                 else np.asarray(data)).view(np.uint8)
        self._check(self.lib.te_upload(self.h, int(buf_id), b.ctypes.data_as(ctypes.c_void_p), b.nbytes))

    def write_words(self, off, data):
        b = np.ascontiguousarray(np.asarray(data)).view(np.uint8)
        self._check(self.lib.te_write_words(self.h, int(off), b.ctypes.data_as(ctypes.c_void_p), b.nbytes))

    def use_step(self, cmds):
        j = _json_bytes(cmds)
        self._check(self.lib.te_use_step(self.h, j, len(j)))
        info = TeInfo()
        self._check(self.lib.te_get_info(self.h, ctypes.byref(info)))
        self.num_ops = info.num_ops

    def encode_steps(self, n=1, with_hashes=False, last_op=None):
        if last_op is None:
            self._check(self.lib.te_run(self.h, int(n), 1 if with_hashes else 0))
        else:
            for _ in range(int(n)):
                self._check(self.lib.te_run_ops(self.h, 0, int(last_op), 1 if with_hashes else 0))

    def run_ops(self, first, last, with_hashes=False):
        self._check(self.lib.te_run_ops(self.h, int(first), int(last), 1 if with_hashes else 0))

    def encode_diag(self):
        self._check(self.lib.te_run_diag(self.h))

    def read(self, words, off_words=0):
        out = np.empty(int(words), dtype=np.uint32)
        self._check(self.lib.te_read(self.h, int(off_words), int(words), out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def read_hashes(self):
        out = np.zeros(max(self.hash_count, 1), dtype=np.uint32)
        self._check(self.lib.te_read_hashes(self.h, out.ctypes.data_as(ctypes.c_void_p), self.hash_count))
        return out[:self.hash_count]

    def clear_hashes(self):
        self._check(self.lib.te_clear_hashes(self.h))

    def set_mode(self, mode):
        self._check(self.lib.te_set_mode(self.h, int(mode)))

    def device_ptr(self, off_words):
        p = ctypes.c_void_p()
        self._check(self.lib.te_device_ptr(self.h, int(off_words), ctypes.byref(p)))
        return p.value

    def op_name(self, i):
        r = self.lib.te_op_name(self.h, int(i))
        return r.decode() if r else None

    def set_stream(self, stream_handle):
        """Launch on a caller-owned CUDA stream (int handle; 0 = the context's own)."""
        self._check(self.lib.te_set_stream(self.h, ctypes.c_void_p(int(stream_handle) or None)))

    def fused_segments(self):
        """Fused-mode segments of the active step: list of (kind, first_op, last_op, kernels)."""
        n = ctypes.c_int()
        self._check(self.lib.te_fused_segments(self.h, None, 0, ctypes.byref(n)))
        arr = (TeSegment * max(n.value, 1))()
        self._check(self.lib.te_fused_segments(self.h, arr, n.value, ctypes.byref(n)))
        return [(s.kind, s.first_op, s.last_op, s.kernels) for s in arr[:n.value]]

    def run_segment(self, seg, part=-1):
        self._check(self.lib.te_run_segment(self.h, int(seg), int(part)))

    def autotune(self, reps=5):
        """Picks the thread-block shape of each per-dispatch op (te_autotune); returns the
        number of ops whose shape changed.  Memory is left as it was."""
        n = ctypes.c_int()
        self._check(self.lib.te_autotune(self.h, int(reps), ctypes.byref(n)))
        return n.value

    # ---- discrete adjoint (te_adjoint_*; no counterpart in the reference)
    def adjoint_forward(self, nsteps, checkpoint_every):
        """Runs nsteps steps keeping checkpoints every checkpoint_every steps; clears the
        adjoint memory."""
        self._check(self.lib.te_adjoint_forward(self.h, int(nsteps), int(checkpoint_every)))

    def adjoint_backward(self):
        """Adjoint memory: d(cost)/d(final state) -> d(cost)/d(initial state); memory
        returns to the initial state."""
        self._check(self.lib.te_adjoint_backward(self.h))

    def adjoint_write_words(self, off, data):
        a = np.ascontiguousarray(np.asarray(data))
        self._check(self.lib.te_adjoint_write_words(self.h, int(off), a.ctypes.data, a.nbytes))

    def adjoint_read(self, words, off_words=0):
        out = np.empty(int(words), dtype=np.float32)
        self._check(self.lib.te_adjoint_read(self.h, int(off_words), int(words), out.ctypes.data))
        return out

    def adjoint_zero(self):
        self._check(self.lib.te_adjoint_zero(self.h))

    def adjoint_memory(self):
        n = ctypes.c_uint64()
        self._check(self.lib.te_adjoint_memory(self.h, ctypes.byref(n)))
        return n.value

    def sync(self):
        self._check(self.lib.te_sync(self.h))


class Ensemble:
    """Independent Replayers on one device advanced together (te_ensemble_*; no
    counterpart in the reference): one graph launch per large step runs every member's
    step, the members' kernels concurrently."""

    def __init__(self, members):
        self.lib = load_library()
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m.h.value if hasattr(m.h, "value") else m.h for m in self.members])
        h = ctypes.c_void_p()
        rc = self.lib.te_ensemble_create(arr, len(self.members), ctypes.byref(h))
        self.h = h
        if rc != 0:
            msg = self.lib.te_ensemble_last_error(h).decode() if h.value else 'te_ensemble_create failed'
            self.close()
            raise RuntimeError('thunderstep error %d: %s' % (rc, msg))

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError('thunderstep error %d: %s' % (rc, self.lib.te_ensemble_last_error(self.h).decode()))

    def run(self, nsteps=1):
        self._check(self.lib.te_ensemble_run(self.h, int(nsteps)))

    def stream(self):
        s = ctypes.c_void_p()
        self._check(self.lib.te_ensemble_stream(self.h, ctypes.byref(s)))
        return s.value

    def sync(self):
        self._check(self.lib.te_ensemble_sync(self.h))

    def close(self):
        if getattr(self, 'h', None) is not None and self.h.value:
            self.lib.te_ensemble_destroy(self.h)
        self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
