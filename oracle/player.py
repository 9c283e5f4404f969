"""CPU tape player with the reference player's memory model (TEST INFRASTRUCTURE).

Only ``tests/`` and ``bench.py``'s CPU-baseline leg use this module; the product is
the CUDA player behind ``include/thunderstep.h``.

It restates ``Replayer`` (web/replay.js:36-396) on host memory:

* every tape buffer is packed into one u32 word memory ``M``, each 64-word aligned
  (replay.js:46-52); then the ``setBytes`` payloads (layoutBytes, replay.js:68-83),
  a 2^18-word spare (replay.js:15, 58-59), then per-thread kernel scratch
  (replay.js:64-66, 100-110);
* each dispatch gets a 64-word ARG slot: [0..2] grid in threads, [3] = 0, [4+n] word
  offset of binding n, [36] scratch base, [37..38] y tile (replay.js:258-288);
* ``copy`` ops move words inside ``M`` (replay.js:95-97, UTIL_WGSL copy_words);
* region hashes use the reference formula (replay.js:407-418) over the region each
  written binding covers (regionLen, replay.js:168-178); buffer checks use FNV-1a
  over u32 words (web/view.js:1063-1068).

Kernels are looked up by name in a ``KernelSet``: a ctypes library exporting
``<prefix><name>(uint32_t *M, const uint32_t *ARG)``.  Two such libraries exist:
``oracle/liboracle.so`` (the hand-written restatement, prefix ``teor_``) and
``oracle/_ref/libteref.so`` (the reference kernels translated, prefix ``teref_``).
"""
import base64
import ctypes
import gzip
import json
import math
import os

import numpy as np

SLOT = 64
ALIGN = 64
BYTES_SPARE = 1 << 18
SCRATCH_CAP = 1 << 26

HERE = os.path.dirname(os.path.abspath(__file__))


def unb64(s):
    return base64.b64decode(s)


def signature(cmds):
    """Step structure without setBytes data (replay.js:31)."""
    out = []
    for c in cmds:
        if c['op'] == 'bytes':
            out.append('b%d:%d' % (c['index'], len(c['data'])))
        elif c['op'] == 'barrier':
            out.append('')
        else:
            out.append(json.dumps(c, sort_keys=True))
    return '|'.join(out)


def region_hash(words):
    """Reference region hash (replay.js:407-418): sum of mixed words, mod 2^32."""
    w = np.asarray(words, dtype=np.uint32)
    i = np.arange(w.size, dtype=np.uint32)
    with np.errstate(over='ignore'):
        h = (w ^ (i * np.uint32(0x9E3779B1))) * np.uint32(0x85EBCA6B)
        h ^= h >> np.uint32(13)
        h *= np.uint32(0xC2B2AE35)
        h ^= h >> np.uint32(16)
    return int(h.sum(dtype=np.uint64) & 0xFFFFFFFF)


def fnv1a(words):
    """FNV-1a over u32 words (web/view.js:1063-1068)."""
    w = np.asarray(words, dtype=np.uint32)
    h = 0x811c9dc5
    # vectorising FNV is not possible; chunked python over numpy ints stays fast enough
    # for fixture-sized buffers (a few 10^7 words) when done in C; fall back to python.
    lib = _fnv_lib()
    if lib is not None:
        return lib.te_fnv1a(w.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(w.size))
    for x in w.tolist():
        h = ((h ^ x) * 0x01000193) & 0xFFFFFFFF
    return h


_FNV = None


def _fnv_lib():
    global _FNV
    if _FNV is None:
        path = os.path.join(HERE, 'liboracle.so')
        if os.path.exists(path):
            lib = ctypes.CDLL(path)
            lib.te_fnv1a.restype = ctypes.c_uint32
            lib.te_fnv1a.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
            _FNV = lib
        else:
            _FNV = False
    return _FNV or None


class KernelSet:
    """Kernels from a ctypes library: name -> fn(M, ARG)."""

    def __init__(self, path, prefix):
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix
        self.cache = {}

    def has(self, name):
        try:
            self.get(name)
            return True
        except AttributeError:
            return False

    def get(self, name):
        f = self.cache.get(name)
        if f is None:
            f = getattr(self.lib, self.prefix + name)
            f.restype = None
            f.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            self.cache[name] = f
        return f


class Op:
    __slots__ = ('kind', 'name', 'grid', 'tg', 'bind', 'hashes', 'tileY', 'src', 'dst', 'n', 'arg', 'index')


class CpuPlayer:
    """Host-memory restatement of web/replay.js ``Replayer``."""

    def __init__(self, tape, kernels_meta):
        self.tape = tape
        self.kmeta = kernels_meta

    # ---- plan (replay.js:46-66)
    def plan(self, with_hashes=True):
        t = self.tape
        top = 0
        self.base = []
        for b in t['buffers']:
            self.base.append(top)
            top += math.ceil(b['length'] / 4 / ALIGN) * ALIGN
        self.buffers_end = top
        self.bytes = []
        self.bytes_top = top
        self.bytes_spare_end = None
        self.scratch_need = 0
        self.hash_count = 0
        e0 = self.layout_bytes(t['steps'][0])
        eD = self.layout_bytes(t.get('diag') or [])
        self.bytes_spare_end = self.bytes_top + BYTES_SPARE
        top = math.ceil(self.bytes_spare_end / ALIGN) * ALIGN
        self.ops = self.build_ops(t['steps'][0], e0, with_hashes)
        self.diag_ops = self.build_ops(t.get('diag') or [], eD, False)
        self.cache = {signature(t['steps'][0]): {'ops': self.ops, 'offs': e0, 'data': {}}}
        for i, c in enumerate(t['steps'][0]):
            if c['op'] == 'bytes':
                self.cache[signature(t['steps'][0])]['data'][i] = c['data']
        self.scratch_base = top
        top += math.ceil(self.scratch_need / ALIGN) * ALIGN
        self.mem_words = top
        # The reference runs a dispatch whose per-thread scratch would pass SCRATCH_CAP in
        # y tiles that share the planned scratch (replay.js:23-29, 104-109, 272-274); the C
        # kernels here run the whole grid at once, so the host array carries the scratch of
        # every thread past mem_words (the layout, mem_words and all hashed regions are
        # the reference's).
        full = self.mem_words
        for o in self.ops + self.diag_ops:
            scr = (self.kmeta.get(o.name) or {}).get('scratch') or 0 if o.kind == 'k' else 0
            if scr:
                full = max(full, self.scratch_base + scr * o.grid[0] * o.grid[1] * o.grid[2])
        self.M = np.zeros(full, dtype=np.uint32)
        for off, data in self.bytes:
            self.write_words(off, data)
        self.hashes = np.zeros(max(self.hash_count, 1), dtype=np.uint32)
        self._build_slots(self.ops + self.diag_ops)

    def layout_bytes(self, cmds):
        offs = {}
        for i, c in enumerate(cmds):
            if c['op'] != 'bytes':
                continue
            raw = unb64(c['data'])
            words = math.ceil(len(raw) / 4)
            padded = raw + b'\0' * (words * 4 - len(raw))
            if self.bytes_spare_end is not None and self.bytes_top + words + 4 > self.bytes_spare_end:
                raise RuntimeError('no room for the bytes of a new step structure (BYTES_SPARE)')
            offs[i] = self.bytes_top
            self.bytes.append((self.bytes_top, padded))
            self.bytes_top += math.ceil(words / 4) * 4 + 4
        return offs

    def region_len(self, off):
        t = self.tape
        if off is None:
            return 0
        for b in range(len(t['buffers']) - 1, -1, -1):
            if off >= self.base[b]:
                end = self.base[b] + t['buffers'][b]['length'] // 4
                if t['buffers'][b]['arena']:
                    return min(t['fieldStride'] // 4, end - off)
                return end - off
        return 0

    def build_ops(self, cmds, offs, hashes):
        ops = []
        bind, last, pipe = {}, {}, None
        for i, c in enumerate(cmds):
            op = c['op']
            if op == 'pipe':
                pipe = c['name']
            elif op == 'buf':
                bind[c['index']] = 0 if c['buf'] < 0 else self.base[c['buf']] + c['offset'] // 4
                last[c['index']] = c['buf']
            elif op == 'bufoff':
                bind[c['index']] = self.base[last[c['index']]] + c['offset'] // 4
            elif op == 'bytes':
                bind[c['index']] = offs[i]
            elif op == 'end':
                bind = {}
            elif op == 'copy':
                o = Op()
                o.kind = 'copy'
                o.src = self.base[c['src']] + c['srcOffset'] // 4
                o.dst = self.base[c['dst']] + c['dstOffset'] // 4
                o.n = c['size'] // 4
                o.index = i
                ops.append(o)
            elif op == 'dispatch':
                k = self.kmeta.get(pipe)
                if k is None:
                    raise RuntimeError('no kernel ' + str(pipe))
                grid = c['grid']
                threads = grid[0] * grid[1] * grid[2]
                tileY = grid[1]
                scr = k.get('scratch') or 0
                if scr and scr * threads > SCRATCH_CAP:
                    row = scr * grid[0] * grid[2]
                    tileY = max(c['tg'][1], (SCRATCH_CAP // row // c['tg'][1]) * c['tg'][1])
                self.scratch_need = max(self.scratch_need, scr * grid[0] * grid[2] * tileY)
                o = Op()
                o.kind = 'k'
                o.name = pipe
                o.grid = list(grid)
                o.tg = list(c['tg'])
                o.bind = dict(bind)
                o.hashes = []
                o.tileY = tileY
                o.index = i
                if hashes:
                    for p in k['params']:
                        if not p['write']:
                            continue
                        off = bind.get(p['index'])
                        o.hashes.append((self.hash_count, off, self.region_len(off)))
                        self.hash_count += 1
                ops.append(o)
        return ops

    def _build_slots(self, ops):
        for o in ops:
            if o.kind != 'k':
                continue
            a = np.zeros(SLOT, dtype=np.uint32)
            a[0:3] = o.grid
            for i, off in o.bind.items():
                a[4 + i] = off
            a[36] = self.scratch_base
            a[37] = 0
            a[38] = o.grid[1]
            o.arg = a

    def write_words(self, off, data):
        b = bytes(data)
        if len(b) % 4:
            b += b'\0' * (4 - len(b) % 4)
        w = np.frombuffer(b, dtype=np.uint32)
        self.M[off:off + w.size] = w

    # ---- state
    def upload(self, buf_id, data):
        self.write_words(self.base[buf_id], data)

    def upload_state_dir(self, state_dir):
        for b in self.tape['buffers']:
            p = os.path.join(state_dir, '%d.bin.gz' % b['id'])
            if os.path.exists(p):
                with gzip.open(p, 'rb') as fh:
                    self.upload(b['id'], fh.read())

    def buffer_words(self, buf_id):
        o = self.base[buf_id]
        return self.M[o:o + self.tape['buffers'][buf_id]['length'] // 4]

    def use_step(self, cmds):
        """Same structure: only new setBytes payloads are written (replay.js:127-146)."""
        sig = signature(cmds)
        e = self.cache.get(sig)
        if e is None:
            offs = self.layout_bytes(cmds)
            ops = self.build_ops(cmds, offs, False)
            e = {'ops': ops, 'offs': offs, 'data': {}}
            self.cache[sig] = e
            need = self.scratch_base + math.ceil(self.scratch_need / ALIGN) * ALIGN
            if need > self.mem_words:
                self.M = np.concatenate([self.M, np.zeros(need - self.mem_words, dtype=np.uint32)])
                self.mem_words = need
            self._build_slots(ops)
        for i, c in enumerate(cmds):
            if c['op'] != 'bytes' or e['data'].get(i) == c['data']:
                continue
            e['data'][i] = c['data']
            self.write_words(e['offs'][i], unb64(c['data']))
        self.ops = e['ops']

    def clear_hashes(self):
        self.hashes[:] = 0

    # ---- execution
    def run(self, kernels, nsteps=1, with_hashes=False, last_op=None, ops=None, on_op=None):
        """Execute the planned ops. ``kernels``: callable name -> fn(M, ARG)."""
        ops = self.ops if ops is None else ops
        mp = self.M.ctypes.data_as(ctypes.c_void_p)
        for _ in range(nsteps):
            for oi, o in enumerate(ops):
                if last_op is not None and oi > last_op:
                    break
                if o.kind == 'copy':
                    self.M[o.dst:o.dst + o.n] = self.M[o.src:o.src + o.n]
                else:
                    kernels(o.name)(mp, o.arg.ctypes.data_as(ctypes.c_void_p))
                    if with_hashes:
                        # slots accumulate across runs like the reference's atomicAdd
                        # into H, which is never cleared (replay.js:199, UTIL_WGSL)
                        for slot, off, ln in o.hashes:
                            if off is not None:
                                self.hashes[slot] = (int(self.hashes[slot]) + region_hash(self.M[off:off + ln])) & 0xFFFFFFFF
                if on_op is not None:
                    on_op(oi, o)


def load_tape(scen_dir):
    with open(os.path.join(scen_dir, 'tape.json')) as fh:
        return json.load(fh)


def load_kernels_meta(path):
    with open(path) as fh:
        return json.load(fh)


class CpuPlayer64(CpuPlayer):
    """The same player over the binary64 twin of the oracle (liboracle64.so): a double
    array ``D`` beside the word memory holds every field value; kernels read parameter
    structs from ``M`` and field values from ``D``.  ``values_from_words()`` widens the
    uploaded binary32 words into ``D``; ``field64(off, n)`` reads values back."""

    def __init__(self, tape, kernels_meta, lib_path=None):
        super().__init__(tape, kernels_meta)
        self.lib64 = ctypes.CDLL(lib_path or os.path.join(HERE, 'liboracle64.so'))
        self.lib64.te64_bind.argtypes = [ctypes.c_void_p]
        self.lib64.te64_bind.restype = None
        self.kernels64 = {}

    def plan(self, with_hashes=False):
        super().plan(False)
        self.D = np.zeros(self.M.size, dtype=np.float64)

    def values_from_words(self):
        self.D[:] = self.M.view(np.float32)

    def kernel(self, name):
        f = self.kernels64.get(name)
        if f is None:
            f = getattr(self.lib64, 'teor_' + name)
            f.restype = None
            f.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            self.kernels64[name] = f
        return f

    def run64(self, nsteps=1):
        self.lib64.te64_bind(self.D.ctypes.data_as(ctypes.c_void_p))
        mp = self.M.ctypes.data_as(ctypes.c_void_p)
        for _ in range(nsteps):
            for o in self.ops:
                if o.kind == 'copy':
                    self.D[o.dst:o.dst + o.n] = self.D[o.src:o.src + o.n]
                    self.M[o.dst:o.dst + o.n] = self.M[o.src:o.src + o.n]
                else:
                    self.kernel(o.name)(mp, o.arg.ctypes.data_as(ctypes.c_void_p))

    def field64(self, off, n):
        return self.D[off:off + n]
