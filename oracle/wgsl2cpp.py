#!/usr/bin/env python3
"""Build recipe for ``oracle/_ref``: the reference's own WGSL kernels compiled as C++.

TEST INFRASTRUCTURE ONLY. Nothing in the product imports or links what this script
writes; only ``tests/`` and ``bench.py``'s CPU-baseline leg may load ``oracle/_ref``.

The reference (ThunderEngine, data/kernels/*.wgsl) ships its compute kernels as
machine-generated WGSL ("generated, do not edit by hand", e.g.
data/kernels/adv_flux_x_weno.wgsl:5).  That WGSL is a small, regular subset:
word-addressed loads/stores on one memory ``M``, a 64-word argument slot ``ARG``,
``opq()``/``nego()`` rounding barriers (adv_flux_x_weno.wgsl:15-21), explicit ``fma``,
``select``, ``bitcast``, ``loop``/``continuing``, small vectors and fixed arrays.
This script rewrites that subset mechanically into C++ so the reference's kernels can
run on host cores against the shipped golden hashes (data/<scenario>/hashes.ref.bin,
step1.json).  It reads the sources where they lie (``--src``) and writes generated
C++ only into ``oracle/_ref/`` (git-ignored); no reference source is committed.

Semantics kept: every f32 operation is one IEEE binary32 operation (compiled with
``-ffp-contract=off``, no fast-math), ``fma`` is a fused multiply-add, i32 wraps
(``-fwrapv``), ``opq(x)`` returns x (the slot word ARG[3] is always 0,
replay.js:266-269) through an empty asm so the compiler cannot fold across it, as the
reference intends (adv_flux_x_weno.wgsl:15-21), ``select(f, t, c)`` evaluates both
operands.

Usage: python oracle/wgsl2cpp.py --src <kernels dir> --out oracle/_ref/gen
"""
import argparse
import json
import os
import re
import sys

PRELUDE = r'''
#pragma once
#include <cstdint>
#include <cstring>
#include <cmath>
#include <array>
typedef float f32; typedef int32_t i32; typedef uint32_t u32;
template <class T> struct vec2 { T x{}, y{}; vec2() {} vec2(T a, T b) : x(a), y(b) {} explicit vec2(T a) : x(a), y(a) {}
  T& operator[](long i) { return (&x)[i]; } T operator[](long i) const { return (&x)[i]; } };
template <class T> struct vec3 { T x{}, y{}, z{}; vec3() {} vec3(T a, T b, T c) : x(a), y(b), z(c) {} explicit vec3(T a) : x(a), y(a), z(a) {}
  vec2<T> xy() const { return vec2<T>(x, y); }
  T& operator[](long i) { return (&x)[i]; } T operator[](long i) const { return (&x)[i]; } };
template <class T> struct vec4 { T x{}, y{}, z{}, w{}; vec4() {} vec4(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {} explicit vec4(T a) : x(a), y(a), z(a), w(a) {}
  T& operator[](long i) { return (&x)[i]; } T operator[](long i) const { return (&x)[i]; } };
#define VOP(OP) \
template <class T> static inline vec2<T> operator OP(vec2<T> a, vec2<T> b) { return vec2<T>(a.x OP b.x, a.y OP b.y); } \
template <class T> static inline vec3<T> operator OP(vec3<T> a, vec3<T> b) { return vec3<T>(a.x OP b.x, a.y OP b.y, a.z OP b.z); } \
template <class T> static inline vec4<T> operator OP(vec4<T> a, vec4<T> b) { return vec4<T>(a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w); } \
template <class T> static inline vec2<T> operator OP(vec2<T> a, T b) { return vec2<T>(a.x OP b, a.y OP b); } \
template <class T> static inline vec3<T> operator OP(vec3<T> a, T b) { return vec3<T>(a.x OP b, a.y OP b, a.z OP b); } \
template <class T> static inline vec4<T> operator OP(vec4<T> a, T b) { return vec4<T>(a.x OP b, a.y OP b, a.z OP b, a.w OP b); } \
template <class T> static inline vec2<T> operator OP(T a, vec2<T> b) { return vec2<T>(a OP b.x, a OP b.y); } \
template <class T> static inline vec3<T> operator OP(T a, vec3<T> b) { return vec3<T>(a OP b.x, a OP b.y, a OP b.z); } \
template <class T> static inline vec4<T> operator OP(T a, vec4<T> b) { return vec4<T>(a OP b.x, a OP b.y, a OP b.z, a OP b.w); }
VOP(+) VOP(-) VOP(*) VOP(/) VOP(|) VOP(&) VOP(^)
#undef VOP
template <class T> static inline vec2<T> operator-(vec2<T> a) { return vec2<T>(-a.x, -a.y); }
template <class T> static inline vec3<T> operator-(vec3<T> a) { return vec3<T>(-a.x, -a.y, -a.z); }
template <class T> static inline vec4<T> operator-(vec4<T> a) { return vec4<T>(-a.x, -a.y, -a.z, -a.w); }
template <class T, size_t N> using array = std::array<T, N>;

template <class T, class S> static inline T W_bitcast(S s) { static_assert(sizeof(T) == sizeof(S), "bitcast"); T t; std::memcpy(&t, &s, sizeof t); return t; }
template <class T> static inline T W_select(T f, T t, bool c) { return c ? t : f; }
static inline f32 W_fma(f32 a, f32 b, f32 c) { return fmaf(a, b, c); }
static inline vec2<f32> W_fma(vec2<f32> a, vec2<f32> b, vec2<f32> c) { return vec2<f32>(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y)); }
static inline vec3<f32> W_fma(vec3<f32> a, vec3<f32> b, vec3<f32> c) { return vec3<f32>(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y), fmaf(a.z, b.z, c.z)); }
static inline vec4<f32> W_fma(vec4<f32> a, vec4<f32> b, vec4<f32> c) { return vec4<f32>(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y), fmaf(a.z, b.z, c.z), fmaf(a.w, b.w, c.w)); }
static inline f32 W_abs(f32 a) { return fabsf(a); }
static inline i32 W_abs(i32 a) { return a < 0 ? -a : a; }
static inline u32 W_abs(u32 a) { return a; }
// WGSL min/max: min(a, b) = b if b < a else a; max(a, b) = b if a < b else a; NaN -> other
static inline f32 W_min(f32 a, f32 b) { return (b < a || a != a) ? b : a; }
static inline f32 W_max(f32 a, f32 b) { return (a < b || a != a) ? b : a; }
static inline i32 W_min(i32 a, i32 b) { return a < b ? a : b; }
static inline i32 W_max(i32 a, i32 b) { return a > b ? a : b; }
static inline u32 W_min(u32 a, u32 b) { return a < b ? a : b; }
static inline u32 W_max(u32 a, u32 b) { return a > b ? a : b; }
static inline f32 W_clamp(f32 e, f32 lo, f32 hi) { return W_min(W_max(e, lo), hi); }
static inline i32 W_clamp(i32 e, i32 lo, i32 hi) { return W_min(W_max(e, lo), hi); }
static inline u32 W_clamp(u32 e, u32 lo, u32 hi) { return W_min(W_max(e, lo), hi); }
static inline f32 W_sqrt(f32 a) { return sqrtf(a); }
static inline f32 W_floor(f32 a) { return floorf(a); }
static inline f32 W_round(f32 a) { return nearbyintf(a); }
static inline f32 W_trunc(f32 a) { return truncf(a); }
#ifdef TE_REF_F64_BUILTINS
// WGSL leaves the precision of exp/log/pow/log2/atan2 to the implementation: this variant
// evaluates them like the CUDA kernels (binary64, rounded once; oracle.c te_*_f64)
extern "C" float te_exp_f64(float x);
extern "C" float te_log_f64(float x);
extern "C" float te_pow_f64(float x, float y);
extern "C" float te_log2_f64(float x);
extern "C" float te_atan2_f64(float y, float x);
static inline f32 W_exp(f32 a) { return te_exp_f64(a); }
static inline f32 W_log(f32 a) { return te_log_f64(a); }
static inline f32 W_pow(f32 a, f32 b) { return te_pow_f64(a, b); }
static inline f32 W_log2(f32 a) { return te_log2_f64(a); }
static inline f32 W_atan2(f32 a, f32 b) { return te_atan2_f64(a, b); }
#else
static inline f32 W_exp(f32 a) { return expf(a); }
static inline f32 W_log(f32 a) { return logf(a); }
static inline f32 W_pow(f32 a, f32 b) { return powf(a, b); }
static inline f32 W_log2(f32 a) { return log2f(a); }
static inline f32 W_atan2(f32 a, f32 b) { return atan2f(a, b); }
#endif
static inline f32 W_sin(f32 a) { return sinf(a); }
static inline f32 W_atan(f32 a) { return atanf(a); }
static inline f32 W_length(vec2<f32> v) { return sqrtf(v.x * v.x + v.y * v.y); }
static inline f32 W_length(vec3<f32> v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
static inline f32 W_dot(vec2<f32> a, vec2<f32> b) { return a.x * b.x + a.y * b.y; }
static inline f32 W_dot(vec3<f32> a, vec3<f32> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
struct W_frexp_t { f32 fract; i32 exp; };
static inline W_frexp_t W_frexp(f32 x) { int e = 0; f32 m = frexpf(x, &e); return W_frexp_t{m, (i32)e}; }
static inline f32 W_ldexp(f32 x, i32 e) { return ldexpf(x, e); }
static inline u32 W_countLeadingZeros(u32 x) { return x ? (u32)__builtin_clz(x) : 32u; }
static inline i32 W_countLeadingZeros(i32 x) { return (i32)W_countLeadingZeros((u32)x); }
static inline i32 W_to_i32(f32 x) { if (!(x == x)) return 0; if (x >= 2147483520.0f) return 2147483647; if (x <= -2147483648.0f) return (-2147483647 - 1); return (i32)x; }
static inline i32 W_to_i32(i32 x) { return x; }
static inline i32 W_to_i32(u32 x) { return (i32)x; }
static inline i32 W_to_i32(bool x) { return x ? 1 : 0; }
static inline u32 W_to_u32(f32 x) { if (!(x > 0.0f)) return 0u; if (x >= 4294967040.0f) return 4294967295u; return (u32)x; }
static inline u32 W_to_u32(i32 x) { return (u32)x; }
static inline u32 W_to_u32(u32 x) { return x; }
static inline u32 W_to_u32(bool x) { return x ? 1u : 0u; }
static inline f32 W_to_f32(f32 x) { return x; }
static inline f32 W_to_f32(i32 x) { return (f32)x; }
static inline f32 W_to_f32(u32 x) { return (f32)x; }
static inline f32 W_to_f32(bool x) { return x ? 1.0f : 0.0f; }
static inline bool W_to_bool(bool x) { return x; }
static inline bool W_to_bool(i32 x) { return x != 0; }
static inline bool W_to_bool(u32 x) { return x != 0; }
static inline bool W_to_bool(f32 x) { return x != 0.0f; }
static inline u32 W_atomicLoad(u32* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
static inline void W_atomicStore(u32* p, u32 v) { __atomic_store_n(p, v, __ATOMIC_RELAXED); }
static inline u32 W_atomicAdd(u32* p, u32 v) { return __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }
static inline u32 W_atomicMax(u32* p, u32 v) { u32 o = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (o < v && !__atomic_compare_exchange_n(p, &o, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {} return o; }
// opq(): the reference's rounding barrier (x | Z0 with Z0 = 0 unknown to the compiler).
// An empty asm on the value keeps the same meaning here: the compiler may not fold or
// reassociate across it (e.g. -fma(a,b,c) -> fma(-a,b,-c), which flips signed zeros).
static inline f32 opq(f32 x) { __asm__("" : "+x"(x)); return x; }
static inline vec2<f32> opq2(vec2<f32> x) { x.x = opq(x.x); x.y = opq(x.y); return x; }
static inline vec3<f32> opq3(vec3<f32> x) { x.x = opq(x.x); x.y = opq(x.y); x.z = opq(x.z); return x; }
static inline vec4<f32> opq4(vec4<f32> x) { x.x = opq(x.x); x.y = opq(x.y); x.z = opq(x.z); x.w = opq(x.w); return x; }
static inline f32 nego(f32 x) { return opq(W_bitcast<f32>(W_bitcast<u32>(x) ^ 0x80000000u)); }
'''

BUILTINS = ['fma', 'abs', 'min', 'max', 'clamp', 'sqrt', 'floor', 'round', 'trunc', 'exp', 'log', 'log2',
            'pow', 'sin', 'atan', 'atan2', 'length', 'dot', 'frexp', 'ldexp', 'countLeadingZeros',
            'atomicLoad', 'atomicStore', 'atomicAdd', 'atomicMax', 'select']
SKIP_FNS = {'opq', 'opq2', 'opq3', 'opq4', 'nego'}


def strip_comments(src):
    return '\n'.join(line.split('//', 1)[0] for line in src.split('\n'))


def match_close(s, i, open_ch, close_ch):
    """Index of the bracket closing the one at s[i]."""
    assert s[i] == open_ch, (s[i:i + 40])
    depth = 0
    for j in range(i, len(s)):
        c = s[j]
        if c == open_ch:
            depth += 1
        elif c == close_ch:
            depth -= 1
            if depth == 0:
                return j
    raise ValueError('unbalanced ' + open_ch)


def split_top(s, sep=','):
    """Split on sep at bracket depth 0 (<>, (), [])."""
    out, depth, cur = [], 0, ''
    for c in s:
        if c in '<([':
            depth += 1
        elif c in '>)]':
            depth -= 1
        if c == sep and depth == 0:
            out.append(cur)
            cur = ''
        else:
            cur += c
    if cur.strip():
        out.append(cur)
    return out


def cpp_type(t):
    t = t.strip()
    m = re.match(r'ptr<\s*function\s*,\s*(.*)>$', t)
    if m:
        return cpp_type(m.group(1)) + '*'
    m = re.match(r'atomic<\s*(.*)>$', t)
    if m:
        return cpp_type(m.group(1))
    return t


def rewrite_loops(body):
    """loop { ... continuing { C } }  ->  for (;; ({ C })) { ... }"""
    while True:
        m = re.search(r'\bloop\s*\{', body)
        if not m:
            return body
        ob = body.index('{', m.start())
        cb = match_close(body, ob, '{', '}')
        inner = body[ob + 1:cb]
        # find a continuing block at depth 0 of this loop
        cont = ''
        depth = 0
        k = 0
        cstart = -1
        while k < len(inner):
            c = inner[k]
            if c == '{':
                depth += 1
            elif c == '}':
                depth -= 1
            elif depth == 0 and inner.startswith('continuing', k) and re.match(r'continuing\s*\{', inner[k:]):
                cstart = k
                break
            k += 1
        if cstart >= 0:
            cob = inner.index('{', cstart)
            ccb = match_close(inner, cob, '{', '}')
            cont = inner[cob + 1:ccb]
            inner = inner[:cstart] + inner[ccb + 1:]
        head = 'for (;; ({ %s })) {' % cont.strip() if cont.strip() else 'for (;;) {'
        body = body[:m.start()] + head + inner + '}' + body[cb + 1:]


def rewrite_switch(body):
    """WGSL cases never fall through: add break after each case block."""
    out = ''
    pos = 0
    for m in re.finditer(r'\b(case\s+default|case\s+([^:{]+)|default)\s*:\s*\{', body):
        if m.start() < pos:
            continue
        ob = body.index('{', m.start())
        cb = match_close(body, ob, '{', '}')
        if m.group(1).startswith('case') and m.group(2) is not None and 'default' not in m.group(1):
            labels = [x.strip() for x in m.group(2).split(',') if x.strip()]
            head = ' '.join('case %s:' % lab for lab in labels)
        else:
            head = 'default:'
        out += body[pos:m.start()] + head + ' ' + rewrite_switch(body[ob:cb + 1]) + ' break;'
        pos = cb + 1
    return out + body[pos:]


def braces_ctor(s):
    """array<T, N>(a, b) / S_X(a) constructors -> brace initialisation."""
    pat = re.compile(r'(array<[^<>]*(?:<[^<>]*>)?[^<>]*>|\bS_\w+)\(')
    pos = 0
    out = ''
    while True:
        m = pat.search(s, pos)
        if not m:
            return out + s[pos:]
        op = m.end() - 1
        cp = match_close(s, op, '(', ')')
        out += s[pos:m.start()] + m.group(1) + '{' + braces_ctor(s[op + 1:cp]) + '}'
        pos = cp + 1


def rewrite_expr(s):
    s = braces_ctor(s)
    s = re.sub(r'\bbitcast<', 'W_bitcast<', s)
    for b in BUILTINS:
        s = re.sub(r'(?<![\w.])%s\s*\(' % b, 'W_%s(' % b, s)
    s = re.sub(r'(?<![\w.<])(i32|u32|f32|bool)\s*\(', r'W_to_\1(', s)
    s = re.sub(r'(?<![\w.])(\d+)i\b', r'\1', s)
    s = re.sub(r'(?<![\w.])(0x[0-9a-fA-F]+)i\b', r'\1', s)
    s = re.sub(r'\.xy\b(?!\s*\()', '.xy()', s)
    s = re.sub(r'(?<![\w.])_\s*=\s*([^;]*);', r'(void)(\1);', s)
    return s


def rewrite_decls(body):
    # var<function>? name: T = e;   var name: T;   var name = e;   let name(: T)? = e;   const
    body = re.sub(r'\bvar\s+(\w+)\s*:\s*([^=;]+?)\s*=', lambda m: '%s %s =' % (cpp_type(m.group(2)), m.group(1)), body)
    body = re.sub(r'\bvar\s+(\w+)\s*:\s*([^=;]+?)\s*;', lambda m: '%s %s{};' % (cpp_type(m.group(2)), m.group(1)), body)
    body = re.sub(r'\bvar\s+(\w+)\s*=', r'auto \1 =', body)
    body = re.sub(r'\blet\s+(\w+)\s*:\s*([^=;]+?)\s*=', lambda m: '%s %s =' % (cpp_type(m.group(2)), m.group(1)), body)
    body = re.sub(r'\blet\s+(\w+)\s*=', r'auto \1 =', body)
    body = re.sub(r'\bconst\s+(\w+)\s*:\s*([^=;]+?)\s*=', lambda m: 'const %s %s =' % (cpp_type(m.group(2)), m.group(1)), body)
    body = re.sub(r'\bconst\s+(\w+)\s*=', r'const auto \1 =', body)
    return body


def fn_header(name, params, ret):
    ps = []
    for p in split_top(params):
        p = p.strip()
        if not p:
            continue
        pn, pt = p.split(':', 1)
        ps.append('%s %s' % (cpp_type(pt), pn.strip()))
    r = cpp_type(ret) if ret else 'void'
    return 'static %s %s(%s)' % (r, name, ', '.join(ps))


def translate(name, src):
    src = strip_comments(src)
    atomic_mem = 'array<atomic<u32>>' in src
    structs, consts, protos, fns = [], [], [], []
    pos = 0
    n = len(src)
    while pos < n:
        m = re.compile(r'\s*').match(src, pos)
        pos = m.end()
        if pos >= n:
            break
        rest = src[pos:]
        if rest.startswith('@group') or rest.startswith('override') or rest.startswith('var<private>'):
            pos = src.index(';', pos) + 1
            continue
        if rest.startswith('@compute'):
            pos = src.index(')', src.index('@workgroup_size', pos)) + 1
            continue
        if rest.startswith('struct'):
            ob = src.index('{', pos)
            cb = match_close(src, ob, '{', '}')
            sname = src[pos:ob].split()[1]
            members = []
            for mem in split_top(src[ob + 1:cb]):
                mem = mem.strip()
                if not mem:
                    continue
                mn, mt = mem.split(':', 1)
                mt = cpp_type(mt)
                members.append('  %s %s{};' % (mt, mn.strip()))
            structs.append('struct %s {\n%s\n};' % (sname, '\n'.join(members)))
            pos = cb + 1
            if pos < n and src[pos] == ';':
                pos += 1
            continue
        if rest.startswith('alias'):
            end = src.index(';', pos)
            am = re.match(r'alias\s+(\w+)\s*=\s*(.*);', src[pos:end + 1], re.S)
            structs.append('using %s = %s;' % (am.group(1), cpp_type(am.group(2))))
            pos = end + 1
            continue
        if rest.startswith('const'):
            end = src.index(';', pos)
            consts.append('static ' + rewrite_expr(rewrite_decls(src[pos:end + 1])))
            pos = end + 1
            continue
        if rest.startswith('fn'):
            m = re.compile(r'fn\s+(\w+)\s*\(').match(src, pos)
            fname = m.group(1)
            op = m.end() - 1
            cp = match_close(src, op, '(', ')')
            params = src[op + 1:cp]
            ob = src.index('{', cp)
            ret = src[cp + 1:ob].strip()
            ret = ret[2:].strip() if ret.startswith('->') else ''
            cb = match_close(src, ob, '{', '}')
            body = src[ob:cb + 1]
            pos = cb + 1
            if fname in SKIP_FNS:
                continue
            if fname == 'main':
                pm = re.match(r'\s*@builtin\(global_invocation_id\)\s*(\w+)\s*:', params)
                header = 'static void main_(vec3<u32> %s)' % pm.group(1)
            else:
                header = fn_header(fname, params, ret)
            body = rewrite_loops(body)
            body = rewrite_switch(body)
            body = rewrite_decls(body)
            body = rewrite_expr(body)
            protos.append(header + ';')
            fns.append(header + ' ' + body)
            continue
        raise ValueError('%s: cannot parse at: %r' % (name, rest[:80]))

    ns = 'k_' + name
    out = ['// generated from the reference kernel %s.wgsl by oracle/wgsl2cpp.py; do not commit' % name,
           '#include "prelude.hpp"',
           'namespace %s {' % ns,
           'static u32* M; static const u32* ARG;',
           'static thread_local u32 Z0; static thread_local u32 SCRB;',
           ]
    out += structs + consts + protos + fns
    out.append('}  // namespace')
    out.append('''extern "C" void teref_%s(uint32_t* mem, const uint32_t* arg) {
  %s::M = mem; %s::ARG = arg;
  const long gx = arg[0], gy = arg[1], gz = arg[2];
  #pragma omp parallel for collapse(2) schedule(static)
  for (long z = 0; z < gz; z++)
    for (long y = 0; y < gy; y++)
      for (long x = 0; x < gx; x++)
        %s::main_(vec3<u32>((u32)x, (u32)y, (u32)z));
}''' % (name, ns, ns, ns))
    _ = atomic_mem
    return '\n'.join(out) + '\n'


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--src', required=True, help='directory of the reference WGSL kernels')
    ap.add_argument('--out', required=True)
    ap.add_argument('--only', nargs='*', default=None)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    with open(os.path.join(a.out, 'prelude.hpp'), 'w') as fh:
        fh.write(PRELUDE)
    names = sorted(f[:-5] for f in os.listdir(a.src) if f.endswith('.wgsl'))
    if a.only:
        names = [x for x in names if x in a.only]
    done = []
    for nm in names:
        with open(os.path.join(a.src, nm + '.wgsl')) as fh:
            src = fh.read()
        try:
            cpp = translate(nm, src)
        except Exception as e:  # pragma: no cover - reported, not fatal
            print('skip %s: %s' % (nm, e), file=sys.stderr)
            continue
        with open(os.path.join(a.out, nm + '.cpp'), 'w') as fh:
            fh.write(cpp)
        done.append(nm)
    with open(os.path.join(a.out, 'kernels.txt'), 'w') as fh:
        fh.write('\n'.join(done) + '\n')
    print('translated %d kernels' % len(done))


if __name__ == '__main__':
    main()
