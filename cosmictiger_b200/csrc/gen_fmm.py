#!/usr/bin/env python3
"""Generator of the Cartesian FMM operators used by the gravity step.

Emits one C++ header per expansion order P (``fmm_p{P}.h``).  Every operator is
a function template on the arithmetic type ``T`` (float on the device and in the
kick, double in the multipole upsweep), callable from host and device code.

Tensor layout (the reference's ``tensor_trless_sym<T,Q>``, ``cosmictiger/tensor.hpp:62-126``):
a symmetric tensor of orders 0..Q-1 is stored through its components (l,m,n)
with n in {0,1} plus the single (0,0,2) component, Q*Q+1 numbers.  Index of
(l,m,n): (l+m)(l+m+1)/2 + m + [n==1]*Q(Q+1)/2 + [n==2]*Q*Q.  Components with
n >= 2 (other than (0,0,2)) follow from tracelessness,
T(l,m,n) = -(T(l+2,m,n-2) + T(l,m+2,n-2)).  Orders >= 3 are traceless; order 2
keeps its trace through the stored (0,0,2) entry, because the Ewald Green's
function has a non-zero Laplacian (uniform background).

Lengths are scaled by 1e3 inside every operator (the reference's SCALE_FACTOR,
``cosmictiger/fmm_kernels.hpp:33-49``) so that high powers stay in float range.

Operators (mathematics restated from ``src/fmm_kernel_codegen.cpp``):
  greens      D(n)  = d^n(-1/r)                                   (codegen.cpp:1265-1306)
  ewald_*     periodic correction d^n(phi_ewald + 1/r)            (codegen.cpp:1036-1216)
  m2l         L(n) += sum_m M(m) D(n+m) / m!                      (codegen.cpp:1311-1451)
  p2m         M(n)  = detrace((-x)^n) / (2|n|-1)!!  (|n|>=3)      (codegen.cpp:1455-1471)
  m2m         M'(n) = detrace(sum_k C(n,k) (-d)^(n-k) M(k))       (codegen.cpp:1473-1586)
  l2l / l2p   L'(n) = sum_k d^k/k! L(n+k)                         (codegen.cpp:683-834)
The code emitted here is this project's own; only the mathematical definitions
and the storage layout are shared with the reference.
"""
import sys
from fractions import Fraction as Fr
from math import factorial, pi, sqrt, exp

SCALE = 1000.0


def vfact(n):
    return factorial(n[0]) * factorial(n[1]) * factorial(n[2])


def dfact(k):
    r = 1
    while k > 1:
        r *= k
        k -= 2
    return r


def full_set(Q):
    """All multi-indices of total order < Q, ordered by order then lexicographically descending."""
    out = []
    for N in range(Q):
        for a in range(N, -1, -1):
            for b in range(N - a, -1, -1):
                out.append((a, b, N - a - b))
    return out


def tl_index(n, Q):
    l, m, k = n
    s = l + m
    base = s * (s + 1) // 2 + m
    if k == 0:
        return base
    if k == 1:
        return Q * (Q + 1) // 2 + base
    if n == (0, 0, 2):
        return Q * Q
    raise ValueError(n)


def tl_stored(Q):
    out = [n for n in full_set(Q) if n[2] <= 1 or n == (0, 0, 2)]
    return sorted(out, key=lambda n: tl_index(n, Q))


def tl_expand(n, Q, memo=None):
    """Express a full component through stored ones: {stored index: integer coefficient}."""
    if n[2] <= 1 or n == (0, 0, 2):
        return {tl_index(n, Q): 1}
    a = tl_expand((n[0] + 2, n[1], n[2] - 2), Q)
    b = tl_expand((n[0], n[1] + 2, n[2] - 2), Q)
    out = {}
    for d in (a, b):
        for k, v in d.items():
            out[k] = out.get(k, 0) - v
    return {k: v for k, v in out.items() if v != 0}


def sym_index(n):
    """Position of a full multi-index in a packed full symmetric tensor of order < Q (order-major)."""
    N = n[0] + n[1] + n[2]
    base = N * (N + 1) * (N + 2) // 6
    # within order N: enumerate like full_set
    i = 0
    for a in range(N, -1, -1):
        for b in range(N - a, -1, -1):
            if (a, b, N - a - b) == n:
                return base + i
            i += 1
    raise ValueError(n)


def sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def add(a, b):
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def half_range(n):
    """All m with 2m <= n componentwise."""
    for a in range(n[0] // 2 + 1):
        for b in range(n[1] // 2 + 1):
            for c in range(n[2] // 2 + 1):
                yield (a, b, c)


def detrace_coef(n, m):
    """Coefficient of x^(n-2m) r^(2|m|) in the order-|n| detracer (without the 1/(2N-1)!! factor)."""
    N = sum(n)
    m0 = sum(m)
    return Fr((-1) ** m0 * dfact(2 * N - 2 * m0 - 1) * vfact(n), (2 ** m0) * vfact(m) * vfact(sub(n, add(m, m))))


def lit(x):
    """Literal for T: exact rationals printed with 17 significant digits."""
    f = float(x)
    if f == int(f) and abs(f) < 2 ** 24:
        return "T(%d)" % int(f)
    return "T(%.17g)" % f


class Emitter:
    def __init__(self):
        self.lines = []
        self.ind = 1

    def __call__(self, s):
        self.lines.append("\t" * self.ind + s)

    def text(self):
        return "\n".join(self.lines) + "\n"


def monomials(em, name, vx, vy, vz, needed, prefix="T"):
    """Emit products x^a y^b z^c for every multi-index in `needed` (built from lower ones)."""
    have = {(0, 0, 0): "T(1)", (1, 0, 0): vx, (0, 1, 0): vy, (0, 0, 1): vz}
    # close `needed` under taking predecessors so every product has its factors
    need = set(needed)
    changed = True
    while changed:
        changed = False
        for n in list(need):
            if sum(n) >= 2:
                # split into two halves of nearly equal order
                a = list(n)
                b = [0, 0, 0]
                k = sum(n) // 2
                for d in range(3):
                    t = min(a[d], k)
                    a[d] -= t
                    b[d] += t
                    k -= t
                for p in (tuple(a), tuple(b)):
                    if sum(p) >= 2 and p not in need:
                        need.add(p)
                        changed = True
    for n in sorted(need, key=lambda n: (sum(n), n)):
        if n in have:
            continue
        a = list(n)
        b = [0, 0, 0]
        k = sum(n) // 2
        for d in range(3):
            t = min(a[d], k)
            a[d] -= t
            b[d] += t
            k -= t
        nm = "%s%d%d%d" % (name, n[0], n[1], n[2])
        em("const T %s = %s * %s;" % (nm, have[tuple(a)], have[tuple(b)]))
        have[n] = nm
    return have


def emit_sum(em, target, terms, init, op="="):
    """target (op) sum(coef * expr); terms: list of (Fraction coef, expr). Groups equal coefficients."""
    groups = {}
    for c, e in terms:
        if c == 0:
            continue
        groups.setdefault(c, []).append(e)
    parts = []
    lead = None
    if init and 1 in groups:
        # products with coefficient 1 go straight onto the initial value as fused multiply-adds
        lead = init
        for e in groups.pop(1):
            lead = "ct_fma(%s, %s, %s)" % (e[0], e[1], lead) if isinstance(e, tuple) else "(%s + %s)" % (lead, e)
        init = lead
    for c in sorted(groups, key=lambda c: (abs(c), c)):
        exprs = groups[c]
        # products are chained through explicit fused multiply-adds, so that host and device
        # builds evaluate the same operation sequence (no compiler contraction choices)
        e0 = exprs[0]
        acc = "(%s * %s)" % e0 if isinstance(e0, tuple) else e0
        for e in exprs[1:]:
            if isinstance(e, tuple):
                acc = "ct_fma(%s, %s, %s)" % (e[0], e[1], acc)
            else:
                acc = "(%s + %s)" % (acc, e)
        parts.append((c, acc))
    if not parts:
        em("%s = %s;" % (target, init if init else "T(0)"))
        return
    expr = None
    for c, acc in parts:
        if c == 1:
            term = acc
        elif c == -1:
            term = "(-%s)" % acc
        else:
            term = None
        if expr is None:
            if init:
                expr = "ct_fma(%s, %s, %s)" % (lit(c), acc, init) if term is None else "(%s + %s)" % (init, term)
            else:
                expr = "(%s * %s)" % (lit(c), acc) if term is None else term
        else:
            expr = "ct_fma(%s, %s, %s)" % (lit(c), acc, expr) if term is None else "(%s + %s)" % (expr, term)
    em("%s = %s;" % (target, expr))


def full_from_stored(em, arr, name, Q, needed):
    """Emit `const T name_abc` for every needed full component of stored tensor `arr`."""
    out = {}
    for n in sorted(needed, key=lambda n: (sum(n), n)):
        ex = tl_expand(n, Q)
        if len(ex) == 1 and list(ex.values())[0] == 1:
            out[n] = "%s[%d]" % (arr, list(ex.keys())[0])
            continue
        terms = [(Fr(v), "%s[%d]" % (arr, k)) for k, v in sorted(ex.items())]
        nm = "%s%d%d%d" % (name, n[0], n[1], n[2])
        emit_sum(em, "const T " + nm, terms, None)
        out[n] = nm
    return out


def gen_greens(P, accumulate=False):
    """D(n) = d^n(-1/r); with accumulate, L[n] += D(n) instead, the final scaling by
    r^-(|n|+1) fused with the add (one FMA per entry)."""
    em = Emitter()
    stored = tl_stored(P)
    em("x *= T(%g); y *= T(%g); z *= T(%g);" % (SCALE, SCALE, SCALE))
    em("const T r2 = ct_fma(x, x, ct_fma(y, y, z * z));")
    em("const T rinv = ct_rinv(r2);")
    em("const T ux = x * rinv, uy = y * rinv, uz = z * rinv;")
    needed = set()
    for n in stored:
        for m in half_range(n):
            needed.add(sub(n, add(m, m)))
    mon = monomials(em, "u", "ux", "uy", "uz", needed)
    em("T rp1 = rinv;")
    for k in range(2, P + 1):
        em("const T rp%d = rp%d * rinv;" % (k, k - 1))
    for n in stored:
        N = sum(n)
        terms = [(detrace_coef(n, m), mon[sub(n, add(m, m))]) for m in half_range(n)]
        sign = -((-1) ** N)
        terms = [(c * sign, e) for c, e in terms]
        em("{")
        em("\tT s;")
        sub_em = Emitter()
        sub_em.ind = em.ind + 1
        emit_sum(sub_em, "s", terms, None)
        em.lines.extend(sub_em.lines)
        if accumulate:
            em("\tL[%d] = ct_fma(s, rp%d, L[%d]);" % (tl_index(n, P), N + 1, tl_index(n, P)))
        else:
            em("\tD[%d] = s * rp%d;" % (tl_index(n, P), N + 1))
        em("}")
    return em.text()


def gen_radial(P, stf_from=3):
    """Add sum_m n!/(2^m0 m!(n-2m)!) u^(n-2m) g_(N-m0) rinv^m0 into the full tensor Dr (all |n| < P).

    For orders N >= stf_from only the m = 0 term u^n g_N is added: every other term carries a
    Kronecker delta, which the traceless projection of those orders (gen_detrace_full) maps to
    zero, so the stored tensor after the projection is the same."""
    em = Emitter()
    full = full_set(P)
    low = [n for n in full if sum(n) < stf_from]
    high = [n for n in full if sum(n) >= stf_from]
    # orders below stf_from: every term; orders from stf_from on: u^n g_N, formed as
    # (ux^a uy^b) (g_N uz^c), which shares the xy monomials and the z powers across orders
    needed = set()
    for n in low:
        for m in half_range(n):
            needed.add(sub(n, add(m, m)))
    for n in high:
        needed.add((n[0], n[1], 0))
        needed.add((0, 0, n[2]))
    mon = monomials(em, "u", "ux", "uy", "uz", needed)
    em("const T ri1 = rinv;")
    for k in range(2, P // 2 + 1):
        em("const T ri%d = ri%d * rinv;" % (k, k - 1))
    pw = {}
    for n in low:
        N = sum(n)
        for m in half_range(n):
            m0 = sum(m)
            pw[(N - m0, m0)] = True
    for (l, m0) in sorted(pw):
        if m0 == 0:
            em("const T G%d_%d = g%d;" % (l, m0, l))
        else:
            em("const T G%d_%d = g%d * ri%d;" % (l, m0, l, m0))
    zs = sorted({(sum(n), n[2]) for n in high})
    for (N, c) in zs:
        em("const T Z%d_%d = %s;" % (N, c, "g%d" % N if c == 0 else "g%d * %s" % (N, mon[(0, 0, c)])))
    for n in full:
        N = sum(n)
        if N >= stf_from:
            xy = mon[(n[0], n[1], 0)]
            z = "Z%d_%d" % (N, n[2])
            if xy == "T(1)":
                em("Dr[%d] = (Dr[%d] + %s);" % (sym_index(n), sym_index(n), z))
            else:
                em("Dr[%d] = ct_fma(%s, %s, Dr[%d]);" % (sym_index(n), xy, z, sym_index(n)))
            continue
        terms = []
        for m in half_range(n):
            m0 = sum(m)
            c = Fr(vfact(n), (2 ** m0) * vfact(m) * vfact(sub(n, add(m, m))))
            terms.append((c, (mon[sub(n, add(m, m))], "G%d_%d" % (N - m0, m0))))
        emit_sum(em, "Dr[%d]" % sym_index(n), terms, "Dr[%d]" % sym_index(n))
    return em.text()


def gen_detrace_full(P, src, dst):
    """dst (stored, order < P) = detrace_d(src full): orders <= 2 copied, higher orders projected."""
    em = Emitter()
    for n in tl_stored(P):
        N = sum(n)
        if N <= 2:
            em("%s[%d] = %s[%d];" % (dst, tl_index(n, P), src, sym_index(n)))
            continue
        terms = []
        for m in half_range(n):
            m0 = sum(m)
            c = detrace_coef(n, m) / dfact(2 * N - 1)
            p = sub(n, add(m, m))
            # m0-fold trace of src at p: sum_{|k|=m0} m0!/k! src[p+2k]
            for ka in range(m0 + 1):
                for kb in range(m0 - ka + 1):
                    k = (ka, kb, m0 - ka - kb)
                    cc = c * Fr(factorial(m0), vfact(k))
                    terms.append((cc, "%s[%d]" % (src, sym_index(add(p, add(k, k))))))
        # merge equal source entries
        merged = {}
        for c, e in terms:
            merged[e] = merged.get(e, 0) + c
        emit_sum(em, "%s[%d]" % (dst, tl_index(n, P)), [(c, e) for e, c in merged.items()], None)
    return em.text()


def gen_m2l(P, Pmax):
    em = Emitter()
    outs = [n for n in tl_stored(Pmax) if sum(n) < Pmax]
    if Pmax == 2:
        outs = [n for n in outs if sum(n) <= 1]
    needM = set()
    needD = set()
    plan = {}
    for n in outs:
        N = sum(n)
        q = min(P - N, P - 1)
        lst = []
        for m in full_set(q):
            needM.add(m)
            needD.add(add(n, m))
            lst.append(m)
        plan[n] = lst
    Mf = full_from_stored(em, "M", "Mf", P - 1, needM)
    Df = full_from_stored(em, "D", "Df", P, needD)
    for n in outs:
        terms = [(Fr(1, vfact(m)), (Mf[m], Df[add(n, m)])) for m in plan[n]]
        idx = tl_index(n, Pmax)
        if n == (0, 0, 0):
            em("if (do_phi) {")
            sub_em = Emitter()
            sub_em.ind = em.ind + 1
            emit_sum(sub_em, "L[%d]" % idx, terms, "L[%d]" % idx)
            em.lines.extend(sub_em.lines)
            em("}")
        else:
            emit_sum(em, "L[%d]" % idx, terms, "L[%d]" % idx)
    return em.text()


def gen_p2m(P):
    Q = P - 1
    em = Emitter()
    em("x *= T(%g); y *= T(%g); z *= T(%g);" % (-SCALE, -SCALE, -SCALE))
    em("const T r2 = ct_fma(x, x, ct_fma(y, y, z * z));")
    stored = tl_stored(Q)
    needed = set()
    maxm0 = 0
    for n in stored:
        if sum(n) <= 2:
            needed.add(n)
        else:
            for m in half_range(n):
                needed.add(sub(n, add(m, m)))
                maxm0 = max(maxm0, sum(m))
    mon = monomials(em, "y", "x", "y", "z", needed)
    em("const T q1 = r2;")
    for k in range(2, maxm0 + 1):
        em("const T q%d = q%d * r2;" % (k, k - 1))
    for n in stored:
        N = sum(n)
        idx = tl_index(n, Q)
        if N <= 2:
            em("M[%d] = %s;" % (idx, mon[n]))
            continue
        terms = []
        for m in half_range(n):
            m0 = sum(m)
            c = detrace_coef(n, m) / dfact(2 * N - 1)
            e = mon[sub(n, add(m, m))]
            if m0 > 0:
                e = (e, "q%d" % m0)
            terms.append((c, e))
        emit_sum(em, "M[%d]" % idx, terms, None)
    return em.text()


def gen_m2m(P):
    Q = P - 1
    em = Emitter()
    em("x *= T(%g); y *= T(%g); z *= T(%g);" % (-SCALE, -SCALE, -SCALE))
    full = full_set(Q)
    Mf = full_from_stored(em, "Ma", "Mf", Q, set(full))
    mon = monomials(em, "y", "x", "y", "z", set(full))
    em("T Mb[%d];" % len(full))
    for n in full:
        terms = []
        for a in range(n[0] + 1):
            for b in range(n[1] + 1):
                for c in range(n[2] + 1):
                    k = (a, b, c)
                    coef = Fr(vfact(n), vfact(k) * vfact(sub(n, k)))
                    d = sub(n, k)
                    e = Mf[k] if d == (0, 0, 0) else (mon[d], Mf[k])
                    terms.append((coef, e))
        emit_sum(em, "Mb[%d]" % sym_index(n), terms, None)
    em.lines.extend(gen_detrace_full(Q, "Mb", "M").splitlines())
    return em.text()


def gen_l2l(P, Qout):
    em = Emitter()
    em("x *= T(%g); y *= T(%g); z *= T(%g);" % (SCALE, SCALE, SCALE))
    outs = [n for n in tl_stored(Qout) if sum(n) < Qout]
    if Qout == 2:
        outs = [n for n in outs if sum(n) <= 1]
    needL = set()
    needX = set()
    plan = {}
    for n in outs:
        N = sum(n)
        lst = []
        for k in full_set(P - N):
            needL.add(add(n, k))
            needX.add(k)
            lst.append(k)
        plan[n] = lst
    Lf = full_from_stored(em, "La", "Lf", P, needL)
    mon = monomials(em, "y", "x", "y", "z", needX)
    for n in outs:
        terms = []
        for k in plan[n]:
            e = Lf[add(n, k)] if k == (0, 0, 0) else (mon[k], Lf[add(n, k)])
            terms.append((Fr(1, vfact(k)), e))
        idx = tl_index(n, Qout)
        if n == (0, 0, 0):
            em("if (do_phi) {")
            sub_em = Emitter()
            sub_em.ind = em.ind + 1
            emit_sum(sub_em, "Lb[%d]" % idx, terms, None)
            em.lines.extend(sub_em.lines)
            em("} else {")
            em("\tLb[%d] = La[%d];" % (idx, tl_index(n, P)))
            em("}")
        else:
            emit_sum(em, "Lb[%d]" % idx, terms, None)
    return em.text()


def gen_header(P):
    Q = P - 1
    nexp = P * P + 1
    nmul = Q * Q + 1
    nfull = P * (P + 1) * (P + 2) // 6
    ns = "ct_p%d" % P
    h = []
    h.append("// Generated by gen_fmm.py for expansion order %d. Do not edit." % P)
    h.append("// Cartesian FMM operators in the reference's trace-reduced symmetric tensor layout")
    h.append("// (cosmictiger/tensor.hpp:62-126); mathematics follow src/fmm_kernel_codegen.cpp.")
    h.append("#pragma once")
    h.append('#include "fmm_common.h"')
    h.append("namespace %s {" % ns)
    h.append("constexpr int ORDER = %d;" % P)
    h.append("constexpr int NEXP = %d;   // local expansion (orders < %d)" % (nexp, P))
    h.append("constexpr int NMULT = %d;  // multipole (orders < %d)" % (nmul, Q))
    h.append("constexpr int NFULL = %d;  // full symmetric tensor (orders < %d)" % (nfull, P))
    h.append("")
    h.append("// D(n) = d^n(-1/r) at (x,y,z) (box units; scaled by 1e3 inside). fmm_kernels.hpp:52-307")
    h.append("template<class T> CT_HD void greens(T* __restrict__ D, T x, T y, T z) {")
    h.append(gen_greens(P).rstrip())
    h.append("}")
    h.append("")
    h.append("// L(n) += D(n) at (x,y,z): P2L of a unit mass, without storing D (each entry's")
    h.append("// r^-(|n|+1) scaling fused with the add). gravity.cu:134-144")
    h.append("template<class T> CT_HD void greens_add(T* __restrict__ L, T x, T y, T z) {")
    h.append(gen_greens(P, accumulate=True).rstrip())
    h.append("}")
    h.append("")
    h.append("// Add the radial-function derivative tensor: Dr[n] += sum_m n!/(2^|m| m!(n-2m)!) u^(n-2m) g_(|n|-|m|) rinv^|m|,")
    h.append("// where g_k = r^k (r^-1 d/dr)^k f and u the unit vector (full packed symmetric storage).  Orders >= 3")
    h.append("// keep only the m = 0 term u^n g_|n|: the others carry a Kronecker delta, which detrace_full's")
    h.append("// traceless projection of those orders maps to zero, so only the projected sum is meaningful there.")
    h.append("template<class T> CT_HD void radial_add(T* __restrict__ Dr, T ux, T uy, T uz, T rinv, const T* g) {")
    gl = ["\tconst T g%d = g[%d];" % (k, k) for k in range(P)]
    h.extend(gl)
    h.append(gen_radial(P).rstrip())
    h.append("}")
    h.append("")
    h.append("// Stored (trace-reduced) tensor from a full symmetric one: orders <= 2 copied, orders >= 3 projected")
    h.append("// onto their traceless part (the reference's 'd' detracer, src/fmm_kernel_codegen.cpp:165-371).")
    h.append("template<class T> CT_HD void detrace_full(T* __restrict__ D, const T* __restrict__ Dr) {")
    h.append(gen_detrace_full(P, "Dr", "D").rstrip())
    h.append("}")
    h.append("")
    h.append("// L(n) += sum_m M(m) D(n+m)/m!  (orders of L < %d). fmm_kernels.hpp:1495-1890" % P)
    h.append("template<class T> CT_HD void m2l(T* __restrict__ L, const T* __restrict__ M, const T* __restrict__ D, bool do_phi) {")
    h.append(gen_m2l(P, P).rstrip())
    h.append("}")
    h.append("")
    h.append("// Second-order variant for M2P: L[0..3] (potential and gradient) at a particle.")
    h.append("template<class T> CT_HD void m2l_2(T* __restrict__ L, const T* __restrict__ M, const T* __restrict__ D, bool do_phi) {")
    h.append(gen_m2l(P, 2).rstrip())
    h.append("}")
    h.append("")
    h.append("// Multipole of a unit mass at offset (x,y,z) from the expansion centre. fmm_kernels.hpp:2863")
    h.append("template<class T> CT_HD void p2m(T* __restrict__ M, T x, T y, T z) {")
    h.append(gen_p2m(P).rstrip())
    h.append("}")
    h.append("")
    h.append("// Shift a multipole whose centre sits at (x,y,z) relative to the new centre. fmm_kernels.hpp:3095")
    h.append("template<class T> CT_HD void m2m(T* __restrict__ M, const T* __restrict__ Ma, T x, T y, T z) {")
    h.append(gen_m2m(P).rstrip())
    h.append("}")
    h.append("")
    h.append("// Taylor shift of a local expansion by (x,y,z). fmm_kernels.hpp:3973")
    h.append("template<class T> CT_HD void l2l(T* __restrict__ Lb, const T* __restrict__ La, T x, T y, T z, bool do_phi) {")
    h.append(gen_l2l(P, P).rstrip())
    h.append("}")
    h.append("")
    h.append("// Potential and gradient of a local expansion at offset (x,y,z). fmm_kernels.hpp:4958")
    h.append("template<class T> CT_HD void l2p(T* __restrict__ Lb, const T* __restrict__ La, T x, T y, T z, bool do_phi) {")
    h.append(gen_l2l(P, 2).rstrip())
    h.append("}")
    h.append("")
    def table(name, ctype, dims, body, comment):
        # one host copy and one __constant__ device copy, read through an accessor
        h.append("// " + comment)
        h.append("static constexpr %s %s_H%s = {%s};" % (ctype, name, dims, body))
        h.append("#ifdef __CUDACC__")
        h.append("static __constant__ %s %s_D%s = {%s};" % (ctype, name, dims, body))
        h.append("#endif")
    table("FULL_IDX", "unsigned char", "[NFULL][3]", ", ".join("{%d,%d,%d}" % n for n in sorted(full_set(P), key=sym_index)),
          "Exponents (x,y,z) of the full packed symmetric tensor components, order-major.")
    table("EXP_IDX", "unsigned char", "[NEXP][3]", ", ".join("{%d,%d,%d}" % n for n in tl_stored(P)),
          "Exponents (x,y,z) of the stored components of a local expansion, in storage order.")
    table("MULT_IDX", "unsigned char", "[NMULT][3]", ", ".join("{%d,%d,%d}" % n for n in tl_stored(Q)),
          "Exponents (x,y,z) of the stored components of a multipole, in storage order.")
    h.append("#ifdef __CUDA_ARCH__")
    h.append("#define CT_TAB(name) name##_D")
    h.append("#else")
    h.append("#define CT_TAB(name) name##_H")
    h.append("#endif")
    h.append("")
    # series of (z^-1 d/dz)^l [erf(z)/z] in w = z^2 (used by ewald_greens for the n = 0 image)
    K = 26
    b = [Fr(2) / Fr(1) * Fr((-1) ** k, factorial(k) * (2 * k + 1)) for k in range(K + P)]
    rows = []
    for l in range(P):
        row = []
        for j in range(K):
            k = j + l
            row.append(float(b[k] * (2 ** l) * Fr(factorial(k), factorial(j))) / sqrt(pi))
        rows.append("{" + ", ".join("%.17g" % v for v in row) + "}")
    h.append("// (z^-1 d/dz)^l [erf(z)/z] = sum_j ERF_SERIES[l][j] z^(2j), |z| <= 1.8 (26 terms)")
    h.append("constexpr int ERF_SERIES_N = %d;" % K)
    body = ",\n\t".join(rows)
    h.append("static constexpr double ERF_SERIES_H[ORDER][ERF_SERIES_N] = {%s};" % body)
    h.append("#ifdef __CUDACC__")
    h.append("static __constant__ double ERF_SERIES_D[ORDER][ERF_SERIES_N] = {%s};" % body)
    h.append("// the same coefficients rounded to float once, for the single-precision evaluation")
    h.append("static __constant__ float ERF_SERIES_DF[ORDER][ERF_SERIES_N] = {%s};" % body)
    h.append("#endif")
    h.append("template<class T> CT_HD T erf_series(int l, int j) {")
    h.append("#ifdef __CUDA_ARCH__")
    h.append("\tif constexpr (sizeof(T) == sizeof(float)) {")
    h.append("\t\treturn ERF_SERIES_DF[l][j];")
    h.append("\t} else {")
    h.append("\t\treturn T(ERF_SERIES_D[l][j]);")
    h.append("\t}")
    h.append("#else")
    h.append("\treturn T(ERF_SERIES_H[l][j]);")
    h.append("#endif")
    h.append("}")
    # Fourier accumulation unrolled: odd-order entries take the sine, even ones the cosine
    acc = "\n".join("\t\tD[%d] = ct_fma(%s, T(tab.four_exp[i][%d]), D[%d]);" % (kk, "sn" if sum(n) & 1 else "cn", kk, kk)
                    for kk, n in enumerate(tl_stored(P)))
    h.append(EWALD_TEMPLATE.replace("@FOURIER_ACC@", acc))
    h.append("}  // namespace %s" % ns)
    return "\n".join(h) + "\n"


EWALD_TEMPLATE = r"""
// Periodic (Ewald) correction to the Green's function, d^n(phi_periodic + 1/r), for a separation
// (x,y,z) inside the unit cell: the n=0 image with the bare 1/r removed (erf series), the
// real-space images inside the CT_EWALD_RCUT_G cutoff (erfc, Abramowitz & Stegun 7.1.26), the Fourier
// sum over 0<|h|^2<=8 and the pi/alpha^2 background term, alpha = 2.
// Follows ewald_greens_function, cosmictiger/fmm_kernels.hpp:310-1491.
template<class T, class Tab> CT_HD int ewald_greens(T* __restrict__ D, T x, T y, T z, const Tab& tab) {
	x *= T(1000); y *= T(1000); z *= T(1000);
	T Dr[NFULL];
	for (int i = 0; i < NFULL; i++) {
		Dr[i] = T(0);
	}
	T g[ORDER];
	int icnt = 0;
	{
		const T r2 = ct_fma(x, x, ct_fma(y, y, z * z));
		const T r = ct_sqrt(r2);
		icnt++;
		if (r > T(0)) {
			// n = 0 image: f = erf(beta r)/r, beta = 2e-3 in scaled units.  The reference's
			// downward recursion (fmm_kernels.hpp:333-356) cancels catastrophically for small r;
			// the same derivatives are taken here from the convergent series of
			// F(z) = erf(z)/z, z = beta r:  g_l = beta^(l+1) z^l F_(l)(z),
			// F_(l) = (z^-1 d/dz)^l F = sum_j ERF_SERIES[l][j] (z^2)^j.
			const T rinv = T(1) / r;
			const T zz = T(2e-3) * r;
			const T w = zz * zz;
			T zl = T(1);
			T bl = T(2e-3);
			for (int l = 0; l < ORDER; l++) {
				T s = erf_series<T>(l, ERF_SERIES_N - 1);
				for (int j = ERF_SERIES_N - 2; j >= 0; j--) {
					s = ct_fma(s, w, erf_series<T>(l, j));
				}
				g[l] = bl * zl * s;
				zl *= zz;
				bl *= T(2e-3);
			}
			radial_add(Dr, x * rinv, y * rinv, z * rinv, rinv, g);
		} else {
			for (int i = 0; i < NFULL; i++) {
				Dr[i] = T(tab.D0[i]);
			}
		}
	}
	// Real images inside the cutoff: a first pass marks them in a bit set, the second evaluates
	// them in increasing order.  Each thread then loops over its own images only, so the
	// threads of a warp (each with its own separation) no longer step through the union of
	// their image sets; the accumulation order is unchanged.
	// Only the first CT_EWALD_NREAL_G images of the table (those within CT_EWALD_RCUT_G of the
	// unit cell) can be inside the cutoff.
	static_assert((CT_EWALD_NREAL_G + 31) / 32 == 4, "four words of image bits");
	unsigned int inside[4];
	int nin = 0;
	for (int wd = 0; wd < 4; wd++) {
		unsigned int m = 0u;
		for (int b = 0; b < 32 && 32 * wd + b < CT_EWALD_NREAL_G; b++) {
			const int i = 32 * wd + b;
			const T dx = x - T(1000) * T(tab.real[i][0]);
			const T dy = y - T(1000) * T(tab.real[i][1]);
			const T dz = z - T(1000) * T(tab.real[i][2]);
			const T r2 = ct_fma(dx, dx, ct_fma(dy, dy, dz * dz));
			m |= (unsigned int) (r2 < T(1000 * 1000 * CT_EWALD_RCUT_G * CT_EWALD_RCUT_G)) << b;
		}
		inside[wd] = m;
		nin += ct_popc(m);
	}
	int wd = 0;
	unsigned int bits = inside[0];
	for (int q = 0; q < nin; q++) {
		while (bits == 0u) {
			wd++;
			bits = ct_word4(inside, wd);
		}
		const int i = 32 * wd + ct_ffs(bits) - 1;
		bits &= bits - 1u;
		{
			const T dx = x - T(1000) * T(tab.real[i][0]);
			const T dy = y - T(1000) * T(tab.real[i][1]);
			const T dz = z - T(1000) * T(tab.real[i][2]);
			const T r2 = ct_fma(dx, dx, ct_fma(dy, dy, dz * dz));
			icnt++;
			T r, rinv;
			ct_dist(r2, &r, &rinv);
			T ec, ex;
			ct_erfcexp(T(2e-3) * r, &ec, &ex);
			T e0 = T(2.2567583341910252e-3) * ex * rinv;
			const T n8r = T(-8e-6) * r;
			g[0] = -ec * rinv;
			for (int l = 1; l < ORDER; l++) {
				g[l] = ct_fma(T(1 - 2 * l) * g[l - 1], rinv, e0);
				e0 *= n8r;
			}
			radial_add(Dr, dx * rinv, dy * rinv, dz * rinv, rinv, g);
		}
	}
	detrace_full(D, Dr);
	// Fourier terms accumulate straight into the detraced real-space sum.  The vectors h and -h
	// add the same term (the order-n derivative tensor changes sign by (-1)^n, the sine with
	// h, so every entry's product is unchanged): the first half of the table holds one vector
	// of each pair (ewald_build_indices), taken twice.
	static_assert(CT_EWALD_NFOUR % 2 == 0, "Fourier vectors come in +h/-h pairs");
#pragma unroll 1
	for (int i = 0; i < CT_EWALD_NFOUR / 2; i++) {
		const T hdotx = ct_fma(T(tab.four[i][0]), x, ct_fma(T(tab.four[i][1]), y, T(tab.four[i][2]) * z));
		T sn, cn;
		ct_sincos_poly(T(6.2831853071795865e-3) * hdotx, &sn, &cn);
		sn *= T(2);
		cn *= T(2);
@FOURIER_ACC@
	}
	D[0] += T(7.8539816339744831e-4);
	return icnt;
}

// Ewald table storage for this order (lives in __constant__ memory on the device).
struct EwaldTab {
	float real[CT_EWALD_NREAL][3];       // real-space image vectors: the CT_EWALD_NREAL_G within CT_EWALD_RCUT_G of the cell first; |n|^2 descending in each part
	float four[CT_EWALD_NFOUR][3];       // Fourier vectors: one of each +h/-h pair, then the negatives (|h|^2 descending in each half)
	float four_exp[CT_EWALD_NFOUR][NEXP];  // detraced derivative tensors of the Fourier terms
	float D0[NFULL];                     // r -> 0 limit of d^n(erf(alpha r)/r), full storage
};

// Fourier-term derivative tensor of vector h in FP64:
// d^n [c0 cos(2 pi h.x)] / {cos|sin}, c0 = -exp(-pi^2 h^2/alpha^2)/(pi h^2), scaled for 1e3 units,
// then detraced (src/ewald_indices.cu:67-86).
CT_HD_FN void ewald_four_entry(double* __restrict__ out, double hx, double hy, double hz) {
	const double h2 = hx * hx + hy * hy + hz * hz;
	const double c0 = -exp(-9.8696044010893586 * h2 / 4.0) / (3.1415926535897932 * h2);
	const double w = 6.2831853071795865e-3;
	const double sgn[4] = { 1.0, -1.0, -1.0, 1.0 };
	double F[NFULL];
	for (int c = 0; c < NFULL; c++) {
		const int a = CT_TAB(FULL_IDX)[c][0], b = CT_TAB(FULL_IDX)[c][1], d = CT_TAB(FULL_IDX)[c][2];
		const int N = a + b + d;
		double v = c0 * 1e-3 * sgn[N % 4];
		for (int k = 0; k < a; k++) v *= hx * w;
		for (int k = 0; k < b; k++) v *= hy * w;
		for (int k = 0; k < d; k++) v *= hz * w;
		F[c] = v;
	}
	detrace_full(out, F);
}

// r -> 0 limit of d^n(erf(alpha r)/r) with alpha = 2 (x1e-3 units), FP64; non-zero only for
// all-even n: 2 (-2)^k beta^(N+1) / ((N+1) sqrt(pi)) prod (n_i-1)!!, N = 2k, beta = 2e-3
// (src/ewald_indices.cu:89-101 stores the negative of this).
CT_HD_FN double ewald_d0_entry(int c) {
	const int a = CT_TAB(FULL_IDX)[c][0], b = CT_TAB(FULL_IDX)[c][1], d = CT_TAB(FULL_IDX)[c][2];
	if ((a & 1) || (b & 1) || (d & 1)) {
		return 0.0;
	}
	const int N = a + b + d;
	const int k = N / 2;
	double v = 2.0 / ((N + 1) * 1.7724538509055160);
	for (int i = 0; i < k; i++) v *= -2.0;
	for (int i = 0; i <= N; i++) v *= 2e-3;
	for (int i = a - 1; i > 1; i -= 2) v *= i;
	for (int i = b - 1; i > 1; i -= 2) v *= i;
	for (int i = d - 1; i > 1; i -= 2) v *= i;
	return v;
}

// Image and Fourier vectors, each list ordered by |n|^2 descending (ties in enumeration order)
// (src/ewald_indices.cu:32-66); the image list is then split at CT_EWALD_RCUT_G from the unit
// cell and the Fourier list into +h and -h halves.
inline void ewald_build_indices(EwaldTab& tab) {
	int cnt = 0;
	for (int i = -4; i <= 4; i++) {
		for (int j = -4; j <= 4; j++) {
			for (int k = -4; k <= 4; k++) {
				const double x = i < 0 ? -i - 0.5 : (i > 0 ? i - 0.5 : 0.0);
				const double y = j < 0 ? -j - 0.5 : (j > 0 ? j - 0.5 : 0.0);
				const double z = k < 0 ? -k - 0.5 : (k > 0 ? k - 0.5 : 0.0);
				const double dd = sqrt(x * x + y * y + z * z);
				if (dd < 2.6 && i * i + j * j + k * k > 0 && cnt < CT_EWALD_NREAL) {
					tab.real[cnt][0] = float(i);
					tab.real[cnt][1] = float(j);
					tab.real[cnt][2] = float(k);
					cnt++;
				}
			}
		}
	}
	cnt = 0;
	for (int i = -3; i <= 3; i++) {
		for (int j = -3; j <= 3; j++) {
			for (int k = -3; k <= 3; k++) {
				const int h2 = i * i + j * j + k * k;
				if (h2 > 0 && h2 <= 8 && cnt < CT_EWALD_NFOUR) {
					tab.four[cnt][0] = float(i);
					tab.four[cnt][1] = float(j);
					tab.four[cnt][2] = float(k);
					cnt++;
				}
			}
		}
	}
	auto sort_desc = [](float (*v)[3], int n) {
		for (int a = 1; a < n; a++) {
			float t[3] = { v[a][0], v[a][1], v[a][2] };
			const float ta = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
			int b = a - 1;
			while (b >= 0 && v[b][0] * v[b][0] + v[b][1] * v[b][1] + v[b][2] * v[b][2] < ta) {
				v[b + 1][0] = v[b][0];
				v[b + 1][1] = v[b][1];
				v[b + 1][2] = v[b][2];
				b--;
			}
			v[b + 1][0] = t[0];
			v[b + 1][1] = t[1];
			v[b + 1][2] = t[2];
		}
	};
	sort_desc(tab.real, CT_EWALD_NREAL);
	// the images within CT_EWALD_RCUT_G of the unit cell first (the only ones the kick's Green's
	// function can reach), the rest after; |n|^2 descending in each part (a stable partition)
	{
		float near_[CT_EWALD_NREAL][3], far_[CT_EWALD_NREAL][3];
		int nn_ = 0, nf_ = 0;
		for (int a = 0; a < CT_EWALD_NREAL; a++) {
			double d2 = 0.0;
			for (int d = 0; d < 3; d++) {
				const double c = tab.real[a][d] < 0.f ? -tab.real[a][d] - 0.5 : (tab.real[a][d] > 0.f ? tab.real[a][d] - 0.5 : 0.0);
				d2 += c * c;
			}
			float* dst = d2 < CT_EWALD_RCUT_G * CT_EWALD_RCUT_G ? near_[nn_++] : far_[nf_++];
			for (int d = 0; d < 3; d++) {
				dst[d] = tab.real[a][d];
			}
		}
		for (int a = 0; a < nn_; a++) {
			for (int d = 0; d < 3; d++) {
				tab.real[a][d] = near_[a][d];
			}
		}
		for (int a = 0; a < nf_; a++) {
			for (int d = 0; d < 3; d++) {
				tab.real[nn_ + a][d] = far_[a][d];
			}
		}
	}
	sort_desc(tab.four, CT_EWALD_NFOUR);
	// one vector of each +h/-h pair (first nonzero component positive) in the first half, the
	// negatives in the second, each half still by |h|^2 descending (a stable partition)
	float pos[CT_EWALD_NFOUR][3], neg[CT_EWALD_NFOUR][3];
	int np = 0, nn = 0;
	for (int a = 0; a < CT_EWALD_NFOUR; a++) {
		const float* v = tab.four[a];
		const bool first = v[0] > 0.f || (v[0] == 0.f && (v[1] > 0.f || (v[1] == 0.f && v[2] > 0.f)));
		float* dst = first ? pos[np++] : neg[nn++];
		dst[0] = v[0];
		dst[1] = v[1];
		dst[2] = v[2];
	}
	for (int a = 0; a < np; a++) {
		for (int d = 0; d < 3; d++) {
			tab.four[a][d] = pos[a][d];
		}
	}
	for (int a = 0; a < nn; a++) {
		for (int d = 0; d < 3; d++) {
			tab.four[np + a][d] = neg[a][d];
		}
	}
}

// Complete table build on the host in FP64 (the device build runs ewald_four_entry and
// ewald_d0_entry in an FP64 kernel instead).
inline void ewald_build_host(EwaldTab& tab) {
	ewald_build_indices(tab);
	for (int i = 0; i < CT_EWALD_NFOUR; i++) {
		double E[NEXP];
		ewald_four_entry(E, tab.four[i][0], tab.four[i][1], tab.four[i][2]);
		for (int k = 0; k < NEXP; k++) {
			tab.four_exp[i][k] = float(E[k]);
		}
	}
	for (int c = 0; c < NFULL; c++) {
		tab.D0[c] = float(ewald_d0_entry(c));
	}
}
"""


if __name__ == "__main__":
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    orders = [int(a) for a in sys.argv[1:]] or [7, 5]
    for P in orders:
        with open(os.path.join(here, "fmm_p%d.h" % P), "w") as f:
            f.write(gen_header(P))
