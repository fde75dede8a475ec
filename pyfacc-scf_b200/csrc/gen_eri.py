#!/usr/bin/env python3
"""Generate eri_classes.cuh: straight-line Obara-Saika / Head-Gordon-Pople
code for every s/p shell-quartet class of STO-nG bases.

For a class (la lb|lc ld) with la >= lb, lc >= ld the generator emits

* ``vrr``  : one primitive quartet, [e0|f0]^(0) for l(e) in [la, la+lb],
             l(f) in [lc, lc+ld] built from I_m = pref*F_m(T) by the OS
             vertical recursion, added into the contracted accumulators;
* ``hrr``  : the horizontal recursion (a b| = (a+1_i b-1_i| + AB_i (a b-1_i|
             on the contracted accumulators, bra then ket, giving (ab|cd);
* ``grad`` : one primitive quartet of the nuclear-gradient contraction
             sum_abcd Gamma_abcd d(ab|cd)/dX for the centres A, B, C
             (D follows from translational invariance), using
             d/dA_x phi_a = 2 alpha phi_{a+1x} - a_x phi_{a-1x}.

It also emits the algorithmic FP operation count (each + - * is one flop)
of every routine; the kernels multiply them by the number of primitive and
contracted quartets they evaluate to report FLOP/s.

The recursions are the textbook ones (Obara & Saika, J. Chem. Phys. 84,
3963 (1986); Head-Gordon & Pople, J. Chem. Phys. 89, 5777 (1988)), the same
algorithm the reference delegates to Libint 2.11.1 (libint_f.f90:303-625).
Cartesian components follow cartesian.f90:7-23 (x descending, then y).
"""
from __future__ import annotations

import os
import sys

AX = 'xyz'


def comps(l):
    out = []
    for ax in range(l, -1, -1):
        for ay in range(l - ax, -1, -1):
            out.append((ax, ay, l - ax - ay))
    return out


def lsum(c):
    return c[0] + c[1] + c[2]


def first_axis(c):
    for i in range(3):
        if c[i] > 0:
            return i
    return -1


def up(c, i):
    c = list(c)
    c[i] += 1
    return tuple(c)


def down(c, i):
    c = list(c)
    c[i] -= 1
    return tuple(c)


def cname(c):
    return f"{c[0]}{c[1]}{c[2]}"


def scaled(c, name):
    """c * name for a small positive integer c, in the kernel's type R."""
    return name if c == 1 else f"(R({c}.0f) * {name})"


def fma_chain(terms, tail=None):
    """sum of the products a * b of terms (+ tail) as nested pf_fma calls,
    so that the code maps onto FMA instructions for every R (double, float
    and the packed float pair, whose pf_fma is one FFMA2)."""
    if tail is None:
        a, b = terms[-1]
        expr = f"{a} * {b}"
        terms = terms[:-1]
    else:
        expr = tail
    for a, b in reversed(terms):
        expr = f"pf_fma({a}, {b}, {expr})"
    return expr


def plain_sum(terms):
    """sum of the products a * b of terms as a plain expression."""
    return " + ".join(f"{a} * {b}" for a, b in terms)


class Emitter:
    def __init__(self):
        self.lines = []
        self.flops = 0
        self.n = 0

    def tmp(self, expr, flops):
        name = f"t{self.n}"
        self.n += 1
        self.lines.append(f"    const R {name} = {expr};")
        self.flops += flops
        return name


class Vrr:
    """Symbolic OS VRR on one primitive quartet."""

    def __init__(self, em: Emitter, L: int, packed: bool = True):
        # packed: pf_fma chains (the J/K routines, instantiated for the packed
        # float pair too); else plain sums, which the compiler contracts and
        # schedules more freely in the large gradient routines (their pf_fma
        # form spilled to local memory)
        self.em = em
        self.L = L
        self.memo = {}
        self.packed = packed

    def V(self, e, f, m):
        key = (e, f, m)
        if key in self.memo:
            return self.memo[key]
        em = self.em
        if lsum(e) == 0 and lsum(f) == 0:
            r = f"I[{m}]"
        elif lsum(f) == 0:
            i = first_axis(e)
            e1 = down(e, i)
            terms, fl = [(f"PA[{i}]", self.V(e1, f, m)), (f"WP[{i}]", self.V(e1, f, m + 1))], 3
            if e1[i] > 0:
                e2 = down(e1, i)
                if self.packed:
                    terms.append((scaled(e1[i], "o2p"), f"pf_fma(nrp, {self.V(e2, f, m + 1)}, {self.V(e2, f, m)})"))
                else:
                    terms.append((scaled(e1[i], "o2p"), f"({self.V(e2, f, m)} + nrp * {self.V(e2, f, m + 1)})"))
                fl += 4 + (1 if e1[i] > 1 else 0)
            r = em.tmp(fma_chain(terms) if self.packed else plain_sum(terms), fl)
        else:
            i = first_axis(f)
            f1 = down(f, i)
            terms, fl = [(f"QC[{i}]", self.V(e, f1, m)), (f"WQ[{i}]", self.V(e, f1, m + 1))], 3
            if f1[i] > 0:
                f2 = down(f1, i)
                if self.packed:
                    terms.append((scaled(f1[i], "o2q"), f"pf_fma(nrq, {self.V(e, f2, m + 1)}, {self.V(e, f2, m)})"))
                else:
                    terms.append((scaled(f1[i], "o2q"), f"({self.V(e, f2, m)} + nrq * {self.V(e, f2, m + 1)})"))
                fl += 4 + (1 if f1[i] > 1 else 0)
            if e[i] > 0:
                terms.append((scaled(e[i], "o2pq"), self.V(down(e, i), f1, m + 1)))
                fl += 2 + (1 if e[i] > 1 else 0)
            r = em.tmp(fma_chain(terms) if self.packed else plain_sum(terms), fl)
        self.memo[key] = r
        return r


class Hrr:
    """Symbolic HGP HRR.  base(e, f) gives the name of [e0|f0]."""

    def __init__(self, em: Emitter, base, packed: bool = True):
        self.em = em
        self.base = base
        self.mb = {}
        self.mk = {}
        self.packed = packed

    def bra(self, a, b, f):
        key = (a, b, f)
        if key in self.mb:
            return self.mb[key]
        if lsum(b) == 0:
            r = self.base(a, f)
        else:
            i = first_axis(b)
            x, y = self.bra(up(a, i), down(b, i), f), self.bra(a, down(b, i), f)
            r = self.em.tmp(f"pf_fma(AB[{i}], {y}, {x})" if self.packed else f"{x} + AB[{i}] * {y}", 2)
        self.mb[key] = r
        return r

    def full(self, a, b, c, d):
        key = (a, b, c, d)
        if key in self.mk:
            return self.mk[key]
        if lsum(d) == 0:
            r = self.bra(a, b, c)
        else:
            i = first_axis(d)
            x, y = self.full(a, b, up(c, i), down(d, i)), self.full(a, b, c, down(d, i))
            r = self.em.tmp(f"pf_fma(CD[{i}], {y}, {x})" if self.packed else f"{x} + CD[{i}] * {y}", 2)
        self.mk[key] = r
        return r


def ecomps(lo, hi):
    out = []
    for l in range(max(lo, 0), hi + 1):
        out.extend(comps(l))
    return out


def gen_class(la, lb, lc, ld):
    L = la + lb + lc + ld
    E = ecomps(la, la + lb)
    F = ecomps(lc, lc + ld)
    acc_index = {}
    for e in E:
        for f in F:
            acc_index[(e, f)] = len(acc_index)
    nacc = len(acc_index)
    nout = len(comps(la)) * len(comps(lb)) * len(comps(lc)) * len(comps(ld))
    tag = f"{la}{lb}{lc}{ld}"
    src = []
    src.append(f"template <typename R> struct EriClass<R, {la}, {lb}, {lc}, {ld}> {{")
    src.append(f"  static constexpr int L = {L};")
    src.append(f"  static constexpr int NACC = {nacc};")
    src.append(f"  static constexpr int NOUT = {nout};")
    # --- vrr
    em = Emitter()
    v = Vrr(em, L)
    acc_lines = []
    for (e, f), k in acc_index.items():
        acc_lines.append(f"    acc[{k}] += {v.V(e, f, 0)};")
        em.flops += 1
    vrr_flops = em.flops
    src.append("  __device__ static __forceinline__ void vrr(const R* __restrict__ I, const R* __restrict__ PA,")
    src.append("      const R* __restrict__ WP, const R* __restrict__ QC, const R* __restrict__ WQ, R o2p, R nrp,")
    src.append("      R o2q, R nrq, R o2pq, R* __restrict__ acc) {")
    src.extend(em.lines)
    src.extend(acc_lines)
    src.append("    (void)PA; (void)WP; (void)QC; (void)WQ; (void)o2p; (void)nrp; (void)o2q; (void)nrq; (void)o2pq;")
    src.append("  }")
    # --- hrr
    em = Emitter()
    h = Hrr(em, lambda e, f: f"acc[{acc_index[(e, f)]}]")
    out_lines = []
    k = 0
    for a in comps(la):
        for b in comps(lb):
            for c in comps(lc):
                for d in comps(ld):
                    out_lines.append(f"    out[{k}] = {h.full(a, b, c, d)};")
                    k += 1
    hrr_flops = em.flops
    src.append("  __device__ static __forceinline__ void hrr(const R* __restrict__ acc, const R* __restrict__ AB,")
    src.append("      const R* __restrict__ CD, R* __restrict__ out) {")
    src.extend(em.lines)
    src.extend(out_lines)
    src.append("    (void)AB; (void)CD;")
    src.append("  }")
    # --- gradient (primitive level, contracted with gam).  Below L = 4 one
    # inlined routine per centre and direction (the compiler merges their
    # common recursion terms); from L = 4 on one out-of-line routine per
    # centre whose three directions share one recursion to L + 1 (half the
    # operations of three separate ones; inlined, the (pp|pp) body exhausts
    # the register file)
    grad_flops = 0
    for ctr in range(3 if L >= 4 else 0):
        em = Emitter()
        v = Vrr(em, L + 1, packed=False)
        h = Hrr(em, lambda e, f, v=v: v.V(e, f, 0), packed=False)
        outs = []
        for x in range(3):
            up_terms, dn_terms = [], []
            k = 0
            for a in comps(la):
                for b in comps(lb):
                    for c in comps(lc):
                        for d in comps(ld):
                            q = [a, b, c, d]
                            qu = list(q)
                            qu[ctr] = up(q[ctr], x)
                            up_terms.append((f"gam[{k}]", h.full(*qu)))
                            cnt = q[ctr][x]
                            if cnt > 0:
                                qd = list(q)
                                qd[ctr] = down(q[ctr], x)
                                dn_terms.append((scaled(cnt, f"gam[{k}]"), h.full(*qd)))
                            k += 1
            su = em.tmp(plain_sum(up_terms), 2 * len(up_terms) - 1)
            expr = f"tw * {su}"
            fl = 2
            if dn_terms:
                sd = em.tmp(plain_sum(dn_terms), 2 * len(dn_terms) - 1)
                expr = f"tw * {su} - {sd}"
                fl += 1
            em.flops += fl
            outs.append(expr)
        grad_flops += em.flops
        c = 'ABC'[ctr]
        src.append(f"  // centre {c}: g[x] += tw * sum gam (..+1x..) - sum gam n_x (..-1x..), tw = 2 exponent")
        src.append(f"  __device__ static __noinline__ void grad{c}(const R* __restrict__ I, const R* __restrict__ PA,")
        src.append("      const R* __restrict__ WP, const R* __restrict__ QC, const R* __restrict__ WQ, R o2p, R nrp,")
        src.append("      R o2q, R nrq, R o2pq, const R* __restrict__ AB, const R* __restrict__ CD,")
        src.append("      R tw, const R* __restrict__ gam, R* __restrict__ g) {")
        src.extend(em.lines)
        for x in range(3):
            src.append(f"    g[{x}] += {outs[x]};")
        src.append("    (void)PA; (void)WP; (void)QC; (void)WQ; (void)o2p; (void)nrp; (void)o2q; (void)nrq; (void)o2pq;")
        src.append("    (void)AB; (void)CD;")
        src.append("  }")
    for ctr in range(0 if L >= 4 else 3):
        for x in range(3):
            em = Emitter()
            v = Vrr(em, L + 1, packed=False)
            h = Hrr(em, lambda e, f, v=v: v.V(e, f, 0), packed=False)
            up_terms, dn_terms = [], []
            k = 0
            for a in comps(la):
                for b in comps(lb):
                    for c in comps(lc):
                        for d in comps(ld):
                            q = [a, b, c, d]
                            qu = list(q)
                            qu[ctr] = up(q[ctr], x)
                            up_terms.append((f"gam[{k}]", h.full(*qu)))
                            cnt = q[ctr][x]
                            if cnt > 0:
                                qd = list(q)
                                qd[ctr] = down(q[ctr], x)
                                dn_terms.append((scaled(cnt, f"gam[{k}]"), h.full(*qd)))
                            k += 1
            su = em.tmp(plain_sum(up_terms), 2 * len(up_terms) - 1)
            expr = f"tw * {su}"
            fl = 2
            if dn_terms:
                sd = em.tmp(plain_sum(dn_terms), 2 * len(dn_terms) - 1)
                expr = f"tw * {su} - {sd}"
                fl += 1
            em.flops += fl
            grad_flops += em.flops
            name = f"grad{'ABC'[ctr]}{'xyz'[x]}"
            src.append(f"  __device__ static __forceinline__ R {name}(const R* __restrict__ I, const R* __restrict__ PA,")
            src.append("      const R* __restrict__ WP, const R* __restrict__ QC, const R* __restrict__ WQ, R o2p, R nrp,")
            src.append("      R o2q, R nrq, R o2pq, const R* __restrict__ AB, const R* __restrict__ CD,")
            src.append("      R tw, const R* __restrict__ gam) {")
            src.extend(em.lines)
            src.append(f"    return {expr};")
            src.append("    (void)PA; (void)WP; (void)QC; (void)WQ; (void)o2p; (void)nrp; (void)o2q; (void)nrq; (void)o2pq;")
            src.append("    (void)AB; (void)CD;")
            src.append("  }")
        c = 'ABC'[ctr]
        src.append(f"  // centre {c}: g[x] += tw * sum gam (..+1x..) - sum gam n_x (..-1x..), tw = 2 exponent")
        src.append(f"  __device__ static __forceinline__ void grad{c}(const R* __restrict__ I, const R* __restrict__ PA,")
        src.append("      const R* __restrict__ WP, const R* __restrict__ QC, const R* __restrict__ WQ, R o2p, R nrp,")
        src.append("      R o2q, R nrq, R o2pq, const R* __restrict__ AB, const R* __restrict__ CD,")
        src.append("      R tw, const R* __restrict__ gam, R* __restrict__ g) {")
        for x in range(3):
            src.append(f"    g[{x}] += grad{c}{'xyz'[x]}(I, PA, WP, QC, WQ, o2p, nrp, o2q, nrq, o2pq, AB, CD, tw, gam);")
        src.append("  }")
    gsrc, ginfo = gen_contracted_grad(la, lb, lc, ld)
    src.extend(gsrc)
    src.append(f"  static constexpr int VRR_FLOPS = {vrr_flops};")
    src.append(f"  static constexpr int HRR_FLOPS = {hrr_flops};")
    src.append(f"  static constexpr int GRAD_FLOPS = {grad_flops};")
    src.append("};")
    return "\n".join(src), dict(tag=tag, L=L, nacc=nacc, nout=nout, vrr=vrr_flops, hrr=hrr_flops, grad=grad_flops,
                                **ginfo)


# Classes whose gradient is contracted before the HRR (gen_contracted_grad):
# their exponent-weighted accumulators fit the register file (10, 25, 69 and
# 66 of them); (pp|ps) and (pp|pp) would need 240 and 585.
GCON_CLASSES = {(0, 0, 0, 0), (1, 0, 0, 0), (1, 0, 1, 0), (1, 1, 0, 0)}


def gen_contracted_grad(la, lb, lc, ld):
    """Nuclear-gradient contraction with the HRR after the primitive sum.

    d/dA_x phi_a = 2 alpha phi_{a+1x} - a_x phi_{a-1x}, and the HRR that
    turns [e0|f0] into (ab|cd) has primitive-independent coefficients (AB,
    CD), so sum_prim 2 alpha (a+1x b|cd)_prim is the HRR of the contracted
    accumulators U_A[e, f] = sum_prim 2 alpha [e0|f0]_prim (likewise U_B with
    2 beta, U_C with 2 gamma, and the plain sum V for the a_x (a-1x b|cd)
    terms).  ``gacc`` adds one primitive quartet into these accumulators
    (VRR to L + 1 and one multiply-add per accumulator); ``gfin`` runs the
    HRR on them once per contracted quartet and contracts with gam, giving
    the same g[0..8] as the per-primitive routines gradA/B/C summed over the
    primitives."""
    if (la, lb, lc, ld) not in GCON_CLASSES:
        return ["  static constexpr bool GCON = false;", "  static constexpr int NGACC = 1;",
                "  static constexpr int GACC_FLOPS = 0;", "  static constexpr int GFIN_FLOPS = 0;"], \
            dict(ngacc=0, gacc=0, gfin=0)
    L = la + lb + lc + ld
    idx, order = {}, []

    def base(kind):
        def f(e, ff):
            key = (kind, e, ff)
            if key not in idx:
                idx[key] = len(order)
                order.append(key)
            return f"acc[{idx[key]}]"
        return f

    em = Emitter()
    hs = [Hrr(em, base(k), packed=False) for k in range(4)]  # U_A, U_B, U_C, V
    out = []
    for ctr in range(3):
        for x in range(3):
            up_terms, dn_terms = [], []
            k = 0
            for a in comps(la):
                for b in comps(lb):
                    for c in comps(lc):
                        for d in comps(ld):
                            q = [a, b, c, d]
                            qu = list(q)
                            qu[ctr] = up(q[ctr], x)
                            up_terms.append((f"gam[{k}]", hs[ctr].full(*qu)))
                            cnt = q[ctr][x]
                            if cnt > 0:
                                qd = list(q)
                                qd[ctr] = down(q[ctr], x)
                                dn_terms.append((scaled(cnt, f"gam[{k}]"), hs[3].full(*qd)))
                            k += 1
            expr = em.tmp(plain_sum(up_terms), 2 * len(up_terms) - 1)
            if dn_terms:
                sd = em.tmp(plain_sum(dn_terms), 2 * len(dn_terms) - 1)
                expr = f"{expr} - {sd}"
                em.flops += 1
            out.append(f"    g[{3 * ctr + x}] += {expr};")
            em.flops += 1
    fin_lines, fin_flops = em.lines, em.flops
    em = Emitter()
    v = Vrr(em, L + 1, packed=False)
    weight = ["ta", "tb", "tc", None]
    acc_lines = []
    for key in order:
        kind, e, ff = key
        val = v.V(e, ff, 0)
        if weight[kind]:
            acc_lines.append(f"    acc[{idx[key]}] += {weight[kind]} * {val};")
            em.flops += 2
        else:
            acc_lines.append(f"    acc[{idx[key]}] += {val};")
            em.flops += 1
    src = ["  static constexpr bool GCON = true;",
           f"  static constexpr int NGACC = {len(order)};",
           "  // one primitive quartet into the exponent-weighted accumulators",
           "  // (ta, tb, tc = 2 alpha, 2 beta, 2 gamma of the primitive)",
           "  __device__ static __forceinline__ void gacc(const R* __restrict__ I, const R* __restrict__ PA,",
           "      const R* __restrict__ WP, const R* __restrict__ QC, const R* __restrict__ WQ, R o2p, R nrp,",
           "      R o2q, R nrq, R o2pq, R ta, R tb, R tc, R* __restrict__ acc) {"]
    src.extend(em.lines)
    src.extend(acc_lines)
    src.append("    (void)PA; (void)WP; (void)QC; (void)WQ; (void)o2p; (void)nrp; (void)o2q; (void)nrq; (void)o2pq;")
    src.append("    (void)ta; (void)tb; (void)tc;")
    src.append("  }")
    src.append("  // the contracted accumulators through the HRR, contracted with gam: g[0..8] += d/dA, d/dB, d/dC")
    src.append("  __device__ static __forceinline__ void gfin(const R* __restrict__ acc, const R* __restrict__ AB,")
    src.append("      const R* __restrict__ CD, const R* __restrict__ gam, R* __restrict__ g) {")
    src.extend(fin_lines)
    src.extend(out)
    src.append("    (void)AB; (void)CD;")
    src.append("  }")
    src.append(f"  static constexpr int GACC_FLOPS = {em.flops};")
    src.append(f"  static constexpr int GFIN_FLOPS = {fin_flops};")
    return src, dict(ngacc=len(order), gacc=em.flops, gfin=fin_flops)


class Vrr1e:
    """OS recursion for the nuclear attraction of one primitive pair and one
    nucleus C: [e|A_C|0]^(m) from I_m = pref * F_m(p |PC|^2)."""

    def __init__(self, em: Emitter):
        self.em = em
        self.memo = {}

    def V(self, e, m):
        key = (e, m)
        if key in self.memo:
            return self.memo[key]
        if lsum(e) == 0:
            r = f"I[{m}]"
        else:
            i = first_axis(e)
            e1 = down(e, i)
            expr = f"PA[{i}] * {self.V(e1, m)} - PC[{i}] * {self.V(e1, m + 1)}"
            fl = 3
            if e1[i] > 0:
                e2 = down(e1, i)
                c = f"{e1[i]}.0 * " if e1[i] > 1 else ""
                expr += f" + {c}o2p * ({self.V(e2, m)} - {self.V(e2, m + 1)})"
                fl += 3 + (1 if e1[i] > 1 else 0)
            r = self.em.tmp(expr, fl)
        self.memo[key] = r
        return r


class Hrr1e:
    def __init__(self, em: Emitter, base):
        self.em = em
        self.base = base
        self.memo = {}

    def ab(self, a, b):
        key = (a, b)
        if key in self.memo:
            return self.memo[key]
        if lsum(b) == 0:
            r = self.base(a)
        else:
            i = first_axis(b)
            r = self.em.tmp(f"{self.ab(up(a, i), down(b, i))} + AB[{i}] * {self.ab(a, down(b, i))}", 2)
        self.memo[key] = r
        return r


def gen_one_electron(la, lb):
    """Nuclear attraction (one nucleus) and its density-contracted
    derivative with respect to the two centres, class (la|lb), la >= lb."""
    L = la + lb
    na, nb = len(comps(la)), len(comps(lb))
    src = [f"template <typename R> struct NucClass<R, {la}, {lb}> {{",
           f"  static constexpr int L = {L};",
           f"  static constexpr int NOUT = {na * nb};"]
    em = Emitter()
    v = Vrr1e(em)
    h = Hrr1e(em, lambda a: v.V(a, 0))
    out = []
    k = 0
    for a in comps(la):
        for b in comps(lb):
            out.append(f"    out[{k}] += {h.ab(a, b)};")
            em.flops += 1
            k += 1
    vflops = em.flops
    src.append("  __device__ static __forceinline__ void vint(const R* __restrict__ I, const R* __restrict__ PA,")
    src.append("      const R* __restrict__ PC, R o2p, const R* __restrict__ AB, R* __restrict__ out) {")
    src.extend(em.lines)
    src.extend(out)
    src.append("    (void)PA; (void)PC; (void)o2p; (void)AB;")
    src.append("  }")
    em = Emitter()
    v = Vrr1e(em)
    h = Hrr1e(em, lambda a: v.V(a, 0))
    lines = []
    for ctr in range(2):
        for x in range(3):
            ups, dns = [], []
            k = 0
            for a in comps(la):
                for b in comps(lb):
                    q = [a, b]
                    qu = list(q)
                    qu[ctr] = up(q[ctr], x)
                    ups.append(f"dens[{k}] * {h.ab(*qu)}")
                    cnt = q[ctr][x]
                    if cnt > 0:
                        qd = list(q)
                        qd[ctr] = down(q[ctr], x)
                        cc = f"{cnt}.0 * " if cnt > 1 else ""
                        dns.append(f"{cc}dens[{k}] * {h.ab(*qd)}")
                    k += 1
            su = em.tmp(" + ".join(ups), 2 * len(ups) - 1)
            expr = f"tw[{ctr}] * {su}"
            if dns:
                sd = em.tmp(" + ".join(dns), 2 * len(dns) - 1)
                expr += f" - {sd}"
            lines.append(f"    g[{3 * ctr + x}] += {expr};")
            em.flops += 3
    gflops = em.flops
    src.append("  // g[0..2] += d/dA, g[3..5] += d/dB of sum_ab dens_ab (a|A_C|b); tw = {2 alpha, 2 beta}")
    src.append("  __device__ static __forceinline__ void vgrad(const R* __restrict__ I, const R* __restrict__ PA,")
    src.append("      const R* __restrict__ PC, R o2p, const R* __restrict__ AB, const R* __restrict__ tw,")
    src.append("      const R* __restrict__ dens, R* __restrict__ g) {")
    src.extend(em.lines)
    src.extend(lines)
    src.append("    (void)PA; (void)PC; (void)o2p; (void)AB;")
    src.append("  }")
    src.append(f"  static constexpr int VINT_FLOPS = {vflops};")
    src.append(f"  static constexpr int VGRAD_FLOPS = {gflops};")
    src.append("};")
    return "\n".join(src)


CLASSES = [(0, 0, 0, 0), (1, 0, 0, 0), (1, 0, 1, 0), (1, 1, 0, 0), (1, 1, 1, 0), (1, 1, 1, 1)]
ONE_E_CLASSES = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]


def generate() -> str:
    parts = ["// Generated by gen_eri.py -- do not edit by hand.",
             "// Obara-Saika VRR / Head-Gordon-Pople HRR for s/p shell quartets.",
             "#pragma once", "",
             "// Multiply-add of the class routines: the scalar FMA for double and float;",
             "// a packed type supplies its own pf_fma (found by argument lookup).",
             "__device__ __forceinline__ double pf_fma(double a, double b, double c) { return __fma_rn(a, b, c); }",
             "__device__ __forceinline__ float pf_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }",
             "",
             "template <typename R, int LA, int LB, int LC, int LD> struct EriClass;",
             "template <typename R, int LA, int LB> struct NucClass;", ""]
    table = []
    for cl in CLASSES:
        s, info = gen_class(*cl)
        parts.append(s)
        parts.append("")
        table.append(info)
    for cl in ONE_E_CLASSES:
        parts.append(gen_one_electron(*cl))
        parts.append("")
    parts.append("// class | L | accumulators | outputs | vrr flops/prim | hrr flops/contr | grad flops/prim"
                 " | contracted-gradient accumulators | flops/prim | flops/contr")
    for t in table:
        parts.append(f"//  {t['tag']}  | {t['L']} | {t['nacc']:3d} | {t['nout']:3d} | {t['vrr']:5d} | {t['hrr']:4d} | {t['grad']:6d}"
                     f" | {t['ngacc']:3d} | {t['gacc']:4d} | {t['gfin']:5d}")
    return "\n".join(parts) + "\n"


def main(out_path=None):
    here = os.path.dirname(os.path.abspath(__file__))
    out_path = out_path or os.path.join(here, "eri_classes.cuh")
    text = generate()
    old = open(out_path).read() if os.path.exists(out_path) else None
    if old != text:
        with open(out_path, "w") as fh:
            fh.write(text)
    return out_path


if __name__ == "__main__":
    print(main(sys.argv[1] if len(sys.argv) > 1 else None))
