#!/usr/bin/env python3
"""Generate eri_programs.cuh: Obara-Saika / Head-Gordon-Pople recursions of
the shell-quartet classes that contain a d shell, as operation lists that
one warp executes cooperatively (kernels_d.cu).

The s/p classes run as straight-line code, one contracted quartet per lane
(gen_eri.py).  A d class has up to 961 contracted accumulators and 2330
recursion intermediates ((dd|dd)), far more than a lane's registers, so its
recursions are flattened here into operation lists grouped in dependency
levels: the 32 lanes of a warp execute the operations of one level at a
time on tables in shared memory, level after level, for one primitive
quartet after another.

Per class (la lb|lc ld), la >= lb, lc >= ld, at least one l = 2:

* VRR ops: [e0|f0]^(m) from I_m = pref F_m(T) (Obara & Saika 1986, the
  same recursion as gen_eri.py), table slots 0..L hold I_0..I_L;
* accumulator map: the VRR slot of every [e0|f0]^(0), e in [la, la+lb],
  f in [lc, lc+ld], summed over the primitive quartets;
* HRR ops (Head-Gordon & Pople 1988) on the contracted accumulators: H
  slots 0..nacc-1 are the accumulators, temporaries follow;
* output map: the H slot of every (ab|cd), a, b, c, d in the Cartesian order
  of cartesian.f90:7-23 (x descending, then y).

For the nuclear gradient of a class the derivative integrals come from the
same VRR run to L+1: the primitive integrals [e0|f0] are summed four ways
(plain, and weighted by 2 alpha, 2 beta, 2 gamma of the primitive), and six
HRR programs build (a+1b|, (a-1b|, (ab+1|, (ab-1|, |c+1d), |c-1d) from
those sums (d/dA phi_a = 2 alpha phi_{a+1} - a_x phi_{a-1}, contracted).

An op is packed into 16 bytes (uint4):
  VRR  x = dst | s1 << 16, y = s2 | s3 << 16, z = s4 | s5 << 16,
       w = axis | ket << 2 | c3 << 4 | c5 << 8   (s3..s5 = 0xffff: absent)
       bra:  dst = PA_i s1 + WP_i s2 + c3 o2p (s3 - rho/p s4)
       ket:  dst = QC_i s1 + WQ_i s2 + c3 o2q (s3 - rho/q s4) + c5 o2pq s5
  HRR  x = dst | sa << 16, y = sb, z = axis | ket << 2, w = 0
       dst = sa + X_i sb, X = A - B (bra) or C - D (ket)
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from gen_eri import comps, down, ecomps, first_axis, lsum, up  # noqa: E402

ABSENT = 0xFFFF


class VrrOps:
    """OS VRR recorded as ops with dependency levels; slots 0..L are I_m."""

    def __init__(self, L):
        self.L = L
        self.memo = {}
        self.ops = []          # (level, dst, kind, axis, s1, s2, s3, s4, s5, c3, c5)
        self.level = {m: 0 for m in range(L + 1)}
        self.nslot = L + 1

    def V(self, e, f, m):
        key = (e, f, m)
        if key in self.memo:
            return self.memo[key]
        if lsum(e) == 0 and lsum(f) == 0:
            r = m
        elif lsum(f) == 0:
            i = first_axis(e)
            e1 = down(e, i)
            s1, s2 = self.V(e1, f, m), self.V(e1, f, m + 1)
            s3 = s4 = ABSENT
            c3 = 0
            if e1[i] > 0:
                e2 = down(e1, i)
                s3, s4, c3 = self.V(e2, f, m), self.V(e2, f, m + 1), e1[i]
            r = self._op(0, i, s1, s2, s3, s4, ABSENT, c3, 0)
        else:
            i = first_axis(f)
            f1 = down(f, i)
            s1, s2 = self.V(e, f1, m), self.V(e, f1, m + 1)
            s3 = s4 = s5 = ABSENT
            c3 = c5 = 0
            if f1[i] > 0:
                f2 = down(f1, i)
                s3, s4, c3 = self.V(e, f2, m), self.V(e, f2, m + 1), f1[i]
            if e[i] > 0:
                s5, c5 = self.V(down(e, i), f1, m + 1), e[i]
            r = self._op(1, i, s1, s2, s3, s4, s5, c3, c5)
        self.memo[key] = r
        return r

    def _op(self, kind, axis, s1, s2, s3, s4, s5, c3, c5):
        dst = self.nslot
        self.nslot += 1
        lev = 1 + max(self.level[s] for s in (s1, s2, s3, s4, s5) if s != ABSENT)
        self.level[dst] = lev
        self.ops.append((lev, dst, kind, axis, s1, s2, s3, s4, s5, c3, c5))
        return dst


class HrrOps:
    """HGP HRR recorded as ops; base(e, f) gives an H slot (an accumulator)."""

    def __init__(self, base, nbase):
        self.base = base
        self.mb, self.mk = {}, {}
        self.ops = []          # (level, dst, kind, axis, sa, sb)
        self.level = {}
        self.nslot = nbase
        self.used = set()      # (e, f) pairs taken from the base

    def _base(self, e, f):
        self.used.add((e, f))
        s = self.base(e, f)
        self.level.setdefault(s, 0)
        return s

    def bra(self, a, b, f):
        key = (a, b, f)
        if key in self.mb:
            return self.mb[key]
        if lsum(b) == 0:
            r = self._base(a, f)
        else:
            i = first_axis(b)
            r = self._op(0, i, self.bra(up(a, i), down(b, i), f), self.bra(a, down(b, i), f))
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
            r = self._op(1, i, self.full(a, b, up(c, i), down(d, i)), self.full(a, b, c, down(d, i)))
        self.mk[key] = r
        return r

    def _op(self, kind, axis, sa, sb):
        dst = self.nslot
        self.nslot += 1
        lev = 1 + max(self.level[sa], self.level[sb])
        self.level[dst] = lev
        self.ops.append((lev, dst, kind, axis, sa, sb))
        return dst


def sorted_ops(ops):
    """ops grouped by level (stable), with the level offsets."""
    ops = sorted(ops, key=lambda o: o[0])
    nlev = (ops[-1][0] if ops else 0)
    off = [0] * (nlev + 1)
    for k in range(1, nlev + 1):
        off[k] = sum(1 for o in ops if o[0] <= k)
    # off[k] = end of level k; levels start at 1: level k spans [off[k-1], off[k])
    return ops, off


def energy_program(la, lb, lc, ld):
    """VRR + accumulate + HRR program of one class (la lb|lc ld)."""
    L = la + lb + lc + ld
    v = VrrOps(L)
    E = ecomps(la, la + lb)
    F = ecomps(lc, lc + ld)
    acc = [(e, f) for e in E for f in F]
    acc_index = {k: n for n, k in enumerate(acc)}
    acc_slot = [v.V(e, f, 0) for e, f in acc]
    h = HrrOps(lambda e, f: acc_index[(e, f)], len(acc))
    outs = [h.full(a, b, c, d) for a in comps(la) for b in comps(lb) for c in comps(lc) for d in comps(ld)]
    return dict(L=L, vrr=v, acc_slot=acc_slot, nacc=len(acc), hrr=h, outs=outs)


def grad_program(la, lb, lc, ld):
    """Derivative integrals of class (la lb|lc ld) for the centres A, B, C:
    VRR to L + 1, four accumulator sets (U plain; WA, WB, WC weighted by
    2 alpha, 2 beta, 2 gamma of the primitive quartet) and six HRR programs
    (A+, A-, B+, B-, C+, C-; the minus ones only for l > 0)."""
    L = la + lb + lc + ld
    v = VrrOps(L + 1)
    shifted = {"A+": ("WA", (la + 1, lb, lc, ld)), "B+": ("WB", (la, lb + 1, lc, ld)),
               "C+": ("WC", (la, lb, lc + 1, ld))}
    if la > 0:
        shifted["A-"] = ("U", (la - 1, lb, lc, ld))
    if lb > 0:
        shifted["B-"] = ("U", (la, lb - 1, lc, ld))
    if lc > 0:
        shifted["C-"] = ("U", (la, lb, lc - 1, ld))
    # pass 1: which (e, f) each accumulator set needs (HRR base calls)
    need = {k: set() for k in ("U", "WA", "WB", "WC")}
    for name, (acc, cl) in shifted.items():
        h = HrrOps(lambda e, f: 0, 1)
        for a in comps(cl[0]):
            for b in comps(cl[1]):
                for c in comps(cl[2]):
                    for d in comps(cl[3]):
                        h.full(a, b, c, d)
        need[acc] |= h.used
    sets = {}
    for k in ("U", "WA", "WB", "WC"):
        pairs = sorted(need[k], key=lambda ef: (lsum(ef[0]), comps(lsum(ef[0])).index(ef[0]),
                                               lsum(ef[1]), comps(lsum(ef[1])).index(ef[1])))
        sets[k] = dict(pairs=pairs, index={ef: n for n, ef in enumerate(pairs)},
                       slot=[v.V(e, f, 0) for e, f in pairs])
    hrrs = {}
    for name, (acc, cl) in shifted.items():
        h = HrrOps(lambda e, f, idx=sets[acc]["index"]: idx[(e, f)], len(sets[acc]["pairs"]))
        outs = [h.full(a, b, c, d) for a in comps(cl[0]) for b in comps(cl[1]) for c in comps(cl[2])
                for d in comps(cl[3])]
        hrrs[name] = dict(acc=acc, cl=cl, hrr=h, outs=outs)
    return dict(L=L, vrr=v, sets=sets, hrrs=hrrs)


def emulate_grad(prog, prims, AB, CD, gam, comp_ratio):
    """Reference execution of a gradient program (tests).  prims: as for
    emulate_energy plus (2 alpha, 2 beta, 2 gamma); gam: the two-particle
    density of the class (la lb|lc ld), row-major; returns g[3][3] for A,
    B, C (x, y, z)."""
    import numpy as np
    la, lb, lc, ld = _base_class(prog)
    vr = prog["vrr"]
    ops, _ = sorted_ops(vr.ops)
    accs = {k: np.zeros(len(v["pairs"])) for k, v in prog["sets"].items()}
    for (I, PA, WP, QC, WQ, o2p, rp, o2q, rq, o2pq, ta, tb, tc) in prims:
        T = np.zeros(vr.nslot)
        T[:prog["L"] + 2] = I
        for (_, dst, kind, i, s1, s2, s3, s4, s5, c3, c5) in ops:
            if kind == 0:
                val = PA[i] * T[s1] + WP[i] * T[s2]
                if c3:
                    val += c3 * o2p * (T[s3] - rp * T[s4])
            else:
                val = QC[i] * T[s1] + WQ[i] * T[s2]
                if c3:
                    val += c3 * o2q * (T[s3] - rq * T[s4])
                if c5:
                    val += c5 * o2pq * T[s5]
            T[dst] = val
        for k, w in (("U", 1.0), ("WA", ta), ("WB", tb), ("WC", tc)):
            if len(accs[k]):
                accs[k] += w * T[prog["sets"][k]["slot"]]
    res = {}
    for name, hp in prog["hrrs"].items():
        h = hp["hrr"]
        H = np.zeros(h.nslot)
        n0 = len(prog["sets"][hp["acc"]]["pairs"])
        H[:n0] = accs[hp["acc"]]
        hops, _ = sorted_ops(h.ops)
        for (_, dst, kind, i, sa, sb) in hops:
            H[dst] = H[sa] + (AB[i] if kind == 0 else CD[i]) * H[sb]
        res[name] = H[hp["outs"]]
    g = np.zeros((3, 3))
    cls = [la, lb, lc, ld]
    k = 0
    for a in comps(la):
        for b in comps(lb):
            for c in comps(lc):
                for d in comps(ld):
                    q = [a, b, c, d]
                    wgt = gam[k] * comp_ratio(a) * comp_ratio(b) * comp_ratio(c) * comp_ratio(d)
                    for ctr, nm in enumerate("ABC"):
                        for x in range(3):
                            qu = list(q)
                            qu[ctr] = up(q[ctr], x)
                            g[ctr][x] += wgt * res[nm + "+"][_index(cls, ctr, +1, qu)]
                            if q[ctr][x] > 0:
                                qd = list(q)
                                qd[ctr] = down(q[ctr], x)
                                g[ctr][x] -= wgt * q[ctr][x] * res[nm + "-"][_index(cls, ctr, -1, qd)]
                    k += 1
    return g


def _base_class(prog):
    la, lb, lc, ld = prog["hrrs"]["A+"]["cl"]
    return la - 1, lb, lc, ld


def _index(cls, ctr, sh, q):
    """Row-major index of components q in the class cls with centre ctr's l
    shifted by sh."""
    ls = list(cls)
    ls[ctr] += sh
    idx = 0
    for l, c in zip(ls, q):
        idx = idx * len(comps(l)) + comps(l).index(c)
    return idx


def emulate_energy(prog, prims, AB, CD):
    """Reference execution of an energy program (tests): prims = list of
    primitive quartets (I[0..L], PA, WP, QC, WQ, o2p, rp, o2q, rq, o2pq)."""
    import numpy as np
    vr, hr = prog["vrr"], prog["hrr"]
    ops, _ = sorted_ops(vr.ops)
    acc = np.zeros(prog["nacc"])
    for (I, PA, WP, QC, WQ, o2p, rp, o2q, rq, o2pq) in prims:
        T = np.zeros(vr.nslot)
        T[:prog["L"] + 1] = I
        for (_, dst, kind, i, s1, s2, s3, s4, s5, c3, c5) in ops:
            if kind == 0:
                v = PA[i] * T[s1] + WP[i] * T[s2]
                if c3:
                    v += c3 * o2p * (T[s3] - rp * T[s4])
            else:
                v = QC[i] * T[s1] + WQ[i] * T[s2]
                if c3:
                    v += c3 * o2q * (T[s3] - rq * T[s4])
                if c5:
                    v += c5 * o2pq * T[s5]
            T[dst] = v
        acc += T[prog["acc_slot"]]
    hops, _ = sorted_ops(hr.ops)
    H = np.zeros(hr.nslot)
    H[:prog["nacc"]] = acc
    for (_, dst, kind, i, sa, sb) in hops:
        H[dst] = H[sa] + (AB[i] if kind == 0 else CD[i]) * H[sb]
    return H[prog["outs"]]


# quartet classes with a d shell, bra class >= ket class in the pair-class
# order ss < ps < pp < ds < dp < dd
PAIR_CLASSES = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]
D_CLASSES = [(pb + pk) for bi, pb in enumerate(PAIR_CLASSES) for ki, pk in enumerate(PAIR_CLASSES)
             if ki <= bi and bi >= 3]


def pack_vrr(op):
    _, dst, kind, axis, s1, s2, s3, s4, s5, c3, c5 = op
    assert max(dst, s1, s2) < ABSENT
    return (dst | (s1 << 16), s2 | (s3 << 16), s4 | (s5 << 16), axis | (kind << 2) | (c3 << 4) | (c5 << 8))


def pack_hrr(op):
    _, dst, kind, axis, sa, sb = op
    assert max(dst, sa, sb) < ABSENT
    return (dst | (sa << 16), sb, axis | (kind << 2), 0)


GRAD_PARTS = ("A+", "A-", "B+", "B-", "C+", "C-")
SETS = ("U", "WA", "WB", "WC")


def generate() -> str:
    vrr_all, hrr_all, lev_all, map_all = [], [], [], []

    def add_vrr(v):
        ops, off = sorted_ops(v.ops)
        r = (len(vrr_all), len(ops), len(lev_all), len(off) - 1)
        vrr_all.extend(pack_vrr(o) for o in ops)
        lev_all.extend(off[1:])
        return r

    def add_hrr(h):
        ops, off = sorted_ops(h.ops)
        r = (len(hrr_all), len(ops), len(lev_all), len(off) - 1)
        hrr_all.extend(pack_hrr(o) for o in ops)
        lev_all.extend(off[1:])
        return r

    def add_map(vals):
        r = len(map_all)
        map_all.extend(vals)
        return r

    rows = []
    for cl in D_CLASSES:
        p = energy_program(*cl)
        v = add_vrr(p["vrr"])
        h = add_hrr(p["hrr"])
        rows.append(dict(cl=cl, L=p["L"], nslot=p["vrr"].nslot, v=v, h=h, nh=p["hrr"].nslot,
                         acc=add_map(p["acc_slot"]), nacc=p["nacc"], out=add_map(p["outs"]), nout=len(p["outs"])))
    grows = []
    for cl in D_CLASSES:
        g = grad_program(*cl)
        la, lb, lc, ld = cl
        v = add_vrr(g["vrr"])
        sets = []
        base = 0
        for k in SETS:
            sl = g["sets"][k]["slot"]
            sets.append((add_map(sl), len(sl), base))
            base += len(sl)
        parts = []
        for name in GRAD_PARTS:
            if name not in g["hrrs"]:
                parts.append(None)
                continue
            hp = g["hrrs"][name]
            h = add_hrr(hp["hrr"])
            # contraction map: for every output (abcd) of the class and
            # direction x, the H slot of the shifted integral and its factor
            ctr = "ABC".index(name[0])
            sign = 1 if name[1] == "+" else -1
            slots, facs = [], []
            for a in comps(la):
                for b in comps(lb):
                    for c in comps(lc):
                        for d in comps(ld):
                            q = [a, b, c, d]
                            for x in range(3):
                                if sign > 0:
                                    qs = list(q)
                                    qs[ctr] = up(q[ctr], x)
                                    slots.append(hp["outs"][_index(cl, ctr, +1, qs)])
                                    facs.append(1)
                                elif q[ctr][x] > 0:
                                    qs = list(q)
                                    qs[ctr] = down(q[ctr], x)
                                    slots.append(hp["outs"][_index(cl, ctr, -1, qs)])
                                    facs.append(q[ctr][x])
                                else:
                                    slots.append(ABSENT)
                                    facs.append(0)
            parts.append(dict(h=h, nh=hp["hrr"].nslot, set=SETS.index(hp["acc"]), cmap=add_map(slots),
                              cfac=add_map(facs)))
        grows.append(dict(cl=cl, L=g["L"] + 1, nslot=g["vrr"].nslot, v=v, sets=sets, nacc_all=base, parts=parts,
                          nout=len(comps(la)) * len(comps(lb)) * len(comps(lc)) * len(comps(ld)),
                          nh=max(pp["nh"] for pp in parts if pp)))

    def arr(name, ctype, vals, per_line=8):
        lines = [f"__device__ const {ctype} {name}[{max(len(vals), 1)}] = {{"]
        for k in range(0, len(vals), per_line):
            lines.append("  " + ", ".join(vals[k:k + per_line]) + ",")
        if not vals:
            lines.append("  0,")
        lines.append("};")
        return lines

    name = lambda cl: "".join("spd"[x] for x in cl[:2]) + "|" + "".join("spd"[x] for x in cl[2:])
    out = ["// Generated by gen_programs.py -- do not edit by hand.",
           "// Operation lists of the d-shell quartet classes (executed by kernels_d.cu).",
           "#pragma once", "", "#include <cuda_runtime.h>", "",
           "namespace pyfacc {", "",
           "struct DOps {",
           "  int begin, n;      // ops [begin, begin + n) of g_dvrr or g_dhrr",
           "  int lev, nlev;     // level k (1-based) ends at g_dlev[lev + k - 1]",
           "};",
           "struct DProg {       // one class, energy integrals",
           "  int la, lb, lc, ld, L;",
           "  int nslot;         // VRR table (doubles); slots 0..L are I_m",
           "  DOps vrr, hrr;",
           "  int nh;            // HRR table (doubles); slots 0..nacc-1 are the accumulators",
           "  int acc, nacc;     // g_dmap[acc + k]: VRR slot of accumulator k",
           "  int out, nout;     // g_dmap[out + o]: H slot of output (abcd) o",
           "};",
           "struct DGradPart {   // one shifted class (A+, A-, B+, B-, C+, C-)",
           "  int present;",
           "  DOps hrr;",
           "  int nh, set;       // HRR table size; accumulator set it starts from",
           "  int cmap, cfac;    // g_dmap[cmap + 3 o + x]: H slot (0xffff: none); g_dmap[cfac + ...]: factor",
           "};",
           "struct DGradProg {   // one class, derivative integrals for the centres A, B, C",
           "  int la, lb, lc, ld, L;   // L: the VRR order (class L + 1)",
           "  int nslot;",
           "  DOps vrr;",
           "  int set_map[4], set_n[4], set_base[4];  // U, WA, WB, WC: VRR slots, sizes, offsets",
           "  int nacc_all, nh, nout;",
           "  DGradPart part[6];",
           "};",
           f"constexpr int PF_NDPROG = {len(rows)};",
           "__device__ const DProg g_dprog[PF_NDPROG] = {"]
    ops = lambda t: "{%d, %d, %d, %d}" % t
    for r in rows:
        out.append("  {%d, %d, %d, %d, %d, %d, %s, %s, %d, %d, %d, %d, %d},  // (%s)" % (
            *r["cl"], r["L"], r["nslot"], ops(r["v"]), ops(r["h"]), r["nh"], r["acc"], r["nacc"], r["out"],
            r["nout"], name(r["cl"])))
    out.append("};")
    out.append("__device__ const DGradProg g_dgrad[PF_NDPROG] = {")
    for r in grows:
        sm = ", ".join(str(x[0]) for x in r["sets"])
        sn = ", ".join(str(x[1]) for x in r["sets"])
        sb = ", ".join(str(x[2]) for x in r["sets"])
        parts = []
        for pp in r["parts"]:
            if pp is None:
                parts.append("{0, {0, 0, 0, 0}, 0, 0, 0, 0}")
            else:
                parts.append("{1, %s, %d, %d, %d, %d}" % (ops(pp["h"]), pp["nh"], pp["set"], pp["cmap"], pp["cfac"]))
        out.append("  {%d, %d, %d, %d, %d, %d, %s, {%s}, {%s}, {%s}, %d, %d, %d,  // (%s)" % (
            *r["cl"], r["L"], r["nslot"], ops(r["v"]), sm, sn, sb, r["nacc_all"], r["nh"], r["nout"], name(r["cl"])))
        out.append("   {" + ", ".join(parts) + "}},")
    out.append("};")
    out.append("// host copies of the table sizes (shared-memory sizing), per class:")
    out.append("// energy {nslot, nacc, nh, nout}, gradient {nslot, nacc_all, nh, nout}")
    out.append("constexpr int PF_DPROG_SIZES[PF_NDPROG][4] = {")
    for r in rows:
        out.append("  {%d, %d, %d, %d}," % (r["nslot"], r["nacc"], r["nh"], r["nout"]))
    out.append("};")
    out.append("constexpr int PF_DGRAD_SIZES[PF_NDPROG][4] = {")
    for r in grows:
        out.append("  {%d, %d, %d, %d}," % (r["nslot"], r["nacc_all"], r["nh"], r["nout"]))
    out.append("};")
    out += arr("g_dvrr", "uint4", ["{%du, %du, %du, %du}" % t for t in vrr_all], 2)
    out += arr("g_dhrr", "uint4", ["{%du, %du, %du, %du}" % t for t in hrr_all], 2)
    out += arr("g_dlev", "int", [str(x) for x in lev_all], 16)
    out += arr("g_dmap", "unsigned short", [str(x) for x in map_all], 16)
    out += ["", "}  // namespace pyfacc", ""]
    return "\n".join(out)


def main(out_path=None):
    out_path = out_path or os.path.join(HERE, "eri_programs.cuh")
    text = generate()
    old = open(out_path).read() if os.path.exists(out_path) else None
    if old != text:
        with open(out_path, "w") as fh:
            fh.write(text)
    return out_path


if __name__ == "__main__":
    print(main(sys.argv[1] if len(sys.argv) > 1 else None))
