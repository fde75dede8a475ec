"""The generated d-shell recursion programs (csrc/gen_programs.py, run by
the warp-cooperative kernels of kernels_d.cu) executed by their reference
interpreter on the CPU, against the oracle's OS/HGP shell quartets
(oracle/oracle.cpp eri_quartet) for every class with a d shell: the program
tables themselves are checked here, without a GPU."""
import math
import os
import sys

import numpy as np
import pytest

from conftest import PKG, basis_file

sys.path.insert(0, os.path.join(PKG, "csrc"))


def _boys(m, T):
    import mpmath
    return float(mpmath.hyp1f1(m + 0.5, m + 1.5, -T) / (2 * m + 1))


def _prim_norm(l, a):
    n = (2.0 * a / math.pi) ** 0.75
    return n * (4.0 * a) ** (l / 2.0) / math.sqrt({0: 1.0, 1: 1.0, 2: 3.0}[l])


def _ratio(c):
    l = sum(c)
    f2 = lambda n: math.prod(range(n, 0, -2)) if n > 0 else 1.0
    return math.sqrt(f2(2 * l - 1) / (f2(2 * c[0] - 1) * f2(2 * c[1] - 1) * f2(2 * c[2] - 1)))


def _contracted(prog, sh, q):
    """(ab|cd) of shells q = (a, b, c, d) through the program."""
    import gen_programs as GP
    from gen_eri import comps
    A, B, C, D = (np.array(sh["cen"][s]) for s in q)
    prims = []
    pa = [(sh["ex"][s], sh["co"][s]) for s in q]
    L = prog["L"]
    for aa, ca in zip(*pa[0]):
        for bb, cb in zip(*pa[1]):
            p = aa + bb
            P = (aa * A + bb * B) / p
            Kab = ca * cb * _prim_norm(sh["l"][q[0]], aa) * _prim_norm(sh["l"][q[1]], bb) * math.exp(
                -aa * bb / p * np.dot(A - B, A - B)) * math.sqrt(2) * math.pi ** 1.25 / p
            for cc, c_c in zip(*pa[2]):
                for dd, cd in zip(*pa[3]):
                    qq = cc + dd
                    Q = (cc * C + dd * D) / qq
                    Kcd = c_c * cd * _prim_norm(sh["l"][q[2]], cc) * _prim_norm(sh["l"][q[3]], dd) * math.exp(
                        -cc * dd / qq * np.dot(C - D, C - D)) * math.sqrt(2) * math.pi ** 1.25 / qq
                    z = p + qq
                    rho = p * qq / z
                    PQ = P - Q
                    T = rho * np.dot(PQ, PQ)
                    pref = Kab * Kcd / math.sqrt(z)
                    I = np.array([pref * _boys(m, T) for m in range(L + 1)])
                    prims.append((I, P - A, -qq / z * PQ, Q - C, p / z * PQ, 0.5 / p, qq / z, 0.5 / qq, p / z,
                                  0.5 / z))
    out = GP.emulate_energy(prog, prims, A - B, C - D)
    k = 0
    ls = [sh["l"][s] for s in q]
    for a in comps(ls[0]):
        for b in comps(ls[1]):
            for c in comps(ls[2]):
                for d in comps(ls[3]):
                    out[k] *= _ratio(a) * _ratio(b) * _ratio(c) * _ratio(d)
                    k += 1
    return out


@pytest.mark.parametrize("cls", range(15))
def test_d_program_matches_oracle(oracle, cls):
    import gen_programs as GP
    la, lb, lc, ld = GP.D_CLASSES[cls]
    # Sc (d shells) and O (s, p) in STO-3G, off-axis so no integral vanishes by symmetry
    sp = ["Sc", "O"]
    xyz = np.array([[0.1, -0.2, 0.3], [1.3, 2.1, -1.7]])
    mol = oracle.molecule(sp, xyz, basis_file("sto-3g"))
    S = mol.shells
    poff = S.poff
    sh = {"l": list(S.l), "cen": [S.center[s] for s in range(len(S.l))],
          "ex": [list(S.exps[poff[s]:poff[s + 1]]) for s in range(len(S.l))],
          "co": [list(S.coefs[poff[s]:poff[s + 1]]) for s in range(len(S.l))]}
    by_l = {}
    for s, l in enumerate(S.l):
        by_l.setdefault(int(l), []).append(s)
    # distinct shells where possible (d on Sc; s, p from both atoms)
    pick = {0: list(reversed(by_l[0])), 1: list(reversed(by_l[1])), 2: by_l[2] * 4}
    q = []
    used = {0: 0, 1: 0, 2: 0}
    for l in (la, lb, lc, ld):
        q.append(pick[l][used[l] % len(pick[l])])
        used[l] += 1
    prog = GP.energy_program(la, lb, lc, ld)
    got = _contracted(prog, sh, q)
    ref = oracle.eri_quartet(mol, *q).ravel()
    assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), (GP.D_CLASSES[cls], q)


def _prims_grad(sh, q, Lp1, shift=None):
    """Primitive quartet data (with 2 alpha, 2 beta, 2 gamma) of shells q;
    shift = (centre, axis, h) displaces one centre."""
    cen = [np.array(sh["cen"][s], dtype=float) for s in q]
    if shift is not None:
        cen[shift[0]] = cen[shift[0]].copy()
        cen[shift[0]][shift[1]] += shift[2]
    A, B, C, D = cen
    pa = [(sh["ex"][s], sh["co"][s]) for s in q]
    out = []
    for aa, ca in zip(*pa[0]):
        for bb, cb in zip(*pa[1]):
            p = aa + bb
            P = (aa * A + bb * B) / p
            Kab = ca * cb * _prim_norm(sh["l"][q[0]], aa) * _prim_norm(sh["l"][q[1]], bb) * math.exp(
                -aa * bb / p * np.dot(A - B, A - B)) * math.sqrt(2) * math.pi ** 1.25 / p
            for cc, c_c in zip(*pa[2]):
                for dd, cd in zip(*pa[3]):
                    qq = cc + dd
                    Q = (cc * C + dd * D) / qq
                    Kcd = c_c * cd * _prim_norm(sh["l"][q[2]], cc) * _prim_norm(sh["l"][q[3]], dd) * math.exp(
                        -cc * dd / qq * np.dot(C - D, C - D)) * math.sqrt(2) * math.pi ** 1.25 / qq
                    z = p + qq
                    PQ = P - Q
                    T = p * qq / z * np.dot(PQ, PQ)
                    pref = Kab * Kcd / math.sqrt(z)
                    I = np.array([pref * _boys(m, T) for m in range(Lp1 + 1)])
                    out.append((I, P - A, -qq / z * PQ, Q - C, p / z * PQ, 0.5 / p, qq / z, 0.5 / qq, p / z,
                                0.5 / z, 2 * aa, 2 * bb, 2 * cc))
    return out, (A - B), (C - D)


@pytest.mark.parametrize("cls", [0, 1, 4, 5, 9])
def test_d_gradient_program_matches_finite_differences(oracle, cls):
    """sum gam (ab|cd) differentiated by the gradient program against
    central differences of the energy program (each centre moved alone)."""
    import gen_programs as GP
    cl = GP.D_CLASSES[cls]
    mol = oracle.molecule(["Sc", "O"], np.array([[0.1, -0.2, 0.3], [1.3, 2.1, -1.7]]), basis_file("sto-3g"))
    S = mol.shells
    poff = S.poff
    sh = {"l": list(S.l), "cen": [S.center[s] for s in range(len(S.l))],
          "ex": [list(S.exps[poff[s]:poff[s + 1]]) for s in range(len(S.l))],
          "co": [list(S.coefs[poff[s]:poff[s + 1]]) for s in range(len(S.l))]}
    by_l = {}
    for s, l in enumerate(S.l):
        by_l.setdefault(int(l), []).append(s)
    used = {0: 0, 1: 0, 2: 0}
    q = []
    for l in cl:
        q.append(by_l[l][::-1][used[l] % len(by_l[l])] if l < 2 else by_l[2][0])
        used[l] += 1
    # give every centre its own position (the quartet's four centres move independently)
    rng = np.random.default_rng(cls)
    sh["cen"] = list(sh["cen"])
    for k, s in enumerate(q):
        sh["cen"].append(np.array(sh["cen"][s]) + rng.normal(0, 0.3, 3))
        for key in ("l", "ex", "co"):
            sh[key].append(sh[key][s])
        q[k] = len(sh["l"]) - 1
    from gen_eri import comps
    nout = math.prod(len(comps(l)) for l in cl)
    gam = rng.normal(0, 1, nout)
    gp = GP.grad_program(*cl)
    prims, AB, CD = _prims_grad(sh, q, gp["L"] + 1)
    g = GP.emulate_grad(gp, prims, AB, CD, gam, _ratio)
    ep = GP.energy_program(*cl)
    h = 1e-4
    for ctr in range(3):
        for x in range(3):
            vals = []
            for sgn in (1, -1):
                pr, ab, cd = _prims_grad(sh, q, ep["L"], (ctr, x, sgn * h))
                out = GP.emulate_energy(ep, [p[:10] for p in pr], ab, cd)
                k = 0
                for a in comps(cl[0]):
                    for b in comps(cl[1]):
                        for c in comps(cl[2]):
                            for d in comps(cl[3]):
                                out[k] *= _ratio(a) * _ratio(b) * _ratio(c) * _ratio(d)
                                k += 1
                vals.append(np.dot(gam, out))
            fd = (vals[0] - vals[1]) / (2 * h)
            assert g[ctr][x] == pytest.approx(fd, abs=1e-7, rel=1e-6), (cl, ctr, x)
