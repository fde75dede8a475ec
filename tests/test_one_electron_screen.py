"""The one-electron pair screen of the engine leaves out shell pairs on two
atoms whose largest primitive-pair prefactor |c_a N_a c_b N_b| exp(-mu R^2)
is below 1e-25, testing each pair with the two smallest exponents and the
largest |c N| of each shell (ONE_E_PAIR_CUT and System::upload_shells).
This checks, with the oracle's S, T and V of a 40-carbon chain, that every
entry of a pair the rule leaves out is below 1e-15 (the engine writes zero
there), and that the rule does leave out a good part of the pairs."""
import math

import numpy as np

from conftest import basis_file

CUT = 1e-25


def _norm(l, a):
    n = (2.0 * a / math.pi) ** 0.75
    return n * 2.0 * math.sqrt(a) if l else n


def test_screened_one_electron_entries_are_negligible(oracle):
    from pyfacc import geometry as G
    sp, xyz = G.alkane(40, seed=40)
    mol = oracle.molecule(sp, xyz, basis_file("sto-3g"))
    sh = mol.shells
    ns = len(sh.l)
    lcn, amin = np.zeros(ns), np.zeros(ns)
    for s in range(ns):
        ex = sh.exps[sh.poff[s]:sh.poff[s + 1]]
        co = sh.coefs[sh.poff[s]:sh.poff[s + 1]]
        lcn[s] = math.log(max(abs(c * _norm(sh.l[s], a)) for a, c in zip(ex, co)))
        amin[s] = ex.min()
    S, T, V = oracle.one_electron(mol)
    nf = [(l + 1) * (l + 2) // 2 for l in sh.l]
    worst, left_out, total = 0.0, 0, 0
    for a in range(ns):
        for b in range(a + 1, ns):
            if sh.atom[a] == sh.atom[b]:
                continue
            total += 1
            r2 = float(np.sum((sh.center[a] - sh.center[b]) ** 2))
            mu = amin[a] * amin[b] / (amin[a] + amin[b])
            if mu * r2 <= lcn[a] + lcn[b] - math.log(CUT):
                continue
            left_out += 1
            ia = slice(sh.bf_off[a], sh.bf_off[a] + nf[a])
            ib = slice(sh.bf_off[b], sh.bf_off[b] + nf[b])
            for M in (S, T, V):
                worst = max(worst, float(np.abs(M[ia, ib]).max()))
    assert left_out > 0.2 * total
    assert worst < 1e-15
