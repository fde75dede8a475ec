"""The Libint-compatible one-body entry points libint_overlap_c,
libint_kinetic_c and libint_potential_c (the reference's unused wrapper,
src/cpp/libint_wrapper.cpp:16-327), called through the C ABI for every
shell pair of ScH3 in STO-3G (s, p and d shells on Sc, s on H, both shell
orders), against the engine's own S, T and V: with the coefficients passed
as c_i N_l(alpha_i) (the engine's primitive normalisation of the x^l
component) a block times the engine's component ratios (sqrt(3) for d_xy,
d_xz, d_yz) is the engine's matrix block, and V = -sum_C Z_C times the
unit-charge potential at nucleus C.  Also: an f shell is refused with NaN
and PYFACC_ERR_UNSUPPORTED_L."""
import ctypes
import math

import numpy as np
import pytest

from conftest import basis_file

pytestmark = pytest.mark.gpu
A2B = 1.8897259886
RATIO = {0: [1.0], 1: [1.0] * 3, 2: [1.0, math.sqrt(3), math.sqrt(3), 1.0, math.sqrt(3), 1.0]}


def _norm(l, a):
    n = (2.0 * a / math.pi) ** 0.75
    return n * (1.0, 2.0 * math.sqrt(a), 4.0 * a / math.sqrt(3))[l]


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _block(fn, la, ea, ca, A, lb, eb, cb, B, C=None):
    nc = lambda l: (l + 1) * (l + 2) // 2
    out = np.full(nc(la) * nc(lb), -1.0)
    keep = [np.ascontiguousarray(x, dtype=np.float64) for x in (A, ea, ca, B, eb, cb)]
    args = [la, len(ea), _p(keep[0]), _p(keep[1]), _p(keep[2]), lb, len(eb), _p(keep[3]), _p(keep[4]), _p(keep[5])]
    if C is not None:
        c = np.ascontiguousarray(C, dtype=np.float64)
        keep.append(c)
        args.append(_p(c))
    fn(*args, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out.reshape(nc(la), nc(lb))


def test_libint_blocks_match_engine_matrices(engine, oracle):
    from pyfacc import _native as N
    lib = N.lib()
    sp = ["Sc", "H", "H", "H"]
    xyz = np.array([[0.0, 0.0, 0.1], [1.8, 0.1, 0.0], [-0.85, 1.55, -0.05], [-0.9, -1.5, 0.05]]) * A2B
    Z = [21.0, 1.0, 1.0, 1.0]
    with engine.System(engine.Molecule(sp, xyz)) as s:
        S, T, V = (x.cpu().numpy() for x in s.one_electron())
    sh = oracle.molecule(sp, xyz, basis_file()).shells
    nc = lambda l: (l + 1) * (l + 2) // 2
    off = np.concatenate([[0], np.cumsum([nc(l) for l in sh.l])])
    assert off[-1] == S.shape[0]
    worst = 0.0
    for a in range(len(sh.l)):
        la, A = int(sh.l[a]), sh.center[a]
        ea = sh.exps[sh.poff[a]:sh.poff[a + 1]]
        ca = np.array([c * _norm(la, e) for c, e in zip(sh.coefs[sh.poff[a]:sh.poff[a + 1]], ea)])
        for b in range(len(sh.l)):
            lb, B = int(sh.l[b]), sh.center[b]
            eb = sh.exps[sh.poff[b]:sh.poff[b + 1]]
            cb = np.array([c * _norm(lb, e) for c, e in zip(sh.coefs[sh.poff[b]:sh.poff[b + 1]], eb)])
            r = np.outer(RATIO[la], RATIO[lb])
            so = _block(lib.libint_overlap_c, la, ea, ca, A, lb, eb, cb, B)
            ko = _block(lib.libint_kinetic_c, la, ea, ca, A, lb, eb, cb, B)
            vo = sum(-z * _block(lib.libint_potential_c, la, ea, ca, A, lb, eb, cb, B, C)
                     for z, C in zip(Z, xyz))
            assert lib.pyfacc_last_status() == N.OK
            blk = (slice(off[a], off[a + 1]), slice(off[b], off[b + 1]))
            for got, ref in ((so * r, S[blk]), (ko * r, T[blk]), (vo * r, V[blk])):
                worst = max(worst, float(np.abs(got - ref).max()))
    assert worst < 1e-10, worst


def test_libint_f_shell_is_refused(engine):
    from pyfacc import _native as N
    lib = N.lib()
    out = _block(lib.libint_overlap_c, 3, [1.0], [1.0], [0.0, 0.0, 0.0], 0, [1.0], [1.0], [0.0, 0.0, 1.0])
    assert np.isnan(out).all()
    assert lib.pyfacc_last_status() == N.ERR_UNSUPPORTED_L
