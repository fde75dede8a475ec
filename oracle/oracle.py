"""CPU oracle for PyFAcc-SCF's hot path (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of
bench.py import this module, as the checker.  The product package never does.

It restates, in NumPy around the C++ kernels of ``oracle.cpp``:

* ``read_xyz`` / ``compute_spin_electrons`` / ``guess_multiplicity``
  (src/python/helper_functions.py:25-87)
* basis construction and shell order (src/fortran/basis.f90:9-190)
* the Roothaan loops (src/fortran/rscf.f90:54-164, src/fortran/uscf.f90:139-213)
  with canonical orthogonalisation X = U s^-1/2 (src/fortran/la.f90:28-57)

Deviations from the literal reference, all intended semantics (the reference
cannot run as shipped):

* D4  J/K use every 8-fold image (rscf.f90:170-184 drops non-canonical ones).
* D5  RHF when n_alpha == n_beta, UHF otherwise (main.f90:57-61 intent).
* D6  converge on |dE| and the DIIS commutator instead of stopping at
      max_iter=10; Pulay DIIS accelerates the same fixed point.
* D7  S is diagonalised once (la.f90:38 re-diagonalises every call).
* D8  basis sections are delimited by '****', so shell lines of elements that
      are absent from the molecule are never read as atom labels
      (basis.f90:30-60 would misread an 'S' shell line as sulphur).

Parity with the reference's own outputs is unpinned: the reference has no
tests or golden vectors and cannot be built here.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
ANG_TO_BOHR = 1.8897259886  # helper_functions.py:7

PERIODIC_TABLE = {  # helper_functions.py:10-19
    'H': 1, 'He': 2, 'Li': 3, 'Be': 4, 'B': 5, 'C': 6, 'N': 7, 'O': 8,
    'F': 9, 'Ne': 10, 'Na': 11, 'Mg': 12, 'Al': 13, 'Si': 14, 'P': 15, 'S': 16,
    'Cl': 17, 'Ar': 18, 'K': 19, 'Ca': 20, 'Sc': 21, 'Ti': 22, 'V': 23,
    'Cr': 24, 'Mn': 25, 'Fe': 26, 'Co': 27, 'Ni': 28, 'Cu': 29, 'Zn': 30,
    'Ga': 31, 'Ge': 32, 'As': 33, 'Se': 34, 'Br': 35, 'Kr': 36, 'Rb': 37,
    'Sr': 38, 'Y': 39, 'Zr': 40, 'Nb': 41, 'Mo': 42, 'Tc': 43, 'Ru': 44,
    'Rh': 45, 'Pd': 46, 'Ag': 47, 'Cd': 48, 'In': 49, 'Sn': 50, 'Sb': 51,
    'Te': 52, 'I': 53, 'Xe': 54,
}


def build_lib() -> str:
    """Compile liboracle.so with the committed Makefile if it is missing."""
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
            os.path.join(HERE, "oracle.cpp")):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(build_lib())
        d, i, p = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        _LIB.orc_boys.restype = d
        _LIB.orc_boys.argtypes = [i, i, d]
        _LIB.orc_norm.restype = d
        _LIB.orc_norm.argtypes = [i, i, i, d]
        _LIB.orc_enuc.restype = d
        _LIB.orc_enuc.argtypes = [i, p, p]
        sh = [i, p, p, p, p, p, p]
        _LIB.orc_one_electron.argtypes = sh + [i, p, p, i, p, p, p]
        _LIB.orc_eri_quartet.argtypes = sh + [i, i, i, i, i, i, p]
        _LIB.orc_eri_tensor.argtypes = sh + [i, p]
        _LIB.orc_schwarz.argtypes = sh + [i, p]
        _LIB.orc_jk.restype = ctypes.c_long
        _LIB.orc_jk.argtypes = sh + [i, i, p, d, p, p]
        _LIB.orc_jk_range.restype = ctypes.c_long
        _LIB.orc_jk_range.argtypes = sh + [i, i, p, d, i, i, p, p]
        _LIB.orc_gradient.argtypes = sh + [i, p, p, i, p, p, p, p, d, p, p, p, p]
        _LIB.orc_jk_sample.restype = ctypes.c_long
        _LIB.orc_jk_sample.argtypes = sh + [i, i, p, d, i, i, p, p]
        _LIB.orc_gradient_sample.argtypes = sh + [i, p, p, i, p, p, p, p, d, i, i, p, p, p, p]
    return _LIB


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


# ---------------------------------------------------------------------------
# Inputs (helper_functions.py:25-87)
# ---------------------------------------------------------------------------
def read_xyz(path: str):
    """helper_functions.py:25-54, on an explicit path.  Returns natoms,
    coords (3, natoms) in bohr, species."""
    with open(path) as fh:
        lines = fh.readlines()
    natoms = int(lines[0].strip())
    species, coords = [], []
    for line in lines[2:2 + natoms]:
        parts = line.strip().split()
        if len(parts) != 4:
            raise ValueError(f"Invalid line in XYZ file: {line}")
        species.append(parts[0])
        coords.append([float(parts[1]), float(parts[2]), float(parts[3])])
    coords = np.array(coords).T * ANG_TO_BOHR
    return natoms, coords, np.array(species, dtype=str)


def guess_multiplicity(atoms, charge=0):
    """helper_functions.py:63-74."""
    total = sum(PERIODIC_TABLE[a] for a in atoms) - charge
    counts = {a: list(atoms).count(a) for a in set(atoms)}
    for (sym, cnt), mult in {('O', 2): 3, ('N', 2): 4}.items():
        if counts.get(sym, 0) == cnt and len(counts) == 1:
            return mult
    return 1 if total % 2 == 0 else 2


def compute_spin_electrons(atoms, charge=0):
    """helper_functions.py:76-87."""
    total = sum(PERIODIC_TABLE[a] for a in atoms) - charge
    mult = guess_multiplicity(atoms, charge)
    s = (mult - 1) / 2
    if (total + 2 * s) % 2 != 0:
        raise ValueError("Inconsistent electron count and spin state.")
    na = int((total + 2 * s) // 2)
    return na, total - na, mult


# ---------------------------------------------------------------------------
# Basis (basis.f90:9-190)
# ---------------------------------------------------------------------------
@dataclass
class Shells:
    l: np.ndarray          # int32 [ns]
    atom: np.ndarray       # int32 [ns] (0-based)
    center: np.ndarray     # float64 [ns, 3]
    poff: np.ndarray       # int32 [ns+1]
    exps: np.ndarray       # float64 [nprim]
    coefs: np.ndarray      # float64 [nprim]
    nbf: int = 0
    bf_off: np.ndarray = field(default=None)

    def args(self):
        return [len(self.l), _ptr(self.l), _ptr(self.atom), _ptr(self.center), _ptr(self.poff),
                _ptr(self.exps), _ptr(self.coefs)]


def _fnum(tok: str) -> float:
    return float(tok.replace('D', 'E').replace('d', 'e'))


def build_basis(basis_file: str, species, coords) -> Shells:
    """Shells in reference order: element sections in file order, shells in
    section order, matching atoms in input order; an SP line yields all its
    S shells, then all its P shells (basis.f90:9-190).  No contraction
    renormalisation."""
    species = [str(s).strip() for s in species]
    coords = np.asarray(coords, dtype=np.float64).reshape(3, -1)
    with open(basis_file) as fh:
        lines = [ln.rstrip('\n') for ln in fh]
    L, A, E, Cf = [], [], [], []
    i = 0
    while i < len(lines):
        ln = lines[i]
        i += 1
        if ln.strip() == '' or ln.startswith('!'):
            continue
        label = ln.split()[0]
        if label == '****':
            continue
        atoms = [k for k, s in enumerate(species) if s == label]
        # consume the section up to '****'
        while i < len(lines):
            ln = lines[i]
            i += 1
            if '****' in ln:
                break
            if not atoms:
                continue
            parts = ln.split()
            kind, nprim = parts[0], int(parts[1])
            prims = [lines[i + k].split() for k in range(nprim)]
            i += nprim
            if kind == 'S':
                groups = [(0, 1)]
            elif kind == 'P':
                groups = [(1, 1)]
            elif kind == 'SP':
                groups = [(0, 1), (1, 2)]
            elif kind == 'D':
                # not read by the reference (basis.f90:76-82 has no D branch);
                # the oracle takes Cartesian d shells (xx, xy, xz, yy, yz, zz)
                # so that the d-shell integrals can be checked
                groups = [(2, 1)]
            else:
                raise ValueError(f"unsupported shell type {kind!r} for element {label}")
            for lval, col in groups:
                ex = [_fnum(p[0]) for p in prims]
                cf = [_fnum(p[col]) for p in prims]
                for a in atoms:
                    L.append(lval); A.append(a); E.append(ex); Cf.append(cf)
    present = set(species)
    found = {species[a] for a in A}
    missing = present - found
    if missing:
        raise ValueError(f"no basis functions for {sorted(missing)} in {basis_file}")
    poff = np.zeros(len(L) + 1, dtype=np.int32)
    poff[1:] = np.cumsum([len(e) for e in E])
    sh = Shells(l=np.array(L, dtype=np.int32), atom=np.array(A, dtype=np.int32),
                center=np.ascontiguousarray(coords.T[np.array(A, dtype=int)]),
                poff=poff, exps=np.array(sum(E, []), dtype=np.float64),
                coefs=np.array(sum(Cf, []), dtype=np.float64))
    ncart = (sh.l + 1) * (sh.l + 2) // 2
    sh.bf_off = np.concatenate([[0], np.cumsum(ncart)]).astype(np.int32)
    sh.nbf = int(sh.bf_off[-1])
    return sh


# ---------------------------------------------------------------------------
# Molecule + integrals
# ---------------------------------------------------------------------------
@dataclass
class Molecule:
    species: list
    Z: np.ndarray          # int32 [natoms]
    xyz: np.ndarray        # float64 [natoms, 3], bohr
    nalpha: int
    nbeta: int
    shells: Shells

    @property
    def natoms(self):
        return len(self.Z)


def molecule(species, xyz_bohr, basis_file, charge=0, nalpha=None, nbeta=None) -> Molecule:
    species = [str(s).strip() for s in species]
    xyz = np.ascontiguousarray(np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3))
    if nalpha is None:
        nalpha, nbeta, _ = compute_spin_electrons(species, charge)
    Z = np.array([PERIODIC_TABLE[s] for s in species], dtype=np.int32)
    sh = build_basis(basis_file, species, xyz.T)
    return Molecule(species, Z, xyz, nalpha, nbeta, sh)


def enuc(mol: Molecule) -> float:
    return lib().orc_enuc(mol.natoms, _ptr(mol.xyz), _ptr(mol.Z))


def boys(m: int, x: float, mode: int = 0) -> float:
    return lib().orc_boys(mode, m, x)


def one_electron(mol: Molecule, boys_mode: int = 0):
    n = mol.shells.nbf
    S, T, V = (np.zeros((n, n)) for _ in range(3))
    lib().orc_one_electron(*mol.shells.args(), mol.natoms, _ptr(mol.xyz), _ptr(mol.Z), boys_mode,
                           _ptr(S), _ptr(T), _ptr(V))
    return S, T, V


def eri_quartet(mol: Molecule, a, b, c, d, method=0, boys_mode=0):
    l = mol.shells.l
    nc = [(int(l[s]) + 1) * (int(l[s]) + 2) // 2 for s in (a, b, c, d)]
    out = np.zeros(nc)
    lib().orc_eri_quartet(*mol.shells.args(), a, b, c, d, method, boys_mode, _ptr(out))
    return out


def eri_tensor(mol: Molecule, boys_mode=0):
    n = mol.shells.nbf
    out = np.zeros((n, n, n, n))
    lib().orc_eri_tensor(*mol.shells.args(), boys_mode, _ptr(out))
    return out


def jk_range(mol: Molecule, dens, ij_begin, ij_end, thresh=1e-12):
    """Partial J/K over bra shell pairs ij_begin <= a(a+1)/2 + b < ij_end."""
    D = np.ascontiguousarray(np.asarray(dens, dtype=np.float64))[None]
    J = np.zeros_like(D)
    K = np.zeros_like(D)
    lib().orc_jk_range(*mol.shells.args(), 0, 1, _ptr(D), thresh, ij_begin, ij_end, _ptr(J), _ptr(K))
    return J[0], K[0]


def schwarz(mol: Molecule, boys_mode=0):
    ns = len(mol.shells.l)
    q = np.zeros(ns * (ns + 1) // 2)
    lib().orc_schwarz(*mol.shells.args(), boys_mode, _ptr(q))
    return q


def jk(mol: Molecule, dens, thresh=1e-12, boys_mode=0):
    """J[d], K[d] for a stack of densities (nd, nbf, nbf).  The SCF always
    uses the exact Boys function for ERIs (deviation D2)."""
    D = np.ascontiguousarray(np.asarray(dens, dtype=np.float64))
    single = D.ndim == 2
    if single:
        D = D[None]
    nd, n = D.shape[0], D.shape[1]
    J = np.zeros_like(D)
    K = np.zeros_like(D)
    lib().orc_jk(*mol.shells.args(), boys_mode, nd, _ptr(D), thresh, _ptr(J), _ptr(K))
    return (J[0], K[0]) if single else (J, K)


def jk_sample(mol: Molecule, dens, stride, phase=0, thresh=1e-12):
    """Partial J/K of the bra pairs ij with ij % stride == phase (a uniform
    sample of one Fock build, ~1/stride of its work; for timing)."""
    D = np.ascontiguousarray(np.asarray(dens, dtype=np.float64))
    if D.ndim == 2:
        D = D[None]
    J = np.zeros_like(D)
    K = np.zeros_like(D)
    lib().orc_jk_sample(*mol.shells.args(), 0, D.shape[0], _ptr(D), thresh, stride, phase, _ptr(J), _ptr(K))
    return J, K


def gradient_sample(mol: Molecule, Pt, Pa, Pb, W, stride, phase=0, thresh=1e-12):
    """Gradient pieces of every stride-th one-electron shell and two-electron
    bra pair (a uniform sample of the analytic gradient; for timing)."""
    na = mol.natoms
    g = [np.zeros((na, 3)) for _ in range(4)]
    c = np.ascontiguousarray
    lib().orc_gradient_sample(*mol.shells.args(), na, _ptr(mol.xyz), _ptr(mol.Z), 0, _ptr(c(Pt)), _ptr(c(Pa)),
                              _ptr(c(Pb)), _ptr(c(W)), thresh, stride, phase, *[_ptr(x) for x in g])
    return g


# ---------------------------------------------------------------------------
# SCF (rscf.f90 / uscf.f90 with DIIS)
# ---------------------------------------------------------------------------
@dataclass
class ScfResult:
    energy: float
    e_elec: float
    e_nuc: float
    converged: bool
    n_iter: int
    uhf: bool
    C: list
    eps: list
    D: list               # spin densities (RHF: [P/2, P/2])
    P: np.ndarray         # total density
    S: np.ndarray
    H: np.ndarray
    history: list


def _diis(fs, es):
    m = len(fs)
    B = -np.ones((m + 1, m + 1))
    B[m, m] = 0.0
    for i in range(m):
        for j in range(m):
            B[i, j] = np.vdot(es[i], es[j])
    rhs = np.zeros(m + 1)
    rhs[m] = -1.0
    try:
        c = np.linalg.solve(B, rhs)[:m]
    except np.linalg.LinAlgError:
        c = np.linalg.lstsq(B, rhs, rcond=None)[0][:m]
    return sum(ci * fi for ci, fi in zip(c, fs))


def scf(mol: Molecule, e_tol=1e-10, d_tol=1e-8, max_iter=200, diis_size=8, boys_mode=0,
        thresh=1e-12, uhf=None, use_diis=True) -> ScfResult:
    if uhf is None:
        uhf = mol.nalpha != mol.nbeta
    S, T, V = one_electron(mol, boys_mode)
    H = T + V
    s, U = np.linalg.eigh(S)
    X = U / np.sqrt(s)
    e0, Cp = np.linalg.eigh(X.T @ H @ X)
    C0 = X @ Cp
    if uhf:
        Cs = [C0, C0]
        occ = [mol.nalpha, mol.nbeta]
    else:
        occ = [(mol.nalpha + mol.nbeta + 1) // 2]
        Cs = [C0]
    def dens(Cs):
        if uhf:
            return [C[:, :o] @ C[:, :o].T for C, o in zip(Cs, occ)]
        P = 2.0 * Cs[0][:, :occ[0]] @ Cs[0][:, :occ[0]].T
        return [0.5 * P, 0.5 * P]
    Ds = dens(Cs)
    en = enuc(mol)
    E_old = 0.0
    fs_hist, es_hist, history = [], [], []
    converged = False
    eps = [e0] * len(Cs)
    for it in range(1, max_iter + 1):
        Pt = Ds[0] + Ds[1]
        if uhf:
            J, K = jk(mol, np.stack(Ds), thresh)
            Jt = J[0] + J[1]
            Fs = [H + Jt - K[0], H + Jt - K[1]]
            E = 0.5 * (np.sum(Pt * H) + np.sum(Ds[0] * Fs[0]) + np.sum(Ds[1] * Fs[1]))
        else:
            J, K = jk(mol, Pt, thresh)
            Fs = [H + J - 0.5 * K]
            E = 0.5 * np.sum(Pt * (H + Fs[0]))
        errs = []
        for F, D in zip(Fs, Ds if uhf else [Pt]):
            errs.append(X.T @ (F @ D @ S - S @ D @ F) @ X)
        err = max(float(np.max(np.abs(e))) for e in errs)
        dE = abs(E - E_old)
        history.append((it, E + en, dE, err))
        if dE < e_tol and err < d_tol:
            converged = True
            break
        E_old = E
        if use_diis:
            fs_hist.append(np.concatenate([F.ravel() for F in Fs]))
            es_hist.append(np.concatenate([e.ravel() for e in errs]))
            fs_hist, es_hist = fs_hist[-diis_size:], es_hist[-diis_size:]
            Fx = _diis(fs_hist, es_hist) if len(fs_hist) > 1 else fs_hist[-1]
            n = H.shape[0]
            Fs = [Fx[k * n * n:(k + 1) * n * n].reshape(n, n) for k in range(len(Fs))]
        Cs, eps = [], []
        for F in Fs:
            e, Cp = np.linalg.eigh(X.T @ F @ X)
            Cs.append(X @ Cp)
            eps.append(e)
        Ds = dens(Cs)
    # final orbitals of the converged Fock matrix (for W in the gradient)
    Cs, eps = [], []
    for F in Fs:
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        Cs.append(X @ Cp)
        eps.append(e)
    return ScfResult(E + en, E, en, converged, it, uhf, Cs, eps, Ds, Ds[0] + Ds[1], S, H, history)


def energy_weighted_density(mol: Molecule, res: ScfResult) -> np.ndarray:
    if res.uhf:
        occ = [mol.nalpha, mol.nbeta]
        return sum((C[:, :o] * e[:o]) @ C[:, :o].T for C, e, o in zip(res.C, res.eps, occ))
    o = (mol.nalpha + mol.nbeta + 1) // 2
    C, e = res.C[0], res.eps[0]
    return 2.0 * (C[:, :o] * e[:o]) @ C[:, :o].T


def gradient(mol: Molecule, res: ScfResult, boys_mode=0, thresh=1e-12, parts=False):
    """Analytic gradient (natoms, 3) from derivative integrals."""
    W = energy_weighted_density(mol, res)
    na = mol.natoms
    g = [np.zeros((na, 3)) for _ in range(4)]
    Pt = np.ascontiguousarray(res.P)
    Pa = np.ascontiguousarray(res.D[0])
    Pb = np.ascontiguousarray(res.D[1])
    lib().orc_gradient(*mol.shells.args(), na, _ptr(mol.xyz), _ptr(mol.Z), boys_mode, _ptr(Pt), _ptr(Pa),
                       _ptr(Pb), _ptr(np.ascontiguousarray(W)), thresh, *[_ptr(x) for x in g])
    total = g[0] + g[1] + g[2] + g[3]
    if parts:
        return total, dict(core=g[0], overlap=g[1], two_electron=g[2], nuclear=g[3])
    return total


def gradient_at_density(mol: Molecule, Ds, uhf: bool, thresh=1e-12):
    """Analytic gradient at given spin densities Ds = [D_alpha, D_beta]
    (RHF: [P/2, P/2]): the Fock matrices from these densities, the energy-
    weighted density W = sum_s D_s F_s D_s (the stationarity identity that
    replaces sum_i eps_i C_i C_i^T at a converged density), then the same
    derivative integrals as gradient().  Compares two programs at one
    density, free of the SCF convergence error of either."""
    S, T, V = one_electron(mol)
    H = T + V
    Ds = [np.ascontiguousarray(D) for D in Ds]
    Pt = Ds[0] + Ds[1]
    if uhf:
        J, K = jk(mol, np.stack(Ds), thresh)
        Jt = J[0] + J[1]
        Fs = [H + Jt - K[0], H + Jt - K[1]]
    else:
        J, K = jk(mol, Pt, thresh)
        Fs = [H + J - 0.5 * K] * 2
    W = Ds[0] @ Fs[0] @ Ds[0] + Ds[1] @ Fs[1] @ Ds[1]
    na = mol.natoms
    g = [np.zeros((na, 3)) for _ in range(4)]
    lib().orc_gradient(*mol.shells.args(), na, _ptr(mol.xyz), _ptr(mol.Z), 0, _ptr(np.ascontiguousarray(Pt)),
                       _ptr(Ds[0]), _ptr(Ds[1]), _ptr(np.ascontiguousarray(W)), thresh, *[_ptr(x) for x in g])
    return g[0] + g[1] + g[2] + g[3]


def energy(species, xyz_bohr, basis_file, **kw) -> float:
    charge = kw.pop('charge', 0)
    mol = molecule(species, xyz_bohr, basis_file, charge=charge)
    return scf(mol, **kw).energy


def fd_gradient(species, xyz_bohr, basis_file, coords=None, h=1e-4, **kw):
    """Central finite differences of the SCF energy (all or selected
    (atom, axis) coordinates)."""
    xyz = np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    if coords is None:
        coords = [(a, x) for a in range(len(xyz)) for x in range(3)]
    out = {}
    for a, x in coords:
        vals = []
        for s in (+1, -1):
            x2 = xyz.copy()
            x2[a, x] += s * h
            vals.append(energy(species, x2, basis_file, **kw))
        out[(a, x)] = (vals[0] - vals[1]) / (2 * h)
    return out
