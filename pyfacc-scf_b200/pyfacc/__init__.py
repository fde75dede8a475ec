"""pyfacc -- B200 Hartree-Fock engine behind PyFAcc-SCF's interface.

The drop-in entry points of the reference (``run_scf`` and the C symbol
``run_scf_c``) live in ``helper_functions.py`` next to this package and in
``libpyfacc_b200.so``.  This module is the extended Python API:

* :class:`Molecule` -- species, atomic numbers, bohr coordinates, basis name
* :func:`run` -- SCF (RHF/UHF) with optional analytic gradient and matrices
* :func:`run_batch` -- many molecules on one GPU
* :class:`System` -- a molecule kept resident on the GPU (one-electron
  matrices, J/K builds on torch CUDA tensors, SCF, gradient)
* :func:`energy` -- differentiable energy: a ``torch.autograd.Function``
  whose backward is the engine's analytic gradient
* :func:`boys` -- the device Boys function
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from ._native import PyfaccError, lib

ANG_TO_BOHR = 1.8897259886  # helper_functions.py:7 of the reference

PERIODIC_TABLE = {
    'H': 1, 'He': 2, 'Li': 3, 'Be': 4, 'B': 5, 'C': 6, 'N': 7, 'O': 8,
    'F': 9, 'Ne': 10, 'Na': 11, 'Mg': 12, 'Al': 13, 'Si': 14, 'P': 15, 'S': 16,
    'Cl': 17, 'Ar': 18, 'K': 19, 'Ca': 20, 'Sc': 21, 'Ti': 22, 'V': 23,
    'Cr': 24, 'Mn': 25, 'Fe': 26, 'Co': 27, 'Ni': 28, 'Cu': 29, 'Zn': 30,
    'Ga': 31, 'Ge': 32, 'As': 33, 'Se': 34, 'Br': 35, 'Kr': 36, 'Rb': 37,
    'Sr': 38, 'Y': 39, 'Zr': 40, 'Nb': 41, 'Mo': 42, 'Tc': 43, 'Ru': 44,
    'Rh': 45, 'Pd': 46, 'Ag': 47, 'Cd': 48, 'In': 49, 'Sn': 50, 'Sb': 51,
    'Te': 52, 'I': 53, 'Xe': 54,
}

__all__ = ["Molecule", "ScfResult", "run", "run_batch", "System", "energy", "boys", "PyfaccError",
           "ANG_TO_BOHR", "PERIODIC_TABLE"]


@dataclass
class Molecule:
    species: list
    coords: np.ndarray            # (natoms, 3) bohr
    basis: str = "sto-3g"
    charge: int = 0
    nalpha: int = -1              # < 0: derived like helper_functions.compute_spin_electrons
    nbeta: int = -1

    def __post_init__(self):
        self.species = [str(s).strip() for s in self.species]
        self.coords = np.ascontiguousarray(np.asarray(self.coords, dtype=np.float64).reshape(-1, 3))
        if len(self.species) != len(self.coords):
            raise ValueError("species and coordinates differ in length")

    @property
    def natoms(self):
        return len(self.species)

    @property
    def z(self):
        return np.array([PERIODIC_TABLE[s] for s in self.species], dtype=np.int32)

    @classmethod
    def from_xyz(cls, path: str, basis: str = "sto-3g", charge: int = 0) -> "Molecule":
        with open(path) as fh:
            lines = fh.readlines()
        n = int(lines[0].strip())
        sp, xyz = [], []
        for line in lines[2:2 + n]:
            parts = line.split()
            if len(parts) != 4:
                raise ValueError(f"Invalid line in XYZ file: {line}")
            sp.append(parts[0])
            xyz.append([float(v) for v in parts[1:]])
        return cls(sp, np.array(xyz) * ANG_TO_BOHR, basis, charge)

    def _struct(self):
        """C struct plus the buffers it points into (kept alive by the caller)."""
        z = self.z
        coords = np.ascontiguousarray(self.coords, dtype=np.float64)
        species = b"".join(s.ljust(2).encode() for s in self.species)
        sp_buf = ctypes.create_string_buffer(species, len(species))
        basis = self.basis.encode()
        m = N.MoleculeC()
        m.natoms = self.natoms
        m.z = z.ctypes.data_as(N.P_int32)
        m.coords = coords.ctypes.data_as(N.P_double)
        m.species = ctypes.cast(sp_buf, ctypes.c_void_p)
        m.charge = self.charge
        m.nalpha = self.nalpha
        m.nbeta = self.nbeta
        m.basis = basis
        return m, (z, coords, sp_buf, basis)


@dataclass
class ScfResult:
    energy: float
    e_elec: float
    e_nuc: float
    converged: bool
    n_iter: int
    uhf: bool
    nbf: int
    n_fock_builds: int
    status: int
    gradient: Optional[np.ndarray] = None
    matrices: dict = field(default_factory=dict)
    timings_ms: dict = field(default_factory=dict)
    quartets: dict = field(default_factory=dict)
    flops: dict = field(default_factory=dict)
    last_delta_e: float = 0.0
    last_diis_error: float = 0.0
    task_width: int = 32


def _options(**kw) -> N.Options:
    prec = kw.pop("precision", None)
    if isinstance(prec, str):
        kw["precision"] = {"fp64": N.PRECISION_FP64, "mixed": N.PRECISION_MIXED}[prec]
    elif prec is not None:
        kw["precision"] = prec
    gp = kw.pop("gradient_precision", None)
    if isinstance(gp, str):
        kw["gradient_precision"] = {"fp64": N.PRECISION_FP64, "mixed": N.PRECISION_MIXED}[gp]
    elif gp is not None:
        kw["gradient_precision"] = gp
    bm = kw.pop("boys_mode", None)
    if isinstance(bm, str):
        kw["boys_mode"] = {"accurate": N.BOYS_ACCURATE, "reference_trapezoid": N.BOYS_REFERENCE_TRAPEZOID}[bm]
    elif bm is not None:
        kw["boys_mode"] = bm
    gs = kw.pop("guess", None)
    if isinstance(gs, str):
        kw["guess"] = {"core": N.GUESS_CORE, "atomic": N.GUESS_ATOMIC}[gs]
    elif gs is not None:
        kw["guess"] = gs
    st = kw.pop("scf_type", None)
    if isinstance(st, str):
        kw["scf_type"] = {"auto": N.SCF_AUTO, "rhf": N.SCF_RHF, "uhf": N.SCF_UHF}[st.lower()]
    elif st is not None:
        kw["scf_type"] = st
    return N.default_options(**kw)


def _result_buffers(nbf: int, natoms: int, gradient: bool, matrices: bool):
    r = N.Result()
    keep = {}
    if gradient:
        keep["gradient"] = np.zeros((natoms, 3))
        r.gradient = keep["gradient"].ctypes.data_as(N.P_double)
    if matrices:
        for k in ("S", "T", "V", "P", "C_alpha", "C_beta"):
            keep[k] = np.zeros((nbf, nbf))
            setattr(r, k, keep[k].ctypes.data_as(N.P_double))
        for k in ("eps_alpha", "eps_beta"):
            keep[k] = np.zeros(nbf)
            setattr(r, k, keep[k].ctypes.data_as(N.P_double))
    return r, keep


def _to_result(r: N.Result, keep: dict, status: int) -> ScfResult:
    mats = {}
    for k, v in keep.items():
        if k == "gradient":
            continue
        if k.startswith("C_"):
            v = v.T.copy()  # the engine writes C column-major: orbital j = column j
        mats[k] = v
    return ScfResult(
        energy=r.energy, e_elec=r.e_elec, e_nuc=r.e_nuc, converged=bool(r.converged), n_iter=r.n_iter,
        uhf=r.scf_type == N.SCF_UHF, nbf=r.nbf, n_fock_builds=r.n_fock_builds, status=status,
        gradient=keep.get("gradient"), matrices=mats,
        timings_ms=dict(total=r.ms_total, one_electron=r.ms_one_electron, fock=r.ms_fock, diag=r.ms_diag,
                        gradient=r.ms_gradient),
        quartets=dict(fp64=r.quartets_fp64, fp32=r.quartets_fp32),
        flops=dict(fock=r.flops_fock, gradient=r.flops_gradient),
        last_delta_e=r.last_delta_e, last_diis_error=r.last_diis_error, task_width=r.task_width)


def _nbf_estimate(mol: Molecule) -> int:
    # an upper bound for output buffers before the basis is parsed: STO-nG
    # gives at most 1 (H, He) or 5 (Li-Ne) or 9 (Na-Ar) ... functions per atom
    return int(sum(1 if z <= 2 else (5 if z <= 10 else 9 if z <= 18 else 13) for z in mol.z))


def run(mol: Molecule, gradient: bool = False, matrices: bool = False, check: bool = True, **options) -> ScfResult:
    """SCF of one molecule on the GPU (RHF if n_alpha == n_beta, else UHF)."""
    opt = _options(compute_gradient=int(gradient), **options)
    m, keep_in = mol._struct()
    if matrices:
        with System(mol, **options) as s:
            nbf = s.nbf
    else:
        nbf = _nbf_estimate(mol)
    r, keep = _result_buffers(nbf, mol.natoms, gradient, matrices)
    status = lib().pyfacc_run(ctypes.byref(m), ctypes.byref(opt), ctypes.byref(r))
    if check:
        N.check(status, "pyfacc_run", allow=(N.OK, N.ERR_NOT_CONVERGED))
    return _to_result(r, keep, status)


def run_batch(mols: Sequence[Molecule], gradient: bool = False, check: bool = True, **options):
    """Many molecules on one GPU; returns one ScfResult per molecule."""
    opt = _options(compute_gradient=int(gradient), **options)
    arr = (N.MoleculeC * len(mols))()
    keep_all, res_keep = [], []
    results = (N.Result * len(mols))()
    for i, mol in enumerate(mols):
        m, k = mol._struct()
        arr[i] = m
        keep_all.append(k)
        r, kk = _result_buffers(0, mol.natoms, gradient, False)
        results[i] = r
        res_keep.append(kk)
    status = lib().pyfacc_run_batch(len(mols), arr, ctypes.byref(opt), results)
    if check:
        N.check(status, "pyfacc_run_batch", allow=(N.OK, N.ERR_NOT_CONVERGED))
    return [_to_result(results[i], res_keep[i], status) for i in range(len(mols))]


_BATCH_STAT_KEYS = ("ms_total", "ms_setup", "ms_one_electron", "ms_tune", "ms_scf", "ms_polish", "ms_gradient",
                    "iterations", "flops_fock", "flops_gradient", "quartets_fp64", "quartets_fp32")
_QCLASS_NAMES = ("ss|ss", "ps|ss", "ps|ps", "pp|ss", "pp|ps", "pp|pp")


def batch_stats() -> dict:
    """Timings, counters and task widths of the last run_batch on this thread."""
    n = len(_BATCH_STAT_KEYS) + len(_QCLASS_NAMES) + 1
    buf = (ctypes.c_double * n)()
    N.check(lib().pyfacc_batch_last_stats(buf, n), "pyfacc_batch_last_stats")
    out = {k: buf[i] for i, k in enumerate(_BATCH_STAT_KEYS)}
    out["task_width"] = {q: int(buf[len(_BATCH_STAT_KEYS) + i]) for i, q in enumerate(_QCLASS_NAMES)}
    out["scf_graph_launches"] = int(buf[n - 1])
    return out


def _torch():
    import torch
    return torch


class System:
    """A molecule resident on the GPU (basis, shell pairs, Schwarz factors).

    Device buffers are torch CUDA tensors of dtype float64; the engine works
    on its own stream and synchronises it before returning.
    """

    def __init__(self, mol: Molecule, **options):
        self.mol = mol
        self.opt = _options(**options)
        m, self._keep = mol._struct()
        h = ctypes.c_void_p()
        N.check(lib().pyfacc_system_create(ctypes.byref(m), ctypes.byref(self.opt), ctypes.byref(h)),
                "pyfacc_system_create")
        self.handle = h
        nbf, ns, na, npair = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        lib().pyfacc_system_info(h, ctypes.byref(nbf), ctypes.byref(ns), ctypes.byref(na), ctypes.byref(npair))
        self.nbf, self.nshell, self.natoms, self.npairs = nbf.value, ns.value, na.value, npair.value

    def close(self):
        if getattr(self, "handle", None) and N is not None and N._lib is not None:
            N._lib.pyfacc_system_destroy(self.handle)
        self.handle = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _sync(self):
        torch = _torch()
        if torch.cuda.is_available():
            torch.cuda.current_stream().synchronize()

    def _empty(self, *shape):
        torch = _torch()
        return torch.zeros(*shape, dtype=torch.float64, device="cuda")

    def one_electron(self):
        S, T, V = self._empty(self.nbf, self.nbf), self._empty(self.nbf, self.nbf), self._empty(self.nbf, self.nbf)
        self._sync()
        N.check(lib().pyfacc_system_one_electron(self.handle, S.data_ptr(), T.data_ptr(), V.data_ptr()),
                "pyfacc_system_one_electron")
        return S, T, V

    def jk(self, Dj, Dk=None, precision="fp64"):
        """J[Dj] and K[Dk] (Dk: (nbf, nbf) or (2, nbf, nbf))."""
        torch = _torch()
        Dj = Dj.to(device="cuda", dtype=torch.float64).contiguous()
        Dk = Dj if Dk is None else Dk.to(device="cuda", dtype=torch.float64).contiguous()
        nk = 1 if Dk.dim() == 2 else Dk.shape[0]
        J = self._empty(self.nbf, self.nbf)
        K = self._empty(nk, self.nbf, self.nbf)
        prec = {"fp64": N.PRECISION_FP64, "mixed": N.PRECISION_MIXED, "fp32": N.PRECISION_FP32}.get(precision,
                                                                                                   precision)
        self._sync()
        N.check(lib().pyfacc_system_jk(self.handle, Dj.data_ptr(), nk, Dk.data_ptr(), J.data_ptr(), K.data_ptr(),
                                       prec), "pyfacc_system_jk")
        return J, (K[0] if Dk.dim() == 2 else K)

    def jk_stats(self) -> dict:
        """Timing (CUDA events on the engine stream) and algorithmic flops of
        the last :meth:`jk` build, split by precision."""
        buf = (ctypes.c_double * 31)()
        N.check(lib().pyfacc_system_jk_stats(self.handle, buf, 31), "pyfacc_system_jk_stats")
        keys = ("ms", "flops_fp64", "flops_fp32", "quartets_fp64", "quartets_fp32", "prims_fp64", "prims_fp32")
        out = dict(zip(keys, list(buf)))
        classes = ("ss|ss", "ps|ss", "ps|ps", "pp|ss", "pp|ps", "pp|pp")
        for i, name in enumerate(("quartets_fp64", "quartets_fp32", "prims_fp64", "prims_fp32")):
            out["by_class_" + name] = dict(zip(classes, list(buf)[7 + 6 * i:13 + 6 * i]))
        return out

    def eri_tensor(self):
        eri = self._empty(self.nbf, self.nbf, self.nbf, self.nbf)
        self._sync()
        N.check(lib().pyfacc_system_eri_tensor(self.handle, eri.data_ptr()), "pyfacc_system_eri_tensor")
        return eri

    def scf(self, gradient=False, matrices=False, check=True) -> ScfResult:
        r, keep = _result_buffers(self.nbf, self.natoms, False, matrices)
        status = lib().pyfacc_system_scf(self.handle, ctypes.byref(r))
        if check:
            N.check(status, "pyfacc_system_scf", allow=(N.OK, N.ERR_NOT_CONVERGED))
        res = _to_result(r, keep, status)
        if gradient:
            res.gradient = self.gradient()
        return res

    def result(self, matrices=False) -> ScfResult:
        """Energies, timings and statistics of the last SCF / gradient."""
        r, keep = _result_buffers(self.nbf, self.natoms, True, matrices)
        N.check(lib().pyfacc_system_result(self.handle, ctypes.byref(r)), "pyfacc_system_result")
        return _to_result(r, keep, N.OK)

    def gradient(self) -> np.ndarray:
        g = np.zeros((self.natoms, 3))
        N.check(lib().pyfacc_system_gradient(self.handle, g.ctypes.data_as(N.P_double)), "pyfacc_system_gradient")
        return g

    def set_coords(self, coords_bohr):
        c = np.ascontiguousarray(np.asarray(coords_bohr, dtype=np.float64).reshape(-1, 3))
        N.check(lib().pyfacc_system_set_coords(self.handle, c.ctypes.data_as(N.P_double)), "pyfacc_system_set_coords")
        self.mol = Molecule(self.mol.species, c, self.mol.basis, self.mol.charge, self.mol.nalpha, self.mol.nbeta)


def boys(x, mmax: int, mode: str = "accurate", fp32: bool = False):
    """F_0..F_mmax at the points x (torch CUDA tensor) -> (n, mmax+1)."""
    torch = _torch()
    x = x.to(device="cuda", dtype=torch.float64).contiguous().reshape(-1)
    out = torch.zeros(x.numel(), mmax + 1, dtype=torch.float64, device="cuda")
    m = {"accurate": N.BOYS_ACCURATE, "reference_trapezoid": N.BOYS_REFERENCE_TRAPEZOID}[mode]
    torch.cuda.current_stream().synchronize()
    N.check(lib().pyfacc_boys_dev(m, int(fp32), mmax, x.numel(), x.data_ptr(), out.data_ptr()), "pyfacc_boys_dev")
    return out


def _energy_function():
    torch = _torch()

    class EnergyFn(torch.autograd.Function):
        """E(R) forward, analytic dE/dR backward (computed with the forward)."""

        @staticmethod
        def forward(ctx, coords, mol_template, options):
            c = coords.detach().to("cpu", torch.float64).numpy().reshape(-1, 3)
            mol = Molecule(mol_template.species, c, mol_template.basis, mol_template.charge, mol_template.nalpha,
                           mol_template.nbeta)
            res = run(mol, gradient=True, **options)
            ctx.save_for_backward(torch.as_tensor(res.gradient, dtype=coords.dtype, device=coords.device))
            return torch.as_tensor(res.energy, dtype=coords.dtype, device=coords.device)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g, None, None

    return EnergyFn


_EnergyFn = None


def energy(coords, mol: Molecule, **options):
    """Differentiable SCF energy of ``mol`` at ``coords`` ((natoms, 3) bohr
    torch tensor); ``energy(...).backward()`` fills ``coords.grad`` with the
    analytic nuclear gradient."""
    global _EnergyFn
    if _EnergyFn is None:
        _EnergyFn = _energy_function()
    return _EnergyFn.apply(coords, mol, options)
