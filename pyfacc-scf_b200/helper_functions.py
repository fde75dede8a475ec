"""Drop-in replacement for PyFAcc-SCF's src/python/helper_functions.py.

Same functions, argument meaning and error behaviour:

* ``read_xyz(filename)``            helper_functions.py:25-54
* ``guess_multiplicity(atoms)``     helper_functions.py:63-74
* ``compute_spin_electrons(atoms)`` helper_functions.py:76-87
* ``run_scf(lib, atom_file, eps_scf, max_iter, final_energy, basis_set,
  charge=0)``                       helper_functions.py:90-149

``run_scf`` marshals the arguments exactly as the reference does and calls
``lib.run_scf_c``; ``lib`` is a ``ctypes.CDLL`` of libpyfacc_b200.so (see
``load_library``) instead of libscf.so.  Molecules are read from
``./data/molecules/<atom_file>`` as in the reference; when that file does
not exist the copy shipped with this package is used.
"""
import ctypes
import os
from ctypes import POINTER, c_char, c_double, c_int

import numpy as np

angtobohr = 1.8897259886

periodic_table = {
    'H': 1, 'He': 2, 'Li': 3, 'Be': 4, 'B': 5, 'C': 6, 'N': 7, 'O': 8,
    'F': 9, 'Ne': 10, 'Na': 11, 'Mg': 12, 'Al': 13, 'Si': 14, 'P': 15, 'S': 16,
    'Cl': 17, 'Ar': 18, 'K': 19, 'Ca': 20, 'Sc': 21, 'Ti': 22, 'V': 23,
    'Cr': 24, 'Mn': 25, 'Fe': 26, 'Co': 27, 'Ni': 28, 'Cu': 29, 'Zn': 30,
    'Ga': 31, 'Ge': 32, 'As': 33, 'Se': 34, 'Br': 35, 'Kr': 36, 'Rb': 37,
    'Sr': 38, 'Y': 39, 'Zr': 40, 'Nb': 41, 'Mo': 42, 'Tc': 43, 'Ru': 44,
    'Rh': 45, 'Pd': 46, 'Ag': 47, 'Cd': 48, 'In': 49, 'Sn': 50, 'Sb': 51,
    'Te': 52, 'I': 53, 'Xe': 54,
}

_HERE = os.path.dirname(os.path.abspath(__file__))


def load_library(path=None):
    """ctypes.CDLL of the engine (the reference loads build/lib/libscf.so)."""
    return ctypes.CDLL(path or os.path.join(_HERE, "lib", "libpyfacc_b200.so"))


def symbols_to_z(species):
    return [periodic_table[s] for s in species]


def _molecule_path(filename):
    path = f"./data/molecules/{filename}"
    if not os.path.exists(path):
        shipped = os.path.join(_HERE, "data", "molecules", filename)
        if os.path.exists(shipped):
            return shipped
    return path


def read_xyz(filename):
    """
    Reads an .xyz file and returns:
    - natoms: int, number of atoms
    - coords: np.ndarray of shape (3, natoms), atomic coordinates in bohr
    - species: np.ndarray of shape (natoms,), element symbols as strings
    """
    with open(_molecule_path(filename), 'r') as file:
        lines = file.readlines()
    natoms = int(lines[0].strip())
    species = []
    coords = []
    for line in lines[2:2 + natoms]:
        parts = line.strip().split()
        if len(parts) != 4:
            raise ValueError(f"Invalid line in XYZ file: {line}")
        species.append(parts[0])
        coords.append([float(parts[1]), float(parts[2]), float(parts[3])])
    # (natoms, 3) transposed: an F-ordered (3, natoms) view whose memory is
    # atom-major x1 y1 z1 x2 ..., the order run_scf_c expects
    coords = np.array(coords).T * angtobohr
    species = np.array(species, dtype=str)
    return natoms, coords, species


known_multiplicities = {
    ('O', 2): 3,  # O2 molecule
    ('N', 2): 4,  # N2 molecule
}


def guess_multiplicity(atoms, charge=0):
    total_electrons = sum(periodic_table[atom] for atom in atoms) - charge
    atom_counts = {atom: list(atoms).count(atom) for atom in set(atoms)}
    for (symbol, count), mult in known_multiplicities.items():
        if atom_counts.get(symbol, 0) == count and len(atom_counts) == 1:
            return mult
    return 1 if total_electrons % 2 == 0 else 2


def compute_spin_electrons(atoms, charge=0):
    """Returns (n_alpha, n_beta, multiplicity)"""
    total_electrons = sum(periodic_table[atom] for atom in atoms) - charge
    multiplicity = guess_multiplicity(atoms, charge)
    S = (multiplicity - 1) / 2
    if (total_electrons + 2 * S) % 2 != 0:
        raise ValueError("Inconsistent electron count and spin state.")
    n_alpha = int((total_electrons + 2 * S) // 2)
    n_beta = total_electrons - n_alpha
    return n_alpha, n_beta, multiplicity


def run_scf(lib, atom_file, eps_scf, max_iter, final_energy, basis_set, charge=0):
    natoms, coords, species_list = read_xyz(atom_file)
    nalpha, nbeta, _ = compute_spin_electrons(species_list, charge)
    nelectrons = nalpha + nbeta
    z_num_list = symbols_to_z(species_list)

    species_fixed = [s.ljust(2) for s in species_list]
    flat_bytes = b''.join(s.encode('utf-8') for s in species_fixed)
    species_c_array = (c_char * (2 * natoms))(*flat_bytes)

    coords_flat = np.array(coords, dtype=np.float64)  # keeps the atom-major memory order
    coords_c = coords_flat.ctypes.data_as(POINTER(c_double))

    z_array = np.array(z_num_list, dtype=np.int32)
    z_num_c = z_array.ctypes.data_as(POINTER(c_int))

    natoms_c = c_int(natoms)
    nelectrons_c = c_int(nelectrons)
    nalpha_c = c_int(nalpha)
    nbeta_c = c_int(nbeta)
    eps_scf_c = c_double(eps_scf)
    max_iter_c = c_int(max_iter)
    charge_c = c_int(charge)
    final_energy_c = c_double(0.0)
    basis_set_c = basis_set.encode('utf-8')

    lib.run_scf_c(natoms_c, nelectrons_c, charge_c, nalpha_c, nbeta_c, species_c_array, coords_c,
                  eps_scf_c, max_iter_c, ctypes.byref(final_energy_c), basis_set_c, z_num_c)

    return final_energy_c.value
