"""Drop-in counterpart of PyFAcc-SCF's single_file.py: H2O / STO-3G through
run_scf and the C entry point run_scf_c of libpyfacc_b200.so."""
import ctypes
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from helper_functions import load_library, run_scf  # noqa: E402

eps_scf = 1e-10
max_iter = 10
final_energy = ctypes.c_double()

lib = load_library()

basis = 'sto-3g'
input_file = 'h2o.xyz'

if __name__ == "__main__":
    energy = run_scf(lib, input_file, eps_scf, max_iter, final_energy, basis)
    print(energy)
