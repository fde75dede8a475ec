"""The C-ABI library loads and exports every symbol include/*.h declares;
host-only entry points work without a GPU; failures are reported, not
faked (no CPU fallback)."""
import ctypes
import glob
import math
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\(", text, flags=re.M):
            line = text[m.start():text.find("\n", m.start())]
            if line.startswith("typedef"):
                continue
            name = m.group(1)
            if name not in ("if", "defined"):
                names.add(name)
    return names


def test_library_exports_every_declared_symbol(engine):
    from pyfacc import _native as N
    L = N.lib()
    decl = declared_symbols()
    assert "run_scf_c" in decl and "pyfacc_run" in decl
    for name in decl:
        assert hasattr(L, name), f"{name} declared in include/ but not exported"
    assert decl <= set(N.SIGNATURES), "every declared symbol has a ctypes signature"


def test_version_and_status_strings(engine):
    from pyfacc import _native as N
    L = N.lib()
    assert b"sm_100a" in L.pyfacc_version()
    for s in range(0, 11):
        assert L.pyfacc_status_string(s)


def test_default_options(engine):
    from pyfacc import _native as N
    o = N.default_options()
    assert o.eps_energy == 1e-10 and o.eps_diis == 1e-8 and o.max_iter == 100 and o.diis_size == 8
    assert o.schwarz_thresh == 1e-12 and o.fp32_thresh == 1e-3 and o.shard_count == 1


def test_partition_balances_costs(engine):
    from pyfacc import _native as N
    L = N.lib()
    cost = np.array([5.0, 1, 1, 1, 1, 1, 3, 3, 1, 1, 2, 4], dtype=np.float64)
    for parts in (1, 2, 3, 5):
        b = (ctypes.c_int * (parts + 1))()
        assert L.pyfacc_partition(len(cost), cost.ctypes.data_as(N.P_double), parts, b) == 0
        b = list(b)
        assert b[0] == 0 and b[-1] == len(cost) and b == sorted(b)
        shares = [cost[b[i]:b[i + 1]].sum() for i in range(parts)]
        assert max(shares) <= cost.sum() / parts + cost.max()
    assert L.pyfacc_partition(-1, None, 2, (ctypes.c_int * 3)()) == N.ERR_INVALID


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", None) is None and
                    __import__("torch").cuda.is_available(), reason="GPU present: covered by gpu tests")
def test_no_device_reports_status_and_nan(engine):
    """Without a GPU the drop-in call writes NaN and records NO_DEVICE --
    it never computes on the CPU."""
    import helper_functions as hf
    from pyfacc import _native as N
    L = N.lib()
    e = hf.run_scf(hf.load_library(), "h2o.xyz", 1e-10, 10, ctypes.c_double(), "sto-3g")
    if L.pyfacc_last_status() == N.ERR_NO_DEVICE:
        assert math.isnan(e)
    mol = engine.Molecule(["H", "H"], [[0, 0, 0], [0, 0, 1.4]])
    with pytest.raises(engine.PyfaccError) as ei:
        engine.run(mol)
    assert ei.value.status in (N.ERR_NO_DEVICE, N.ERR_CUDA)
