"""The C-ABI library loads without a GPU and exports every entry point that
include/cpsd_b200.h declares; the host-side size math matches Python's."""
import ctypes
import os
import re

import numpy as np

from cpsd_b200 import api
from cpsd_b200.dpd import Symmetry, xor_dirprd

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "cpsd_b200.h")


def declared_symbols():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b((?:cpsd_|vv2v_)\w+)\s*\(", src))
    names |= {"cpsd_" + k for k in re.findall(r"CPSD_KERNEL\((\w+)\);", src)}
    return sorted(n for n in names if not n.startswith("CPSD"))


def test_every_declared_symbol_is_exported():
    lib = api.lib()
    names = declared_symbols()
    assert len(names) >= 50
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_size_math_matches_python():
    lib = api.lib()
    for nirrep in (1, 2, 4, 8):
        d = xor_dirprd(nirrep)
        api.init(nirrep, d)
        sym = Symmetry(nirrep, d)
        rng = np.random.default_rng(nirrep)
        p = rng.integers(0, 6, 8)
        q = rng.integers(0, 6, 8)
        for s in range(1, nirrep + 1):
            for iop in (0, 1, 2):
                assert lib.cpsd_irpdso(ctypes.c_int64(s), api.arr8(p), api.arr8(p), ctypes.c_int64(iop)) == \
                    sym.irpdso(s, p, p, iop)
                assert lib.cpsd_idsymsoc(ctypes.c_int64(s), api.arr8(p), api.arr8(p), ctypes.c_int64(iop),
                                         api.arr8(q), api.arr8(p), ctypes.c_int64(1)) == \
                    sym.idsymsoc(s, p, p, iop, q, p, 1)
                for h in range(1, nirrep + 1):
                    assert lib.cpsd_isymoffso(ctypes.c_int64(h), ctypes.c_int64(s), api.arr8(p), api.arr8(q),
                                              ctypes.c_int64(iop)) == sym.isymoffso(h, s, p, q, iop)


def test_errors_are_returned_not_fatal():
    lib = api.lib()
    rc = lib.cpsd_init(ctypes.c_int64(9), api.arr8([0] * 8))
    assert rc != 0 and lib.cpsd_last_error()
