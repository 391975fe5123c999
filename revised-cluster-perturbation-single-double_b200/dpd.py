"""DPD size math on the host (int64, 1-based irreps).

Mirrors the reference's size functions so the host can size buffers:
irpdso (src/libsrint/irpdso.f:1-52), idsymsoc (src/libsrint/idsymsoc.f:1-30),
isymoffso (src/libsrint/isymoffso.f:1-54).
"""
import numpy as np

ZORB = (1, 0, 0, 0, 0, 0, 0, 0)


def xor_dirprd(nirrep):
    """Direct-product table of an abelian point group with XOR-ordered irreps
    (C1, Cs/C2/Ci, C2v/C2h/D2, D2h), column-major 8x8, 1-based values."""
    d = np.zeros((8, 8), dtype=np.int64)
    for i in range(8):
        for j in range(8):
            d[i, j] = ((i ^ j) + 1) if (i < nirrep and j < nirrep) else 0
    return d.T.reshape(-1).copy()  # column-major: d[(j)*8 + i] = DIRPRD(i+1, j+1)


class Symmetry:
    def __init__(self, nirrep, dirprd):
        self.nirrep = int(nirrep)
        self.dirprd = np.asarray(dirprd, dtype=np.int64).reshape(8, 8).T  # [i-1, j-1]

    def dp(self, i, j):
        return int(self.dirprd[i - 1, j - 1])

    def irpdso(self, sym, popp, popq, iop):
        n = 0
        for r in range(1, self.nirrep + 1):
            l = self.dp(r, sym)
            if iop == 1:
                n += popp[l - 1] * popq[r - 1]
            elif iop in (0, 2):
                if l > r:
                    continue
                if l < r:
                    n += popp[l - 1] * popq[r - 1]
                elif iop == 0:
                    n += popp[l - 1] * (popq[r - 1] - 1) // 2
                else:
                    n += popp[l - 1] * (popq[r - 1] + 1) // 2
        return int(n)

    def idsymsoc(self, irrepx, popp, popq, ioppq, popr, pops, ioprs):
        n = 0
        for r in range(1, self.nirrep + 1):
            l = self.dp(r, irrepx)
            n += self.irpdso(l, popp, popq, ioppq) * self.irpdso(r, popr, pops, ioprs)
        return int(n)

    def isymoffso(self, irrepq1, irrep, popp, popq, iop):
        off = 1
        for q in range(1, irrepq1):
            p = self.dp(q, irrep)
            if iop == 1:
                off += popp[p - 1] * popq[q - 1]
            elif p < q:
                off += popp[p - 1] * popq[q - 1]
            elif p == q:
                off += popp[p - 1] * (popp[q - 1] + (1 if iop == 2 else -1)) // 2
        return int(off)
