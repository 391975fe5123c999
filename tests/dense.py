"""Independent dense numpy reference for the DPD layout and the spin-orbital
formulas (test infrastructure).

Written from the layout rules (irrep blocks ordered by the right pair's
irrep, column-major, left index fastest, p<q packing within one irrep and
irrep(p) < irrep(q) across irreps) and textbook spin-orbital algebra, with
no code shared with the C oracle.
"""
import numpy as np


def pair_list(sym, popp, popq, iop, irr):
    """Stored (ip, p, iq, q) of the pair space of irrep `irr`, storage order."""
    out = []
    for iq in range(1, sym.nirrep + 1):
        ip = sym.dp(iq, irr)
        if iop != 1 and ip > iq:
            continue
        for q in range(popq[iq - 1]):
            pmax = popp[ip - 1]
            if iop == 0 and ip == iq:
                pmax = q
            for p in range(pmax):
                out.append((ip, p, iq, q))
    return out


def goff(pop):
    o = np.zeros(9, np.int64)
    o[1:] = np.cumsum(pop)
    return o


def dpd_index_lists(sym, pops, iops, tsym):
    """For every stored element: (offset, g0, g1, g2, g3) global indices."""
    offs = [goff(p) for p in pops]
    rows = []
    off = 0
    for R in range(1, sym.nirrep + 1):
        L = sym.dp(R, tsym)
        right = pair_list(sym, pops[2], pops[3], iops[1], R)
        left = pair_list(sym, pops[0], pops[1], iops[0], L)
        for ri, (i2, p2, i3, p3) in enumerate(right):
            g2, g3 = offs[2][i2 - 1] + p2, offs[3][i3 - 1] + p3
            for li, (i0, p0, i1, p1) in enumerate(left):
                rows.append((off + ri * len(left) + li, offs[0][i0 - 1] + p0, offs[1][i1 - 1] + p1, g2, g3))
        off += len(right) * len(left)
    return np.array(rows, dtype=np.int64).reshape(-1, 5), off


def dpd_to_dense(vec, sym, pops, iops, tsym):
    n = [int(np.sum(p)) for p in pops]
    D = np.zeros(n)
    rows, total = dpd_index_lists(sym, pops, iops, tsym)
    assert total == vec.size, (total, vec.size)
    o, a, b, c, d = rows.T
    D[a, b, c, d] = vec[o]
    if iops[0] == 0:
        D[b, a, c, d] = -vec[o]
    if iops[1] == 0:
        D[a, b, d, c] = -vec[o]
    if iops[0] == 0 and iops[1] == 0:
        D[b, a, d, c] = vec[o]
    return D


def dense_to_dpd(D, sym, pops, iops, tsym):
    rows, total = dpd_index_lists(sym, pops, iops, tsym)
    o, a, b, c, d = rows.T
    v = np.zeros(total)
    v[o] = D[a, b, c, d]
    return v


def orbital_irreps(pop):
    return np.concatenate([np.full(int(pop[h]), h + 1) for h in range(8)]).astype(np.int64)


def random_dpd(rng, sym, pops, iops, tsym, antisym=True):
    """Random DPD vector; with antisym the dense form is consistent
    (packed pairs imply antisymmetry)."""
    rows, total = dpd_index_lists(sym, pops, iops, tsym)
    return rng.standard_normal(total)


def spin_orbitals(s):
    """(mo, spin) lists of the spin-free occupied / virtual orbitals."""
    occ, vir = [], []
    for h in range(1, s.nirrep + 1):
        for spin, nocc in ((0, s.nocc_a), (1, s.nocc_b)):
            occ += [(m, spin) for m in range(s.nmo) if s.mo_irrep[m] == h and m < nocc]
        for spin, nocc in ((0, s.nocc_a), (1, s.nocc_b)):
            vir += [(m, spin) for m in range(s.nmo) if s.mo_irrep[m] == h and m >= nocc]
    return occ, vir


def antisym_integrals(s):
    """Dense <pq||rs> blocks over spin-free occ (o) / vir (v) orbitals."""
    eri = np.einsum("Ppq,Prs->pqrs", s.L, s.L)  # (pq|rs)
    occ, vir = spin_orbitals(s)
    so = occ + vir
    mo = np.array([m for m, _ in so])
    sp = np.array([x for _, x in so])
    # <pq|rs> = (pr|qs) d(sp,sr) d(sq,ss)
    phys = eri[np.ix_(mo, mo, mo, mo)].transpose(0, 2, 1, 3)
    d = (sp[:, None] == sp[None, :]).astype(float)
    phys = phys * d[:, None, :, None] * d[None, :, None, :]
    g = phys - phys.transpose(0, 1, 3, 2)
    no = len(occ)
    O, V = slice(0, no), slice(no, len(so))
    eps = np.array([s.eps_a[m] if x == 0 else s.eps_b[m] for m, x in so])
    return g, O, V, eps[O], eps[V]
