"""CPU verification of the sliced-integer (int8 digit) contraction plans.

The gather / scatter tables and the digit-buffer layout that the library
builds for the tensor-core digit path (cpsd_debug_ozaki_plan) are executed
here in numpy with the kernels' arithmetic: per-row / per-column power-of-two
scales from frexp, truncated 7-bit digits, exact integer diagonal sums
(checked against the int32 range per K chunk) and the FP64 combination of
the diagonals.  Every source read, digit tile, exponent and output address
is bounds-checked, output addresses are checked to be written once, and the
result is compared with the CPU oracle within the method's error bound
(digits + 1) K 128^-digits max|a_row| max|b_col|."""
import ctypes

import numpy as np
import pytest

import kernel_specs as ks
import oracle_ffi as of
from cpsd_b200 import api, synth
from test_plan_emulation import KSPEC, to_engine, norm, I64

BK = 64


class OzGroup(ctypes.Structure):
    _fields_ = [("M", I64), ("N", I64), ("K", I64), ("KT", ctypes.c_int), ("nI", ctypes.c_int),
                ("nL", ctypes.c_int)] + [(k, I64) for k in ("aoff", "boff", "eaoff", "eboff", "moff", "noff",
                                                             "crowoff", "ccoloff")]


class OzTile(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int) for k in ("g", "mt", "nt", "pad")]


class OzSliceJob(ctypes.Structure):
    _fields_ = [("R", I64), ("K", I64)] + [(k, ctypes.c_int) for k in ("KT", "rt", "nJ", "nI")] + \
               [(k, I64) for k in ("roff", "koff", "rcoff", "kcoff", "eoff", "doff")] + \
               [("affine", ctypes.c_int), ("rc", ctypes.c_int), ("sr", I64), ("soff", I64)]


class OzStage(ctypes.Structure):
    _fields_ = [("ko0", I64), ("sk", I64), ("j", ctypes.c_int), ("ok", ctypes.c_int)]


def get_oz_plan(o1, t1, o2, t2, o3, t3, nb, sA, sB, sC, digits):
    tabs = (ctypes.c_void_p * 22)()
    sizes = (I64 * 22)()
    api.check(api.lib().cpsd_debug_ozaki_plan(ctypes.byref(o1), t1.encode(), ctypes.byref(o2), t2.encode(),
                                              ctypes.byref(o3), t3.encode(), I64(nb), I64(sA), I64(sB), I64(sC),
                                              ctypes.c_int(digits), tabs, sizes), "ozaki plan")
    if not tabs[0]:
        return None
    n = [sizes[i] for i in range(22)]

    def arr(i, ct):
        return np.ctypeslib.as_array((ct * n[i]).from_address(tabs[i])).copy() if n[i] else np.zeros(0, np.int64)

    return dict(groups=list((OzGroup * n[0]).from_address(tabs[0])), tiles=list((OzTile * n[1]).from_address(tabs[1])),
                ajobs=list((OzSliceJob * n[2]).from_address(tabs[2])) if n[2] else [],
                bjobs=list((OzSliceJob * n[3]).from_address(tabs[3])) if n[3] else [],
                aroff=arr(4, I64), akoff=arr(5, I64), broff=arr(6, I64), bkoff=arr(7, I64), crow=arr(8, I64),
                ccol=arr(9, I64), mcombo=arr(10, ctypes.c_int), ncombo=arr(11, ctypes.c_int),
                kcombo=arr(12, ctypes.c_int), adig=n[13], bdig=n[14], nea=n[15], neb=n[16], kt_chunk=n[17],
                kt_max=n[18], BN=n[19],
                astage=list((OzStage * n[20]).from_address(tabs[20])) if n[20] else [],
                bstage=list((OzStage * n[21]).from_address(tabs[21])) if n[21] else [])


def digits_of(X, S):
    """rows of X -> exponents e (|x| < 2^e) and S truncated 7-bit digits"""
    _, ex = np.frexp(X)
    ex = np.where(X != 0, ex, -100000)
    e = ex.max(axis=1) if X.shape[1] else np.zeros(X.shape[0], int)
    e = np.where(e == -100000, 0, e)
    y = X * np.ldexp(1.0, -e)[:, None]
    q = []
    for _ in range(S):
        y = y * 128.0
        d = np.trunc(y)
        y = y - d
        assert np.abs(d).max(initial=0) <= 127
        q.append(d.astype(np.int64))
    return e, q


def check_affine(plan, jb, stage, roff, koff, rcombo, RT):
    """the kernels' affine gather of an affine job and stage (base + row and
    column steps) must read exactly the table address of every element"""
    r0, r1 = jb.rt * RT, min(jb.R, (jb.rt + 1) * RT)
    r = np.arange(r0, r1)[:, None]
    assert (rcombo[jb.rcoff + r] == jb.rc).all()
    n_fast = 0
    for kt in range(jb.KT):
        st = stage[jb.soff + kt * jb.nI + jb.rc]
        if not st.ok:
            continue
        n_fast += 1
        k = np.arange(kt * BK, min(jb.K, (kt + 1) * BK))[None, :]
        kc = plan["kcombo"][jb.kcoff + k]
        idx = roff[jb.roff + r * jb.nJ + kc] + koff[jb.koff + k * jb.nI + jb.rc]
        fast = roff[jb.roff + r0 * jb.nJ + st.j] + st.ko0 + (r - r0) * jb.sr + (k - kt * BK) * st.sk
        assert (fast == idx).all(), "affine gather differs from the tables"
    return n_fast


def side(plan, jobs, roff, koff, rcombo, src, S, RT, total_bytes, nexp, stage=None):
    """gather one operand side per group (bounds-checked) -> {doff: (e, digits)}"""
    out = {}
    for jb in jobs:
        assert jb.doff + (jb.rt * jb.KT + jb.KT) * S * RT * BK <= total_bytes
        assert jb.eoff + min(jb.R, (jb.rt + 1) * RT) <= nexp
        if stage is not None and jb.affine:
            check_affine(plan, jb, stage, roff, koff, rcombo, RT)
        if jb.rt:
            continue
        R, K = jb.R, jb.K
        r = np.arange(R)[:, None]
        k = np.arange(K)[None, :]
        kc = plan["kcombo"][jb.kcoff + k]
        rc = rcombo[jb.rcoff + r]
        idx = roff[jb.roff + r * jb.nJ + kc] + koff[jb.koff + k * jb.nI + rc]
        assert idx.min(initial=0) >= 0 and idx.max(initial=0) < src.size, "source read out of bounds"
        out[jb.doff] = digits_of(src[idx], S)
    return out


def emulate(plan, A, B, C, alpha, S):
    C = C.copy()
    BN = plan["BN"]
    adig = side(plan, plan["ajobs"], plan["aroff"], plan["akoff"], plan["mcombo"], A, S, 128, plan["adig"],
                plan["nea"], plan["astage"])
    bdig = side(plan, plan["bjobs"], plan["broff"], plan["bkoff"], plan["ncombo"], B, S, BN, plan["bdig"],
                plan["neb"], plan["bstage"])
    for t in plan["tiles"]:
        g = plan["groups"][t.g]
        assert g.aoff + (t.mt * g.KT + g.KT) * S * 128 * BK <= plan["adig"]
        assert g.boff + (t.nt * g.KT + g.KT) * S * BN * BK <= plan["bdig"]
    written = set()
    kchunk = plan["kt_chunk"] * BK
    for gi, g in enumerate(plan["groups"]):
        ea, qa = adig[g.aoff]
        eb, qb = bdig[g.boff]
        val = np.zeros((g.M, g.N))
        for k0 in range(0, max(g.K, 1), kchunk):
            ks_ = slice(k0, min(k0 + kchunk, g.K))
            for d in range(S):
                acc = np.zeros((g.M, g.N), np.int64)
                for tt in range(d + 1):
                    acc += qa[tt][:, ks_] @ qb[d - tt][:, ks_].T
                assert np.abs(acc).max(initial=0) < 2 ** 31, "int32 accumulator overflow"
                val += acc * 128.0 ** -(d + 2)
        val = np.ldexp(val, ea[:, None] + eb[None, :])
        m = np.arange(g.M)[:, None]
        n = np.arange(g.N)[None, :]
        addr = plan["crow"][g.crowoff + m * g.nL + plan["ncombo"][g.noff + n]] + \
            plan["ccol"][g.ccoloff + n * g.nI + plan["mcombo"][g.moff + m]]
        assert addr.min(initial=0) >= 0 and addr.max(initial=0) < C.size, "C out of bounds"
        flat = addr.ravel().tolist()
        assert len(set(flat)) == len(flat) and not (written & set(flat)), "C element written twice"
        written |= set(flat)
        np.add.at(C, addr.ravel(), alpha * val.ravel())
    return C


@pytest.mark.parametrize("digits", [4, 7])
@pytest.mark.parametrize("nirrep", [1, 4, 8])
@pytest.mark.parametrize("name", sorted(KSPEC))
@pytest.mark.parametrize("nb", [1, 3])
def test_kernel_ozaki_plans(name, nirrep, nb, digits):
    s = synth.System(nmo=16 if nirrep < 8 else 24, nocc_a=3, nocc_b=2, nirrep=nirrep, seed=2)
    api.init(s.nirrep, s.dirprd)
    of.set_symmetry(s.nirrep, s.dirprd)
    sym = s.sym
    w, order, t1, t2, t3, anti = KSPEC[name]
    lo, la, lb = ks.KERNELS[name][:3]
    symR = min(2, nirrep)
    sa, sb = (symR, 1) if not name.startswith("c2_r2") else (1, symR)
    po, io = ks.pops_of(lo, s.popo, s.popv)
    pa, ia = ks.pops_of(la, s.popo, s.popv)
    pb, ib = ks.pops_of(lb, s.popo, s.popv)
    so = sym.dp(sa, sb)
    if order == "ab":
        (p1, i1, y1, ba), (p2, i2, y2, bb) = (pa, ia, sa, True), (pb, ib, sb, False)
    else:
        (p1, i1, y1, ba), (p2, i2, y2, bb) = (pb, ib, sb, False), (pa, ia, sa, True)
    e1, e2, e3, j1, j2, j3 = to_engine(w, t1, t2, t3, i1, i2, io)
    e2 = e2 + ".." if len(e2) == 2 else e2
    e3 = e3 + ".." if len(e3) == 2 else e3
    e1, e2, e3 = norm(e1), norm(e2), norm(e3)
    l1 = sym.idsymsoc(y1, p1[0], p1[1], j1[0], p1[2], p1[3], j1[1])
    l2 = sym.idsymsoc(y2, p2[0], p2[1], j2[0], p2[2], p2[3], j2[1])
    l3 = sym.idsymsoc(so, po[0], po[1], j3[0], po[2], po[3], j3[1])
    rng = np.random.default_rng(11)
    n1 = nb if ba and nb > 1 else 1
    n2 = nb if bb and nb > 1 else 1
    A = rng.standard_normal(l1 * n1) * np.exp(rng.uniform(-3, 3, l1 * n1))
    B = rng.standard_normal(l2 * n2)
    C = rng.standard_normal(l3 * nb)
    o = [api.Opt() for _ in range(3)]
    for oo, p, i, y in ((o[0], p1, j1, y1), (o[1], p2, j2, y2), (o[2], po, j3, so)):
        api.check(api.lib().cpsd_opt_init(ctypes.byref(oo), api.arr8(p[0]), api.arr8(p[1]), api.arr8(p[2]),
                                           api.arr8(p[3]), I64(i[0]), I64(i[1]), I64(y), None), "opt")
    plan = get_oz_plan(o[0], e1, o[1], e2, o[2], e3, nb, l1 if n1 > 1 else 0, l2 if n2 > 1 else 0,
                       l3 if nb > 1 else 0, digits)
    if plan is None:
        pytest.skip("contraction does not regroup into dense GEMMs")
    if name == "c2_r2abcd":
        # the particle-particle ladder streams the largest operand, (ab|cd):
        # every row tile and K stage of that side must take the table-free
        # gather (the amplitude side's tiles may straddle batch copies)
        big = max(((plan["ajobs"], plan["astage"]), (plan["bjobs"], plan["bstage"])),
                  key=lambda js: sum(jb.R * jb.K for jb in js[0] if jb.rt == 0))
        jobs, stage = big
        assert all(jb.affine for jb in jobs)
        assert all(stage[jb.soff + kt * jb.nI + jb.rc].ok for jb in jobs for kt in range(jb.KT))
    out = emulate(plan, A, B, C, 0.9, digits)
    kmax = max(g.K for g in plan["groups"])
    bound = (digits + 1) * kmax * 128.0 ** -digits * np.abs(A).max() * np.abs(B).max() * 0.9 * 4 + 1e-12
    for c in range(nb):
        ref = C[c * l3:(c + 1) * l3].copy()
        Ac = A[c * l1:(c + 1) * l1] if n1 > 1 else A
        Bc = B[c * l2:(c + 1) * l2] if n2 > 1 else B
        rc = of.vv2v_dpd(Ac, of.desc(p1, j1, y1), e1, Bc, of.desc(p2, j2, y2), e2, ref, of.desc(po, j3, so), e3, 0.9,
                         1.0)
        assert rc == 0
        np.testing.assert_allclose(out[c * l3:(c + 1) * l3], ref, rtol=0, atol=bound)
