"""CPU verification of the GPU planner (no GPU needed).

The grouped-GEMM tables the library's planner builds (cpsd_debug_contract_plan)
are executed here in numpy with exactly the kernel's index arithmetic
(mixed-radix decode of M/N/K, first index fastest), every gather / scatter
offset is bounds-checked, the tiles are checked to cover each task once,
and the result is compared with the CPU oracle.  Covered: every engine call
the 22 lib_cc kernels issue (after the wrappers' pair expansion), batched
and unbatched, nirrep 1, 4 and 8; and the pair-map tables of the layout
transforms."""
import ctypes

import numpy as np
import pytest

import kernel_specs as ks
import oracle_ffi as of
from cpsd_b200 import api, synth

I64 = ctypes.c_int64
MAXU = 4


class TaskDev(ctypes.Structure):
    _fields_ = [("M", I64), ("N", I64), ("baseC", I64), ("Ktot", I64), ("mExt", I64 * MAXU), ("mSC", I64 * MAXU),
                ("nExt", I64 * MAXU), ("nSC", I64 * MAXU), ("nm", ctypes.c_int), ("nn", ctypes.c_int),
                ("seg0", ctypes.c_int), ("nseg", ctypes.c_int)]


class SegDev(ctypes.Structure):
    _fields_ = [("baseA", I64), ("baseB", I64), ("K", I64), ("kstart", I64), ("mSA", I64 * MAXU),
                ("nSB", I64 * MAXU), ("kExt", I64 * MAXU), ("kSA", I64 * MAXU), ("kSB", I64 * MAXU),
                ("nk", ctypes.c_int), ("aMfast", ctypes.c_int), ("bKfast", ctypes.c_int), ("pad", ctypes.c_int)]


class TileDev(ctypes.Structure):
    _fields_ = [("task", ctypes.c_int), ("mt", ctypes.c_int), ("nt", ctypes.c_int), ("nsplit", ctypes.c_int),
                ("k_lo", I64), ("k_hi", I64), ("part", I64)]


class PMBlockDev(ctypes.Structure):
    _fields_ = [(k, I64) for k in ("outBase", "nlo", "nro", "inBase", "nli", "lmap", "rmap", "start")]


def decode(x, ext, st):
    off = np.zeros_like(x)
    for e, s in zip(ext, st):
        off += (x % e) * s
        x = x // e
    return off


def get_plan(o1, t1, o2, t2, o3, t3, nb=1, sA=0, sB=0, sC=0):
    P = [ctypes.c_void_p() for _ in range(3)]
    N = [I64() for _ in range(3)]
    bm, bn = I64(), I64()
    rc = api.lib().cpsd_debug_contract_plan(ctypes.byref(o1), t1.encode(), ctypes.byref(o2), t2.encode(),
                                            ctypes.byref(o3), t3.encode(), I64(nb), I64(sA), I64(sB), I64(sC),
                                            ctypes.byref(P[0]), ctypes.byref(N[0]), ctypes.byref(P[1]),
                                            ctypes.byref(N[1]), ctypes.byref(P[2]), ctypes.byref(N[2]),
                                            ctypes.byref(bm), ctypes.byref(bn))
    api.check(rc, "plan")
    tasks = (TaskDev * N[0].value).from_address(P[0].value) if N[0].value else []
    segs = (SegDev * N[1].value).from_address(P[1].value) if N[1].value else []
    tiles = (TileDev * N[2].value).from_address(P[2].value) if N[2].value else []
    return tasks, segs, tiles, (bm.value, bn.value)


def emulate(tasks, segs, tiles, A, B, C, alpha, tile=(64, 64)):
    """C += alpha * contraction, exactly as k_contract indexes; bounds-checked."""
    C = C.copy()
    for ti, tk in enumerate(tasks):
        m = np.arange(tk.M)
        n = np.arange(tk.N)
        offMC = decode(m, tk.mExt[:tk.nm], tk.mSC[:tk.nm])
        offNC = decode(n, tk.nExt[:tk.nn], tk.nSC[:tk.nn])
        cidx = tk.baseC + offMC[:, None] + offNC[None, :]
        assert cidx.min() >= 0 and cidx.max() < C.size, "C out of bounds"
        assert len(np.unique(cidx)) == cidx.size, "C elements written twice within a task"
        acc = np.zeros((tk.M, tk.N))
        ksum = 0
        for s in segs[tk.seg0:tk.seg0 + tk.nseg]:
            k = np.arange(s.K)
            offMA = s.baseA + decode(m, tk.mExt[:tk.nm], s.mSA[:tk.nm])
            offNB = s.baseB + decode(n, tk.nExt[:tk.nn], s.nSB[:tk.nn])
            offKA = decode(k, s.kExt[:s.nk], s.kSA[:s.nk])
            offKB = decode(k, s.kExt[:s.nk], s.kSB[:s.nk])
            ai = offMA[:, None] + offKA[None, :]
            bi = offKB[:, None] + offNB[None, :]
            assert ai.min() >= 0 and ai.max() < A.size, "A out of bounds"
            assert bi.min() >= 0 and bi.max() < B.size, "B out of bounds"
            assert s.kstart == ksum
            ksum += s.K
            acc += A[ai] @ B[bi]
        assert ksum == tk.Ktot
        C[cidx] += alpha * acc
    # tiles: every (task, m-tile, n-tile) covers K exactly once
    cover = {}
    for t in tiles:
        cover.setdefault((t.task, t.mt, t.nt), []).append((t.k_lo, t.k_hi))
    bm, bn = tile
    for ti, tk in enumerate(tasks):
        for a in range((tk.M + bm - 1) // bm):
            for b in range((tk.N + bn - 1) // bn):
                r = sorted(cover.pop((ti, a, b)))
                assert r[0][0] == 0 and r[-1][1] == tk.Ktot
                for (x0, x1), (y0, y1) in zip(r, r[1:]):
                    assert x1 == y0
    assert not cover
    return C


def flat(pairs):
    return [all(p != q for j, q in enumerate(pairs) if j != i) for i, p in enumerate(pairs)]


def engine_calls(name):
    """(wrapper args) of the kernel -> the engine-level (t1, t2, t3, exp flags)."""
    return KSPEC[name]


# kernel -> (wrapper, order, t1, t2, t3, anti): order 'ba' = wrapper(b, a, out), 'ab' = wrapper(a, b, out)
KSPEC = {
    "c1_r1iabj": ("422", "ba", "fnai", "fn", "ai", 0), "c1_r1Fae": ("222", "ba", "ae", "ei", "ai", 0),
    "c1_r1Fmi": ("222", "ab", "am", "mi", "ai", 0), "c1_r2abci": ("442", "ba", "feam", "feim", "ai", 0),
    "c1_r2ijka": ("442", "ab", "aemn", "mnie", "ai", 0), "c2_r1abci": ("424", "ba", "abej", "ei", "abij", 2),
    "c2_r1ijka": ("424", "ba", "ijmb", "am", "abij", 1), "c2_r2Wmbej": ("444", "ab", "aeim", "embj", "abij", 3),
    "c2_r2Wmnij": ("444", "ab", "abmn", "mnij", "abij", 0), "c2_r2abcd": ("444", "ba", "abef", "efij", "abij", 0),
    "c2_r2Fae": ("424", "ab", "aeij", "be", "abij", 1), "c2_r2Fmi": ("424", "ab", "abim", "mj", "abij", 2),
    "Fmi_r2abij": ("442", "ba", "efmn", "efin", "mi", 0), "Fae_r2abij": ("442", "ab", "afmn", "efmn", "ae", 0),
    "Fmi_r1ijka": ("422", "ba", "mnie", "en", "mi", 0), "Fae_r1abci": ("422", "ba", "efam", "fm", "ae", 0),
    "Wkbij_r2ijka": ("444", "ba", "klic", "bcjl", "ijkb", 1),
    "Wmbej_r2abij": ("444", "ba", "fenm", "bfjn", "embj", 0),
    "Wmbej_r1abci": ("424", "ba", "febm", "fj", "embj", 0), "Wmbej_r1ijka": ("424", "ba", "nmje", "bn", "embj", 0),
    "Wmnij_r1ijka": ("424", "ba", "mnie", "ej", "mnij", 2),
    "Wmnij_r2abij": ("444", "ba", "efmn", "efij", "mnij", 0),
    "Wkbij_r1iabj": ("424", "ba", "ckbj", "ci", "ijkb", 1), "Wabdj_r1abcd": ("424", "ba", "abdc", "cj", "abdj", 0),
    "Wkbij_r1Uklij": ("424", "ba", "klij", "bl", "ijkb", 0), "Fme_r1abij": ("422", "ba", "efmn", "fn", "em", 0),
    "c1_r2Fme": ("422", "ab", "aeim", "em", "ai", 0),
    "c1d_l1Wibaj": ("422", "ba", "aibj", "bj", "ai", 0),
    "c1d_l1fab": ("222", "ba", "ba", "bi", "ai", 0),
    "c1d_l1fij": ("222", "ab", "aj", "ij", "ai", 0),
    "Fae_r1fia": ("222", "ab", "al", "el", "ae", 0),
    "Fmi_r1fia": ("222", "ba", "dm", "di", "mi", 0),
    "Wkbij_r2Fkc": ("424", "ab", "cbij", "ck", "ijkb", 0),
    "Wlkjd_r1abij": ("424", "ba", "cdlk", "cj", "lkjd", 0),
}


def to_engine(w, t1, t2, t3, i1, i2, i3):
    """wrapper-level types and iops -> engine types and the iops after expansion"""
    if w == "422":
        w, t2, t3 = "444", t2 + "+-", t3 + "+-"
    if w == "222":
        w, t1, t2, t3 = "444", t1 + "=+", t2 + "=-", t3 + "+-"
    if w == "444":
        pairs = [t1[:2], t1[2:], t2[:2], t2[2:], t3[:2], t3[2:]]
        f = flat(pairs)
        io = [i1[0], i1[1], i2[0], i2[1], i3[0], i3[1]]
        io = [1 if (f[k] and io[k] != 1) else io[k] for k in range(6)]
        return t1, t2, t3, (io[0], io[1]), (io[2], io[3]), (io[4], io[5])
    if w == "424":
        pairs = [t1[:2], t1[2:], t3[:2], t3[2:]]
        f = flat(pairs)
        io = [i1[0], i1[1], i3[0], i3[1]]
        io = [1 if (f[k] and io[k] != 1) else io[k] for k in range(4)]
        return t1, t2 + "..", t3, (io[0], io[1]), i2, (io[2], io[3])
    if w == "442":
        pairs = [t1[:2], t1[2:], t2[:2], t2[2:]]
        f = flat(pairs)
        io = [i1[0], i1[1], i2[0], i2[1]]
        io = [1 if (f[k] and io[k] != 1) else io[k] for k in range(4)]
        return t1, t2, t3 + "..", (io[0], io[1]), (io[2], io[3]), i3
    raise AssertionError(w)


def norm(t):
    return "".join("." if c in "+-=" else c for c in t)


@pytest.mark.parametrize("nirrep", [1, 4, 8])
@pytest.mark.parametrize("name", sorted(KSPEC))
@pytest.mark.parametrize("nb", [1, 3])
def test_kernel_engine_plans(name, nirrep, nb):
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
    # wrapper operands in call order
    if order == "ab":
        (p1, i1, y1, ba), (p2, i2, y2, bb) = (pa, ia, sa, True), (pb, ib, sb, False)
    else:
        (p1, i1, y1, ba), (p2, i2, y2, bb) = (pb, ib, sb, False), (pa, ia, sa, True)
    e1, e2, e3, j1, j2, j3 = to_engine(w, t1, t2, t3, i1, i2, io)
    if len(e2) == 2:
        e2 = e2 + ".."
    if len(e3) == 2:
        e3 = e3 + ".."
    e1, e2, e3 = norm(e1), norm(e2), norm(e3)
    if w in ("424",) and len(t2) == 2:
        p2 = [p2[0], p2[1], p2[2], p2[3]]
    l1 = sym.idsymsoc(y1, p1[0], p1[1], j1[0], p1[2], p1[3], j1[1])
    l2 = sym.idsymsoc(y2, p2[0], p2[1], j2[0], p2[2], p2[3], j2[1])
    l3 = sym.idsymsoc(so, po[0], po[1], j3[0], po[2], po[3], j3[1])
    rng = np.random.default_rng(7)
    n1 = nb if ba and nb > 1 else 1
    n2 = nb if bb and nb > 1 else 1
    A = rng.standard_normal(l1 * n1)
    B = rng.standard_normal(l2 * n2)
    C = rng.standard_normal(l3 * nb)
    z = np.zeros(1)
    o1 = api.Opt(); o2 = api.Opt(); o3 = api.Opt()
    for o, p, i, y in ((o1, p1, j1, y1), (o2, p2, j2, y2), (o3, po, j3, so)):
        api.check(api.lib().cpsd_opt_init(ctypes.byref(o), api.arr8(p[0]), api.arr8(p[1]), api.arr8(p[2]),
                                           api.arr8(p[3]), I64(i[0]), I64(i[1]), I64(y), None), "opt")
    tasks, segs, tiles, tile = get_plan(o1, e1, o2, e2, o3, e3, nb, l1 if n1 > 1 else 0, l2 if n2 > 1 else 0,
                                        l3 if nb > 1 else 0)
    assert tile in ((128, 64), (128, 32), (64, 128), (64, 64))
    out = emulate(tasks, segs, tiles, A, B, C, 0.9, tile)
    for c in range(nb):
        ref = C[c * l3:(c + 1) * l3].copy()
        Ac = A[c * l1:(c + 1) * l1] if n1 > 1 else A
        Bc = B[c * l2:(c + 1) * l2] if n2 > 1 else B
        rc = of.vv2v_dpd(Ac, of.desc(p1, j1, y1), e1, Bc, of.desc(p2, j2, y2), e2, ref, of.desc(po, j3, so), e3, 0.9,
                         1.0)
        assert rc == 0
        np.testing.assert_allclose(out[c * l3:(c + 1) * l3], ref, rtol=0, atol=1e-12)


@pytest.mark.parametrize("nirrep", [1, 4, 8])
def test_pairmap_plans_in_bounds_and_match_oracle(nirrep):
    s = synth.System(nmo=16 if nirrep < 8 else 24, nocc_a=3, nocc_b=2, nirrep=nirrep, seed=2)
    api.init(s.nirrep, s.dirprd)
    of.set_symmetry(s.nirrep, s.dirprd)
    sym, o, v = s.sym, s.popo, s.popv
    rng = np.random.default_rng(1)
    cases = [  # (pops, iops, sym, op0, op1, t0, t1)
        ([v, v, o, o], (0, 0), 2 if nirrep > 1 else 1, 1, 1, 1, 1),    # expand both
        ([v, v, o, o], (0, 1), 1, 1, 0, 1, 1),                          # expand pq
        ([v, v, o, o], (1, 1), 1, 4, 4, 0, 0),                          # anti+compress both
        ([v, v, o, o], (1, 1), 1, 3, 0, 1, 1),                          # anti pq (full)
        ([o, o, v, o], (0, 1), 1, 0, 5, 1, 1),                          # swap rs
        ([v, v, o, o], (1, 1), 1, 2, 0, 0, 1),                          # compress pq
    ]
    for pops, iops, y, op0, op1, t0, t1 in cases:
        oin = api.Opt()
        api.check(api.lib().cpsd_opt_init(ctypes.byref(oin), *[api.arr8(p) for p in pops], I64(iops[0]),
                                          I64(iops[1]), I64(y), None), "opt")
        P = [ctypes.c_void_p() for _ in range(3)]
        nbk, nidx, lt, rt = I64(), I64(), I64(), I64()
        api.check(api.lib().cpsd_debug_pairmap_plan(ctypes.byref(oin), I64(op0), I64(op1), I64(t0), I64(t1),
                                                    ctypes.byref(P[0]), ctypes.byref(nbk), ctypes.byref(P[1]),
                                                    ctypes.byref(P[2]), ctypes.byref(nidx), ctypes.byref(lt),
                                                    ctypes.byref(rt)), "pairmap plan")
        blocks = (PMBlockDev * nbk.value).from_address(P[0].value)
        idx = np.ctypeslib.as_array((ctypes.c_longlong * nidx.value).from_address(P[1].value))
        sgn = np.ctypeslib.as_array((ctypes.c_double * nidx.value).from_address(P[2].value))
        lin = sym.idsymsoc(y, pops[0], pops[1], iops[0], pops[2], pops[3], iops[1])
        x = rng.standard_normal(lin)
        # output descriptor
        pout = list(pops)
        iout = list(iops)
        for k, op, t in ((0, op0, t0), (1, op1, t1)):
            if op == 1:
                iout[k] = 1
            if op in (2, 4):
                iout[k] = t
            if op == 5:
                pout[2 * k], pout[2 * k + 1] = pout[2 * k + 1], pout[2 * k]
        lout = sym.idsymsoc(y, pout[0], pout[1], iout[0], pout[2], pout[3], iout[1])
        out = np.zeros(lout)
        for b in blocks:
            for r in range(b.nro):
                for l in range(b.nlo):
                    val = 0.0
                    for tr in range(rt.value):
                        ri = idx[b.rmap + r * rt.value + tr]
                        if ri < 0:
                            continue
                        for tq in range(lt.value):
                            li = idx[b.lmap + l * lt.value + tq]
                            if li < 0:
                                continue
                            assert 0 <= li < b.nli
                            p = b.inBase + ri * b.nli + li
                            assert 0 <= p < lin
                            val += sgn[b.rmap + r * rt.value + tr] * sgn[b.lmap + l * lt.value + tq] * x[p]
                    q = b.outBase + r * b.nlo + l
                    assert 0 <= q < lout
                    out[q] = val
        # oracle equivalent
        din = of.desc(pops, iops, y)
        ref = np.zeros(lout)
        lib = of.lib()
        if op0 == 1 or op1 == 1:
            lib.o_iexpso(of.ptr(x), of.ptr(ref), ctypes.byref(din), I64(op0 == 1), I64(op1 == 1))
        elif op1 == 5:
            lib.o_isymtrso(of.ptr(x), of.ptr(ref), ctypes.byref(din), I64(0), I64(1))
        elif op0 == 2:
            lib.o_icompso(of.ptr(x), of.ptr(ref), ctypes.byref(din), I64(t0), I64(1))
        elif op0 == 3:
            sw = np.zeros(lin)
            lib.o_isymtrso(of.ptr(x), of.ptr(sw), ctypes.byref(din), I64(1), I64(0))
            ref = x - sw
        else:  # anti + compress both pairs
            sw = np.zeros(lin)
            lib.o_isymtrso(of.ptr(x), of.ptr(sw), ctypes.byref(din), I64(1), I64(0))
            y1 = x - sw
            sw2 = np.zeros(lin)
            lib.o_isymtrso(of.ptr(y1), of.ptr(sw2), ctypes.byref(din), I64(0), I64(1))
            y2 = y1 - sw2
            lib.o_icompso(of.ptr(y2), of.ptr(ref), ctypes.byref(din), I64(0), I64(0))
        np.testing.assert_allclose(out, ref, rtol=0, atol=1e-13)
