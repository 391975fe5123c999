"""CPU verification of the narrow-output contraction plans (no GPU needed).

For every engine call of the 22 kernels whose output block has at most 16
columns (or rows), the work items of the narrow kernels
(cpsd_debug_narrow_plan) are executed in numpy with the kernels' index
arithmetic over the planner's task / segment tables: every operand read
and output write is bounds-checked, each output element is produced by
exactly one item (or one fixed-order reduction of K-split items that
partition the task's contracted range), and the result is compared with
the CPU oracle."""
import ctypes

import numpy as np
import pytest

import kernel_specs as ks
import oracle_ffi as of
from cpsd_b200 import api, synth
from test_plan_emulation import KSPEC, to_engine, norm, I64, get_plan, decode

COLS = 8  # short-K items: 32 rows x 8 columns


class NarrowItem(ctypes.Structure):
    _fields_ = [("task", ctypes.c_int), ("c0", ctypes.c_int), ("r0", I64), ("k0", I64), ("k1", I64), ("part", I64)]


class NarrowRed(ctypes.Structure):
    _fields_ = [("task", ctypes.c_int), ("c0", ctypes.c_int), ("nparts", ctypes.c_int), ("pad", ctypes.c_int),
                ("r0", I64), ("part0", I64)]


def get_narrow(o1, t1, o2, t2, o3, t3, nb, sA, sB, sC):
    it, ni, rd, nr = ctypes.c_void_p(), I64(), ctypes.c_void_p(), I64()
    flags = (I64 * 5)()
    api.check(api.lib().cpsd_debug_narrow_plan(ctypes.byref(o1), t1.encode(), ctypes.byref(o2), t2.encode(),
                                               ctypes.byref(o3), t3.encode(), I64(nb), I64(sA), I64(sB), I64(sC),
                                               ctypes.byref(it), ctypes.byref(ni), ctypes.byref(rd), ctypes.byref(nr),
                                               flags), "narrow plan")
    if not flags[0]:
        return None
    items = list((NarrowItem * ni.value).from_address(it.value)) if ni.value else []
    reds = list((NarrowRed * nr.value).from_address(rd.value)) if nr.value else []
    return dict(items=items, reds=reds, swap=bool(flags[1]), longk=bool(flags[2]), nparts=flags[3], kc=int(flags[4]))


def emulate(tasks, segs, plan, A, B, C, alpha):
    C = C.copy()
    swap = plan["swap"]
    X, Y = (B, A) if swap else (A, B)
    # long K: items of 32 / kc rows x kc columns; short K: 32 rows x 8 columns
    kc = plan.get("kc", COLS) if plan["longk"] else COLS
    assert kc in (4, 5, 6, 8)
    krows = 32 // kc
    partial = np.full((plan["nparts"], krows, kc), np.nan)
    written = set()

    def views(tk):
        if swap:
            return tk.N, tk.M, (tk.nn, tk.nExt, tk.nSC), (tk.nm, tk.mExt, tk.mSC)
        return tk.M, tk.N, (tk.nm, tk.mExt, tk.mSC), (tk.nn, tk.nExt, tk.nSC)

    def block(tk, r0, nrow, c0, ncol, k0, k1):
        acc = np.zeros((nrow, ncol))
        for si in range(tk.nseg):
            sg = segs[tk.seg0 + si]
            kb, ke = max(k0 - sg.kstart, 0), min(k1 - sg.kstart, sg.K)
            if kb >= ke:
                continue
            r = np.arange(r0, r0 + nrow)
            c = np.arange(c0, c0 + ncol)
            k = np.arange(kb, ke)
            if swap:
                ox = sg.baseB + decode(r, tk.nExt[:tk.nn], sg.nSB[:tk.nn])
                oy = sg.baseA + decode(c, tk.mExt[:tk.nm], sg.mSA[:tk.nm])
                kx, ky = sg.kSB, sg.kSA
            else:
                ox = sg.baseA + decode(r, tk.mExt[:tk.nm], sg.mSA[:tk.nm])
                oy = sg.baseB + decode(c, tk.nExt[:tk.nn], sg.nSB[:tk.nn])
                kx, ky = sg.kSA, sg.kSB
            fx = decode(k, sg.kExt[:sg.nk], kx[:sg.nk])
            fy = decode(k, sg.kExt[:sg.nk], ky[:sg.nk])
            ix, iy = ox[:, None] + fx[None, :], oy[:, None] + fy[None, :]
            assert ix.min() >= 0 and ix.max() < X.size, "row operand read out of bounds"
            assert iy.min() >= 0 and iy.max() < Y.size, "column operand read out of bounds"
            acc += X[ix] @ Y[iy].T
        return acc

    def store(tk, r0, nrow, c0, ncol, val):
        _, _, rv, cv = views(tk)
        r = np.arange(r0, r0 + nrow)
        c = np.arange(c0, c0 + ncol)
        addr = tk.baseC + decode(r, rv[1][:rv[0]], rv[2][:rv[0]])[:, None] + \
            decode(c, cv[1][:cv[0]], cv[2][:cv[0]])[None, :]
        assert addr.min() >= 0 and addr.max() < C.size, "output out of bounds"
        flat = addr.ravel().tolist()
        assert not (written & set(flat)) and len(set(flat)) == len(flat), "output written twice"
        written.update(flat)
        C[addr.ravel()] += alpha * val.ravel()

    for it in plan["items"]:
        tk = tasks[it.task]
        R, CN, _, _ = views(tk)
        nrow = min(krows if plan["longk"] else 32, R - it.r0)
        ncol = min(kc, CN - it.c0)
        assert nrow > 0 and ncol > 0 and 0 <= it.k0 <= it.k1 <= tk.Ktot
        val = block(tk, it.r0, nrow, it.c0, ncol, it.k0, it.k1)
        if it.part >= 0:
            assert plan["longk"] and np.isnan(partial[it.part]).all()
            partial[it.part] = 0.0
            partial[it.part, :nrow, :ncol] = val
        else:
            assert it.k0 == 0 and it.k1 == tk.Ktot
            store(tk, it.r0, nrow, it.c0, ncol, val)
    for rd in plan["reds"]:
        tk = tasks[rd.task]
        R, CN, _, _ = views(tk)
        nrow, ncol = min(krows, R - rd.r0), min(kc, CN - rd.c0)
        parts = [it for it in plan["items"] if it.part >= rd.part0 and it.part < rd.part0 + rd.nparts]
        assert len(parts) == rd.nparts and all(p.task == rd.task and p.r0 == rd.r0 and p.c0 == rd.c0 for p in parts)
        ranges = sorted((p.k0, p.k1) for p in parts)
        assert ranges[0][0] == 0 and ranges[-1][1] == tk.Ktot and all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
        val = sum(partial[rd.part0 + q] for q in range(rd.nparts))[:nrow, :ncol]
        store(tk, rd.r0, nrow, rd.c0, ncol, val)
    return C, written


@pytest.mark.parametrize("nirrep", [1, 4, 8])
@pytest.mark.parametrize("name", sorted(KSPEC))
@pytest.mark.parametrize("nb", [1, 3])
def test_kernel_narrow_plans(name, nirrep, nb):
    check_kernel(name, nirrep, nb, 16 if nirrep < 8 else 24)


@pytest.mark.parametrize("name", ["c1_r2abci", "Fmi_r2abij", "c1_r2ijka"])
def test_long_k_split_plans(name):
    """contracted ranges long enough for the K split and its reduction"""
    plan = check_kernel(name, 1, 2, 40)
    assert plan["longk"] and plan["nparts"] > 0 and plan["reds"]


def check_kernel(name, nirrep, nb, nmo):
    s = synth.System(nmo=nmo, nocc_a=3, nocc_b=2, nirrep=nirrep, seed=2)
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
    rng = np.random.default_rng(3)
    n1 = nb if ba and nb > 1 else 1
    n2 = nb if bb and nb > 1 else 1
    A = rng.standard_normal(l1 * n1)
    B = rng.standard_normal(l2 * n2)
    C = rng.standard_normal(l3 * nb)
    o = [api.Opt() for _ in range(3)]
    for oo, p, i, y in ((o[0], p1, j1, y1), (o[1], p2, j2, y2), (o[2], po, j3, so)):
        api.check(api.lib().cpsd_opt_init(ctypes.byref(oo), api.arr8(p[0]), api.arr8(p[1]), api.arr8(p[2]),
                                           api.arr8(p[3]), I64(i[0]), I64(i[1]), I64(y), None), "opt")
    args = (o[0], e1, o[1], e2, o[2], e3, nb, l1 if n1 > 1 else 0, l2 if n2 > 1 else 0, l3 if nb > 1 else 0)
    plan = get_narrow(*args)
    if plan is None:
        pytest.skip("output side wider than 16: tensor-core tiles")
    tasks, segs, _, _ = get_plan(*args)
    out, written = emulate(tasks, segs, plan, A, B, C, 0.9)
    assert len(written) == sum(t.M * t.N for t in tasks)
    for c in range(nb):
        ref = C[c * l3:(c + 1) * l3].copy()
        Ac = A[c * l1:(c + 1) * l1] if n1 > 1 else A
        Bc = B[c * l2:(c + 1) * l2] if n2 > 1 else B
        rc = of.vv2v_dpd(Ac, of.desc(p1, j1, y1), e1, Bc, of.desc(p2, j2, y2), e2, ref, of.desc(po, j3, so), e3, 0.9,
                         1.0)
        assert rc == 0
        np.testing.assert_allclose(out[c * l3:(c + 1) * l3], ref, rtol=0, atol=1e-11)
    return plan
