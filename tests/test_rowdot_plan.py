"""CPU verification of the row-dot contraction plans (no GPU needed).

For every engine call of the 22 kernels that the engine sends to the
row-dot kernel (a narrow output side whose rows are strided in the row
operand, contiguous along one contracted unit of at most 128, one segment
per task), each warp's run of cpsd_debug_rowdot_plan is executed in numpy
with the kernel's index arithmetic: column operand at k * stride, row
operand at row offset + k, outputs (row, column) for columns below the
item's count; reads and writes are bounds-checked, every output element is
written once, and the result is compared with the CPU oracle."""
import ctypes

import numpy as np
import pytest

import kernel_specs as ks
import oracle_ffi as of
from cpsd_b200 import api, synth
from test_narrow_plan import get_narrow
from test_plan_emulation import KSPEC, to_engine, norm, I64, get_plan, decode, TaskDev, SegDev


class RowDotItem(ctypes.Structure):
    _fields_ = [("task", ctypes.c_int), ("seg", ctypes.c_int), ("c0", ctypes.c_int), ("ncol", ctypes.c_int),
                ("r0", I64), ("r1", I64)]


def get_rowdot(o1, t1, o2, t2, o3, t3, nb, sA, sB, sC, ntasks, nsegs):
    it, ni, tp, sp = ctypes.c_void_p(), I64(), ctypes.c_void_p(), ctypes.c_void_p()
    flags = (I64 * 4)()
    api.check(api.lib().cpsd_debug_rowdot_plan(ctypes.byref(o1), t1.encode(), ctypes.byref(o2), t2.encode(),
                                               ctypes.byref(o3), t3.encode(), I64(nb), I64(sA), I64(sB), I64(sC),
                                               ctypes.byref(it), ctypes.byref(ni), ctypes.byref(tp),
                                               ctypes.byref(sp), flags), "row-dot plan")
    if not flags[0]:
        return None
    items = list((RowDotItem * ni.value).from_address(it.value)) if ni.value else []
    tasks = list((TaskDev * ntasks).from_address(tp.value))
    segs = list((SegDev * nsegs).from_address(sp.value))
    return dict(items=items, swap=bool(flags[1]), kq=int(flags[2]), nc=int(flags[3]), tasks=tasks, segs=segs)


def emulate(tasks, segs, plan, A, B, C, alpha):
    C = C.copy()
    swap = plan["swap"]
    X, Y = (B, A) if swap else (A, B)
    written = set()
    for it in plan["items"]:
        tk = tasks[it.task]
        assert it.seg == tk.seg0 and tk.nseg == 1
        sg = segs[it.seg]
        assert sg.nk == 1 and sg.K <= 32 * plan["kq"] and 1 <= it.ncol <= plan["nc"] <= 8
        if swap:
            rext, rsx, rsc, cext, csy, csc = tk.nExt[:tk.nn], sg.nSB[:tk.nn], tk.nSC[:tk.nn], tk.mExt[:tk.nm], \
                sg.mSA[:tk.nm], tk.mSC[:tk.nm]
            xb, yb, kx, ky = sg.baseB, sg.baseA, sg.kSB[0], sg.kSA[0]
        else:
            rext, rsx, rsc, cext, csy, csc = tk.mExt[:tk.nm], sg.mSA[:tk.nm], tk.mSC[:tk.nm], tk.nExt[:tk.nn], \
                sg.nSB[:tk.nn], tk.nSC[:tk.nn]
            xb, yb, kx, ky = sg.baseA, sg.baseB, sg.kSA[0], sg.kSB[0]
        assert kx == 1, "row operand not contiguous along K"
        rows = np.arange(it.r0, it.r1)
        cols = np.arange(it.c0, it.c0 + it.ncol)
        k = np.arange(sg.K)
        ix = (xb + decode(rows, rext, rsx))[:, None] + k[None, :]
        iy = (yb + decode(cols, cext, csy))[:, None] + k[None, :] * ky
        assert ix.min() >= 0 and ix.max() < X.size and iy.min() >= 0 and iy.max() < Y.size
        val = X[ix] @ Y[iy].T
        addr = tk.baseC + decode(rows, rext, rsc)[:, None] + decode(cols, cext, csc)[None, :]
        assert addr.min() >= 0 and addr.max() < C.size
        flat = addr.ravel().tolist()
        assert not (written & set(flat)) and len(set(flat)) == len(flat), "output written twice"
        written.update(flat)
        C[addr.ravel()] += alpha * val.ravel()
    return C, written


@pytest.mark.parametrize("nirrep", [1, 4, 8])
@pytest.mark.parametrize("name", sorted(KSPEC))
@pytest.mark.parametrize("nb", [1, 3])
def test_kernel_rowdot_plans(name, nirrep, nb):
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
    rng = np.random.default_rng(6)
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
    if get_narrow(*args) is not None:
        pytest.skip("narrow kernels take it")
    ptasks, psegs, _, _ = get_plan(*args)
    plan = get_rowdot(*args, len(ptasks), len(psegs))
    if plan is None:
        pytest.skip("not a row-dot contraction")
    # the kernel's tables: the plan's, row units reordered by ascending stride
    tasks, segs = plan["tasks"], plan["segs"]
    for t, pt in zip(tasks, ptasks):
        sg = segs[t.seg0]
        n, sx = (t.nn, sg.nSB) if plan["swap"] else (t.nm, sg.mSA)
        assert list(sx[:n]) == sorted(sx[:n])
        assert t.M == pt.M and t.N == pt.N and t.baseC == pt.baseC
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
