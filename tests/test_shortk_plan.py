"""CPU verification of the short-K contraction plans (no GPU needed).

For every engine call of the 22 kernels that the engine sends to the
short-K kernel (not narrow, every task's contracted range at most 64), the
work items of cpsd_debug_shortk_plan are executed in numpy with the
kernel's index arithmetic over the planner's task / segment tables: each
item is one BF x BS output tile (BF = 2048 / BS along the output side that
is contiguous in C), every operand read and output write is bounds-checked,
the shared-memory K slots of a task stay below the plan's kmax, each output
element is written by exactly one item, and the result is compared with
the CPU oracle."""
import ctypes

import numpy as np
import pytest

import kernel_specs as ks
import oracle_ffi as of
from cpsd_b200 import api, synth
from test_narrow_plan import get_narrow
from test_plan_emulation import KSPEC, to_engine, norm, I64, get_plan, decode


class ShortKItem(ctypes.Structure):
    _fields_ = [("task", ctypes.c_int), ("seg0", ctypes.c_int), ("f0", I64), ("s0", I64)]


def get_shortk(o1, t1, o2, t2, o3, t3, nb, sA, sB, sC):
    it, ni = ctypes.c_void_p(), I64()
    flags = (I64 * 4)()
    api.check(api.lib().cpsd_debug_shortk_plan(ctypes.byref(o1), t1.encode(), ctypes.byref(o2), t2.encode(),
                                               ctypes.byref(o3), t3.encode(), I64(nb), I64(sA), I64(sB), I64(sC),
                                               ctypes.byref(it), ctypes.byref(ni), flags), "short-K plan")
    if not flags[0]:
        return None
    items = list((ShortKItem * ni.value).from_address(it.value)) if ni.value else []
    return dict(items=items, fm=bool(flags[1]), bs=int(flags[2]), kmax=int(flags[3]))


def emulate(tasks, segs, plan, A, B, C, alpha):
    C = C.copy()
    bs = plan["bs"]
    bf = 2048 // bs
    assert bs in (8, 16, 32) and 1 <= plan["kmax"] <= 64
    written = set()
    for it in plan["items"]:
        tk = tasks[it.task]
        F, S = (tk.M, tk.N) if plan["fm"] else (tk.N, tk.M)
        assert 0 <= it.f0 < F and 0 <= it.s0 < S and it.f0 % bf == 0 and it.s0 % bs == 0
        assert it.seg0 == tk.seg0 and tk.nseg >= 1
        f = np.arange(it.f0, min(it.f0 + bf, F))
        s = np.arange(it.s0, min(it.s0 + bs, S))
        m, n = (f, s) if plan["fm"] else (s, f)
        acc = np.zeros((len(m), len(n)))
        kk = 0
        for si in range(tk.nseg):
            sg = segs[tk.seg0 + si]
            k = np.arange(sg.K)
            oa = sg.baseA + decode(m, tk.mExt[:tk.nm], sg.mSA[:tk.nm])
            ob = sg.baseB + decode(n, tk.nExt[:tk.nn], sg.nSB[:tk.nn])
            ka = decode(k, sg.kExt[:sg.nk], sg.kSA[:sg.nk])
            kb = decode(k, sg.kExt[:sg.nk], sg.kSB[:sg.nk])
            ia, ib = oa[:, None] + ka[None, :], ob[:, None] + kb[None, :]
            if sg.K:
                assert ia.min() >= 0 and ia.max() < A.size, "A read out of bounds"
                assert ib.min() >= 0 and ib.max() < B.size, "B read out of bounds"
                acc += A[ia] @ B[ib].T
            kk += sg.K
        assert kk == tk.Ktot and kk <= plan["kmax"], "K slots beyond the plan's kmax"
        addr = tk.baseC + decode(m, tk.mExt[:tk.nm], tk.mSC[:tk.nm])[:, None] + \
            decode(n, tk.nExt[:tk.nn], tk.nSC[:tk.nn])[None, :]
        assert addr.min() >= 0 and addr.max() < C.size, "output out of bounds"
        flat = addr.ravel().tolist()
        assert not (written & set(flat)) and len(set(flat)) == len(flat), "output written twice"
        written.update(flat)
        C[addr.ravel()] += alpha * acc.ravel()
    return C, written


@pytest.mark.parametrize("nirrep", [1, 4, 8])
@pytest.mark.parametrize("name", sorted(KSPEC))
@pytest.mark.parametrize("nb", [1, 3])
def test_kernel_shortk_plans(name, nirrep, nb):
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
    rng = np.random.default_rng(4)
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
        pytest.skip("narrow output: the narrow kernels take it")
    plan = get_shortk(*args)
    if plan is None:
        pytest.skip("contracted range above 64: tensor-core tiles")
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
