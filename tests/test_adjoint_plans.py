"""CPU verification of the contraction launches made by the adjoint
contractions (vjp444 in ops.cpp) on the SF-CIS(D) gradient path.

For every kernel of that path and each of its two operands, the engine call
of the adjoint is rebuilt here with the layouts vjp444 derives (the
result's cotangent with its packed pairs expanded, the other operand
expanded as in the forward call, the operand's own expanded layout), and
the library's plan for it (tiled FP64 tables, and the narrow-output plan
when the engine would take that path) is executed in numpy with the
kernels' indexing, bounds-checked, and compared with the oracle's engine.
The outer-product adjoints (no contracted index, K = 1) are among them."""
import ctypes

import numpy as np
import pytest

import kernel_specs as ks
import oracle_ffi as of
import test_narrow_plan as tn
import test_plan_emulation as te
from cpsd_b200 import api, synth

I64 = ctypes.c_int64

# kernel -> (v1 is operand 'a' or 'b', padded t1, t2, t3): the forward form
# each vjp_<name> reverses
ADJ = {
    "c1_r1iabj": ("b", "fnai", "fn+-", "ai+-"),
    "c1_r1Fae": ("b", "ae=+", "ei=-", "ai+-"),
    "c1_r1Fmi": ("a", "am=+", "mi=-", "ai+-"),
    "c1_r2abci": ("b", "feam", "feim", "ai.."),
    "c1_r2ijka": ("a", "aemn", "mnie", "ai.."),
    "c2_r1abci": ("b", "abej", "ei..", "abij"),
    "c2_r1ijka": ("b", "ijmb", "am..", "abij"),
    "Fmi_r2abij": ("b", "efmn", "efin", "mi.."),
    "Fae_r2abij": ("a", "afmn", "efmn", "ae.."),
    "Wmbej_r2abij": ("b", "fenm", "bfjn", "embj"),
    # the further ones of the third-order correction
    "c2_r2Wmbej": ("a", "aeim", "embj", "abij"),
    "c2_r2Wmnij": ("a", "abmn", "mnij", "abij"),
    "c2_r2abcd": ("b", "abef", "efij", "abij"),
    "c2_r2Fae": ("a", "aeij", "be..", "abij"),
    "c2_r2Fmi": ("a", "abim", "mj..", "abij"),
    "Fmi_r1ijka": ("b", "mnie", "en+-", "mi+-"),
    "Fae_r1abci": ("b", "efam", "fm+-", "ae+-"),
    "Wkbij_r2ijka": ("b", "klic", "bcjl", "ijkb"),
    "Wmbej_r1abci": ("b", "febm", "fj..", "embj"),
    "Wmbej_r1ijka": ("b", "nmje", "bn..", "embj"),
    "Wmnij_r1ijka": ("b", "mnie", "ej..", "mnij"),
}


def norm(t):
    return "".join("." if c in "+-=" else c for c in t)


def opt_of(pops, iops, sym):
    o = api.Opt()
    api.check(api.lib().cpsd_opt_init(ctypes.byref(o), api.arr8(pops[0]), api.arr8(pops[1]), api.arr8(pops[2]),
                                       api.arr8(pops[3]), I64(iops[0]), I64(iops[1]), I64(sym), None), "opt")
    return o


@pytest.mark.parametrize("nirrep", [1, 2, 4, 8])
@pytest.mark.parametrize("which", [0, 1])
@pytest.mark.parametrize("name", sorted(ADJ))
def test_adjoint_engine_plans(name, which, nirrep):
    s = synth.System(nmo=16 if nirrep < 8 else 24, nocc_a=3, nocc_b=2, nirrep=nirrep, seed=2)
    api.init(s.nirrep, s.dirprd)
    of.set_symmetry(s.nirrep, s.dirprd)
    sym = s.sym
    first, t1, t2, t3 = ADJ[name]
    lo, la, lb = ks.KERNELS[name][:3]
    symR = min(2, nirrep)
    # amplitude operand in irrep symR, integral / intermediate totally symmetric
    sa, sb = symR, 1
    if name in ("Fmi_r2abij", "Fae_r2abij", "Wmbej_r2abij"):
        sa = 1
    pa, ia = ks.pops_of(la, s.popo, s.popv)
    pb, ib = ks.pops_of(lb, s.popo, s.popv)
    po, io = ks.pops_of(lo, s.popo, s.popv)
    so = sym.dp(sa, sb)
    ops = {"a": (pa, list(ia), sa), "b": (pb, list(ib), sb)}
    v1, v2 = (ops["a"], ops["b"]) if first == "a" else (ops["b"], ops["a"])
    v3 = (po, list(io), so)
    T = [t1, t2, t3]
    pairs = [t1[:2], t1[2:], t2[:2], t2[2:], t3[:2], t3[2:]]
    iop = v1[1] + v2[1] + v3[1]
    iexp = [all(pairs[i] != pairs[j] for j in range(6) if j != i) and iop[i] != 1 for i in range(6)]
    full = [1 if iexp[i] else iop[i] for i in range(6)]
    X = (po, full[4:6], so)                      # the result's cotangent, expanded
    V = [(v1[0], full[0:2], v1[2]), (v2[0], full[2:4], v2[2])]
    self_, other = V[which], V[1 - which]
    ts, to = T[which], T[1 - which]
    e = [(X, norm(t3)), (other, norm(to)), (self_, norm(ts))]
    o = [opt_of(*d) for d, _ in e]
    lens = [sym.idsymsoc(d[2], d[0][0], d[0][1], d[1][0], d[0][2], d[0][3], d[1][1]) for d, _ in e]
    rng = np.random.default_rng(3)
    A, B, C = (rng.standard_normal(n) for n in lens)
    tasks, segs, tiles, tile = te.get_plan(o[0], e[0][1], o[1], e[1][1], o[2], e[2][1])
    ref = C.copy()
    rc = of.vv2v_dpd(A, of.desc(*X), e[0][1], B, of.desc(*other), e[1][1], ref, of.desc(*self_), e[2][1], 0.7, 1.0)
    assert rc == 0
    out = te.emulate(tasks, segs, tiles, A, B, C, 0.7, tile)
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12)
    nplan = tn.get_narrow(o[0], e[0][1], o[1], e[1][1], o[2], e[2][1], 1, 0, 0, 0)
    if nplan is not None:
        out, _ = tn.emulate(tasks, segs, nplan, A, B, C, 0.7)
        np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12)
