"""The CPU oracle's DPD engine, layout transforms and every lib_cc kernel on
the path, against independent dense numpy formulas (nirrep 1, 2 and 4,
non-totally-symmetric operands included)."""
import numpy as np
import pytest

import dense
import kernel_specs as ks
import oracle_ffi as of
from cpsd_b200 import synth
from cpsd_b200.dpd import Symmetry, xor_dirprd


def _sys(nirrep):
    return synth.System(nmo=12 if nirrep < 4 else 16, nocc_a=3, nocc_b=2, nirrep=nirrep, seed=3)


def test_generator_matches_dense():
    s = synth.System(nmo=14, nocc_a=3, nocc_b=2, nirrep=4, seed=11)
    g, O, V, eo, ev = dense.antisym_integrals(s)
    sym, o, v = s.sym, s.popo, s.popv
    checks = {
        "ijkl": ([o, o, o, o], (0, 0), g[O, O, O, O]),
        "ijka": ([o, o, o, v], (0, 1), g[O, O, O, V]),
        "abij": ([v, v, o, o], (0, 0), g[V, V, O, O]),
        "iabj": ([v, o, v, o], (1, 1), g[O, V, V, O].transpose(2, 0, 1, 3)),
        "abci": ([v, v, v, o], (0, 1), g[V, V, V, O]),
        "abcd": ([v, v, v, v], (0, 0), g[V, V, V, V]),
    }
    for k, (pops, iops, D) in checks.items():
        vec = dense.dense_to_dpd(D, sym, pops, iops, 1)
        np.testing.assert_allclose(s.ints[k], vec, rtol=0, atol=1e-14, err_msg=k)
    np.testing.assert_allclose(s.eorb, np.concatenate([eo, ev]), atol=0)


def test_size_math_matches_python():
    s = _sys(4)
    of.set_symmetry(s.nirrep, s.dirprd)
    for iops in [(0, 0), (1, 1), (0, 1), (2, 1)]:
        for sym in range(1, 5):
            d = of.desc([s.popv, s.popv, s.popo, s.popo], iops, sym)
            assert of.desc_len(d) == s.sym.idsymsoc(sym, s.popv, s.popv, iops[0], s.popo, s.popo, iops[1])


@pytest.mark.parametrize("nirrep", [1, 2, 4])
def test_engine_general_einsum(nirrep):
    """vv2v_dpd with all-full pairs and crossed indices ('3142*3546->1256'
    style, the reference's fallback) and with intact packed pairs (fast path)."""
    rng = np.random.default_rng(nirrep)
    s = _sys(nirrep)
    of.set_symmetry(s.nirrep, s.dirprd)
    sym, o, v = s.sym, s.popo, s.popv
    cases = [
        # (t1, pops1, iops1, s1), (t2,...), (t3,...), einsum
        (("aeim", [v, v, o, o], (1, 1), 2), ("embj", [v, o, v, o], (1, 1), 1),
         ("abij", [v, v, o, o], (1, 1), 2), "aeim,embj->abij"),
        (("abef", [v, v, v, v], (0, 0), 1), ("efij", [v, v, o, o], (0, 0), nirrep),
         ("abij", [v, v, o, o], (0, 0), nirrep), "abef,efij->abij"),
        (("mbie", [o, v, o, v], (1, 1), 1), ("ajme", [v, o, o, v], (1, 1), 2),
         ("abij", [v, v, o, o], (1, 1), 2), "mbie,ajme->abij"),
    ]
    for (t1, p1, i1, s1), (t2, p2, i2, s2), (t3, p3, i3, s3), es in cases:
        if nirrep == 1:
            s1 = s2 = s3 = 1
        a = rng.standard_normal(sym.idsymsoc(s1, p1[0], p1[1], i1[0], p1[2], p1[3], i1[1]))
        b = rng.standard_normal(sym.idsymsoc(s2, p2[0], p2[1], i2[0], p2[2], p2[3], i2[1]))
        c = rng.standard_normal(sym.idsymsoc(s3, p3[0], p3[1], i3[0], p3[2], p3[3], i3[1]))
        A = dense.dpd_to_dense(a, sym, p1, i1, s1)
        B = dense.dpd_to_dense(b, sym, p2, i2, s2)
        C = dense.dpd_to_dense(c, sym, p3, i3, s3)
        fac = 1.0
        for pair_iop in (i1[0], i1[1]):
            pass
        # intact packed contracted pairs sum over p<q only: 1/2 of the full sum
        k_half = 0.5 if es.startswith("abef") else 1.0
        ref = 0.7 * k_half * np.einsum(es, A, B) + 0.3 * C
        out = c.copy()
        rc = of.vv2v_dpd(a, of.desc(p1, i1, s1), t1, b, of.desc(p2, i2, s2), t2,
                         out, of.desc(p3, i3, s3), t3, 0.7, 0.3)
        assert rc == 0
        np.testing.assert_allclose(out, dense.dense_to_dpd(ref, sym, p3, i3, s3), atol=1e-12)
        # beta = 0 overwrites even dirty output (the reference's 999 injection check)
        out = np.full_like(c, 999.0)
        rc = of.vv2v_dpd(a, of.desc(p1, i1, s1), t1, b, of.desc(p2, i2, s2), t2,
                         out, of.desc(p3, i3, s3), t3, 1.0, 0.0)
        assert rc == 0
        np.testing.assert_allclose(out, dense.dense_to_dpd(k_half * np.einsum(es, A, B), sym, p3, i3, s3),
                                   atol=1e-12)


def test_engine_rejects_broken_packed_pair():
    s = _sys(2)
    of.set_symmetry(s.nirrep, s.dirprd)
    o, v = s.popo, s.popv
    a = np.zeros(s.sym.idsymsoc(1, v, v, 0, o, o, 0))
    b = np.zeros(s.sym.idsymsoc(1, v, o, 1, v, o, 1))
    c = np.zeros(s.sym.idsymsoc(1, v, v, 1, o, o, 1))
    # 'ae' packed in v1 but split in the output: the reference STOPs, the oracle returns an error
    rc = of.vv2v_dpd(a, of.desc([v, v, o, o], (0, 0), 1), "aeim", b, of.desc([v, o, v, o], (1, 1), 1), "embj",
                     c, of.desc([v, v, o, o], (1, 1), 1), "abij", 1.0, 1.0)
    assert rc != 0


@pytest.mark.parametrize("nirrep", [1, 4])
@pytest.mark.parametrize("name", sorted(ks.KERNELS))
def test_kernel_vs_dense(name, nirrep):
    rng = np.random.default_rng(hash(name) % 1000 + nirrep)
    s = _sys(nirrep)
    of.set_symmetry(s.nirrep, s.dirprd)
    sym = s.sym
    lo, la, lb = ks.KERNELS[name][:3]
    fn = ks.KERNELS[name][3]
    symR = 2 if nirrep > 1 else 1
    # the R-like operand (a) carries symR; integral-like operands carry 1
    syms = {"a": symR, "b": 1}
    # W/F intermediates built from R carry symR as the output; operands that
    # are outputs of R-dependent intermediates in calC_VTR also carry symR
    if name in ("c2_r2Wmbej", "c2_r2Wmnij", "c2_r2Fae", "c2_r2Fmi", "c1_r1Fae", "c1_r1Fmi", "c1_r1iabj"):
        syms = {"a": 1, "b": symR} if name.startswith("c2_r2") else {"a": symR, "b": 1}
    so = sym.dp(syms["a"], syms["b"])
    po, io = ks.pops_of(lo, s.popo, s.popv)
    pa, ia = ks.pops_of(la, s.popo, s.popv)
    pb, ib = ks.pops_of(lb, s.popo, s.popv)
    va = rng.standard_normal(sym.idsymsoc(syms["a"], pa[0], pa[1], ia[0], pa[2], pa[3], ia[1]))
    vb = rng.standard_normal(sym.idsymsoc(syms["b"], pb[0], pb[1], ib[0], pb[2], pb[3], ib[1]))
    vo = rng.standard_normal(sym.idsymsoc(so, po[0], po[1], io[0], po[2], po[3], io[1]))
    A = ks.squeeze2(dense.dpd_to_dense(va, sym, pa, ia, syms["a"]), la)
    B = ks.squeeze2(dense.dpd_to_dense(vb, sym, pb, ib, syms["b"]), lb)
    Oref = ks.squeeze2(dense.dpd_to_dense(vo, sym, po, io, so), lo) + fn(A, B, 0.8)
    out = vo.copy()
    oo = of.opt(po, io, so, out)
    oa = of.opt(pa, ia, syms["a"], va)
    ob = of.opt(pb, ib, syms["b"], vb)
    rc = of.call_kernel(name, oo, oa, ob, 0.8)
    assert rc == 0
    np.testing.assert_allclose(out, dense.dense_to_dpd(ks.expand2(Oref, lo), sym, po, io, so), atol=1e-12,
                               err_msg=name)
