"""The int8-digit tensor-core contraction path (tcgen05 kind::i8) on the GPU
against the CPU oracle, through the C-ABI.

Contractions: the engine cases and all 22 kernels with every contraction
routed through the digit path (min_gflop = 0), compared within the method's
bound (digits + 1) K 128^-digits max|a| max|b| (x4 margin).  Pipeline: the
excitation energies and their second / third order corrections with 7
digits to 1e-9 Eh of the oracle, with 5 digits to 1 micro-Eh."""
import numpy as np
import pytest

import kernel_specs as ks
import oracle_ffi as of
from cpsd_b200 import api, synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.fixture(autouse=True)
def _mixed():
    api.use_torch_stream()
    yield
    api.set_mixed(0)


def bound(digits, K, a, b, f):
    return (digits + 1) * K * 128.0 ** -digits * np.abs(a).max() * np.abs(b).max() * abs(f) * 4 + 1e-12


@pytest.mark.parametrize("digits", [4, 7])
@pytest.mark.parametrize("nirrep", [1, 4, 8])
def test_engine_digits_match_oracle(nirrep, digits):
    s = synth.System(nmo=24, nocc_a=4, nocc_b=2, nirrep=nirrep, seed=nirrep)
    api.init(s.nirrep, s.dirprd)
    of.set_symmetry(s.nirrep, s.dirprd)
    api.set_mixed(digits, 0.0)
    sym, o, v = s.sym, s.popo, s.popv
    rng = np.random.default_rng(0)
    s2 = 2 if nirrep > 1 else 1
    z = np.array([1, 0, 0, 0, 0, 0, 0, 0])
    cases = [
        ("aeim", [v, v, o, o], (1, 1), s2, "embj", [v, o, v, o], (1, 1), 1, "abij", [v, v, o, o], (1, 1), s2, 400),
        ("abef", [v, v, v, v], (0, 0), 1, "efij", [v, v, o, o], (0, 0), s2, "abij", [v, v, o, o], (0, 0), s2, 200),
        ("mbie", [o, v, o, v], (1, 1), 1, "ajme", [v, o, o, v], (1, 1), s2, "abij", [v, v, o, o], (1, 1), s2, 200),
        ("ijmb", [o, o, o, v], (0, 1), 1, "am..", [v, o, z, z], (1, 1), s2, "abij", [v, v, o, o], (1, 0), s2, 100),
    ]
    for (t1, p1, i1, y1, t2, p2, i2, y2, t3, p3, i3, y3, K) in cases:
        a = rng.standard_normal(sym.idsymsoc(y1, p1[0], p1[1], i1[0], p1[2], p1[3], i1[1]))
        b = rng.standard_normal(sym.idsymsoc(y2, p2[0], p2[1], i2[0], p2[2], p2[3], i2[1]))
        c = rng.standard_normal(sym.idsymsoc(y3, p3[0], p3[1], i3[0], p3[2], p3[3], i3[1]))
        for f2 in (1.0, 0.0):
            ref = c.copy() if f2 != 0.0 else np.full_like(c, 999.0)
            assert of.vv2v_dpd(a, of.desc(p1, i1, y1), t1, b, of.desc(p2, i2, y2), t2, ref, of.desc(p3, i3, y3),
                               t3, 0.7, f2) == 0
            out = dev(c if f2 != 0.0 else np.full_like(c, 999.0))
            api.vv2v_dpd_444(dev(a), (p1, i1, y1), t1, dev(b), (p2, i2, y2), t2, out, (p3, i3, y3), t3, 0.7, f2)
            np.testing.assert_allclose(host(out), ref, rtol=0, atol=bound(digits, K, a, b, 0.7),
                                       err_msg=f"{t1}*{t2}->{t3} f2={f2}")
    assert api.mixed_error() == 0


@pytest.mark.parametrize("nirrep", [1, 4])
@pytest.mark.parametrize("name", sorted(ks.KERNELS))
def test_kernel_digits_match_oracle(name, nirrep):
    digits = 6
    rng = np.random.default_rng(abs(hash(name)) % 1000 + nirrep)
    s = synth.System(nmo=16, nocc_a=3, nocc_b=1, nirrep=nirrep, seed=5)
    api.init(s.nirrep, s.dirprd)
    of.set_symmetry(s.nirrep, s.dirprd)
    api.set_mixed(digits, 0.0)
    sym = s.sym
    lo, la, lb = ks.KERNELS[name][:3]
    symR = 2 if nirrep > 1 else 1
    syms = {"a": symR, "b": 1}
    if name.startswith("c2_r2"):
        syms = {"a": 1, "b": symR}
    so = sym.dp(syms["a"], syms["b"])
    po, io = ks.pops_of(lo, s.popo, s.popv)
    pa, ia = ks.pops_of(la, s.popo, s.popv)
    pb, ib = ks.pops_of(lb, s.popo, s.popv)
    va = rng.standard_normal(sym.idsymsoc(syms["a"], pa[0], pa[1], ia[0], pa[2], pa[3], ia[1]))
    vb = rng.standard_normal(sym.idsymsoc(syms["b"], pb[0], pb[1], ib[0], pb[2], pb[3], ib[1]))
    vo = rng.standard_normal(sym.idsymsoc(so, po[0], po[1], io[0], po[2], po[3], io[1]))
    ref = vo.copy()
    assert of.call_kernel(name, of.opt(po, io, so, ref), of.opt(pa, ia, syms["a"], va),
                          of.opt(pb, ib, syms["b"], vb), 0.8) == 0
    ta, tb, to = dev(va), dev(vb), dev(vo)
    api.kernel(name, api.opt(po, io, so, to), api.opt(pa, ia, syms["a"], ta), api.opt(pb, ib, syms["b"], tb), 0.8)
    # K of these small systems is below 16^3; antisymmetrisation adds at most 4 terms
    np.testing.assert_allclose(host(to), ref, rtol=0, atol=4 * bound(digits, 4096, va, vb, 0.8), err_msg=name)
    assert api.mixed_error() == 0


@pytest.mark.parametrize("digits,tol", [(7, 1e-9), (5, 1e-6)])
def test_pipeline_digits_match_oracle(digits, tol):
    s = synth.make("c2v_nmo48")
    api.init(s.nirrep, s.dirprd)
    ints = api.DeviceIntegrals(s)
    sc, par = api.make_system(s), api.make_params(s, batch_roots=1)
    api.set_mixed(digits, 0.0)
    api.contract_timing(True)
    try:
        om, w2, w3 = api.pipeline(s, sc, ints, par)
        kinds = api.contract_records()[2]
    finally:
        api.contract_timing(False)
    assert api.mixed_error() == 0
    # the int8 digit GEMM (kind 12) and the digit slicing (10 / 11) ran: a
    # silent fall-back to the FP64 tiles would also pass the energy checks
    assert np.sum(kinds == 12) > 0 and np.sum((kinds == 10) | (kinds == 11)) > 0
    oom, ow2, ow3 = of.Oracle(s).pipeline()
    np.testing.assert_allclose(om, oom, rtol=0, atol=tol)
    np.testing.assert_allclose(w2, ow2, rtol=0, atol=tol)
    np.testing.assert_allclose(w3, ow3, rtol=0, atol=tol)


@pytest.mark.parametrize("digits,tol", [(7, 1e-10), (5, 1e-7)])
def test_all_digit_routing_follows_fp64_roots(digits, tol):
    """Ten small molecules of the batching draw (one of them C1, nmo 45, 7
    roots, max-overlap root tracking) with every regrouping contraction on
    the digit path: same roots as FP64 and no NaN.  Root tracking that could
    give one eigenvector to two roots made the collapse of that C1 molecule
    divide by zero."""
    import test_gpu_batch as tb
    mols = tb.molecules(10, 42)
    out = {}
    for mode in (0, digits):
        res = []
        for s in mols:
            api.init(s.nirrep, s.dirprd)
            d, p = api.DeviceIntegrals(s), api.make_params(s)
            api.set_mixed(mode, 0.0 if mode else 1.0)
            try:
                res.append(api.pipeline(s, api.make_system(s), d, p)[0])
            finally:
                api.set_mixed(0)
        out[mode] = res
    for a, b in zip(out[digits], out[0]):
        assert not np.isnan(a).any()
        np.testing.assert_allclose(a, b, rtol=0, atol=tol)
