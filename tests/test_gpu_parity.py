"""GPU (libcpsd_b200 through the C-ABI) against the CPU oracle on the same
seeded inputs.  FP64 throughout: contractions to 1e-12 absolute on O(1)
data, excitation energies and (D) corrections to 1e-9 Eh; vectors from
iterative solvers are compared up to sign and to their convergence
thresholds (Davidson residual 1e-8, DIIS 1e-7)."""
import numpy as np
import pytest

import kernel_specs as ks
import oracle_ffi as of
from cpsd_b200 import api, synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_E = 1e-9


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def small(nirrep, roots=2, seed=5, nmo=None):
    return synth.System(nmo=nmo or (14 if nirrep <= 2 else 16), nocc_a=3, nocc_b=1, nirrep=nirrep, seed=seed,
                        roots=roots)


@pytest.fixture(autouse=True)
def _stream():
    api.use_torch_stream()
    yield


@pytest.mark.parametrize("nirrep", [1, 4, 8])
def test_engine_matches_oracle(nirrep):
    s = synth.System(nmo=24, nocc_a=4, nocc_b=2, nirrep=nirrep, seed=nirrep)
    api.init(s.nirrep, s.dirprd)
    of.set_symmetry(s.nirrep, s.dirprd)
    sym, o, v = s.sym, s.popo, s.popv
    rng = np.random.default_rng(0)
    s2 = 2 if nirrep > 1 else 1
    z = np.array([1, 0, 0, 0, 0, 0, 0, 0])
    cases = [
        ("aeim", [v, v, o, o], (1, 1), s2, "embj", [v, o, v, o], (1, 1), 1, "abij", [v, v, o, o], (1, 1), s2),
        ("abef", [v, v, v, v], (0, 0), 1, "efij", [v, v, o, o], (0, 0), s2, "abij", [v, v, o, o], (0, 0), s2),
        ("mbie", [o, v, o, v], (1, 1), 1, "ajme", [v, o, o, v], (1, 1), s2, "abij", [v, v, o, o], (1, 1), s2),
        ("ijmb", [o, o, o, v], (0, 1), 1, "am..", [v, o, z, z], (1, 1), s2, "abij", [v, v, o, o], (1, 0), s2),
    ]
    for (t1, p1, i1, y1, t2, p2, i2, y2, t3, p3, i3, y3) in cases:
        a = rng.standard_normal(sym.idsymsoc(y1, p1[0], p1[1], i1[0], p1[2], p1[3], i1[1]))
        b = rng.standard_normal(sym.idsymsoc(y2, p2[0], p2[1], i2[0], p2[2], p2[3], i2[1]))
        c = rng.standard_normal(sym.idsymsoc(y3, p3[0], p3[1], i3[0], p3[2], p3[3], i3[1]))
        for f2 in (1.0, 0.0, 0.5):
            ref = c.copy() if f2 != 0.0 else np.full_like(c, 999.0)
            rc = of.vv2v_dpd(a, of.desc(p1, i1, y1), t1, b, of.desc(p2, i2, y2), t2, ref, of.desc(p3, i3, y3), t3,
                             0.7, f2)
            assert rc == 0
            out = dev(c if f2 != 0.0 else np.full_like(c, 999.0))
            api.vv2v_dpd_444(dev(a), (p1, i1, y1), t1, dev(b), (p2, i2, y2), t2, out, (p3, i3, y3), t3, 0.7, f2)
            np.testing.assert_allclose(host(out), ref, rtol=0, atol=1e-12, err_msg=f"{t1}*{t2}->{t3} f2={f2}")


@pytest.mark.parametrize("nirrep", [1, 4])
@pytest.mark.parametrize("name", sorted(ks.KERNELS))
def test_kernel_matches_oracle(name, nirrep):
    rng = np.random.default_rng(abs(hash(name)) % 1000 + nirrep)
    s = small(nirrep)
    api.init(s.nirrep, s.dirprd)
    of.set_symmetry(s.nirrep, s.dirprd)
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
    rc = of.call_kernel(name, of.opt(po, io, so, ref), of.opt(pa, ia, syms["a"], va), of.opt(pb, ib, syms["b"], vb),
                        0.8)
    assert rc == 0
    ta, tb, to = dev(va), dev(vb), dev(vo)
    api.kernel(name, api.opt(po, io, so, to), api.opt(pa, ia, syms["a"], ta), api.opt(pb, ib, syms["b"], tb), 0.8)
    np.testing.assert_allclose(host(to), ref, rtol=0, atol=1e-12, err_msg=name)


@pytest.mark.parametrize("nocc", [(3, 2), (4, 2)])
@pytest.mark.parametrize("nirrep", [1, 4, 8])
@pytest.mark.parametrize("name,kind", [("Wmbej_r1abci", 23), ("Wmbej_r1ijka", 22), ("c2_r2Fae", 22),
                                       ("c1_r2abci", 21)])
def test_streaming_kernels_ran_and_match_oracle(name, kind, nirrep, nocc):
    """The row-dot (kind 23), short-K (kind 22) and long-K narrow (kind 21)
    kernels are the ones that ran for these shapes (their timing records),
    and they match the oracle (at nirrep 1 the row-dot's and the long-K
    kernel's outputs have 5 or 6 columns: their 5- and 6-column item
    shapes)."""
    rng = np.random.default_rng(17 + nirrep)
    s = synth.System(nmo=16 if nirrep < 8 else 24, nocc_a=nocc[0], nocc_b=nocc[1], nirrep=nirrep, seed=2)
    api.init(s.nirrep, s.dirprd)
    of.set_symmetry(s.nirrep, s.dirprd)
    sym = s.sym
    lo, la, lb = ks.KERNELS[name][:3]
    symR = min(2, nirrep)
    sa, sb = (symR, 1) if not name.startswith("c2_r2") else (1, symR)
    so = sym.dp(sa, sb)
    po, io = ks.pops_of(lo, s.popo, s.popv)
    pa, ia = ks.pops_of(la, s.popo, s.popv)
    pb, ib = ks.pops_of(lb, s.popo, s.popv)
    va = rng.standard_normal(sym.idsymsoc(sa, pa[0], pa[1], ia[0], pa[2], pa[3], ia[1]))
    vb = rng.standard_normal(sym.idsymsoc(sb, pb[0], pb[1], ib[0], pb[2], pb[3], ib[1]))
    vo = rng.standard_normal(sym.idsymsoc(so, po[0], po[1], io[0], po[2], po[3], io[1]))
    ref = vo.copy()
    assert of.call_kernel(name, of.opt(po, io, so, ref), of.opt(pa, ia, sa, va), of.opt(pb, ib, sb, vb), 0.8) == 0
    ta, tb, to = dev(va), dev(vb), dev(vo)
    api.contract_timing(True)
    try:
        api.kernel(name, api.opt(po, io, so, to), api.opt(pa, ia, sa, ta), api.opt(pb, ib, sb, tb), 0.8)
        _, _, kinds, _ = api.contract_records()
    finally:
        api.contract_timing(False)
    assert kind in set(int(k) for k in kinds), (name, sorted(set(int(k) for k in kinds)))
    np.testing.assert_allclose(host(to), ref, rtol=0, atol=1e-12, err_msg=name)


def test_tile_autotune_matches_oracle():
    """With the empirical tile-shape choice on, the FP64 pipeline still
    matches the oracle and the tuner timed the tile plans it met."""
    s = synth.make("c2v_nmo48")
    ints, sc, par, orc = _run_both(s)
    api.set_mixed(0, 1.0)
    t0, _ = api.tile_autotune_stats()
    api.set_tile_autotune(True)
    try:
        om, w2, w3 = api.pipeline(s, sc, ints, par)
    finally:
        api.set_tile_autotune(False)
    t1, c1 = api.tile_autotune_stats()
    assert t1 > t0
    oom, ow2, ow3 = orc.pipeline()
    np.testing.assert_allclose(om, oom, rtol=0, atol=TOL_E)
    np.testing.assert_allclose(w2, ow2, rtol=0, atol=TOL_E)
    np.testing.assert_allclose(w3, ow3, rtol=0, atol=TOL_E)


def _run_both(s, batch_roots=1, **kw):
    api.init(s.nirrep, s.dirprd)
    ints = api.DeviceIntegrals(s)
    return ints, api.make_system(s), api.make_params(s, batch_roots=batch_roots, **kw), of.Oracle(s, **kw)


@pytest.mark.parametrize("nirrep", [1, 2, 4])
def test_cis_matches_oracle(nirrep):
    s = small(nirrep, roots=3)
    ints, sc, par, orc = _run_both(s)
    om, R, it = api.cis_run(s, sc, ints, par)
    oom, oR, oit = orc.cis()
    np.testing.assert_allclose(om, oom, rtol=0, atol=1e-10)
    l1 = s.r1_len(1)
    Rg = host(R)
    for k in range(len(om)):
        a, b = Rg[k * l1:(k + 1) * l1], oR[k * l1:(k + 1) * l1]
        sgn = np.sign(np.dot(a, b))
        np.testing.assert_allclose(sgn * a, b, rtol=0, atol=1e-7)


@pytest.mark.parametrize("nirrep", [1, 4])
def test_cis_nonsymmetric_matches_oracle(nirrep):
    """A non-symmetric CIS matrix: the Davidson step solves the general Ritz
    problem, as the reference's dgeev does (mod_davidson.f90:185-219), and
    matches the oracle.  The matrix is A' = D A D^-1 with a positive
    diagonal D far from the identity (V'(fn,ai) = V(fn,ai) d(ai) / d(fn) in
    every irrep block of iabj): strongly non-symmetric, with the real
    eigenvalues of the symmetric A, and right eigenvectors D R.  An
    eigenvalue's error is first order in the residual for a non-symmetric
    matrix, so both run to a residual of 1e-12 (davidson_conv = 12).  With
    the symmetric integrals every step takes the symmetric solve."""
    s = small(nirrep, roots=3)
    s.run_opts["davidson_conv"] = 12
    ints, sc, par, orc = _run_both(s)
    api.davidson_stats(reset=True)
    sym_om, sym_R, _ = api.cis_run(s, sc, ints, par)
    assert api.davidson_stats()[0] == 0
    rng = np.random.default_rng(11 + nirrep)
    iabj = s.ints["iabj"].copy()
    dvec, off = [], 0
    for h in range(1, s.nirrep + 1):
        n = s.sym.irpdso(h, s.popv, s.popo, 1)
        d = 1.0 + 0.3 * rng.uniform(-1.0, 1.0, n)
        blk = iabj[off:off + n * n].reshape(n, n, order="F")  # (fn, ai), column-major
        iabj[off:off + n * n] = (blk * d[None, :] / d[:, None]).reshape(-1, order="F")
        dvec.append(d)
        off += n * n
    assert off == len(iabj)
    s.ints["iabj"] = iabj
    ints, sc, par, orc = _run_both(s)
    om, R, it = api.cis_run(s, sc, ints, par)
    nonsym, imag = api.davidson_stats()
    assert nonsym > 0 and imag == 0
    oom, oR, oit = orc.cis()
    np.testing.assert_allclose(om, oom, rtol=0, atol=1e-10)
    np.testing.assert_allclose(om, sym_om, rtol=0, atol=1e-9)
    l1 = s.r1_len(1)
    Rg, Rs = host(R), host(sym_R)
    for k in range(len(om)):
        a, b = Rg[k * l1:(k + 1) * l1], oR[k * l1:(k + 1) * l1]
        sgn = np.sign(np.dot(a, b))
        np.testing.assert_allclose(sgn * a, b, rtol=0, atol=1e-9)
        # right eigenvector of D A D^-1: D R (irrep 1 block of the roots)
        dr = dvec[0] * Rs[k * l1:(k + 1) * l1]
        dr /= np.linalg.norm(dr)
        np.testing.assert_allclose(np.sign(np.dot(a, dr)) * a, dr, rtol=0, atol=1e-8)


@pytest.mark.parametrize("lowest", [0, 1])
@pytest.mark.parametrize("nirrep", [1, 4, 8])
def test_cisdoo_matches_oracle(nirrep, lowest):
    """CIS(D-infinity) (src/CISdoo.SD.SF/run.f90): the non-symmetric (R1, R2)
    problem; roots and vectors against the oracle, both converged to a
    residual of 1e-12, every Ritz step through the general eigen-solve."""
    s = small(nirrep, roots=2) if nirrep < 8 else synth.System(nmo=24, nocc_a=4, nocc_b=2, nirrep=8, seed=3, roots=2)
    s.run_opts["davidson_conv"] = 12
    s.run_opts["lowest"] = lowest
    ints, sc, par, orc = _run_both(s)
    api.davidson_stats(reset=True)
    om, R, it = api.cisdoo_run(s, sc, ints, par)
    nonsym, imag = api.davidson_stats()
    assert nonsym > 0 and imag == 0
    oom, oR, oit = orc.cisdoo()
    np.testing.assert_allclose(om, oom, rtol=0, atol=1e-10)
    assert abs(it - oit) <= 1
    Rg = host(R)
    off, k = 0, 0
    for h in range(8):
        n = s.r1_len(h + 1) + s.r2_len(h + 1)
        for _ in range(int(s.estate_sym[h])):
            a, b = Rg[off:off + n], oR[off:off + n]
            sgn = np.sign(np.dot(a, b))
            np.testing.assert_allclose(sgn * a, b, rtol=0, atol=1e-9)
            off += n
            k += 1
    assert k == len(om) > 0


@pytest.mark.parametrize("nirrep", [1, 4])
def test_ground_and_intermediates_match_oracle(nirrep):
    s = small(nirrep)
    ints, sc, par, orc = _run_both(s)
    g = api.ground(s, sc, ints, par)
    og = orc.ground()
    assert abs(g["E2"] - og["E2"]) < 1e-11 and abs(g["E3"] - og["E3"]) < 1e-11
    np.testing.assert_allclose(host(g["T2_1"]), og["T2_1"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(host(g["T2_2"]), og["T2_2"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(host(g["T1_2"]), og["T1_2"], rtol=0, atol=1e-9)
    assert g["iters"] == og["iters"]
    J, js = api.calJ(s, sc, ints, g)
    oJ = orc.jints(og)
    for k in oJ:
        np.testing.assert_allclose(host(J[k]), oJ[k], rtol=0, atol=1e-9, err_msg=k)


@pytest.mark.parametrize("nirrep", [1, 4, 8])
def test_ground_third_order_matches_oracle(nirrep):
    """run3.f90: T2^(3) and E^(4) to the oracle's rounding, T1^(3) to the
    DIIS tolerance, the same DIIS step count."""
    s = small(nirrep) if nirrep < 8 else synth.System(nmo=24, nocc_a=4, nocc_b=2, nirrep=8, seed=3)
    ints, sc, par, orc = _run_both(s)
    g = api.ground(s, sc, ints, par)
    g3 = api.ground3(s, sc, ints, par, g)
    og = orc.ground()
    og3 = orc.ground3(og)
    assert abs(g3["E4"] - og3["E4"]) < 1e-11
    np.testing.assert_allclose(host(g3["T2_3"]), og3["T2_3"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(host(g3["T1_3"]), og3["T1_3"], rtol=0, atol=1e-8)
    assert g3["iters"] == og3["iters"]


@pytest.mark.parametrize("nirrep", [1, 4, 8])
def test_grcpsd_ground_matches_oracle(nirrep):
    """grCPS(D) (src/grCPSd.SF): the three orders' (T1, T2) and E^(2..4)
    against the oracle, the same DIIS iteration counts."""
    s = small(nirrep) if nirrep < 8 else synth.System(nmo=24, nocc_a=4, nocc_b=2, nirrep=8, seed=3)
    s.run_opts["diis_max_err"] = 1e-10
    ints, sc, par, orc = _run_both(s)
    g = api.grcpsd_ground(s, sc, ints, par)
    og = orc.grcpsd()
    np.testing.assert_allclose(g["E"], og["E"], rtol=0, atol=1e-11)
    for k in range(3):
        np.testing.assert_allclose(host(g["T1"][k]), og["T1"][k], rtol=0, atol=1e-9, err_msg=str(k))
        np.testing.assert_allclose(host(g["T2"][k]), og["T2"][k], rtol=0, atol=1e-9, err_msg=str(k))
    assert g["iters"] == og["iters"]


@pytest.mark.parametrize("nirrep", [1, 2, 4])
def test_eegrcpsd_matches_oracle(nirrep):
    """EE-grCPS(D) (src/EE-grCPSd.SF): the device chain CIS(D-infinity) ->
    grCPS(D) -> left vectors and w^(1..3) against the oracle's, every loop
    converged tightly (Davidson 1e-12, DIIS 1e-11)."""
    s = synth.System(nmo=10 if nirrep < 4 else 14, nocc_a=3, nocc_b=1, nirrep=nirrep, seed=7, roots=2)
    s.run_opts.update(lowest=1, davidson_conv=12, diis_max_err=1e-11, diis_cyc=400)
    ints, sc, par, orc = _run_both(s)
    om, R0, _ = api.cisdoo_run(s, sc, ints, par)
    g = api.grcpsd_ground(s, sc, ints, par)
    e = api.eegrcpsd_roots(s, sc, ints, par, g, om, R0)
    oom, oR0, _ = orc.cisdoo()
    og = orc.grcpsd()
    oe = orc.eegrcpsd(og, oom, oR0)
    np.testing.assert_allclose(om, oom, rtol=0, atol=1e-10)
    np.testing.assert_allclose(e["w"], oe["w"], rtol=0, atol=1e-8)
    # vectors up to the sign of each root's R0 (and so of L, R^(1), R^(2))
    Rg, L, R1, R2 = host(R0), host(e["L"]), host(e["R1"]), host(e["R2"])
    off = 0
    for h in range(8):
        n = s.r1_len(h + 1) + s.r2_len(h + 1)
        for _ in range(int(s.estate_sym[h])):
            sl = slice(off, off + n)
            sg = np.sign(np.dot(Rg[sl], oR0[sl]))
            np.testing.assert_allclose(sg * L[sl], oe["L"][sl], rtol=0, atol=1e-7)
            np.testing.assert_allclose(sg * R1[sl], oe["R1"][sl], rtol=0, atol=1e-7)
            np.testing.assert_allclose(sg * R2[sl], oe["R2"][sl], rtol=0, atol=1e-7)
            off += n
    assert np.all(np.abs(e["w"]) > 1e-7)


@pytest.mark.parametrize("batch", [0, 1])
@pytest.mark.parametrize("nirrep", [1, 4])
def test_eecpsd_roots_match_oracle(nirrep, batch):
    s = small(nirrep, roots=3)
    ints, sc, par, orc = _run_both(s, batch_roots=batch)
    om, R, _ = api.cis_run(s, sc, ints, par)
    g = api.ground(s, sc, ints, par)
    J, js = api.calJ(s, sc, ints, g)
    w, outs, it = api.eecpsd_roots(s, sc, ints, par, g, js, 1, om, R, want_vectors=True)
    og = orc.ground()
    oJ = orc.jints(og)
    oom, oR, _ = orc.cis()
    l1, l2 = s.r1_len(1), s.r2_len(1)
    Rg = host(R)
    for k in range(len(om)):
        L = Rg[k * l1:(k + 1) * l1]
        r = orc.root(og, oJ, 1, om[k], L)
        np.testing.assert_allclose(w[k], r["w"], rtol=0, atol=TOL_E)
        np.testing.assert_allclose(host(outs["R2_1"])[k * l2:(k + 1) * l2], r["R2_1"], rtol=0, atol=1e-11)
        np.testing.assert_allclose(host(outs["R2_2"])[k * l2:(k + 1) * l2], r["R2_2"], rtol=0, atol=1e-10)
        np.testing.assert_allclose(host(outs["R1_2"])[k * l1:(k + 1) * l1], r["R1_2"], rtol=0, atol=1e-6)
        assert abs(np.dot(L, host(outs["R1_2"])[k * l1:(k + 1) * l1])) < 1e-10


@pytest.mark.parametrize("batch", [0, 1])
def test_pipeline_c2v_nmo48(batch):
    """The plain-FP64 configuration (C2v, nmo 48, nocc 5/3, 3 roots)."""
    s = synth.make("c2v_nmo48")
    ints, sc, par, orc = _run_both(s, batch_roots=batch)
    om, w2, w3 = api.pipeline(s, sc, ints, par)
    oom, ow2, ow3 = orc.pipeline()
    np.testing.assert_allclose(om, oom, rtol=0, atol=TOL_E)
    np.testing.assert_allclose(w2, ow2, rtol=0, atol=TOL_E)
    np.testing.assert_allclose(w3, ow3, rtol=0, atol=TOL_E)


def test_full_size_d2h_nmo200_properties():
    """The precision-form shapes (D2h, nmo 200, nocc 10/8, 5 roots): checks
    that need no full-size oracle run — Davidson eigen residual, batched vs
    per-root identity, <L|R1^(2)> = 0 — plus one root of the oracle on the
    same inputs."""
    s = synth.make("d2h_nmo200")
    api.init(s.nirrep, s.dirprd)
    ints = api.DeviceIntegrals(s)
    sc = api.make_system(s)
    par1 = api.make_params(s, batch_roots=1)
    om, R, it = api.cis_run(s, sc, ints, par1)
    l1 = s.r1_len(1)
    # eigen residual with the library's own sigma: AR = e(a,i) R + V R
    Rg = R.view(len(om), l1)
    z = np.array([1, 0, 0, 0, 0, 0, 0, 0])
    for k in range(len(om)):
        AR = torch.zeros(l1, dtype=torch.float64, device="cuda")
        api.kernel("c1_r1iabj", api.opt([s.popv, s.popo, z, z], (1, 1), 1, AR),
                   api.opt([s.popv, s.popo, z, z], (1, 1), 1, Rg[k].contiguous()),
                   api.opt([s.popv, s.popo, s.popv, s.popo], (1, 1), 1, ints.t["iabj"]), 1.0)
        oed = np.zeros(l1)
        of.set_symmetry(s.nirrep, s.dirprd)
        of.lib().o_eorb_diff1(of.ptr(oed), of.ptr(s.eorb), of.arr8(s.popv), of.arr8(s.popo), of.I64(1))
        r = host(Rg[k])
        res = host(AR) + oed * r - om[k] * r
        assert np.max(np.abs(res)) < 1e-8
        assert abs(np.linalg.norm(r) - 1.0) < 1e-10
    g = api.ground(s, sc, ints, par1)
    J, js = api.calJ(s, sc, ints, g)
    wb, ob, itb = api.eecpsd_roots(s, sc, ints, par1, g, js, 1, om, R, want_vectors=True)
    par0 = api.make_params(s, batch_roots=0)
    # one root per batch: the order-3 solves still run for all roots at once
    wu, ou, itu = api.eecpsd_roots(s, sc, ints, par0, g, js, 1, om, R, want_vectors=True)
    np.testing.assert_allclose(wb, wu, rtol=0, atol=1e-12)
    assert itb == itu
    for key in ("R2_1", "R2_2"):
        a, b = host(ob[key]), host(ou[key])
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * max(1.0, np.abs(a).max()))
    # R1^(2) is DIIS-converged (diis_max_err): rounding-level differences in
    # its right-hand side move it within that tolerance, relative to its size
    a, b = host(ob["R1_2"]), host(ou["R1_2"])
    np.testing.assert_allclose(a, b, rtol=0, atol=1e-6 * max(1.0, np.abs(a).max()))
    R12 = host(ob["R1_2"]).reshape(len(om), l1)
    for k in range(len(om)):
        assert abs(np.dot(host(Rg[k]), R12[k])) < 1e-10
    assert np.all(np.isfinite(wb))
    # oracle on the first root (same integrals / CIS vector / ground T)
    orc = of.Oracle(s, nthreads=8)
    og = dict(T2_1=host(g["T2_1"]), T1_2=host(g["T1_2"]), T2_2=host(g["T2_2"]))
    oJ = {k: host(v) for k, v in J.items()}
    r = orc.root(og, oJ, 1, om[0], host(Rg[0]))
    np.testing.assert_allclose(wb[0], r["w"], rtol=0, atol=TOL_E)


@pytest.mark.parametrize("digits", [0, 5])
def test_d2h_nmo200_every_root_matches_oracle(digits):
    """The precision-form workload (D2h, nmo 200, nocc 10/8, 5 roots),
    every root against the oracle's whole pipeline on the same inputs: the
    FP64 path to 1e-9 Eh in each of w0, w^(2), w^(3); the mixed path (5
    int8 digits on the tensor cores) to 1 micro-Eh, with the per-root
    errors printed."""
    import os
    s = synth.make("d2h_nmo200")
    api.init(s.nirrep, s.dirprd)
    ints = api.DeviceIntegrals(s)
    sc, par = api.make_system(s), api.make_params(s, batch_roots=1)
    api.set_mixed(digits, 1.0)
    try:
        om, w2, w3 = api.pipeline(s, sc, ints, par)
        assert api.mixed_error() == 0
    finally:
        api.set_mixed(0)
    oom, ow2, ow3 = of.Oracle(s, nthreads=os.cpu_count() or 1).pipeline()
    tol = TOL_E if digits == 0 else 1e-6
    err = np.abs(np.stack([om - oom, w2 - ow2, w3 - ow3]))
    print(f"digits={digits} per-root |gpu - oracle| (w0, w2, w3 rows):\n{err}")
    assert len(om) == 5
    assert err.max() < tol, err
