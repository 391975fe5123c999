"""CPU oracle pipeline (SF-CIS Davidson, ground CPS(D), J^(2)/J^(3),
EE-CPS(D-3) per root) against the dense numpy equations."""
import numpy as np
import pytest

import dense
import dense_pipeline as dp
import oracle_ffi as of
from cpsd_b200 import synth


def small(nirrep, seed=5, roots=2):
    return synth.System(nmo=14 if nirrep <= 2 else 16, nocc_a=3, nocc_b=1, nirrep=nirrep, seed=seed, roots=roots)


def vo_dense(s, vec, symR):
    z = np.array([1, 0, 0, 0, 0, 0, 0, 0])
    return dense.dpd_to_dense(vec, s.sym, [s.popv, s.popo, z, z], (1, 1), symR)[:, :, 0, 0]


def vvoo_dense(s, vec, symR):
    return dense.dpd_to_dense(vec, s.sym, [s.popv, s.popv, s.popo, s.popo], (0, 0), symR)


@pytest.mark.parametrize("lowest", [0, 1])
@pytest.mark.parametrize("nirrep", [1, 2, 4])
def test_cis_matches_dense_diagonalisation(nirrep, lowest):
    s = small(nirrep)
    orc = of.Oracle(s, lowest=lowest)
    om, R, it = orc.cis()
    ds = dp.DenseSystem(s)
    A, idx = ds.cis_matrix(1, spin_flip=True)
    ev = np.linalg.eigvalsh(0.5 * (A + A.T))
    if lowest:
        np.testing.assert_allclose(om, ev[:len(om)], atol=1e-9)
    else:
        # default root tracking (mod_davidson.f90:227-251) follows the
        # eigenvector of largest overlap with each initial guess: every
        # root is an eigenvalue, not necessarily one of the lowest
        for w in om:
            assert np.min(np.abs(ev - w)) < 1e-9
    # Davidson self-test (src/lib_cc/mod_davidson.f90:525-542): |AR - wR|_inf < 1e-8
    l1 = s.r1_len(1)
    for k in range(len(om)):
        r = vo_dense(s, R[k * l1:(k + 1) * l1], 1)
        x = r[idx[:, 0], idx[:, 1]]
        assert abs(np.linalg.norm(x) - 1) < 1e-10
        assert np.max(np.abs(A @ x - om[k] * x)) < 1e-8


@pytest.mark.parametrize("nirrep", [1, 4])
def test_ground_third_order_matches_dense(nirrep):
    """run3.f90: T2^(3) and E^(4) exactly (closed form), T1^(3) to the
    DIIS convergence of its loop; every term of C2^(3) is exercised."""
    s = small(nirrep)
    orc = of.Oracle(s, diis_max_err=1e-12, diis_cyc=200)
    g = orc.ground()
    g3 = orc.ground3(g)
    ds = dp.DenseSystem(s)
    d = ds.ground()
    # the dense third order from the oracle's own (DIIS-converged) T1^(2)
    d3 = ds.ground3(dict(T2_1=d["T2_1"], T1_2=vo_dense(s, g["T1_2"], 1), T2_2=d["T2_2"]))
    np.testing.assert_allclose(vvoo_dense(s, g3["T2_3"], 1), d3["T2_3"], rtol=0, atol=1e-12)
    assert abs(g3["E4"] - d3["E4"]) < 1e-12
    np.testing.assert_allclose(vo_dense(s, g3["T1_3"], 1), d3["T1_3"], rtol=0, atol=1e-10)
    assert abs(g3["E4"]) > 1e-8  # the terms are not trivially zero


@pytest.mark.parametrize("nirrep", [1, 4])
def test_ground_matches_dense(nirrep):
    s = small(nirrep)
    g = of.Oracle(s).ground()
    d = dp.DenseSystem(s).ground()
    assert abs(g["E2"] - d["E2"]) < 1e-12
    assert abs(g["E3"] - d["E3"]) < 1e-12
    np.testing.assert_allclose(vvoo_dense(s, g["T2_1"], 1), d["T2_1"], atol=1e-13)
    np.testing.assert_allclose(vvoo_dense(s, g["T2_2"], 1), d["T2_2"], atol=1e-13)
    # T1^(2) from DIIS converged to 1e-7 (diis_max_err)
    np.testing.assert_allclose(vo_dense(s, g["T1_2"], 1), d["T1_2"], atol=5e-7)


@pytest.mark.parametrize("nirrep", [1, 2, 4])
def test_eecpsd_roots_match_dense(nirrep):
    s = small(nirrep)
    orc = of.Oracle(s)
    om, R, _ = orc.cis()
    g = orc.ground()
    J = orc.jints(g)
    ds = dp.DenseSystem(s)
    # feed the oracle's own T^(2) to the dense J^(3) so only the EE equations are compared
    gd = ds.ground()
    gd["T1_2"] = vo_dense(s, g["T1_2"], 1)
    Jd = ds.jints(gd)
    l1 = s.r1_len(1)
    for k in range(len(om)):
        L = R[k * l1:(k + 1) * l1]
        r = orc.root(g, J, 1, om[k], L)
        d = ds.root(gd, Jd, 1, om[k], vo_dense(s, L, 1))
        assert r["w"][0] == 0.0
        assert abs(r["w"][1] - d["w"][1]) < 1e-11, (r["w"], d["w"])
        assert abs(r["w"][2] - d["w"][2]) < 1e-10, (r["w"], d["w"])
        np.testing.assert_allclose(vvoo_dense(s, r["R2_1"], 1), d["R2_1"], atol=1e-12)
        np.testing.assert_allclose(vvoo_dense(s, r["R2_2"], 1), d["R2_2"], atol=1e-11)
        # R1^(2) from the DIIS solver (residual 1e-7); <L|R1^(2)> = 0
        np.testing.assert_allclose(vo_dense(s, r["R1_2"], 1), d["R1_2"], atol=2e-6)
        assert abs(np.dot(L, r["R1_2"])) < 1e-12


def test_intermediates_match_dense():
    s = small(4)
    orc = of.Oracle(s)
    g = orc.ground()
    J = orc.jints(g)
    ds = dp.DenseSystem(s)
    gd = ds.ground()
    gd["T1_2"] = vo_dense(s, g["T1_2"], 1)
    Jd = ds.jints(gd)
    z = np.array([1, 0, 0, 0, 0, 0, 0, 0])
    o, v, sym = s.popo, s.popv, s.sym
    lay = {"J2_Foo": ([o, o, z, z], (1, 1)), "J2_Fvv": ([v, v, z, z], (1, 1)),
           "J2_Wovvo": ([v, o, v, o], (1, 1)), "J2_Wovoo": ([o, o, o, v], (0, 1)),
           "J3_Foo": ([o, o, z, z], (1, 1)), "J3_Fvv": ([v, v, z, z], (1, 1)),
           "J3_Wovvo": ([v, o, v, o], (1, 1))}
    for k, (pops, iops) in lay.items():
        D = Jd[k]
        if D.ndim == 2:
            D = D[:, :, None, None]
        np.testing.assert_allclose(J[k], dense.dense_to_dpd(D, sym, pops, iops, 1), atol=1e-12, err_msg=k)


@pytest.mark.parametrize("nirrep", [1, 4])
def test_cisdoo_matches_dense_eigenvalues(nirrep):
    """CIS(D-infinity): the (R1, R2) sigma is not symmetric (Fac, Fki and
    Wkaci carry the MP2 amplitudes); the oracle's lowest roots are the
    lowest eigenvalues of the dense operator on the spin-flip sector and
    each returned vector satisfies the Davidson self-test."""
    s = synth.System(nmo=10, nocc_a=3, nocc_b=1, nirrep=nirrep, seed=7, roots=2)
    orc = of.Oracle(s, lowest=1, davidson_conv=10)
    om, R, it = orc.cisdoo()
    ds = dp.DenseSystem(s)
    off = 0
    k = 0
    for h in range(8):
        nr = int(s.estate_sym[h])
        if nr == 0:
            continue
        A, dms = ds.cisdoo_matrix(h + 1)
        assert np.max(np.abs(A - A.T)) > 1e-6  # the operator is not symmetric
        sel = np.flatnonzero(dms == 1)
        ev = np.linalg.eigvals(A[np.ix_(sel, sel)])
        assert np.max(np.abs(ev.imag)) < 1e-9
        ev = np.sort(ev.real)
        n = A.shape[0]
        for r in range(nr):
            x = R[off + r * n:off + (r + 1) * n]
            assert abs(np.linalg.norm(x) - 1) < 1e-10
            assert np.max(np.abs(A @ x - om[k + r] * x)) < 1e-8
            assert np.all(x[dms != 1] == 0)
        np.testing.assert_allclose(om[k:k + nr], ev[:nr], rtol=0, atol=1e-9)
        off += nr * n
        k += nr
    assert k == len(om) and k > 0


@pytest.mark.parametrize("nirrep", [1, 4])
def test_grcpsd_ground_matches_dense(nirrep):
    """grCPS(D) (src/grCPSd.SF): every order's coupled (T1, T2) and the
    energies E^(2), E^(3), E^(4) against the exact dense solution; the DIIS
    loops run to 1e-12."""
    s = small(nirrep)
    orc = of.Oracle(s, diis_max_err=1e-12, diis_cyc=300)
    g = orc.grcpsd()
    d = dp.DenseSystem(s).grcpsd()
    for k in range(3):
        np.testing.assert_allclose(vo_dense(s, g["T1"][k], 1), d["T1"][k], rtol=0, atol=1e-9, err_msg=str(k))
        np.testing.assert_allclose(vvoo_dense(s, g["T2"][k], 1), d["T2"][k], rtol=0, atol=1e-9, err_msg=str(k))
    np.testing.assert_allclose(g["E"], d["E"], rtol=0, atol=1e-10)
    assert np.all(np.abs(d["E"]) > 1e-8) and np.abs(d["T1"][0]).max() > 1e-6


@pytest.mark.parametrize("nirrep", [1, 2])
def test_eegrcpsd_matches_dense(nirrep):
    """EE-grCPS(D) (src/EE-grCPSd.SF): the left vector of each CIS(D-infinity)
    root is the left eigenvector of the dense (R1, R2) operator with
    <L|R> = 1, and w^(1), w^(2), w^(3) and R^(1), R^(2) match the dense
    chain solved exactly with <L|R^(n)> = 0; all DIIS loops run to 1e-12."""
    s = synth.System(nmo=10, nocc_a=3, nocc_b=1, nirrep=nirrep, seed=7, roots=2)
    orc = of.Oracle(s, lowest=1, davidson_conv=12, diis_max_err=1e-12, diis_cyc=400)
    om, R0, _ = orc.cisdoo()
    g = orc.grcpsd()
    e = orc.eegrcpsd(g, om, R0)
    ds = dp.DenseSystem(s)
    dg = ds.grcpsd()
    off, k = 0, 0
    for h in range(8):
        for _ in range(int(s.estate_sym[h])):
            n = s.r1_len(h + 1) + s.r2_len(h + 1)
            A, _ = ds.cisdoo_matrix(h + 1)
            R, L = R0[off:off + n], e["L"][off:off + n]
            assert abs(L @ R - 1.0) < 1e-10
            np.testing.assert_allclose(A.T @ L, om[k] * L, rtol=0, atol=1e-8 * np.abs(L).max())
            w, R1, R2 = ds.eegrcpsd(h + 1, om[k], R, L, dg)
            np.testing.assert_allclose(e["w"][k], w, rtol=0, atol=1e-9, err_msg=str(k))
            np.testing.assert_allclose(e["R1"][off:off + n], R1, rtol=0, atol=1e-8)
            np.testing.assert_allclose(e["R2"][off:off + n], R2, rtol=0, atol=1e-8)
            assert np.all(np.abs(w) > 1e-7)
            off += n
            k += 1
    assert k == len(om) > 0
