"""The DPD lists as a function of the spatial integrals (pq|rs) and the
gradient chained back to them (cpsd_eri_lists / cpsd_eri_adjoint):

* the forward map rebuilds the six lists of a synthetic molecule from its
  dense (pq|rs) (the synthetic generator builds them from the same
  integrals by its own code);
* the adjoint is the transpose of the forward map: <adj(g), D> = <g, fwd(D)>
  for random g and D;
* d(g0.w0 + g2.w^(2))/d(pq|rs) (cpsd_cisd_gradient chained through the
  adjoint) matches central finite differences of the device energies along
  seeded (pq|rs) directions.
"""
import numpy as np
import pytest
import torch

from cpsd_b200 import api, synth

pytestmark = pytest.mark.gpu

LISTS = ("ijkl", "ijka", "abij", "iabj", "abci", "abcd")
TIGHT = dict(davidson_conv=12, davidson_cyc=100, diis_max_err=1e-12, diis_cyc=200)


def dense_eri(s):
    return np.einsum("Ppr,Pqs->prqs", s.L, s.L)


def build(s, eri_t):
    mo, sp = api.orbital_map(s)
    out = {k: torch.zeros(len(s.ints[k]), dtype=torch.float64, device="cuda") for k in LISTS}
    api.eri_lists(api.make_system(s), mo, sp, s.nmo, eri_t, out)
    return out


@pytest.mark.parametrize("nirrep", [1, 2, 4, 8])
def test_forward_reproduces_lists(nirrep):
    s = synth.System(nmo=14 if nirrep < 8 else 20, nocc_a=4, nocc_b=2, nirrep=nirrep, seed=4)
    api.init(s.nirrep, s.dirprd)
    eri = torch.from_numpy(dense_eri(s).reshape(-1)).cuda()
    out = build(s, eri)
    for k in LISTS:
        ref = s.ints[k]
        np.testing.assert_allclose(out[k].cpu().numpy(), ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max()),
                                   err_msg=k)


@pytest.mark.parametrize("nirrep", [1, 4])
def test_adjoint_is_transpose(nirrep):
    s = synth.System(nmo=12, nocc_a=3, nocc_b=2, nirrep=nirrep, seed=5)
    api.init(s.nirrep, s.dirprd)
    rng = np.random.default_rng(nirrep)
    n = s.nmo
    D = torch.from_numpy(rng.standard_normal(n ** 4)).cuda()
    fD = build(s, D)
    g = {k: torch.from_numpy(rng.standard_normal(len(s.ints[k]))).cuda() for k in LISTS}
    G = torch.zeros(n ** 4, dtype=torch.float64, device="cuda")
    mo, sp = api.orbital_map(s)
    api.eri_adjoint(api.make_system(s), mo, sp, n, g, G)
    lhs = float(torch.dot(G, D))
    rhs = sum(float(torch.dot(g[k], fD[k])) for k in LISTS)
    assert abs(lhs - rhs) < 1e-10 * max(1.0, abs(rhs))


def energies(s, t, symR, nroot):
    par = api.make_params(s, **TIGHT)
    w0, w2, L = api.cisd_energies(s, api.make_system(s), api.integrals_struct(t), par, symR, nroot)
    return w0, w2, L, par


@pytest.mark.parametrize("nirrep,symR", [(1, 1), (2, 2)])
def test_gradient_wrt_eri_matches_finite_differences(nirrep, symR):
    s = synth.System(nmo=14, nocc_a=4, nocc_b=2, nirrep=nirrep, seed=3, roots={symR: 2})
    api.init(s.nirrep, s.dirprd)
    n = s.nmo
    eri0 = dense_eri(s)
    eorb = torch.from_numpy(s.eorb).cuda()
    mo, sp = api.orbital_map(s)

    def lists_of(e):
        t = build(s, torch.from_numpy(e.reshape(-1)).cuda())
        t["eorb"] = eorb
        return t

    t = lists_of(eri0)
    w0, w2, L, par = energies(s, t, symR, 2)
    rng = np.random.default_rng(9)
    g0, g2 = rng.uniform(0.5, 1.5, 2), rng.uniform(0.5, 1.5, 2)
    grads = {k: torch.zeros_like(t[k]) for k in ("ijka", "abij", "iabj", "abci", "eorb")}
    api.cisd_gradient(api.make_system(s), api.integrals_struct(t), par, symR, w0, L, g0, g2, grads)
    G = torch.zeros(n ** 4, dtype=torch.float64, device="cuda")
    api.eri_adjoint(api.make_system(s), mo, sp, n, {k: grads[k] for k in ("ijka", "abij", "iabj", "abci")}, G)
    Gh = G.cpu().numpy()
    for trial in range(3):
        D = rng.standard_normal((n, n, n, n))
        # a perturbation with the integrals' 8-fold symmetry
        D = D + D.transpose(1, 0, 2, 3)
        D = D + D.transpose(0, 1, 3, 2)
        D = D + D.transpose(2, 3, 0, 1)
        D /= np.abs(D).max()
        h = 1e-5
        wp0, wp2, _, _ = energies(s, lists_of(eri0 + h * D), symR, 2)
        wm0, wm2, _, _ = energies(s, lists_of(eri0 - h * D), symR, 2)
        fd = (np.dot(g0, wp0 - wm0) + np.dot(g2, wp2 - wm2)) / (2 * h)
        an = float(np.dot(Gh, D.reshape(-1)))
        assert abs(fd - an) < 1e-6 * max(abs(an), 1e-8), (trial, fd, an)
