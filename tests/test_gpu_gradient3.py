"""GPU parity of the third-order EE-CPS(D-3) energies and their adjoint
gradient (cpsd_cpsd3_energies / cpsd_cpsd3_gradient):

* the energies equal those of the full pipeline (cpsd_pipeline) and of the
  oracle;
* the gradient of g0.w0 + g2.w^(2) + g3.w^(3) with respect to all six DPD
  lists and Eorb equals, element by element, the FP64 reference gradient of
  tests/dense_grad.py (torch autograd of the dense order-3 chain, itself
  pinned to oracle finite differences in test_grad_reference.py);
* chained through cpsd_eri_adjoint at the differentiation workload (C2v,
  nmo 120, nocc 8/6, 4 roots; the lists built on the device from a dense
  (pq|rs)), its directional derivatives equal central finite differences of
  the device energies along seeded random (pq|rs) directions with the
  integrals' 8-fold symmetry, within 1e-6 relative;
* the torch.autograd.Function wrapper returns the same gradient.
"""
import numpy as np
import pytest
import torch

import dense_grad as dg
import oracle_ffi as of
from cpsd_b200 import api, autograd, synth

pytestmark = pytest.mark.gpu

TIGHT = dict(davidson_conv=12, davidson_cyc=100, diis_max_err=1e-12, diis_cyc=200)
LISTS = ("ijkl", "ijka", "abij", "iabj", "abci", "abcd")
KEYS = LISTS + ("eorb",)


def device_tensors(s):
    t = {k: torch.from_numpy(s.ints[k]).cuda() for k in LISTS}
    t["eorb"] = torch.from_numpy(s.eorb).cuda()
    return t


def energies(s, symR, nroot, t=None):
    t = device_tensors(s) if t is None else t
    par = api.make_params(s, **TIGHT)
    w0, w2, w3, L = api.cpsd3_energies(s, api.make_system(s), api.integrals_struct(t), par, symR, nroot)
    return w0, w2, w3, L, t, par


def gradient(s, symR, w0, L, t, par, g0, g2, g3):
    grads = {k: torch.zeros_like(v) for k, v in t.items()}
    api.cpsd3_gradient(api.make_system(s), api.integrals_struct(t), par, symR, w0, L, g0, g2, g3, grads)
    return grads


def test_energies_match_pipeline_and_oracle():
    s = synth.make("c2v_nmo48")
    ints = api.DeviceIntegrals(s)
    par = api.make_params(s, **TIGHT)
    om, w2p, w3p = api.pipeline(s, api.make_system(s), ints, par)
    w0, w2, w3 = energies(s, 1, s.nroots)[:3]
    assert np.abs(w0 - om).max() < 1e-12
    assert np.abs(w2 - w2p).max() < 1e-12
    assert np.abs(w3 - w3p).max() < 1e-11
    of.set_symmetry(s.nirrep, s.dirprd)
    o0, o2, o3 = of.Oracle(s, **TIGHT).pipeline()
    assert np.abs(w0 - o0).max() < 1e-9 and np.abs(w2 - o2).max() < 1e-9 and np.abs(w3 - o3).max() < 1e-9


CASES = [
    (dict(nmo=12, nocc_a=3, nocc_b=1, nirrep=1, seed=4), 1, 2),
    (dict(nmo=14, nocc_a=4, nocc_b=2, nirrep=2, seed=3), 2, 1),
    (dict(nmo=20, nocc_a=5, nocc_b=3, nirrep=4, seed=7), 1, 2),
    (dict(nmo=20, nocc_a=5, nocc_b=3, nirrep=4, seed=7), 3, 1),
    (dict(nmo=24, nocc_a=5, nocc_b=3, nirrep=8, seed=8), 2, 1),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_gradient_matches_reference(case):
    kw, symR, nroot = CASES[case]
    s = synth.System(roots={symR: nroot}, **kw)
    w0, w2, w3, L, t, par = energies(s, symR, nroot)
    rng = np.random.default_rng(case)
    g0, g2, g3 = (rng.uniform(0.5, 1.5, nroot) for _ in range(3))
    G = {k: v.cpu().numpy() for k, v in gradient(s, symR, w0, L, t, par, g0, g2, g3).items()}
    ref = dg.DenseCpsd3(s, symR)
    l1 = s.r1_len(symR)
    Lh = L.cpu().numpy()
    R = {k: 0.0 for k in KEYS}
    for r in range(nroot):
        Gr, a, b, c = ref.gradient3(s, Lh[r * l1:(r + 1) * l1], w0[r], g0[r], g2[r], g3[r])
        assert abs(a - w0[r]) < 1e-11 and abs(b - w2[r]) < 1e-11 and abs(c - w3[r]) < 1e-11
        for k in KEYS:
            R[k] = R[k] + Gr[k]
    for k in KEYS:
        scale = np.abs(R[k]).max()
        assert np.abs(G[k] - R[k]).max() <= 1e-8 * scale + 1e-13, (k, np.abs(G[k] - R[k]).max(), scale)


def test_gradient_wrt_eri_fd_c2v_nmo120():
    s = synth.System(nmo=120, nocc_a=8, nocc_b=6, nirrep=4, roots={1: 4}, seed=0, skip_abcd=True, host_ints=False)
    api.init(s.nirrep, s.dirprd)
    n, symR, nroot = s.nmo, 1, 4
    Lf = torch.from_numpy(s.L).cuda()
    eri0 = torch.einsum("Ppr,Pqs->prqs", Lf, Lf).contiguous().reshape(-1)
    del Lf
    eorb = torch.from_numpy(s.eorb).cuda()
    mo, sp = api.orbital_map(s)
    lens = s.lengths()

    def lists_of(e):
        out = {k: torch.zeros(lens[k], dtype=torch.float64, device="cuda") for k in LISTS}
        api.eri_lists(api.make_system(s), mo, sp, n, e, out)
        out["eorb"] = eorb
        return out

    w0, w2, w3, L, t, par = energies(s, symR, nroot, t=lists_of(eri0))
    rng = np.random.default_rng(12)
    g0, g2, g3 = (rng.uniform(0.5, 1.5, nroot) for _ in range(3))
    grads = gradient(s, symR, w0, L, t, par, g0, g2, g3)
    del t
    G = torch.zeros(n ** 4, dtype=torch.float64, device="cuda")
    api.eri_adjoint(api.make_system(s), mo, sp, n, {k: grads[k] for k in LISTS}, G)
    del grads
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7)
    h = 1e-5
    for trial in range(2):
        D = torch.randn((n, n, n, n), generator=gen, dtype=torch.float64, device="cuda")
        D = D + D.permute(1, 0, 2, 3)
        D = D + D.permute(0, 1, 3, 2)
        D = D + D.permute(2, 3, 0, 1)
        D = (D / D.abs().max()).reshape(-1)
        vals = []
        for sgn in (1.0, -1.0):
            a, b, c = energies(s, symR, nroot, t=lists_of(eri0 + sgn * h * D))[:3]
            vals.append(np.dot(g0, a) + np.dot(g2, b) + np.dot(g3, c))
        fd = (vals[0] - vals[1]) / (2 * h)
        an = float(torch.dot(G, D))
        del D
        assert abs(fd - an) < 1e-6 * abs(an), (trial, fd, an)


def test_autograd_function():
    s = synth.System(nmo=16, nocc_a=4, nocc_b=2, nirrep=2, seed=5, roots={1: 2})
    t = device_tensors(s)
    leaves = {k: v.clone().requires_grad_(True) for k, v in t.items()}
    w0, w2, w3 = autograd.cpsd3_energies(s, leaves, 1, 2, **TIGHT)
    (w0.sum() + 2.0 * w2.sum() + 3.0 * w3.sum()).backward()
    a, b, c, L, _, par = energies(s, 1, 2, t=t)
    G = gradient(s, 1, a, L, t, par, np.ones(2), 2.0 * np.ones(2), 3.0 * np.ones(2))
    for k in KEYS:
        g = G[k].cpu().numpy()
        assert np.abs(leaves[k].grad.cpu().numpy() - g).max() <= 1e-12 * (np.abs(g).max() + 1)
