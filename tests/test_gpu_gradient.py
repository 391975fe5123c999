"""GPU parity of the SF-CIS(D) energies and their adjoint gradient.

* cpsd_cisd_energies gives the same w0 / w^(2) as the full EE-CPS(D-3) path
  and the oracle;
* cpsd_cisd_gradient equals, element by element, the FP64 reference gradient
  of tests/dense_grad.py (torch autograd of a dense restatement, itself
  pinned to oracle finite differences in test_grad_reference.py);
* at the differentiation workload (C2v, nmo 120, nocc 8/6, 4 roots) its
  directional derivatives equal central finite differences of the device
  energies (step 1e-5) along seeded integral-perturbation directions within
  1e-6 relative;
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
KEYS = ("ijka", "abij", "iabj", "abci", "eorb")


def device_tensors(s):
    t = {k: torch.from_numpy(s.ints[k]).cuda() for k in KEYS[:4]}
    t["eorb"] = torch.from_numpy(s.eorb).cuda()
    return t


def energies(s, symR, nroot, **kw):
    t = device_tensors(s)
    par = api.make_params(s, **{**TIGHT, **kw})
    w0, w2, L = api.cisd_energies(s, api.make_system(s), api.integrals_struct(t), par, symR, nroot)
    return w0, w2, L, t, par


def gradient(s, symR, w0, L, t, par, g0, g2):
    grads = {k: torch.zeros_like(v) for k, v in t.items()}
    api.cisd_gradient(api.make_system(s), api.integrals_struct(t), par, symR, w0, L, g0, g2, grads)
    return {k: v.cpu().numpy() for k, v in grads.items()}


def test_energies_match_pipeline_and_oracle():
    s = synth.make("c2v_nmo48")
    ints = api.DeviceIntegrals(s)
    par = api.make_params(s, **TIGHT)
    om, w2p, _ = api.pipeline(s, api.make_system(s), ints, par)
    n = s.nroots
    w0, w2, _, _, _ = energies(s, 1, n)
    assert np.abs(w0 - om).max() < 1e-12
    assert np.abs(w2 - w2p).max() < 1e-12
    of.set_symmetry(s.nirrep, s.dirprd)
    o0, o2, _ = of.Oracle(s, **TIGHT).pipeline()
    assert np.abs(w0 - o0).max() < 1e-9 and np.abs(w2 - o2).max() < 1e-9


CASES = [
    (dict(nmo=14, nocc_a=4, nocc_b=2, nirrep=2, seed=3), 1, 2),
    (dict(nmo=14, nocc_a=4, nocc_b=2, nirrep=2, seed=3), 2, 1),
    (dict(nmo=12, nocc_a=3, nocc_b=1, nirrep=1, seed=4), 1, 2),
    (dict(nmo=20, nocc_a=5, nocc_b=3, nirrep=4, seed=7), 1, 2),
    (dict(nmo=20, nocc_a=5, nocc_b=3, nirrep=4, seed=7), 3, 1),
    (dict(nmo=24, nocc_a=5, nocc_b=3, nirrep=8, seed=8), 2, 1),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_gradient_matches_reference(case):
    kw, symR, nroot = CASES[case]
    s = synth.System(roots={symR: nroot}, **kw)
    w0, w2, L, t, par = energies(s, symR, nroot)
    rng = np.random.default_rng(case)
    g0, g2 = rng.uniform(0.5, 1.5, nroot), rng.uniform(0.5, 1.5, nroot)
    G = gradient(s, symR, w0, L, t, par, g0, g2)
    ref = dg.DenseCisd(s, symR)
    l1 = s.r1_len(symR)
    Lh = L.cpu().numpy()
    R = {k: 0.0 for k in KEYS}
    for r in range(nroot):
        Gr, a, b = ref.gradient(s, Lh[r * l1:(r + 1) * l1], w0[r], g0[r], g2[r])
        assert abs(a - w0[r]) < 1e-11 and abs(b - w2[r]) < 1e-11
        for k in KEYS:
            R[k] = R[k] + Gr[k]
    for k in KEYS:
        scale = np.abs(R[k]).max()
        assert np.abs(G[k] - R[k]).max() <= 1e-8 * scale + 1e-13, (k, np.abs(G[k] - R[k]).max(), scale)


def test_gradient_fd_c2v_nmo120():
    s = synth.make("c2v_nmo120", skip_abcd=True)
    symR, nroot = 1, 4
    w0, w2, L, t, par = energies(s, symR, nroot)
    rng = np.random.default_rng(11)
    h = 1e-5
    Gs = []
    for r in range(nroot):
        g = np.zeros(nroot)
        g[r] = 1.0
        Gs.append(gradient(s, symR, w0, L, t, par, g, g))
    worst = 0.0
    for _ in range(3):
        d = s.integral_direction(*s.input_direction(rng))
        vals = []
        for ints, eo in (dg.shifted(s, d, h), dg.shifted(s, d, -h)):
            saved = s.ints, s.eorb
            s.ints, s.eorb = ints, eo
            try:
                a, b = energies(s, symR, nroot)[:2]
            finally:
                s.ints, s.eorb = saved
            vals.append(a + b)
        fd = (vals[0] - vals[1]) / (2 * h)
        for r in range(nroot):
            pred = sum(float(np.dot(Gs[r][k], d[k])) for k in KEYS)
            rel = abs(pred - fd[r]) / abs(fd[r])
            worst = max(worst, rel)
            assert rel < 1e-6, (r, pred, fd[r])


def test_autograd_function():
    s = synth.System(nmo=16, nocc_a=4, nocc_b=2, nirrep=2, seed=5, roots={1: 2})
    t = device_tensors(s)
    leaves = {k: v.clone().requires_grad_(True) for k, v in t.items()}
    w0, w2 = autograd.cisd_energies(s, leaves, 1, 2, **TIGHT)
    (w0.sum() + 2.0 * w2.sum()).backward()
    par = api.make_params(s, **TIGHT)
    a, b, L = api.cisd_energies(s, api.make_system(s), api.integrals_struct(t), par, 1, 2)
    G = gradient(s, 1, a, L, t, par, np.ones(2), 2.0 * np.ones(2))
    for k in KEYS:
        assert np.abs(leaves[k].grad.cpu().numpy() - G[k]).max() <= 1e-12 * (np.abs(G[k]).max() + 1)
