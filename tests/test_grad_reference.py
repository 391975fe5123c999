"""The FP64 reference gradient of the SF-CIS(D) energies (dense torch
autograd, tests/dense_grad.py) pinned against the oracle: its energies equal
the oracle pipeline's w0 / w^(2), and its directional derivatives equal
central finite differences of the oracle pipeline along seeded integral-
perturbation directions (the DPD images of moves of the generator's (pq|rs)
factor L and of the orbital energies, step 1e-5)."""
import numpy as np
import pytest
import torch

import dense_grad as dg
import oracle_ffi as of
from cpsd_b200 import synth

TIGHT = dict(davidson_conv=12, davidson_cyc=100, diis_max_err=1e-12, diis_cyc=200)
CASES = [
    dict(nmo=14, nocc_a=4, nocc_b=2, nirrep=2, seed=3, roots={1: 2, 2: 1}),
    dict(nmo=12, nocc_a=3, nocc_b=1, nirrep=1, seed=4, roots={1: 2}),
    dict(nmo=16, nocc_a=4, nocc_b=2, nirrep=4, seed=6, roots={1: 1, 3: 1}),
]


def oracle_run(s):
    of.set_symmetry(s.nirrep, s.dirprd)
    o = of.Oracle(s, **TIGHT)
    om, R, _ = o.cis()
    w0, w2, _ = o.pipeline()
    assert np.allclose(om, w0, rtol=0, atol=1e-13)
    return w0, w2, R


def roots_of(s, R):
    """(symR, root index in irrep, global root index, packed L) of every root"""
    off = k = 0
    for symR in range(1, s.nirrep + 1):
        n, l1 = int(s.estate_sym[symR - 1]), s.r1_len(symR)
        for r in range(n):
            yield symR, r, k, R[off + r * l1: off + (r + 1) * l1]
            k += 1
        off += n * l1


@pytest.mark.parametrize("case", range(len(CASES)))
def test_dense_energies_match_oracle(case):
    s = synth.System(**CASES[case])
    w0, w2, R = oracle_run(s)
    for symR, r, k, L0 in roots_of(s, R):
        ref = dg.DenseCisd(s, symR)
        ints = {key: torch.tensor(s.ints[key]) for key in ref.LAYOUTS}
        a, b, L = ref.energies(ints, torch.tensor(s.eorb), L0, w0[k])
        assert abs(float(a) - w0[k]) < 1e-12
        assert abs(float(b) - w2[k]) < 1e-12
        assert np.abs(np.abs(L.numpy()) - np.abs(L0)).max() < 1e-10


@pytest.mark.parametrize("case", range(len(CASES)))
def test_reference_gradient_matches_oracle_fd(case):
    s = synth.System(**CASES[case])
    w0, w2, R = oracle_run(s)
    rng = np.random.default_rng(100 + case)
    h = 1e-5
    for symR, r, k, L0 in roots_of(s, R):
        ref = dg.DenseCisd(s, symR)
        g0, g2 = rng.uniform(0.5, 1.5, 2)
        G, _, _ = ref.gradient(s, L0, w0[k], g0, g2)
        for _ in range(2):
            d = s.integral_direction(*s.input_direction(rng))
            pred = sum(float(np.dot(G[key], d[key])) for key in G)
            vals = []
            for ints, eo in (dg.shifted(s, d, h), dg.shifted(s, d, -h)):
                saved = s.ints, s.eorb
                s.ints, s.eorb = ints, eo
                try:
                    a, b = oracle_run(s)[:2]
                finally:
                    s.ints, s.eorb = saved
                vals.append(g0 * a[k] + g2 * b[k])
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(pred - fd) <= 1e-7 * abs(fd) + 1e-10, (symR, r, pred, fd)


def oracle_run3(s):
    of.set_symmetry(s.nirrep, s.dirprd)
    o = of.Oracle(s, **TIGHT)
    _, R, _ = o.cis()
    w0, w2, w3 = o.pipeline()
    return w0, w2, w3, R


CASES3 = [
    dict(nmo=12, nocc_a=3, nocc_b=1, nirrep=1, seed=4, roots={1: 2}),
    dict(nmo=14, nocc_a=4, nocc_b=2, nirrep=2, seed=3, roots={1: 1, 2: 1}),
]


@pytest.mark.parametrize("case", range(len(CASES3)))
def test_dense_order3_matches_oracle(case):
    """the dense w^(3) chain (DenseCpsd3) gives the oracle pipeline's w0, w^(2), w^(3)"""
    s = synth.System(**CASES3[case])
    w0, w2, w3, R = oracle_run3(s)
    for symR, r, k, L0 in roots_of(s, R):
        ref = dg.DenseCpsd3(s, symR)
        ints = {key: torch.tensor(s.ints[key]) for key in ref.LAYOUTS}
        a, b, c, _ = ref.energies3(ints, torch.tensor(s.eorb), L0, w0[k])
        assert abs(float(a) - w0[k]) < 1e-12
        assert abs(float(b) - w2[k]) < 1e-12
        assert abs(float(c) - w3[k]) < 1e-11 * max(1.0, abs(w3[k])), (float(c), w3[k])


@pytest.mark.parametrize("case", range(len(CASES3)))
def test_reference_order3_gradient_matches_oracle_fd(case):
    """its autograd gradient of g0 w0 + g2 w2 + g3 w3 (all six lists and
    Eorb) equals central finite differences of the oracle pipeline"""
    s = synth.System(**CASES3[case])
    w0, w2, w3, R = oracle_run3(s)
    rng = np.random.default_rng(200 + case)
    h = 1e-5
    for symR, r, k, L0 in roots_of(s, R):
        ref = dg.DenseCpsd3(s, symR)
        g0, g2, g3 = rng.uniform(0.5, 1.5, 3)
        G, _, _, _ = ref.gradient3(s, L0, w0[k], g0, g2, g3)
        assert set(G) == {"ijkl", "ijka", "abij", "iabj", "abci", "abcd", "eorb"}
        d = s.integral_direction(*s.input_direction(rng))
        pred = sum(float(np.dot(G[key], d[key])) for key in G)
        vals = []
        for ints, eo in (dg.shifted(s, d, h), dg.shifted(s, d, -h)):
            saved = s.ints, s.eorb
            s.ints, s.eorb = ints, eo
            try:
                a, b, c = oracle_run3(s)[:3]
            finally:
                s.ints, s.eorb = saved
            vals.append(g0 * a[k] + g2 * b[k] + g3 * c[k])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(pred - fd) <= 1e-7 * abs(fd) + 1e-10, (symR, r, pred, fd)
