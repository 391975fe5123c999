"""GPU parity of the independent-molecule batch (cpsd_pipeline_batch).

Molecules drawn like the batching workload (nocc_beta = nocc_alpha - 2,
irrep count from {1, 2, 4, 8}, 4-8 roots each) at sizes the oracle finishes
quickly run concurrently on several worker streams; every molecule's
energies must equal the single-molecule pipeline's (FP64 and the int8-digit
mixed mode), and two of them are checked against the oracle."""
import numpy as np
import pytest

import oracle_ffi as of
from cpsd_b200 import api, synth

pytestmark = pytest.mark.gpu


def molecules(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nirrep = int(rng.choice([1, 2, 4, 8]))
        nmo = int(rng.integers(24, 49))
        na = int(rng.integers(4, 8))
        roots = int(rng.integers(4, 9))
        out.append(synth.System(nmo=nmo, nocc_a=na, nocc_b=na - 2, nirrep=nirrep, seed=int(rng.integers(1 << 30)),
                                roots=roots))
    return out


@pytest.mark.parametrize("digits", [0, 5])
def test_batch_equals_single_molecule_runs(digits):
    mols = molecules(10, 42)
    ints = [api.DeviceIntegrals(s) for s in mols]
    pars = [api.make_params(s) for s in mols]
    # digit path for contractions of at least 10 MFLOP that pass its padding
    # and K filters (the production routing rule at a lower threshold)
    api.set_mixed(digits, 0.01 if digits else 1.0)
    try:
        single = [api.pipeline(s, api.make_system(s), d, p) for s, d, p in zip(mols, ints, pars)]
        for workers in (1, 4):
            batch = api.pipeline_batch(mols, ints, pars, nworkers=workers)
            for (a0, a2, a3), (b0, b2, b3) in zip(single, batch):
                assert len(a0) == len(b0)
                assert np.abs(a0 - b0).max() < 1e-12
                assert np.abs(a2 - b2).max() < 1e-12
                assert np.abs(a3 - b3).max() < 1e-12
    finally:
        api.set_mixed(0)


def test_batch_matches_oracle():
    mols = molecules(6, 7)
    ints = [api.DeviceIntegrals(s) for s in mols]
    pars = [api.make_params(s) for s in mols]
    batch = api.pipeline_batch(mols, ints, pars, nworkers=3)
    for s, (om, w2, w3) in list(zip(mols, batch))[:2]:
        of.set_symmetry(s.nirrep, s.dirprd)
        o0, o2, o3 = of.Oracle(s).pipeline()
        assert np.abs(om - o0).max() < 1e-9
        assert np.abs(w2 - o2).max() < 1e-9
        assert np.abs(w3 - o3).max() < 1e-9
