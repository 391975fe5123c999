"""The pipeline fed from the reference's input files: the interface node
file and the six spin-free integral lists of a run directory (written for
the plain-FP64 configuration, C2v nmo 48), read by cpsd_load_system /
cpsd_load_inputs and run through cpsd_pipeline; the energies equal the
oracle's on the generator's arrays to 1e-9 Eh and the GPU run on those
arrays bit for bit."""
import numpy as np
import pytest

import oracle_ffi as of
from cpsd_b200 import api, synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_pipeline_from_reference_files(tmp_path):
    api.use_torch_stream()
    s = synth.make("c2v_nmo48")
    ipath = str(tmp_path / "interface")
    api.write_inputs(str(tmp_path), ipath, s)
    sc = api.load_system(ipath)
    host = api.load_inputs(str(tmp_path), ipath, sc, s.lengths(), len(s.eorb))
    ints = api.DeviceIntegrals.from_tensors({k: torch.from_numpy(v).cuda() for k, v in host.items()})
    par = api.make_params(s)
    om, w2, w3 = api.pipeline(s, sc, ints, par)
    ref = api.pipeline(s, api.make_system(s), api.DeviceIntegrals(s), par)
    for a, b in zip((om, w2, w3), ref):
        np.testing.assert_array_equal(a, b)
    oom, ow2, ow3 = of.Oracle(s).pipeline()
    np.testing.assert_allclose(om, oom, rtol=0, atol=1e-9)
    np.testing.assert_allclose(w2, ow2, rtol=0, atol=1e-9)
    np.testing.assert_allclose(w3, ow3, rtol=0, atol=1e-9)
