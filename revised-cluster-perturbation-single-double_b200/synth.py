"""Seeded synthetic SF-CIS / SF-CPS(D) inputs.

The reference builds its integrals with PySCF (src/pyscf2cc/py2cc.py:10) and
xgetHF (src/getHF/main.f90:3); neither is available, so this module draws a
synthetic high-spin open-shell reference:

* nmo spatial orbitals, irreps assigned round-robin (MO k -> irrep k % nirrep + 1);
  alpha-occupied for k < nocc_a, beta-occupied for k < nocc_b;
* orbital energies occ ~ U[-1.5, -0.3] Eh and vir ~ U[0.1, 3.0] Eh, sorted,
  drawn independently for alpha and beta (canonical, diagonal Fock);
* (pq|rs) = sum_P L_pq^P L_rs^P, L ~ N(0, 0.05^2), naux = 4 nmo, symmetric in
  pq; aux function P carries irrep P % nirrep + 1 and L_pq^P = 0 unless
  irrep(p) x irrep(q) = irrep(P), so (pq|rs) vanishes wherever the irrep
  product is not A1 and every symmetry-allowed block is populated;
* Gamma(R_y) = A1, so a spin-free irrep equals the spatial irrep.

The antisymmetrised spin-free DPD tensors are assembled by the C routine in
csrc/synth.c.  Draw order (fixed): eps_a occ, eps_a vir, eps_b occ, eps_b vir, L.
"""
import ctypes
import os

import numpy as np

from .dpd import Symmetry, ZORB, xor_dirprd

_HERE = os.path.dirname(os.path.abspath(__file__))
_SYNTH_SO = os.path.join(_HERE, "_build", "libcpsd_synth.so")
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_SYNTH_SO):
            raise RuntimeError(f"synthetic front end not built: {_SYNTH_SO} (run __graft_entry__.build())")
        _lib = ctypes.CDLL(_SYNTH_SO)
        _lib.cpsd_synth_build.restype = ctypes.c_int
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class System:
    """Orbital spaces, symmetry and integrals of one synthetic molecule."""

    def __init__(self, nmo, nocc_a, nocc_b, nirrep, seed=0, naux=None, roots=None,
                 spin_flip=1, skip_abcd=False, run_opts=None, host_ints=True):
        self.nmo, self.nocc_a, self.nocc_b, self.nirrep = int(nmo), int(nocc_a), int(nocc_b), int(nirrep)
        # program keywords of this workload (CCSOINP keys of mod_common.f90)
        self.run_opts = dict(run_opts or {})
        self.seed = int(seed)
        self.naux = int(naux) if naux is not None else 4 * self.nmo
        self.dirprd = xor_dirprd(self.nirrep)
        self.sym = Symmetry(self.nirrep, self.dirprd)
        self.symry = 1
        self.spin_flip = int(spin_flip)
        mo_irrep = np.array([k % self.nirrep + 1 for k in range(self.nmo)], dtype=np.int64)
        self.mo_irrep = mo_irrep
        self.popa = np.zeros(8, np.int64)
        self.popb = np.zeros(8, np.int64)
        self.vrta = np.zeros(8, np.int64)
        self.vrtb = np.zeros(8, np.int64)
        for k in range(self.nmo):
            h = mo_irrep[k] - 1
            if k < self.nocc_a:
                self.popa[h] += 1
            else:
                self.vrta[h] += 1
            if k < self.nocc_b:
                self.popb[h] += 1
            else:
                self.vrtb[h] += 1
        self.popo = self.popa + self.popb
        self.popv = self.vrta + self.vrtb
        rng = np.random.default_rng(self.seed)
        ea = np.concatenate([np.sort(rng.uniform(-1.5, -0.3, self.nocc_a)),
                             np.sort(rng.uniform(0.1, 3.0, self.nmo - self.nocc_a))])
        eb = np.concatenate([np.sort(rng.uniform(-1.5, -0.3, self.nocc_b)),
                             np.sort(rng.uniform(0.1, 3.0, self.nmo - self.nocc_b))])
        self.eps_a, self.eps_b = ea, eb
        L = rng.normal(0.0, 0.05, (self.naux, self.nmo, self.nmo))
        L = np.triu(L) + np.transpose(np.triu(L, 1), (0, 2, 1))
        aux_irrep = np.array([P % self.nirrep + 1 for P in range(self.naux)], dtype=np.int64)
        ip = mo_irrep[:, None] - 1
        iq = mo_irrep[None, :] - 1
        pq_irrep = (ip ^ iq) + 1  # XOR-ordered abelian groups
        mask = pq_irrep[None, :, :] == aux_irrep[:, None, None]
        L = np.where(mask, L, 0.0)
        self.L = np.ascontiguousarray(L)
        self.aux_irrep = aux_irrep
        # roots: dict irrep -> count (estate_sym)
        self.estate_sym = np.zeros(8, np.int64)
        if roots is not None:
            if isinstance(roots, int):
                self.estate_sym[0] = roots
            else:
                for h, n in dict(roots).items():
                    self.estate_sym[int(h) - 1] = int(n)
        self._build(skip_abcd, host_ints)

    # DPD lengths of the integral tensors (iop = 0 on antisymmetric pairs)
    def lengths(self):
        s, o, v = self.sym, self.popo, self.popv
        return {
            "ijkl": s.idsymsoc(1, o, o, 0, o, o, 0),
            "ijka": s.idsymsoc(1, o, o, 0, o, v, 1),
            "abij": s.idsymsoc(1, v, v, 0, o, o, 0),
            "iabj": s.idsymsoc(1, v, o, 1, v, o, 1),
            "abci": s.idsymsoc(1, v, v, 0, v, o, 1),
            "abcd": s.idsymsoc(1, v, v, 0, v, v, 0),
        }

    def _build(self, skip_abcd, host_ints=True):
        lib = _load()
        lens = self.lengths()
        self.ints = {k: np.zeros(n, np.float64) if host_ints else None for k, n in lens.items()}
        if skip_abcd:
            self.ints["abcd"] = None
        self.eorb = np.zeros(int(self.popo.sum() + self.popv.sum()), np.float64)
        popo = np.zeros(8, np.int64)
        popv = np.zeros(8, np.int64)
        rc = lib.cpsd_synth_build(
            ctypes.c_int64(self.nmo), ctypes.c_int64(self.nirrep), _p(self.dirprd), _p(self.mo_irrep),
            ctypes.c_int64(self.nocc_a), ctypes.c_int64(self.nocc_b), _p(self.eps_a), _p(self.eps_b),
            ctypes.c_int64(self.naux), _p(self.aux_irrep), _p(self.L),
            _p(popo), _p(popv), _p(self.eorb),
            _p(self.ints["ijkl"]), _p(self.ints["ijka"]), _p(self.ints["abij"]), _p(self.ints["iabj"]),
            _p(self.ints["abci"]), _p(self.ints["abcd"]))
        if rc != 0:
            raise RuntimeError(f"cpsd_synth_build failed: {rc}")
        assert np.array_equal(popo, self.popo) and np.array_equal(popv, self.popv)

    def input_direction(self, rng):
        """Seeded direction in the generator's inputs that keeps the
        integrals' structure: L' symmetric in pq under the aux-irrep mask of
        L, and orbital-energy moves for eps_a / eps_b."""
        dL = rng.normal(0.0, 0.05, self.L.shape)
        dL = np.triu(dL) + np.transpose(np.triu(dL, 1), (0, 2, 1))
        dL = np.where(self.L != 0, dL, 0.0)
        return dL, rng.normal(0.0, 0.1, self.eps_a.shape), rng.normal(0.0, 0.1, self.eps_b.shape)

    def integral_direction(self, dL, deps_a, deps_b):
        """The direction in the DPD integrals and Eorb of a generator-input
        direction: the integrals are quadratic in L, so with the symmetric
        bilinear form B, ints(L + L') - ints(L - L') = 4 B(L, L') exactly;
        Eorb is linear in the orbital energies.  Returns {name: array}
        (abcd None when it is not built)."""
        L0, ea0, eb0 = self.L, self.eps_a, self.eps_b
        out = []
        try:
            for sgn in (1.0, -1.0):
                self.L = np.ascontiguousarray(L0 + sgn * dL)
                self.eps_a, self.eps_b = ea0 + sgn * deps_a, eb0 + sgn * deps_b
                self._build(self.ints["abcd"] is None)
                out.append(({k: (None if v is None else v.copy()) for k, v in self.ints.items()}, self.eorb.copy()))
        finally:
            self.L, self.eps_a, self.eps_b = L0, ea0, eb0
            self._build(self.ints["abcd"] is None)
        (ip, ep), (im, em) = out
        d = {k: (None if ip[k] is None else 0.5 * (ip[k] - im[k])) for k in ip}
        d["eorb"] = 0.5 * (ep - em)
        return d

    @property
    def nroots(self):
        return int(self.estate_sym.sum())

    def r1_len(self, sym):
        return self.sym.irpdso(sym, self.popv, self.popo, 1)

    def r2_len(self, sym):
        return self.sym.idsymsoc(sym, self.popv, self.popv, 0, self.popo, self.popo, 0)


_SYNTH_DEV_SO = os.path.join(_HERE, "_build", "libcpsd_synth_dev.so")
_dev_lib = None


def device_integrals(s, keys=("ijkl", "ijka", "abij", "iabj", "abci", "abcd"), stream=None):
    """The integral tensors of s built on the current CUDA device (float64
    torch tensors; same values as the host build up to the summation order of
    the (pq|rs) dot products) plus Eorb; for molecules whose integrals are
    too large to assemble on the host (csrc/synth_dev.cu)."""
    global _dev_lib
    import torch
    if _dev_lib is None:
        if not os.path.exists(_SYNTH_DEV_SO):
            raise RuntimeError(f"device generator not built: {_SYNTH_DEV_SO} (run __graft_entry__.build())")
        _dev_lib = ctypes.CDLL(_SYNTH_DEV_SO)
        _dev_lib.cpsd_synth_build_device.restype = ctypes.c_int
    lens = s.lengths()
    out = {k: torch.empty(lens[k], dtype=torch.float64, device="cuda") for k in keys}
    L = torch.from_numpy(s.L).cuda()
    st = stream if stream is not None else torch.cuda.current_stream()

    def ptr(k):
        return ctypes.c_void_p(out[k].data_ptr()) if k in out else None

    rc = _dev_lib.cpsd_synth_build_device(
        ctypes.c_int64(s.nmo), ctypes.c_int64(s.nirrep), _p(s.dirprd), _p(s.mo_irrep), ctypes.c_int64(s.nocc_a),
        ctypes.c_int64(s.nocc_b), ctypes.c_int64(s.naux), _p(s.aux_irrep), ctypes.c_void_p(L.data_ptr()),
        ptr("ijkl"), ptr("ijka"), ptr("abij"), ptr("iabj"), ptr("abci"), ptr("abcd"), ctypes.c_void_p(st.cuda_stream))
    del L
    if rc != 0:
        raise RuntimeError(f"cpsd_synth_build_device failed: {rc}")
    out["eorb"] = torch.from_numpy(s.eorb).cuda()
    return out


# named workloads (shapes of the benchmark configurations).  With these
# random integrals the spin-flip CIS spectrum at nmo >= 200 has roots below
# the guess energies, where the reference's default root tracking
# (mod_davidson.f90:227-251) breaks down; those workloads set the
# reference's `lowest=t` keyword (mod_common.f90:41), which targets the
# lowest roots.
CONFIGS = {
    # plain FP64 SF-CIS + SF-CPS(D), C2v: nmo 48, nocc 5/3, 3 roots
    "c2v_nmo48": dict(nmo=48, nocc_a=5, nocc_b=3, nirrep=4, roots=3),
    # precision form, single molecule, D2h: nmo 200, nocc 10/8, 5 roots
    "d2h_nmo200": dict(nmo=200, nocc_a=10, nocc_b=8, nirrep=8, roots=5, run_opts={"lowest": 1}),
    # differentiation form shapes, C2v: nmo 120, nocc 8/6, 4 roots
    "c2v_nmo120": dict(nmo=120, nocc_a=8, nocc_b=6, nirrep=4, roots=4),
    # large EE run, D2h: nmo 400, nocc 20/18, 10 roots
    "d2h_nmo400": dict(nmo=400, nocc_a=20, nocc_b=18, nirrep=8, roots=10, run_opts={"lowest": 1}),
}


def config_integral_bytes(name):
    """bytes of the six FP64 integral tensors of a named workload (from its
    orbital populations alone, without drawing the integrals)"""
    cfg = CONFIGS[name]
    nmo, na, nb, nirrep = cfg["nmo"], cfg["nocc_a"], cfg["nocc_b"], cfg["nirrep"]
    o = np.zeros(8, np.int64)
    v = np.zeros(8, np.int64)
    for k in range(nmo):
        h = k % nirrep
        o[h] += (k < na) + (k < nb)
        v[h] += (k >= na) + (k >= nb)
    sym = Symmetry(nirrep, xor_dirprd(nirrep))
    n = (sym.idsymsoc(1, o, o, 0, o, o, 0) + sym.idsymsoc(1, o, o, 0, o, v, 1) + sym.idsymsoc(1, v, v, 0, o, o, 0) +
         sym.idsymsoc(1, v, o, 1, v, o, 1) + sym.idsymsoc(1, v, v, 0, v, o, 1) + sym.idsymsoc(1, v, v, 0, v, v, 0))
    return 8 * int(n)


def batch_draw(n=64, seed=0):
    """Shapes of the batching workload: n independent molecules with
    nmo ~ U{60..240}, nocc_alpha ~ U{4..12}, nocc_beta = nocc_alpha - 2,
    irrep count from {1, 2, 4, 8} and 4-8 roots (irrep 1) each; molecule k
    uses generator seed 1000 + k."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nmo = int(rng.integers(60, 241))
        na = int(rng.integers(4, 13))
        nirrep = int(rng.choice([1, 2, 4, 8]))
        roots = int(rng.integers(4, 9))
        out.append(dict(nmo=nmo, nocc_a=na, nocc_b=na - 2, nirrep=nirrep, roots=roots, seed=1000 + k))
    return out


def make(name, seed=0, **kw):
    cfg = dict(CONFIGS[name])
    cfg.update(kw)
    return System(seed=seed, **cfg)
