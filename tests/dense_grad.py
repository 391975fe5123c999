"""FP64 reference gradient of the SF-CIS(D) energies (test infrastructure).

The energies w0 (SF-CIS) and w^(2) (order 2 of src/EE-CPSd.SF/run_order.f90)
are restated densely in torch (float64, CPU) from the packed DPD integral
vectors and Eorb, and differentiated by torch autograd; no hand-written
adjoint is involved.  The packed -> dense expansion is an index scatter with
the pair signs of the DPD layout (tests/dense.py), so autograd returns the
gradient with respect to the packed storage the library differentiates.

The CIS vector is the converged right eigenvector of A(ai,fn) = e(a,i) d +
V(fn,ai) on the irrep's (a,i) space, obtained by shifted inverse iteration
started from a converged root (unrolled, so autograd differentiates the
eigenvector itself, also for perturbations that make A non-symmetric); w0 is
its Rayleigh quotient, which agrees with the eigenvalue to first order.
The dense kernel formulas are those of tests/kernel_specs.py.
"""
import numpy as np
import torch

import dense

T = torch.float64


def _pq(X):
    return X - X.permute(1, 0, 2, 3)


def _rs(X):
    return X - X.permute(0, 1, 3, 2)


class DenseCisd:
    """Dense w0 / w^(2) of the roots of irrep symR of a synth.System."""

    LAYOUTS = {  # tensor -> (pop letters, iops)
        "ijka": ("ooov", (0, 1)),
        "abij": ("vvoo", (0, 0)),
        "iabj": ("vovo", (1, 1)),
        "abci": ("vvvo", (0, 1)),
    }

    def __init__(self, s, symR):
        self.s, self.symR = s, symR
        sym = s.sym
        self.no, self.nv = int(s.popo.sum()), int(s.popv.sum())
        pm = {"o": s.popo, "v": s.popv}
        self.maps = {}
        for k, (letters, iops) in self.LAYOUTS.items():
            pops = [pm[c] for c in letters]
            rows, total = dense.dpd_index_lists(sym, pops, iops, 1)
            self.maps[k] = (torch.from_numpy(rows), total, iops, tuple(int(np.sum(p)) for p in pops))
        z = np.array([1, 0, 0, 0, 0, 0, 0, 0], np.int64)
        rows, self.l1 = dense.dpd_index_lists(sym, [s.popv, s.popo, z, z], (1, 1), symR)
        self.r1_rows = torch.from_numpy(rows)
        irr_o, irr_v = dense.orbital_irreps(s.popo), dense.orbital_irreps(s.popv)
        mask = np.array([[sym.dp(a, i) == symR for i in irr_o] for a in irr_v])
        self.idx = torch.from_numpy(np.argwhere(mask))

    def to_dense(self, key, vec):
        rows, total, iops, shape = self.maps[key]
        assert vec.numel() == total
        o, a, b, c, d = rows.T
        x = vec[o]
        D = torch.zeros(shape, dtype=T)
        D = D.index_put((a, b, c, d), x, accumulate=True)
        if iops[0] == 0:
            D = D.index_put((b, a, c, d), -x, accumulate=True)
        if iops[1] == 0:
            D = D.index_put((a, b, d, c), -x, accumulate=True)
        if iops[0] == 0 and iops[1] == 0:
            D = D.index_put((b, a, d, c), x, accumulate=True)
        return D

    def r1_to_dense(self, vec):
        o, a, b = self.r1_rows.T[:3]
        return torch.zeros((self.nv, self.no), dtype=T).index_put((a, b), vec[o], accumulate=True)

    def r1_to_dpd(self, M):
        o, a, b = self.r1_rows.T[:3]
        out = torch.zeros(self.l1, dtype=T)
        out[o] = M[a, b]
        return out

    def energies(self, ints, eorb, L0, w0_start, iters=4, shift=1e-7):
        """ints: dict of packed torch vectors; eorb: torch vector; L0: packed
        converged CIS vector (start of the inverse iteration); returns
        (w0, w2, L packed)."""
        ijka = self.to_dense("ijka", ints["ijka"])
        abij = self.to_dense("abij", ints["abij"])
        iabj = self.to_dense("iabj", ints["iabj"])
        abci = self.to_dense("abci", ints["abci"])
        eo, ev = eorb[:self.no], eorb[self.no:]
        e1 = ev[:, None] - eo[None, :]
        e2 = ev[:, None, None, None] + ev[None, :, None, None] - eo[None, None, :, None] - eo[None, None, None, :]
        # CIS: A(ai,fn) = V(fn,ai) + e(a,i) on the (a,i) pairs of irrep symR
        a, i = self.idx[:, 0], self.idx[:, 1]
        A = iabj[:, :, a, i][a, i].T + torch.diag(e1[a, i])  # rows (ai), columns (fn)
        x = self.r1_to_dense(torch.as_tensor(L0, dtype=T))[a, i]
        x = x / torch.linalg.norm(x)
        sig = float(w0_start) + shift
        M = A - sig * torch.eye(len(a), dtype=T)
        for _ in range(iters):
            x = torch.linalg.solve(M, x)
            x = x / torch.linalg.norm(x)
        if float(torch.dot(x.detach(), self.r1_to_dense(torch.as_tensor(L0, dtype=T))[a, i])) < 0:
            x = -x
        w0 = torch.dot(x, A @ x)
        L = torch.zeros((self.nv, self.no), dtype=T).index_put((a, i), x)
        # T2^(1) and J^(2) (run1.f90, calJ.f90)
        T2 = -abij / e2
        Foo = 0.5 * torch.einsum("efin,efmn->mi", T2, abij)
        Fvv = -0.5 * torch.einsum("afmn,efmn->ae", T2, abij)
        Wvo = torch.einsum("bfjn,fenm->embj", T2, abij)
        # order 1 / 2 of run_order.f90
        C2 = -_pq(torch.einsum("ijmb,am->abij", ijka, L)) + _rs(torch.einsum("abej,ei->abij", abci, L))
        R2 = -C2 / (e2 - w0)
        C1 = (0.5 * torch.einsum("feam,feim->ai", abci, R2) - 0.5 * torch.einsum("aemn,mnie->ai", R2, ijka)
              + torch.einsum("fn,fnai->ai", L, Wvo) + torch.einsum("ae,ei->ai", Fvv, L)
              - torch.einsum("am,mi->ai", L, Foo))
        w2 = torch.sum(L * C1)
        return w0, w2, self.r1_to_dpd(L.detach())

    def gradient(self, s, L0, w0_start, g0, g2):
        """d(g0 w0 + g2 w2) / d(ijka, abij, iabj, abci, eorb) as numpy vectors."""
        leaves = {k: torch.tensor(s.ints[k], dtype=T, requires_grad=True) for k in self.LAYOUTS}
        eorb = torch.tensor(s.eorb, dtype=T, requires_grad=True)
        w0, w2, _ = self.energies(leaves, eorb, L0, w0_start)
        E = g0 * w0 + g2 * w2
        grads = torch.autograd.grad(E, [leaves[k] for k in self.LAYOUTS] + [eorb])
        out = {k: g.numpy() for k, g in zip(self.LAYOUTS, grads[:4])}
        out["eorb"] = grads[4].numpy()
        return out, float(w0.detach()), float(w2.detach())



def shifted(s, d, h):
    """integrals and Eorb of s moved by h along the DPD direction d"""
    ints = {k: (None if v is None else v + h * d[k]) if k in d else v for k, v in s.ints.items()}
    return ints, s.eorb + h * d["eorb"]


def _e(spec, *ops):
    return torch.einsum(spec, *ops)


# the kernels' dense formulas (tests/kernel_specs.py) on torch tensors:
# name -> fn(a, b, f) with a, b in the kernel's operand order
TK = {
    "c1_r1iabj": lambda r, V, f: f * _e("fn,fnai->ai", r, V),
    "c1_r1Fae": lambda r, F, f: f * _e("ae,ei->ai", F, r),
    "c1_r1Fmi": lambda r, F, f: -f * _e("am,mi->ai", r, F),
    "c1_r2abci": lambda r, V, f: 0.5 * f * _e("feam,feim->ai", V, r),
    "c1_r2ijka": lambda r, V, f: -0.5 * f * _e("aemn,mnie->ai", r, V),
    "c2_r1abci": lambda r, V, f: f * _rs(_e("abej,ei->abij", V, r)),
    "c2_r1ijka": lambda r, V, f: -f * _pq(_e("ijmb,am->abij", V, r)),
    "c2_r2Wmbej": lambda r, W, f: f * _rs(_pq(_e("aeim,embj->abij", r, W))),
    "c2_r2Wmnij": lambda r, W, f: 0.5 * f * _e("abmn,mnij->abij", r, W),
    "c2_r2abcd": lambda r, V, f: 0.5 * f * _e("abef,efij->abij", V, r),
    "c2_r2Fae": lambda r, F, f: f * _pq(_e("aeij,be->abij", r, F)),
    "c2_r2Fmi": lambda r, F, f: -f * _rs(_e("abim,mj->abij", r, F)),
    "Fmi_r2abij": lambda r, V, f: 0.5 * f * _e("efin,efmn->mi", r, V),
    "Fae_r2abij": lambda r, V, f: -0.5 * f * _e("afmn,efmn->ae", r, V),
    "Fmi_r1ijka": lambda r, V, f: f * _e("en,mnie->mi", r, V),
    "Fae_r1abci": lambda r, V, f: f * _e("fm,efam->ae", r, V),
    "Wkbij_r2ijka": lambda r, V, f: f * _pq(_e("klic,bcjl->ijkb", V, r)),
    "Wkbij_r2abci": lambda r, V, f: 0.5 * f * _e("dcbk,cdij->ijkb", V, r),
    "Wmbej_r2abij": lambda r, V, f: 0.5 * f * _e("bfjn,fenm->embj", r, V),
    "Wmbej_r1abci": lambda r, V, f: f * _e("fj,febm->embj", r, V),
    "Wmbej_r1ijka": lambda r, V, f: -f * _e("bn,nmje->embj", r, V),
    "Wmnij_r1ijka": lambda r, V, f: f * _rs(_e("ej,mnie->mnij", r, V)),
}


def K(name, a, b, f=1.0):
    return TK[name](a, b, f)


class DenseCpsd3(DenseCisd):
    """Dense w0 / w^(2) / w^(3) of the roots of irrep symR: the order-3 chain
    of src/EE-CPSd.SF/run_order.f90 (calE_C.f90, calC_JR.f90, calC_VTR.f90)
    with the ground state of src/CPSd.SF/run1.f90 / run2.f90 (T1^(2) by an
    exact dense solve) and calJ.f90's J^(2) / J^(3), all six lists read."""

    LAYOUTS = dict(DenseCisd.LAYOUTS, ijkl=("oooo", (0, 0)), abcd=("vvvv", (0, 0)))

    def __init__(self, s, symR):
        super().__init__(s, symR)
        sym = s.sym
        irr_o, irr_v = dense.orbital_irreps(s.popo), dense.orbital_irreps(s.popv)
        mask = np.array([[sym.dp(a, i) == 1 for i in irr_o] for a in irr_v])
        self.idx1 = torch.from_numpy(np.argwhere(mask))

    def energies3(self, ints, eorb, L0, w0_start, iters=4, shift=1e-7):
        D = {k: self.to_dense(k, ints[k]) for k in self.LAYOUTS}
        ijkl, ijka, abij, iabj, abci, abcd = (D[k] for k in ("ijkl", "ijka", "abij", "iabj", "abci", "abcd"))
        eo, ev = eorb[:self.no], eorb[self.no:]
        e1 = ev[:, None] - eo[None, :]
        e2 = ev[:, None, None, None] + ev[None, :, None, None] - eo[None, None, :, None] - eo[None, None, None, :]
        # SF-CIS root by shifted inverse iteration (as DenseCisd.energies)
        a, i = self.idx[:, 0], self.idx[:, 1]
        A = iabj[:, :, a, i][a, i].T + torch.diag(e1[a, i])
        L0d = self.r1_to_dense(torch.as_tensor(L0, dtype=T))[a, i]
        x = L0d / torch.linalg.norm(L0d)
        M = A - (float(w0_start) + shift) * torch.eye(len(a), dtype=T)
        for _ in range(iters):
            x = torch.linalg.solve(M, x)
            x = x / torch.linalg.norm(x)
        if float(torch.dot(x.detach(), L0d)) < 0:
            x = -x
        w0 = torch.dot(x, A @ x)
        L = torch.zeros((self.nv, self.no), dtype=T).index_put((a, i), x)
        # ground state: T2^(1), T2^(2), T1^(2) (run1.f90, run2.f90)
        T2 = -abij / e2
        C1g = K("c1_r2abci", T2, abci) + K("c1_r2ijka", T2, ijka)
        C2g = K("c2_r2Wmbej", T2, iabj) + K("c2_r2Wmnij", T2, ijkl) + K("c2_r2abcd", T2, abcd)
        T2b = -C2g / e2
        a1, i1 = self.idx1[:, 0], self.idx1[:, 1]
        A1 = iabj[:, :, a1, i1][a1, i1].T + torch.diag(e1[a1, i1])
        T1b = torch.zeros((self.nv, self.no), dtype=T).index_put((a1, i1), torch.linalg.solve(A1, -C1g[a1, i1]))
        # J^(2), J^(3) (calJ.f90)
        Foo, Fvv = K("Fmi_r2abij", T2, abij), K("Fae_r2abij", T2, abij)
        Woo = K("Wkbij_r2ijka", T2, ijka) + K("Wkbij_r2abci", T2, abci)
        Wvo = K("Wmbej_r2abij", T2, abij, 2.0)
        Foo3 = K("Fmi_r1ijka", T1b, ijka) + K("Fmi_r2abij", T2b, abij)
        Fvv3 = K("Fae_r1abci", T1b, abci) + K("Fae_r2abij", T2b, abij)
        Wvo3 = K("Wmbej_r1ijka", T1b, ijka) + K("Wmbej_r1abci", T1b, abci) + K("Wmbej_r2abij", T2b, abij, 2.0)
        # orders 1-3 of run_order.f90
        C2 = K("c2_r1ijka", L, ijka) + K("c2_r1abci", L, abci)
        R2 = -C2 / (e2 - w0)
        C1 = (K("c1_r2abci", R2, abci) + K("c1_r2ijka", R2, ijka) + K("c1_r1iabj", L, Wvo)
              + K("c1_r1Fmi", L, Foo) + K("c1_r1Fae", L, Fvv))
        w2 = torch.sum(L * C1)
        C2b = (K("c2_r2Wmbej", R2, iabj) + K("c2_r2Wmnij", R2, ijkl) + K("c2_r2abcd", R2, abcd)
               + K("c2_r1ijka", L, Woo)
               + K("c2_r2Wmnij", T2, K("Wmnij_r1ijka", L, ijka)) + K("c2_r2Wmbej", T2, K("Wmbej_r1abci", L, abci))
               + K("c2_r2Fmi", T2, K("Fmi_r1ijka", L, ijka)) + K("c2_r2Fae", T2, K("Fae_r1abci", L, abci)))
        R22 = -C2b / (e2 - w0)
        C1c = (K("c1_r2abci", R22, abci) + K("c1_r2ijka", R22, ijka) + K("c1_r1iabj", L, Wvo3)
               + K("c1_r1Fmi", L, Foo3) + K("c1_r1Fae", L, Fvv3))
        w3 = torch.sum(L * C1c)
        return w0, w2, w3, self.r1_to_dpd(L.detach())

    def gradient3(self, s, L0, w0_start, g0, g2, g3):
        """d(g0 w0 + g2 w2 + g3 w3) / d(six lists, eorb) as numpy vectors."""
        keys = list(self.LAYOUTS)
        leaves = {k: torch.tensor(s.ints[k], dtype=T, requires_grad=True) for k in keys}
        eorb = torch.tensor(s.eorb, dtype=T, requires_grad=True)
        w0, w2, w3, _ = self.energies3(leaves, eorb, L0, w0_start)
        E = g0 * w0 + g2 * w2 + g3 * w3
        grads = torch.autograd.grad(E, [leaves[k] for k in keys] + [eorb])
        out = {k: g.numpy() for k, g in zip(keys, grads[:-1])}
        out["eorb"] = grads[-1].numpy()
        return out, float(w0.detach()), float(w2.detach()), float(w3.detach())
