"""Dense numpy SF-CIS / CPS(D) / EE-CPS(D-3) equations on small systems
(test infrastructure): an independent check of the drivers' bookkeeping.

Equations follow the reference's programs (src/EE-CIS.SF/calAR.f90,
src/CPSd.SF/run1.f90, run2.f90, src/EE-CPSd.SF/run_order.f90, calE_C.f90,
calJ.f90, calC_JR.f90, calC_VTR.f90, solver.f90) with the kernels' dense
formulas from kernel_specs; linear solves are done exactly (numpy.linalg)
instead of DIIS, which the iterative solvers converge to.
"""
import numpy as np

import dense
from kernel_specs import KERNELS


def K(name, a, b, f=1.0):
    return KERNELS[name][3](a, b, f)


class DenseSystem:
    def __init__(self, s):
        self.s = s
        g, O, V, eo, ev = dense.antisym_integrals(s)
        self.eo, self.ev = eo, ev
        self.ijkl = g[O, O, O, O]
        self.ijka = g[O, O, O, V]
        self.abij = g[V, V, O, O]
        self.iabj = g[O, V, V, O].transpose(2, 0, 1, 3)  # (b,i,a,j)
        self.abci = g[V, V, V, O]
        self.abcd = g[V, V, V, V]
        self.irr_o = dense.orbital_irreps(s.popo)
        self.irr_v = dense.orbital_irreps(s.popv)
        occ, vir = dense.spin_orbitals(s)
        self.spin_o = np.array([x for _, x in occ])
        self.spin_v = np.array([x for _, x in vir])
        self.e1 = ev[:, None] - eo[None, :]
        self.e2 = ev[:, None, None, None] + ev[None, :, None, None] - eo[None, None, :, None] - eo[None, None, None, :]

    def mask1(self, symR):
        sym = self.s.sym
        return np.array([[sym.dp(a, i) == symR for i in self.irr_o] for a in self.irr_v])

    def cis_matrix(self, symR, spin_flip=True):
        m = self.mask1(symR)
        if spin_flip:
            m = m & (self.spin_v[:, None] == 1) & (self.spin_o[None, :] == 0)
        idx = np.argwhere(m)
        nv, no = self.e1.shape
        Afull = np.einsum("fnai->aifn", self.iabj).reshape(nv * no, nv * no)
        Afull = Afull + np.diag(self.e1.reshape(-1))
        flat = idx[:, 0] * no + idx[:, 1]
        return Afull[np.ix_(flat, flat)], idx

    def ground(self):
        T2_1 = -self.abij / self.e2
        E2 = 0.25 * np.sum(T2_1 * self.abij)
        C1 = K("c1_r2abci", T2_1, self.abci) + K("c1_r2ijka", T2_1, self.ijka)
        C2 = (K("c2_r2Wmbej", T2_1, self.iabj) + K("c2_r2Wmnij", T2_1, self.ijkl)
              + K("c2_r2abcd", T2_1, self.abcd))
        T2_2 = -C2 / self.e2
        E3 = 0.25 * np.sum(T2_2 * self.abij)
        # T1^(2): -e T1 = C1 + V T1 on the totally symmetric (a,i) space
        A, idx = self._sigma_matrix(1)
        rhs = -C1[idx[:, 0], idx[:, 1]]
        x = np.linalg.solve(A, rhs)
        T1_2 = np.zeros_like(C1)
        T1_2[idx[:, 0], idx[:, 1]] = x
        return dict(T2_1=T2_1, T1_2=T1_2, T2_2=T2_2, E2=E2, E3=E3)

    def ground3(self, g):
        """run3.f90: T^(3) and E^(4) from T2^(1), T1^(2), T2^(2) (T1^(1) = 0)"""
        T2_1, T1_2, T2_2 = g["T2_1"], g["T1_2"], g["T2_2"]
        C1 = K("c1_r2abci", T2_2, self.abci) + K("c1_r2ijka", T2_2, self.ijka)
        C2 = (K("c2_r1ijka", T1_2, self.ijka) + K("c2_r1abci", T1_2, self.abci)
              + K("c2_r2Wmbej", T2_2, self.iabj) + K("c2_r2Wmnij", T2_2, self.ijkl)
              + K("c2_r2abcd", T2_2, self.abcd))
        Fli = K("Fmi_r2abij", T2_1, self.abij)
        C2 = C2 + K("c2_r2Fmi", T2_1, Fli)
        Fad = K("Fae_r2abij", T2_1, self.abij)
        C2 = C2 + K("c2_r2Fae", T2_1, Fad)
        Wkaci = K("Wmbej_r2abij", T2_1, self.abij)
        C2 = C2 + K("c2_r2Wmbej", T2_1, Wkaci)
        Wklij = K("Wmnij_r2abij", T2_1, self.abij, 0.5)
        C2 = C2 + K("c2_r2Wmnij", T2_1, Wklij, 2.0)
        T2_3 = -C2 / self.e2
        E4 = 0.25 * np.sum(T2_3 * self.abij)
        A, idx = self._sigma_matrix(1)
        x = np.linalg.solve(A, -C1[idx[:, 0], idx[:, 1]])
        T1_3 = np.zeros_like(C1)
        T1_3[idx[:, 0], idx[:, 1]] = x
        return dict(T1_3=T1_3, T2_3=T2_3, E4=E4)

    def _sigma_matrix(self, symR):
        m = self.mask1(symR)
        idx = np.argwhere(m)
        nv, no = self.e1.shape
        Afull = np.einsum("fnai->aifn", self.iabj).reshape(nv * no, nv * no) + np.diag(self.e1.reshape(-1))
        flat = idx[:, 0] * no + idx[:, 1]
        return Afull[np.ix_(flat, flat)], idx

    def jints(self, g):
        T2_1, T1_2, T2_2 = g["T2_1"], g["T1_2"], g["T2_2"]
        J = {}
        J["J2_Foo"] = K("Fmi_r2abij", T2_1, self.abij)
        J["J2_Fvv"] = K("Fae_r2abij", T2_1, self.abij)
        J["J2_Wovoo"] = K("Wkbij_r2ijka", T2_1, self.ijka) + K("Wkbij_r2abci", T2_1, self.abci)
        J["J2_Wovvo"] = K("Wmbej_r2abij", T2_1, self.abij, 2.0)
        J["J3_Foo"] = K("Fmi_r1ijka", T1_2, self.ijka) + K("Fmi_r2abij", T2_2, self.abij)
        J["J3_Fvv"] = K("Fae_r1abci", T1_2, self.abci) + K("Fae_r2abij", T2_2, self.abij)
        J["J3_Wovvo"] = (K("Wmbej_r1ijka", T1_2, self.ijka) + K("Wmbej_r1abci", T1_2, self.abci)
                         + K("Wmbej_r2abij", T2_2, self.abij, 2.0))
        return J

    def root(self, g, J, symR, w0, L):
        """L: dense (v,o) CIS vector; returns w^(1..3), R2^(1), R1^(2), R2^(2)."""
        T2 = g["T2_1"]
        # order 1: C^(1) = J^(1) R^(0): C2 only
        C1_1 = np.zeros_like(L)
        C2_1 = K("c2_r1ijka", L, self.ijka) + K("c2_r1abci", L, self.abci)
        w1 = np.sum(L * C1_1)
        # order 2
        R2_1 = -C2_1 / (self.e2 - w0)
        C1_2 = K("c1_r2abci", R2_1, self.abci) + K("c1_r2ijka", R2_1, self.ijka)
        C2_2 = (K("c2_r2Wmbej", R2_1, self.iabj) + K("c2_r2Wmnij", R2_1, self.ijkl)
                + K("c2_r2abcd", R2_1, self.abcd))
        C2_2 = C2_2 + K("c2_r1ijka", L, J["J2_Wovoo"])
        C1_2 = C1_2 + K("c1_r1iabj", L, J["J2_Wovvo"]) + K("c1_r1Fmi", L, J["J2_Foo"]) + K("c1_r1Fae", L, J["J2_Fvv"])
        # calC_VTR with T^(1) = (0, T2^(1))
        Wmn = K("Wmnij_r1ijka", L, self.ijka)
        C2_2 = C2_2 + K("c2_r2Wmnij", T2, Wmn)
        Wmb = K("Wmbej_r1abci", L, self.abci)
        C2_2 = C2_2 + K("c2_r2Wmbej", T2, Wmb)
        G = K("Fmi_r1ijka", L, self.ijka)
        C2_2 = C2_2 + K("c2_r2Fmi", T2, G)
        Gv = K("Fae_r1abci", L, self.abci)
        C2_2 = C2_2 + K("c2_r2Fae", T2, Gv)
        w2 = np.sum(L * C1_2)
        # order 3
        Ct1 = -C1_2 + w2 * L
        Ct2 = -C2_2
        R2_2 = Ct2 / (self.e2 - w0)
        # fixed point of solver.f90: R1 = P[(C' - w0 R1 + V R1)/(-e)] with
        # P = 1 - L L^T, i.e. (A - w0) R1 + c e*L = Ct1, L.R1 = 0
        A, idx = self._sigma_matrix(symR)
        l = L[idx[:, 0], idx[:, 1]]
        el = self.e1[idx[:, 0], idx[:, 1]] * l
        n = len(l)
        M = np.zeros((n + 1, n + 1))
        M[:n, :n] = A - w0 * np.eye(n)
        M[:n, n] = el
        M[n, :n] = l
        rhs = np.zeros(n + 1)
        rhs[:n] = Ct1[idx[:, 0], idx[:, 1]]
        x = np.linalg.solve(M, rhs)[:n]
        R1_2 = np.zeros_like(L)
        R1_2[idx[:, 0], idx[:, 1]] = x
        C1_3 = K("c1_r2abci", R2_2, self.abci) + K("c1_r2ijka", R2_2, self.ijka)
        C1_3 = C1_3 + K("c1_r1iabj", L, J["J3_Wovvo"]) + K("c1_r1Fmi", L, J["J3_Foo"]) + K("c1_r1Fae", L, J["J3_Fvv"])
        w3 = np.sum(L * C1_3)
        return dict(w=np.array([w1, w2, w3]), R2_1=R2_1, R1_2=R1_2, R2_2=R2_2)

    def cisdoo_matrix(self, symR):
        """CIS(D-infinity) (src/CISdoo.SD.SF/run.f90:25-39, calAR.f90:19-49)
        as a dense matrix over the packed (R1, R2) coordinates of irrep symR,
        with each coordinate's spin change (occupied spin 0 -> virtual spin 1
        counts +1)."""
        s, sym = self.s, self.s.sym
        z = np.array([1, 0, 0, 0, 0, 0, 0, 0])
        MP2t = -self.abij / self.e2
        Fac = np.diag(self.ev) + K("Fae_r2abij", MP2t, self.abij)
        Fki = np.diag(self.eo) + K("Fmi_r2abij", MP2t, self.abij)
        W = self.iabj + K("Wmbej_r2abij", MP2t, self.abij, 2.0)
        p1 = ([s.popv, s.popo, z, z], (1, 1), symR)
        p2 = ([s.popv, s.popv, s.popo, s.popo], (0, 0), symR)
        l1, l2 = s.r1_len(symR), s.r2_len(symR)
        n = l1 + l2
        A = np.zeros((n, n))
        for k in range(n):
            x = np.zeros(n)
            x[k] = 1.0
            R1 = dense.dpd_to_dense(x[:l1], sym, *p1)[:, :, 0, 0]
            R2 = dense.dpd_to_dense(x[l1:], sym, *p2)
            C1 = (K("c1_r1Fae", R1, Fac) + K("c1_r1Fmi", R1, Fki) + K("c1_r1iabj", R1, W)
                  + K("c1_r2abci", R2, self.abci) + K("c1_r2ijka", R2, self.ijka))
            C2 = self.e2 * R2 + K("c2_r1abci", R1, self.abci) + K("c2_r1ijka", R1, self.ijka)
            A[:l1, k] = dense.dense_to_dpd(C1[:, :, None, None], sym, *p1)
            A[l1:, k] = dense.dense_to_dpd(C2, sym, *p2)
        rows1, _ = dense.dpd_index_lists(sym, *p1)
        rows2, _ = dense.dpd_index_lists(sym, *p2)
        dms = np.zeros(n, np.int64)
        dms[rows1[:, 0]] = self.spin_v[rows1[:, 1]] - self.spin_o[rows1[:, 2]]
        dms[l1 + rows2[:, 0]] = (self.spin_v[rows2[:, 1]] + self.spin_v[rows2[:, 2]]
                                 - self.spin_o[rows2[:, 3]] - self.spin_o[rows2[:, 4]])
        return A, dms

    def grcpsd(self):
        """grCPS(D) ground state (src/grCPSd.SF/run.f90, solver.f90) with
        each order's coupled (T1, T2) equations solved exactly: T2 =
        -(C2 + A0R2 T1) / e2 eliminated, the (a,i) system of irrep 1 solved
        densely.  Returns T1, T2 per order and E^(2..4)."""
        e1, e2 = self.e1, self.e2
        MP2t = -self.abij / e2
        Fli = K("Fmi_r2abij", MP2t, self.abij, -1.0)
        Fad = K("Fae_r2abij", MP2t, self.abij, -1.0)
        W = self.iabj + K("Wmbej_r2abij", MP2t, self.abij, 2.0)

        def a0r1(T1, T2):
            return (K("c1_r1iabj", T1, W) + K("c1_r1Fmi", T1, Fli, -1.0) + K("c1_r1Fae", T1, Fad, -1.0)
                    + K("c1_r2ijka", T2, self.ijka) + K("c1_r2abci", T2, self.abci))

        def a0r2(T1):
            return K("c2_r1ijka", T1, self.ijka) + K("c2_r1abci", T1, self.abci)

        def a1r2(T2):
            return (K("c2_r2Wmbej", T2, self.iabj) + K("c2_r2Wmnij", T2, self.ijkl)
                    + K("c2_r2abcd", T2, self.abcd))

        def a2r1(T1):
            return (K("c1_r1iabj", T1, W - self.iabj, -1.0) + K("c1_r1Fmi", T1, Fli, 1.0)
                    + K("c1_r1Fae", T1, Fad, 1.0))

        def l1_vtt(T1, T2):
            Gli = K("Fmi_r1ijka", T1, self.ijka, -1.0) + K("Fmi_r2abij", T2, self.abij, -1.0)
            Gad = K("Fae_r1abci", T1, self.abci, -1.0) + K("Fae_r2abij", T2, self.abij, -1.0)
            Gld = K("Fme_r1abij", T1, self.abij, 1.0)
            return K("c1_r1Fmi", T1, Gli, -1.0) + K("c1_r1Fae", T1, Gad, -1.0) + K("c1_r2Fme", T2, Gld, 1.0)

        def l2_vtt(T1, T2):
            L = K("c2_r1ijka", T1, K("Wkbij_r1iabj", T1, self.iabj), -1.0)
            L = L + K("c2_r1abci", T1, K("Wabdj_r1abcd", T1, self.abcd), 0.5)
            L = L + K("c2_r1ijka", T1, K("Wkbij_r1Uklij", T1, self.ijkl), 0.5)
            G = K("Fmi_r1ijka", T1, self.ijka) + K("Fmi_r2abij", T2, self.abij)
            L = L + K("c2_r2Fmi", T2, G)
            G = K("Fae_r1abci", T1, self.abci) + K("Fae_r2abij", T2, self.abij)
            L = L + K("c2_r2Fae", T2, G)
            G = (K("Wmbej_r1ijka", T1, self.ijka) + K("Wmbej_r1abci", T1, self.abci)
                 + K("Wmbej_r2abij", T2, self.abij))
            L = L + K("c2_r2Wmbej", T2, G)
            L = L + K("c2_r1ijka", T1, K("Wkbij_r2abci", T2, self.abci))
            G = K("Wmnij_r1ijka", T1, self.ijka, 0.5) + K("Wmnij_r2abij", T2, self.abij, 0.5)
            return L + K("c2_r2Wmnij", T2, G, 2.0)

        idx = np.argwhere(self.mask1(1))

        def solve(C1, C2):
            # -e1 T1 = C1 + a0r1(T1, T2), T2 = -(C2 + a0r2(T1)) / e2
            def t2_of(T1):
                return -(C2 + a0r2(T1)) / e2

            def resid(x):
                T1 = np.zeros_like(e1)
                T1[idx[:, 0], idx[:, 1]] = x
                r = e1 * T1 + C1 + a0r1(T1, t2_of(T1))
                return r[idx[:, 0], idx[:, 1]]

            n = len(idx)
            r0 = resid(np.zeros(n))
            M = np.column_stack([resid(np.eye(n)[k]) - r0 for k in range(n)])
            x = np.linalg.solve(M, -r0)
            T1 = np.zeros_like(e1)
            T1[idx[:, 0], idx[:, 1]] = x
            return T1, t2_of(T1)

        out = []
        zero1, zero2 = np.zeros_like(e1), np.zeros_like(e2)
        T1a, T2a = solve(zero1, self.abij)
        E2 = 0.25 * np.sum(T2a * self.abij)
        T1b, T2b = solve(zero1, a1r2(T2a))
        tau = T2b + (np.einsum("ai,bj->abij", T1a, T1a) - np.einsum("aj,bi->abij", T1a, T1a))
        E3 = 0.25 * np.sum(tau * self.abij)
        T1c, T2c = solve(a2r1(T1a) + l1_vtt(T1a, T2a), a1r2(T2b) + l2_vtt(T1a, T2a))
        X = np.einsum("ai,bj->abij", T1b, T1a)
        tau = T2c + (X - X.transpose(0, 1, 3, 2) - X.transpose(1, 0, 2, 3) + X.transpose(1, 0, 3, 2))
        E4 = 0.25 * np.sum(tau * self.abij)
        return dict(T1=[T1a, T1b, T1c], T2=[T2a, T2b, T2c], E=np.array([E2, E3, E4]))

    # ---------------------------------------------------------- EE-grCPS(D)
    def _gr_intermediates(self):
        MP2t = -self.abij / self.e2
        Fli = K("Fmi_r2abij", MP2t, self.abij, -1.0)
        Fad = K("Fae_r2abij", MP2t, self.abij, -1.0)
        W = self.iabj + K("Wmbej_r2abij", MP2t, self.abij, 2.0)
        return Fli, Fad, W

    def _jset(self, t1, t2):
        """the [V,T] part of calJ2 / calJ3 (src/EE-grCPSd.SF/calJ.f90)"""
        return dict(
            Foo=K("Fmi_r1ijka", t1, self.ijka) + K("Fmi_r2abij", t2, self.abij),
            Fvv=K("Fae_r1abci", t1, self.abci) + K("Fae_r2abij", t2, self.abij),
            Fov=K("Fme_r1abij", t1, self.abij),
            Wovoo=(K("Wkbij_r1iabj", t1, self.iabj, -1.0) + K("Wkbij_r1Uklij", t1, self.ijkl)
                   + K("Wkbij_r2ijka", t2, self.ijka) + K("Wkbij_r2abci", t2, self.abci)),
            Wovvo=(K("Wmbej_r1ijka", t1, self.ijka) + K("Wmbej_r1abci", t1, self.abci)
                   + K("Wmbej_r2abij", t2, self.abij, 2.0)),
            Woooo=K("Wmnij_r1ijka", t1, self.ijka) + K("Wmnij_r2abij", t2, self.abij),
            Wooov=K("Wlkjd_r1abij", t1, self.abij))

    def _jset_vtt(self, J, t1, t2):
        """the [[V,T^(1)],T^(1)] part of calJ3"""
        w = K("Fme_r1abij", t1, self.abij)
        J["Foo"] = J["Foo"] + K("Fmi_r1fia", t1, w)
        J["Fvv"] = J["Fvv"] + K("Fae_r1fia", t1, w)
        J["Wovoo"] = J["Wovoo"] + K("Wkbij_r2Fkc", t2, w, -1.0)
        w = K("Wlkjd_r1abij", t1, self.abij)
        J["Wovvo"] = J["Wovvo"] + K("Wmbej_r1ijka", t1, w)
        J["Woooo"] = J["Woooo"] + K("Wmnij_r1ijka", t1, w, 0.5)
        J["Wovoo"] = J["Wovoo"] + K("Wkbij_r2ijka", t2, w)
        w = K("Wmnij_r1ijka", t1, self.ijka) + K("Wmnij_r2abij", t2, self.abij)
        J["Wovoo"] = J["Wovoo"] + K("Wkbij_r1Uklij", t1, w)
        w = K("Wmbej_r1abci", t1, self.abci)
        J["Wovoo"] = J["Wovoo"] + K("Wkbij_r1iabj", t1, w, -0.5)
        return J

    def _cjr(self, J, r1, r2):
        c1 = (K("c1_r1iabj", r1, J["Wovvo"]) + K("c1_r1Fmi", r1, J["Foo"]) + K("c1_r1Fae", r1, J["Fvv"])
              + K("c1_r2ijka", r2, J["Wooov"]) + K("c1_r2Fme", r2, J["Fov"]))
        c2 = (K("c2_r1ijka", r1, J["Wovoo"]) + K("c2_r2Wmbej", r2, J["Wovvo"]) + K("c2_r2Wmnij", r2, J["Woooo"])
              + K("c2_r2Fmi", r2, J["Foo"]) + K("c2_r2Fae", r2, J["Fvv"]))
        return c1, c2

    def _vtr(self, t1, t2, r1, r2):
        c1 = K("c1_r1Fmi", t1, K("Fmi_r2abij", r2, self.abij))
        c2 = K("c2_r1ijka", t1, K("Wkbij_r1iabj", r1, self.iabj, -1.0) + K("Wkbij_r2abci", r2, self.abci))
        c2 = c2 + K("c2_r1abci", r1, K("Wabdj_r1abcd", t1, self.abcd))
        c2 = c2 + K("c2_r2Wmnij", t2, K("Wmnij_r2abij", r2, self.abij) + K("Wmnij_r1ijka", r1, self.ijka))
        c2 = c2 + K("c2_r2Wmbej", t2, K("Wmbej_r1abci", r1, self.abci))
        c2 = c2 + K("c2_r2Fmi", t2, K("Fmi_r1ijka", r1, self.ijka) + K("Fmi_r2abij", r2, self.abij))
        c2 = c2 + K("c2_r2Fae", t2, K("Fae_r1abci", r1, self.abci) + K("Fae_r2abij", r2, self.abij))
        return c1, c2

    def _vttr(self, t1, t2, r1, r2):
        a = K("Fme_r1abij", r1, self.abij)
        c2 = K("c2_r2Fae", t2, K("Fae_r1fia", t1, a))
        b = K("Fmi_r1fia", t1, a) + K("Fmi_r1fia", r1, K("Fme_r1abij", t1, self.abij))
        c2 = c2 + K("c2_r2Fmi", t2, b)
        c2 = c2 + K("c2_r2Wmnij", t2, K("Wmnij_r1ijka", t1, K("Wlkjd_r1abij", r1, self.abij)))
        W = (K("Wkbij_r1Uklij", t1, K("Wmnij_r2abij", r2, self.abij) + K("Wmnij_r1ijka", r1, self.ijka), 0.5)
             + K("Wkbij_r1iabj", r1, K("Wmbej_r1abci", t1, self.abci), -1.0)
             + K("Wkbij_r2ijka", t2, K("Wlkjd_r1abij", r1, self.abij)))
        return c2 + K("c2_r1ijka", t1, W)

    def eegrcpsd(self, symR, w0, R0, L, T):
        """EE-grCPS(D) orders of one root (src/EE-grCPSd.SF): R0, L packed
        (R1, R2) vectors of irrep symR with <L|R0> = 1, T the dense grCPS(D)
        amplitudes (dict of grcpsd()).  Each order's (A - w0) R^(n) =
        sum_k w^(k) R^(n-k) - C^(n) is solved exactly with <L|R^(n)> = 0.
        Returns w^(1..3) and the packed R^(1), R^(2)."""
        s, sym = self.s, self.s.sym
        z = np.array([1, 0, 0, 0, 0, 0, 0, 0])
        p1 = ([s.popv, s.popo, z, z], (1, 1), symR)
        p2 = ([s.popv, s.popv, s.popo, s.popo], (0, 0), symR)
        l1 = s.r1_len(symR)

        def unpack(x):
            return dense.dpd_to_dense(x[:l1], sym, *p1)[:, :, 0, 0], dense.dpd_to_dense(x[l1:], sym, *p2)

        def pack(c1, c2):
            return np.concatenate([dense.dense_to_dpd(c1[:, :, None, None], sym, *p1), dense.dense_to_dpd(c2, sym, *p2)])

        A, _ = self.cisdoo_matrix(symR)
        n = A.shape[0]
        Fli, Fad, W = self._gr_intermediates()
        t1a, t2a, t1b, t2b = T["T1"][0], T["T2"][0], T["T1"][1], T["T2"][1]
        J2 = self._jset(t1a, t2a)
        J3 = self._jset_vtt(self._jset(t1b, t2b), t1a, t2a)

        def c2vr2(r2):
            return (K("c2_r2Wmbej", r2, self.iabj) + K("c2_r2Wmnij", r2, self.ijkl) + K("c2_r2abcd", r2, self.abcd))

        def vmp2r1(r1):
            return (K("c1_r1iabj", r1, W - self.iabj, -1.0) + K("c1_r1Fmi", r1, Fli, 1.0)
                    + K("c1_r1Fae", r1, Fad, 1.0))

        def cterm(order, R):
            r1, r2 = unpack(R[order - 1])
            c1, c2 = np.zeros_like(r1), c2vr2(r2)
            if order >= 2:
                r1, r2 = unpack(R[order - 2])
                c1 = c1 + vmp2r1(r1)
                x1, x2 = self._cjr(J2, r1, r2)
                y1, y2 = self._vtr(t1a, t2a, r1, r2)
                c1, c2 = c1 + x1 + y1, c2 + x2 + y2
            if order == 3:
                r1, r2 = unpack(R[0])
                x1, x2 = self._cjr(J3, r1, r2)
                y1, y2 = self._vtr(t1b, t2b, r1, r2)
                c1, c2 = c1 + x1 + y1, c2 + x2 + y2 + self._vttr(t1a, t2a, r1, r2)
            return pack(c1, c2)

        M = np.zeros((n + 1, n + 1))
        M[:n, :n] = A - w0 * np.eye(n)
        M[:n, n] = L
        M[n, :n] = L
        R = [np.asarray(R0, float)]
        w = []
        C = cterm(1, R)
        w.append(L @ C)
        for order in (1, 2):
            rhs = -C + sum(w[k - 1] * R[order - k] for k in range(1, order + 1))
            x = np.linalg.solve(M, np.concatenate([rhs, [0.0]]))
            R.append(x[:n])
            C = cterm(order + 1, R)
            w.append(L @ C)
        return np.array(w), R[1], R[2]
