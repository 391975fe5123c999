"""The spin-free lib_cc contraction kernels of the SF-CIS / SF-CPS(D-3) path:
operand layouts and independent dense formulas (test infrastructure).

Each entry: out tensor kind, operand kinds, and the dense result of
`out += fact * kernel(a, b)` written from the kernel's documented formula
(header comment of src/lib_cc/<name>.f90).
Kinds: (pops letters, iops) with 'o'/'v'/'z' (zorb) populations.
"""
import numpy as np

# tensor layouts: name -> (pop letters, iops)
LAYOUT = {
    "ai": ("vozz", (1, 1)),
    "oo": ("oozz", (1, 1)),
    "vv": ("vvzz", (1, 1)),
    "abij": ("vvoo", (0, 0)),
    "ijkl": ("oooo", (0, 0)),
    "ijka": ("ooov", (0, 1)),
    "iabj": ("vovo", (1, 1)),   # (bi,aj); also Wmbej (em,bj)
    "abci": ("vvvo", (0, 1)),
    "abcd": ("vvvv", (0, 0)),
}


def PQ(X):  # antisymmetrise first pair
    return X - X.transpose(1, 0, 2, 3)


def RS(X):
    return X - X.transpose(0, 1, 3, 2)


# name -> (out layout, a layout, b layout, dense fn(a, b, f) -> increment)
# a is the first operand passed to the kernel after `out`, b the second.
KERNELS = {
    "c1_r1iabj": ("ai", "ai", "iabj", lambda r, V, f: f * np.einsum("fn,fnai->ai", r, V)),
    "c1_r1Fae": ("ai", "ai", "vv", lambda r, F, f: f * np.einsum("ae,ei->ai", F, r)),
    "c1_r1Fmi": ("ai", "ai", "oo", lambda r, F, f: -f * np.einsum("am,mi->ai", r, F)),
    "c1_r2abci": ("ai", "abij", "abci", lambda r, V, f: 0.5 * f * np.einsum("feam,feim->ai", V, r)),
    "c1_r2ijka": ("ai", "abij", "ijka", lambda r, V, f: -0.5 * f * np.einsum("aemn,mnie->ai", r, V)),
    "c2_r1abci": ("abij", "ai", "abci", lambda r, V, f: f * RS(np.einsum("abej,ei->abij", V, r))),
    "c2_r1ijka": ("abij", "ai", "ijka", lambda r, V, f: -f * PQ(np.einsum("ijmb,am->abij", V, r))),
    "c2_r2Wmbej": ("abij", "abij", "iabj", lambda r, W, f: f * RS(PQ(np.einsum("aeim,embj->abij", r, W)))),
    "c2_r2Wmnij": ("abij", "abij", "ijkl", lambda r, W, f: 0.5 * f * np.einsum("abmn,mnij->abij", r, W)),
    "c2_r2abcd": ("abij", "abij", "abcd", lambda r, V, f: 0.5 * f * np.einsum("abef,efij->abij", V, r)),
    "c2_r2Fae": ("abij", "abij", "vv", lambda r, F, f: f * PQ(np.einsum("aeij,be->abij", r, F))),
    "c2_r2Fmi": ("abij", "abij", "oo", lambda r, F, f: -f * RS(np.einsum("abim,mj->abij", r, F))),
    "Fmi_r2abij": ("oo", "abij", "abij", lambda r, V, f: 0.5 * f * np.einsum("efin,efmn->mi", r, V)),
    "Fae_r2abij": ("vv", "abij", "abij", lambda r, V, f: -0.5 * f * np.einsum("afmn,efmn->ae", r, V)),
    "Fmi_r1ijka": ("oo", "ai", "ijka", lambda r, V, f: f * np.einsum("en,mnie->mi", r, V)),
    "Fae_r1abci": ("vv", "ai", "abci", lambda r, V, f: f * np.einsum("fm,efam->ae", r, V)),
    "Wkbij_r2ijka": ("ijka", "abij", "ijka", lambda r, V, f: f * PQ(np.einsum("klic,bcjl->ijkb", V, r))),
    "Wkbij_r2abci": ("ijka", "abij", "abci", lambda r, V, f: 0.5 * f * np.einsum("dcbk,cdij->ijkb", V, r)),
    "Wmbej_r2abij": ("iabj", "abij", "abij", lambda r, V, f: 0.5 * f * np.einsum("bfjn,fenm->embj", r, V)),
    "Wmbej_r1abci": ("iabj", "ai", "abci", lambda r, V, f: f * np.einsum("fj,febm->embj", r, V)),
    "Wmbej_r1ijka": ("iabj", "ai", "ijka", lambda r, V, f: -f * np.einsum("bn,nmje->embj", r, V)),
    "Wmnij_r1ijka": ("ijkl", "ai", "ijka", lambda r, V, f: f * RS(np.einsum("ej,mnie->mnij", r, V))),
    "Wmnij_r2abij": ("ijkl", "abij", "abij", lambda r, V, f: 0.5 * f * np.einsum("efmn,efij->mnij", V, r)),
    # the second-order ground state's (src/grCPSd.SF/calL1_VTT.f90, calL2_VTT.f90)
    "Wkbij_r1iabj": ("ijka", "ai", "iabj", lambda r, V, f: -f * PQ(np.einsum("ckbj,ci->ijkb", V, r))),
    "Wabdj_r1abcd": ("abci", "ai", "abcd", lambda r, V, f: f * np.einsum("abdc,cj->abdj", V, r)),
    "Wkbij_r1Uklij": ("ijka", "ai", "ijkl", lambda r, U, f: -f * np.einsum("klij,bl->ijkb", U, r)),
    "Fme_r1abij": ("ai", "ai", "abij", lambda r, V, f: f * np.einsum("efmn,fn->em", V, r)),
    "c1_r2Fme": ("ai", "abij", "ai", lambda r, F, f: f * np.einsum("aeim,em->ai", r, F)),
    # the excited-state grCPS(D)'s (src/EE-grCPSd.SF)
    "c1d_l1Wibaj": ("ai", "ai", "iabj", lambda l, W, f: f * np.einsum("aibj,bj->ai", W, l)),
    "c1d_l1fab": ("ai", "ai", "vv", lambda l, F, f: -f * np.einsum("ba,bi->ai", F, l)),
    "c1d_l1fij": ("ai", "ai", "oo", lambda l, F, f: f * np.einsum("aj,ij->ai", l, F)),
    "Fae_r1fia": ("vv", "ai", "ai", lambda r, F, f: -f * np.einsum("al,el->ae", r, F)),
    "Fmi_r1fia": ("oo", "ai", "ai", lambda r, F, f: f * np.einsum("dm,di->mi", F, r)),
    "Wkbij_r2Fkc": ("ijka", "abij", "ai", lambda r, F, f: -f * np.einsum("cbij,ck->ijkb", r, F)),
    "Wlkjd_r1abij": ("ijka", "ai", "abij", lambda r, V, f: f * np.einsum("cdlk,cj->lkjd", V, r)),
}


def pops_of(layout, popo, popv):
    zorb = np.array([1, 0, 0, 0, 0, 0, 0, 0], np.int64)
    m = {"o": popo, "v": popv, "z": zorb}
    letters, iops = LAYOUT[layout]
    return [m[c] for c in letters], iops


def squeeze2(D, layout):
    """dense 4-index array of a 2-index layout -> 2-index matrix"""
    return D[:, :, 0, 0] if LAYOUT[layout][0][2:] == "zz" else D


def expand2(M, layout):
    return M[:, :, None, None] if LAYOUT[layout][0][2:] == "zz" else M
