/*
 * Synthetic spin-free integral front end.
 *
 * Stands in for the reference's integral front ends (pyscf2cc.py2cc ->
 * xgetHF, src/pyscf2cc/py2cc.py:10, src/getHF/main.f90:3-149), which need
 * PySCF.  From density-fitting factors L[P][p][q] and alpha/beta orbital
 * energies it writes the six antisymmetrised spin-orbital integral tensors
 * in the spin-free DPD layout the programs load (src/getHF/loadSCF.f90,
 * src/EE-CPSd.SF/allocate_mem.f90):
 *
 *   ijkl(ij,kl) = <ij||kl>   (o,o,o,o) iop 0,0
 *   ijka(ij,ka) = <ij||ka>   (o,o,o,v) iop 0,1
 *   abij(ab,ij) = <ab||ij>   (v,v,o,o) iop 0,0
 *   iabj(bi,aj) = <ia||bj>   (v,o,v,o) iop 1,1   stored as (bi,aj)
 *   abci(ab,ci) = <ab||ci>   (v,v,v,o) iop 0,1
 *   abcd(ab,cd) = <ab||cd>   (v,v,v,v) iop 0,0
 *
 * with <pq||rs> = <pq|rs> - <pq|sr>, <pq|rs> = (pr|qs) d(sp,sr) d(sq,ss),
 * (pr|qs) = sum_P L[P][p][r] L[P][q][s].  Spin-free orbitals of one irrep
 * are the alpha spin-orbitals of that irrep followed by the beta ones
 * (src/getHF/resortV.f90:100-200, Gamma(R_y) = A1), occupied irreps first
 * in the orbital-energy array (src/lib_cc/seperateEorb.f90).
 *
 * Host code only (OpenMP); it prepares inputs, it is not on the timed path.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t i64;

static i64 D8[8][8];
static i64 NIRR;

static i64 dp(i64 a, i64 b) { return D8[a - 1][b - 1]; }

static i64 irpd(i64 sym, const i64 *pp, const i64 *pq, i64 iop)
{
    i64 n = 0;
    for (i64 r = 1; r <= NIRR; r++) {
        i64 l = dp(r, sym);
        if (iop == 1) n += pp[l - 1] * pq[r - 1];
        else if (l < r) n += pp[l - 1] * pq[r - 1];
        else if (l == r) n += pp[l - 1] * (pq[r - 1] - 1) / 2;
    }
    return n;
}

typedef struct {
    i64 n;
    i64 *ip, *p, *iq, *q;
} pairs_t;

static void pairs(pairs_t *pl, const i64 *pp, const i64 *pq, i64 iop, i64 irr)
{
    i64 n = irpd(irr, pp, pq, iop);
    pl->n = n;
    pl->ip = (i64 *)malloc(sizeof(i64) * (size_t)(n + 1) * 4);
    pl->p = pl->ip + n; pl->iq = pl->p + n; pl->q = pl->iq + n;
    i64 k = 0;
    for (i64 iq = 1; iq <= NIRR; iq++) {
        i64 ip = dp(iq, irr);
        if (iop != 1 && ip > iq) continue;
        for (i64 q = 0; q < pq[iq - 1]; q++) {
            i64 pmax = (iop == 0 && ip == iq) ? q : pp[ip - 1];
            for (i64 p = 0; p < pmax; p++) {
                pl->ip[k] = ip; pl->p[k] = p; pl->iq[k] = iq; pl->q[k] = q;
                k++;
            }
        }
    }
}

typedef struct {
    i64 nmo, naux;
    const double *Lt; /* [p][q][P], P contiguous */
    const i64 *aux_irrep;
    i64 *auxoff, *auxcnt; /* P range per irrep in the sorted aux list */
    const i64 *mo_irrep;
    /* spin-free orbital -> (mo, spin) for occupied / virtual per irrep */
    i64 *occ_mo[8], *occ_sp[8], *vir_mo[8], *vir_sp[8];
} gen_t;

/* (pr|qs) over aux functions of irrep(p) x irrep(r) */
static double eri(const gen_t *g, i64 p, i64 r, i64 q, i64 s)
{
    i64 h = dp(g->mo_irrep[p], g->mo_irrep[r]);
    if (h != dp(g->mo_irrep[q], g->mo_irrep[s])) return 0.0;
    const double *a = g->Lt + (p * g->nmo + r) * g->naux + g->auxoff[h - 1];
    const double *b = g->Lt + (q * g->nmo + s) * g->naux + g->auxoff[h - 1];
    double acc = 0.0;
    i64 n = g->auxcnt[h - 1];
    for (i64 k = 0; k < n; k++) acc += a[k] * b[k];
    return acc;
}

/* <pq||rs> for spin-orbitals (mo, spin) */
static double asym(const gen_t *g, i64 mp, i64 sp, i64 mq, i64 sq, i64 mr, i64 sr, i64 ms, i64 ss)
{
    double v = 0.0;
    if (sp == sr && sq == ss) v += eri(g, mp, mr, mq, ms);
    if (sp == ss && sq == sr) v -= eri(g, mp, ms, mq, mr);
    return v;
}

/* fill a DPD tensor; kind[k] = 'o'/'v' per slot; perm maps <pq||rs>
 * positions to slots: integral = <slot perm[0] slot perm[1] || slot perm[2] slot perm[3]> */
static void fill(const gen_t *g, double *out, const char *kind, const i64 *pops[4],
                 i64 iop0, i64 iop1, const int perm[4])
{
    i64 off = 0;
    for (i64 R = 1; R <= NIRR; R++) {
        i64 L = R; /* sym = 1 */
        pairs_t pr, pl;
        pairs(&pr, pops[2], pops[3], iop1, R);
        pairs(&pl, pops[0], pops[1], iop0, L);
        i64 nl = pl.n;
#pragma omp parallel for schedule(dynamic, 16)
        for (i64 r = 0; r < pr.n; r++) {
            i64 irr[4], idx[4], mo[4], sp[4];
            irr[2] = pr.ip[r]; idx[2] = pr.p[r]; irr[3] = pr.iq[r]; idx[3] = pr.q[r];
            for (int k = 2; k < 4; k++) {
                i64 h = irr[k] - 1;
                mo[k] = (kind[k] == 'o') ? g->occ_mo[h][idx[k]] : g->vir_mo[h][idx[k]];
                sp[k] = (kind[k] == 'o') ? g->occ_sp[h][idx[k]] : g->vir_sp[h][idx[k]];
            }
            for (i64 l = 0; l < nl; l++) {
                irr[0] = pl.ip[l]; idx[0] = pl.p[l]; irr[1] = pl.iq[l]; idx[1] = pl.q[l];
                for (int k = 0; k < 2; k++) {
                    i64 h = irr[k] - 1;
                    mo[k] = (kind[k] == 'o') ? g->occ_mo[h][idx[k]] : g->vir_mo[h][idx[k]];
                    sp[k] = (kind[k] == 'o') ? g->occ_sp[h][idx[k]] : g->vir_sp[h][idx[k]];
                }
                out[off + r * nl + l] = asym(g, mo[perm[0]], sp[perm[0]], mo[perm[1]], sp[perm[1]],
                                             mo[perm[2]], sp[perm[2]], mo[perm[3]], sp[perm[3]]);
            }
        }
        off += pr.n * nl;
        free(pr.ip);
        free(pl.ip);
    }
}

/*
 * nmo spatial orbitals with irreps mo_irrep[k] (1-based); MO k is alpha-
 * occupied iff k < nocc_a and beta-occupied iff k < nocc_b; eps_a/eps_b are
 * the alpha/beta orbital energies by MO index.  L is naux x nmo x nmo.
 * dirprd is column-major 8x8.  popo/popv (out, 8 each) receive the
 * spin-free populations.  Any output pointer may be NULL to skip it.
 * Returns 0 on success.
 */
int cpsd_synth_build(i64 nmo, i64 nirrep, const i64 *dirprd, const i64 *mo_irrep,
                     i64 nocc_a, i64 nocc_b, const double *eps_a, const double *eps_b,
                     i64 naux, const i64 *aux_irrep, const double *L,
                     i64 *popo, i64 *popv, double *eorb,
                     double *ijkl, double *ijka, double *abij, double *iabj,
                     double *abci, double *abcd)
{
    if (nirrep < 1 || nirrep > 8) return -1;
    NIRR = nirrep;
    for (int j = 0; j < 8; j++)
        for (int i = 0; i < 8; i++) D8[i][j] = dirprd[j * 8 + i];
    gen_t g;
    memset(&g, 0, sizeof(g));
    g.nmo = nmo;
    g.naux = naux;
    g.mo_irrep = mo_irrep;
    g.aux_irrep = aux_irrep;
    /* aux functions sorted by irrep, Lt[p][q][P] */
    i64 *order = (i64 *)malloc(sizeof(i64) * (size_t)naux);
    i64 auxoff[8] = {0}, auxcnt[8] = {0};
    i64 k = 0;
    for (i64 h = 1; h <= nirrep; h++) {
        auxoff[h - 1] = k;
        for (i64 P = 0; P < naux; P++)
            if (aux_irrep[P] == h) order[k++] = P;
        auxcnt[h - 1] = k - auxoff[h - 1];
    }
    g.auxoff = auxoff;
    g.auxcnt = auxcnt;
    double *Lt = (double *)malloc(sizeof(double) * (size_t)(nmo * nmo * naux));
    if (!Lt || !order) { free(Lt); free(order); return -2; }
#pragma omp parallel for
    for (i64 pq = 0; pq < nmo * nmo; pq++)
        for (i64 j = 0; j < naux; j++) Lt[pq * naux + j] = L[order[j] * nmo * nmo + pq];
    g.Lt = Lt;
    /* spin-free orbital lists */
    for (i64 h = 1; h <= nirrep; h++) {
        i64 no = 0, nv = 0;
        g.occ_mo[h - 1] = (i64 *)malloc(sizeof(i64) * (size_t)(2 * nmo + 1));
        g.occ_sp[h - 1] = (i64 *)malloc(sizeof(i64) * (size_t)(2 * nmo + 1));
        g.vir_mo[h - 1] = (i64 *)malloc(sizeof(i64) * (size_t)(2 * nmo + 1));
        g.vir_sp[h - 1] = (i64 *)malloc(sizeof(i64) * (size_t)(2 * nmo + 1));
        for (int spin = 0; spin < 2; spin++) {
            i64 nocc = spin == 0 ? nocc_a : nocc_b;
            for (i64 m = 0; m < nmo; m++)
                if (mo_irrep[m] == h && m < nocc) { g.occ_mo[h - 1][no] = m; g.occ_sp[h - 1][no++] = spin; }
            for (i64 m = 0; m < nmo; m++)
                if (mo_irrep[m] == h && m >= nocc) { g.vir_mo[h - 1][nv] = m; g.vir_sp[h - 1][nv++] = spin; }
        }
        popo[h - 1] = no;
        popv[h - 1] = nv;
    }
    for (i64 h = nirrep + 1; h <= 8; h++) popo[h - 1] = popv[h - 1] = 0;
    if (eorb) {
        i64 e = 0;
        for (i64 h = 0; h < nirrep; h++)
            for (i64 i = 0; i < popo[h]; i++) {
                i64 m = g.occ_mo[h][i];
                eorb[e++] = g.occ_sp[h][i] == 0 ? eps_a[m] : eps_b[m];
            }
        for (i64 h = 0; h < nirrep; h++)
            for (i64 i = 0; i < popv[h]; i++) {
                i64 m = g.vir_mo[h][i];
                eorb[e++] = g.vir_sp[h][i] == 0 ? eps_a[m] : eps_b[m];
            }
    }
    const int id[4] = {0, 1, 2, 3};
    const int iabj_perm[4] = {1, 2, 0, 3}; /* slots (b,i,a,j) -> <i a || b j> */
    const i64 *P_oooo[4] = {popo, popo, popo, popo};
    const i64 *P_ooov[4] = {popo, popo, popo, popv};
    const i64 *P_vvoo[4] = {popv, popv, popo, popo};
    const i64 *P_vovo[4] = {popv, popo, popv, popo};
    const i64 *P_vvvo[4] = {popv, popv, popv, popo};
    const i64 *P_vvvv[4] = {popv, popv, popv, popv};
    if (ijkl) fill(&g, ijkl, "oooo", P_oooo, 0, 0, id);
    if (ijka) fill(&g, ijka, "ooov", P_ooov, 0, 1, id);
    if (abij) fill(&g, abij, "vvoo", P_vvoo, 0, 0, id);
    if (iabj) fill(&g, iabj, "vovo", P_vovo, 1, 1, iabj_perm);
    if (abci) fill(&g, abci, "vvvo", P_vvvo, 0, 1, id);
    if (abcd) fill(&g, abcd, "vvvv", P_vvvv, 0, 0, id);
    for (i64 h = 0; h < nirrep; h++) {
        free(g.occ_mo[h]); free(g.occ_sp[h]); free(g.vir_mo[h]); free(g.vir_sp[h]);
    }
    free(Lt);
    free(order);
    return 0;
}
