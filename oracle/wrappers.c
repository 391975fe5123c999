/*
 * CPU ORACLE (test infrastructure only): the mod_contract wrappers
 * (src/lib_cc/mod_contract.f90:10-455) and the spin-free lib_cc kernels
 * that the SF-CIS / SF-CPS(D-3) path calls (src/lib_cc/<name>.f90).
 */
#include "cpsd_oracle.h"
#include <stdlib.h>
#include <string.h>

static const i64 ZORB[8] = {1, 0, 0, 0, 0, 0, 0, 0};

void o_opt_view(o_opt *t, const i64 *popp, const i64 *popq, const i64 *popr,
                const i64 *pops, i64 ioppq, i64 ioprs, i64 sym, double *arr)
{
    o_desc_init(&t->d, popp, popq, popr, pops, ioppq, ioprs, sym);
    t->len = o_desc_len(&t->d);
    t->arr = arr;
}

/* map the reference's placeholder characters ('+', '-', '=') to the
 * engine's dummy slot '.' */
static void norm_type(const char *in, int n, char out[5])
{
    for (int i = 0; i < 4; i++) {
        char c = (i < n) ? in[i] : '.';
        if (c == '+' || c == '-' || c == '=') c = '.';
        out[i] = c;
    }
    out[4] = 0;
}

/* check_flat (src/lib_cc/mod_contract.f90:495-513) */
static int check_flat(const char *cur, const char pairs[][2], int n, int self)
{
    for (int i = 0; i < n; i++) {
        if (i == self) continue;
        if (pairs[i][0] == cur[0] && pairs[i][1] == cur[1]) return 0;
    }
    return 1;
}

static double *xalloc(i64 n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

static void axpy(i64 n, double a, const double *x, double *y)
{
    for (i64 i = 0; i < n; i++) y[i] += a * x[i];
}

/* expand the flagged pairs of v (iexpso) into a fresh buffer */
static int expand_opt(const o_opt *v, i64 e0, i64 e1, o_desc *dout, double **buf)
{
    *dout = v->d;
    if (!e0 && !e1) { *buf = NULL; return O_OK; }
    if (e0) dout->iop[0] = 1;
    if (e1) dout->iop[1] = 1;
    *buf = xalloc(o_desc_len(dout));
    if (!*buf) return O_EMEM;
    return o_iexpso(v->arr, *buf, &v->d, e0, e1);
}

/* vv2v_444 (src/lib_cc/mod_contract.f90:10-162):
 * v3 += fact * P1 P2 { v1 * v2 } */
int o_vv2v_444(const o_opt *v1, const o_opt *v2, o_opt *v3, double fact,
               const char *t1, const char *t2, const char *t3, i64 anti)
{
    if (anti < 0 || anti > 3) return O_EARG;
    char pair[6][2] = {{t1[0], t1[1]}, {t1[2], t1[3]}, {t2[0], t2[1]},
                       {t2[2], t2[3]}, {t3[0], t3[1]}, {t3[2], t3[3]}};
    i64 iop[6] = {v1->d.iop[0], v1->d.iop[1], v2->d.iop[0], v2->d.iop[1], v3->d.iop[0], v3->d.iop[1]};
    i64 iexp[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 6; i++)
        if (check_flat(pair[i], pair, 6, i) && iop[i] != 1) { iexp[i] = 1; iop[i] = 1; }
    /* v3 packed but not antisymmetrised is undefined in the reference */
    if (anti == 0 && (iexp[4] || iexp[5])) return O_ELAYOUT;
    char n1[5], n2[5], n3[5];
    norm_type(t1, 4, n1); norm_type(t2, 4, n2); norm_type(t3, 4, n3);
    o_desc e1, e2;
    double *b1 = NULL, *b2 = NULL;
    int rc = expand_opt(v1, iexp[0], iexp[1], &e1, &b1);
    if (rc == O_OK) rc = expand_opt(v2, iexp[2], iexp[3], &e2, &b2);
    if (rc != O_OK) { free(b1); free(b2); return rc; }
    const double *p1 = b1 ? b1 : v1->arr;
    const double *p2 = b2 ? b2 : v2->arr;
    if (anti == 0) {
        rc = o_vv2v_dpd(p1, &e1, n1, p2, &e2, n2, v3->arr, &v3->d, n3, fact, 1.0);
        free(b1); free(b2);
        return rc;
    }
    o_desc d3 = v3->d;
    d3.iop[0] = iop[4];
    d3.iop[1] = iop[5];
    i64 nfull = o_desc_len(&d3);
    double *X = xalloc(nfull), *Y = xalloc(nfull);
    if (!X || !Y) { free(b1); free(b2); free(X); free(Y); return O_EMEM; }
    rc = o_vv2v_dpd(p1, &e1, n1, p2, &e2, n2, X, &d3, n3, fact, 1.0);
    free(b1); free(b2);
    if (rc != O_OK) { free(X); free(Y); return rc; }
    /* antisymmetrise the 1st pair */
    if (anti == 1 || anti == 3) {
        if (d3.iop[0] != 1 || memcmp(d3.pop[0], d3.pop[1], sizeof(d3.pop[0])) != 0) { rc = O_ELAYOUT; goto done; }
        o_isymtrso(X, Y, &d3, 1, 0);
        axpy(nfull, -1.0, Y, X);
    }
    if (iexp[4]) { /* compress the 1st pair */
        o_desc dc = d3;
        dc.iop[0] = v3->d.iop[0];
        if ((rc = o_icompso(X, Y, &d3, v3->d.iop[0], 1)) != O_OK) goto done;
        double *t = X; X = Y; Y = t;
        d3 = dc;
    }
    if (anti == 2 || anti == 3) {
        if (d3.iop[1] != 1 || memcmp(d3.pop[2], d3.pop[3], sizeof(d3.pop[0])) != 0) { rc = O_ELAYOUT; goto done; }
        i64 n = o_desc_len(&d3);
        o_isymtrso(X, Y, &d3, 0, 1);
        axpy(n, -1.0, Y, X);
    }
    if (iexp[5]) {
        o_desc dc = d3;
        dc.iop[1] = v3->d.iop[1];
        if ((rc = o_icompso(X, Y, &d3, 1, v3->d.iop[1])) != O_OK) goto done;
        double *t = X; X = Y; Y = t;
        d3 = dc;
    }
    axpy(v3->len, 1.0, X, v3->arr);
done:
    free(X); free(Y);
    return rc;
}

/* vv2v_222 (src/lib_cc/mod_contract.f90:166-182) */
int o_vv2v_222(const o_opt *v1, const o_opt *v2, o_opt *v3, double fact,
               const char *t1, const char *t2, const char *t3)
{
    char a[5] = {t1[0], t1[1], '=', '+', 0}, b[5] = {t2[0], t2[1], '=', '-', 0}, c[5] = {t3[0], t3[1], '+', '-', 0};
    return o_vv2v_444(v1, v2, v3, fact, a, b, c, 0);
}

/* vv2v_422 (src/lib_cc/mod_contract.f90:184-200) */
int o_vv2v_422(const o_opt *v1, const o_opt *v2, o_opt *v3, double fact,
               const char *t1, const char *t2, const char *t3)
{
    char b[5] = {t2[0], t2[1], '+', '-', 0}, c[5] = {t3[0], t3[1], '+', '-', 0};
    return o_vv2v_444(v1, v2, v3, fact, t1, b, c, 0);
}

/* vv2v_224 (src/lib_cc/mod_contract.f90:202-218) */
int o_vv2v_224(const o_opt *v1, const o_opt *v2, o_opt *v3, double fact,
               const char *t1, const char *t2, const char *t3, i64 anti)
{
    char a[5] = {t1[0], t1[1], '+', '-', 0}, b[5] = {t2[0], t2[1], '+', '-', 0};
    return o_vv2v_444(v1, v2, v3, fact, a, b, t3, anti);
}

/* vv2v_424 (src/lib_cc/mod_contract.f90:220-367) */
int o_vv2v_424(const o_opt *v1, const o_opt *v2, o_opt *v3, double fact,
               const char *t1, const char *t2, const char *t3, i64 anti)
{
    if (anti < 0 || anti > 2) return O_EARG;
    char pair[4][2] = {{t1[0], t1[1]}, {t1[2], t1[3]}, {t3[0], t3[1]}, {t3[2], t3[3]}};
    i64 iop[4] = {v1->d.iop[0], v1->d.iop[1], v3->d.iop[0], v3->d.iop[1]};
    i64 iexp[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; i++)
        if (check_flat(pair[i], pair, 4, i) && iop[i] != 1) { iexp[i] = 1; iop[i] = 1; }
    if ((anti != 1 && iexp[2]) || (anti != 2 && iexp[3])) return O_ELAYOUT;
    char n1[5], n2[5], n3[5];
    norm_type(t1, 4, n1); norm_type(t2, 2, n2); norm_type(t3, 4, n3);
    o_desc e1;
    double *b1 = NULL;
    int rc = expand_opt(v1, iexp[0], iexp[1], &e1, &b1);
    if (rc != O_OK) return rc;
    const double *p1 = b1 ? b1 : v1->arr;
    if (anti == 0) {
        rc = o_vv2v_dpd(p1, &e1, n1, v2->arr, &v2->d, n2, v3->arr, &v3->d, n3, fact, 1.0);
        free(b1);
        return rc;
    }
    o_desc d3 = v3->d;
    d3.iop[0] = iop[2];
    d3.iop[1] = iop[3];
    i64 nfull = o_desc_len(&d3);
    double *X = xalloc(nfull), *Y = xalloc(nfull);
    if (!X || !Y) { free(b1); free(X); free(Y); return O_EMEM; }
    rc = o_vv2v_dpd(p1, &e1, n1, v2->arr, &v2->d, n2, X, &d3, n3, fact, 1.0);
    free(b1);
    if (rc != O_OK) { free(X); free(Y); return rc; }
    if (anti == 1) {
        if (d3.iop[0] != 1 || memcmp(d3.pop[0], d3.pop[1], sizeof(d3.pop[0])) != 0) { rc = O_ELAYOUT; goto done; }
        o_isymtrso(X, Y, &d3, 1, 0);
        axpy(nfull, -1.0, Y, X);
        if (iexp[2]) {
            o_desc dc = d3;
            dc.iop[0] = v3->d.iop[0];
            if ((rc = o_icompso(X, Y, &d3, v3->d.iop[0], 1)) != O_OK) goto done;
            double *t = X; X = Y; Y = t;
            d3 = dc;
        }
    }
    if (anti == 2) {
        if (d3.iop[1] != 1 || memcmp(d3.pop[2], d3.pop[3], sizeof(d3.pop[0])) != 0) { rc = O_ELAYOUT; goto done; }
        i64 n = o_desc_len(&d3);
        o_isymtrso(X, Y, &d3, 0, 1);
        axpy(n, -1.0, Y, X);
        if (iexp[3]) {
            o_desc dc = d3;
            dc.iop[1] = v3->d.iop[1];
            if ((rc = o_icompso(X, Y, &d3, 1, v3->d.iop[1])) != O_OK) goto done;
            double *t = X; X = Y; Y = t;
            d3 = dc;
        }
    }
    axpy(v3->len, 1.0, X, v3->arr);
done:
    free(X); free(Y);
    return rc;
}

/* vv2v_442 (src/lib_cc/mod_contract.f90:369-455) */
int o_vv2v_442(const o_opt *v1, const o_opt *v2, o_opt *v3, double fact,
               const char *t1, const char *t2, const char *t3)
{
    char pair[4][2] = {{t1[0], t1[1]}, {t1[2], t1[3]}, {t2[0], t2[1]}, {t2[2], t2[3]}};
    i64 iop[4] = {v1->d.iop[0], v1->d.iop[1], v2->d.iop[0], v2->d.iop[1]};
    i64 iexp[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; i++)
        if (check_flat(pair[i], pair, 4, i) && iop[i] != 1) { iexp[i] = 1; iop[i] = 1; }
    char n1[5], n2[5], n3[5];
    norm_type(t1, 4, n1); norm_type(t2, 4, n2); norm_type(t3, 2, n3);
    o_desc e1, e2;
    double *b1 = NULL, *b2 = NULL;
    int rc = expand_opt(v1, iexp[0], iexp[1], &e1, &b1);
    if (rc == O_OK) rc = expand_opt(v2, iexp[2], iexp[3], &e2, &b2);
    if (rc == O_OK)
        rc = o_vv2v_dpd(b1 ? b1 : v1->arr, &e1, n1, b2 ? b2 : v2->arr, &e2, n2, v3->arr, &v3->d, n3, fact, 1.0);
    free(b1); free(b2);
    return rc;
}

/* ======================= lib_cc kernels (spin-free) ======================= */

/* c1_r1iabj.f90:3-17: c(a,i) += f*r(f,n)*V(fn,ai) */
int o_c1_r1iabj(o_opt *c1, const o_opt *r1, const o_opt *iabj, double f)
{ return o_vv2v_422(iabj, r1, c1, f, "fnai", "fn", "ai"); }

/* c1_r1Fae.f90:3-17: c(a,i) += f*r(e,i)*F(a,e) */
int o_c1_r1Fae(o_opt *c1, const o_opt *r1, const o_opt *Fae, double f)
{ return o_vv2v_222(Fae, r1, c1, f, "ae", "ei", "ai"); }

/* c1_r1Fmi.f90:3-17: c(a,i) -= f*r(a,m)*F(m,i) */
int o_c1_r1Fmi(o_opt *c1, const o_opt *r1, const o_opt *Fmi, double f)
{ return o_vv2v_222(r1, Fmi, c1, -f, "am", "mi", "ai"); }

/* c1_r2abci.f90:3-27: c(a,i) += f*0.5*r(fe,im)*V(fe,am) */
int o_c1_r2abci(o_opt *c1, const o_opt *r2, const o_opt *abci, double f)
{ return o_vv2v_442(abci, r2, c1, r2->d.iop[0] == 0 ? f : 0.5 * f, "feam", "feim", "ai"); }

/* c1_r2ijka.f90:3-20: c(a,i) -= f*0.5*r(ae,mn)*V(mn,ie) */
int o_c1_r2ijka(o_opt *c1, const o_opt *r2, const o_opt *ijka, double f)
{ return o_vv2v_442(r2, ijka, c1, r2->d.iop[1] == 0 ? -f : -0.5 * f, "aemn", "mnie", "ai"); }

/* c2_r1abci.f90:3-25: c(ab,ij) += f*P(ij){r(e,i)*V(ab,ej)} */
int o_c2_r1abci(o_opt *c2, const o_opt *r1, const o_opt *abci, double f)
{ return o_vv2v_424(abci, r1, c2, f, "abej", "ei", "abij", 2); }

/* c2_r1ijka.f90:3-17: c(ab,ij) -= f*P(ab){r(a,m)*V(ij,mb)} */
int o_c2_r1ijka(o_opt *c2, const o_opt *r1, const o_opt *ijka, double f)
{ return o_vv2v_424(ijka, r1, c2, -f, "ijmb", "am", "abij", 1); }

/* c2_r2Wmbej.f90:3-17: c(ab,ij) += f*P(ab|ij){r(ae,im)*W(em,bj)} */
int o_c2_r2Wmbej(o_opt *c2, const o_opt *r2, const o_opt *W, double f)
{ return o_vv2v_444(r2, W, c2, f, "aeim", "embj", "abij", 3); }

/* c2_r2Wmnij.f90:3-21: c(ab,ij) += 0.5*f*r(ab,mn)*W(mn,ij) */
int o_c2_r2Wmnij(o_opt *c2, const o_opt *r2, const o_opt *W, double f)
{ return o_vv2v_444(r2, W, c2, r2->d.iop[0] == 0 ? f : 0.5 * f, "abmn", "mnij", "abij", 0); }

/* c2_r2abcd.f90:3-27 (incore branch; the out-of-core p_c2_r2abcd_h at
 * c2_r2abcd.f90:29-104 computes the same sum): c(ab,ij) += 0.5*f*r(ef,ij)*V(ab,ef) */
int o_c2_r2abcd(o_opt *c2, const o_opt *r2, const o_opt *abcd, double f)
{ return o_vv2v_444(abcd, r2, c2, r2->d.iop[0] == 1 ? 0.5 * f : f, "abef", "efij", "abij", 0); }

/* c2_r2Fae.f90:3-17: c(ab,ij) += f*P(ab){r(ae,ij)*F(b,e)} */
int o_c2_r2Fae(o_opt *c2, const o_opt *r2, const o_opt *F, double f)
{ return o_vv2v_424(r2, F, c2, f, "aeij", "be", "abij", 1); }

/* c2_r2Fmi.f90:3-17: c(ab,ij) -= f*P(ij){r(ab,im)*F(m,j)} */
int o_c2_r2Fmi(o_opt *c2, const o_opt *r2, const o_opt *F, double f)
{ return o_vv2v_424(r2, F, c2, -f, "abim", "mj", "abij", 2); }

/* Fmi_r2abij.f90:3-21: F(m,i) += f*0.5*r(ef,in)*V(ef,mn) */
int o_Fmi_r2abij(o_opt *F, const o_opt *r2, const o_opt *abij, double f)
{ return o_vv2v_442(abij, r2, F, r2->d.iop[0] == 1 ? 0.5 * f : f, "efmn", "efin", "mi"); }

/* Fae_r2abij.f90:3-21: F(a,e) -= f*0.5*r(af,mn)*V(ef,mn) */
int o_Fae_r2abij(o_opt *F, const o_opt *r2, const o_opt *abij, double f)
{ return o_vv2v_442(r2, abij, F, r2->d.iop[1] == 0 ? -f : -0.5 * f, "afmn", "efmn", "ae"); }

/* Fmi_r1ijka.f90:3-17: F(m,i) += f*r(e,n)*V(mn,ie) */
int o_Fmi_r1ijka(o_opt *F, const o_opt *r1, const o_opt *ijka, double f)
{ return o_vv2v_422(ijka, r1, F, f, "mnie", "en", "mi"); }

/* Fae_r1abci.f90:3-24: F(a,e) += f*r(f,m)*V(ef,am) */
int o_Fae_r1abci(o_opt *F, const o_opt *r1, const o_opt *abci, double f)
{ return o_vv2v_422(abci, r1, F, f, "efam", "fm", "ae"); }

/* Wkbij_r2ijka.f90:3-17: W(ij,kb) += f*P(ij){V(kl,ic)*r(bc,jl)} */
int o_Wkbij_r2ijka(o_opt *W, const o_opt *r2, const o_opt *ijka, double f)
{ return o_vv2v_444(ijka, r2, W, f, "klic", "bcjl", "ijkb", 1); }

/* Wkbij_r2abci.f90:3-43: W(ij,kb) += f*0.5*V(dc,bk)*r(cd,ij) via tmp(ij,bk) */
int o_Wkbij_r2abci(o_opt *W, const o_opt *r2, const o_opt *abci, double f)
{
    o_opt tmp;
    o_desc_init(&tmp.d, W->d.pop[0], W->d.pop[1], W->d.pop[3], W->d.pop[2], W->d.iop[0], 1, W->d.sym);
    tmp.len = o_desc_len(&tmp.d);
    tmp.arr = xalloc(tmp.len);
    double *sw = xalloc(tmp.len);
    if (!tmp.arr || !sw) { free(tmp.arr); free(sw); return O_EMEM; }
    int rc = o_vv2v_444(r2, abci, &tmp, r2->d.iop[0] == 0 ? -f : -0.5 * f, "cdij", "cdbk", "ijbk", 0);
    if (rc == O_OK) rc = o_isymtrso(tmp.arr, sw, &tmp.d, 0, 1);
    if (rc == O_OK) axpy(W->len, 1.0, sw, W->arr);
    free(tmp.arr); free(sw);
    return rc;
}

/* Wmbej_r2abij.f90:3-17: W(em,bj) += f*0.5*r(bf,jn)*V(fe,nm) */
int o_Wmbej_r2abij(o_opt *W, const o_opt *r2, const o_opt *abij, double f)
{ return o_vv2v_444(abij, r2, W, 0.5 * f, "fenm", "bfjn", "embj", 0); }

/* Wmbej_r1abci.f90:3-24: W(em,bj) += f*r(f,j)*V(fe,bm) */
int o_Wmbej_r1abci(o_opt *W, const o_opt *r1, const o_opt *abci, double f)
{ return o_vv2v_424(abci, r1, W, f, "febm", "fj", "embj", 0); }

/* Wmbej_r1ijka.f90:3-17: W(em,bj) -= f*r(b,n)*V(nm,je) */
int o_Wmbej_r1ijka(o_opt *W, const o_opt *r1, const o_opt *ijka, double f)
{ return o_vv2v_424(ijka, r1, W, -f, "nmje", "bn", "embj", 0); }

/* Wmnij_r1ijka.f90:3-17: W(mn,ij) += f*P(ij){r(e,j)*V(mn,ie)} */
int o_Wmnij_r1ijka(o_opt *W, const o_opt *r1, const o_opt *ijka, double f)
{ return o_vv2v_424(ijka, r1, W, f, "mnie", "ej", "mnij", 2); }

/* Wmnij_r2abij.f90:1-20: W(mn,ij) += f*0.5*V(ef,mn)*r(ef,ij) (full e,f sums;
 * a packed ef pair sums each pair once, so the factor is f there) */
int o_Wmnij_r2abij(o_opt *W, const o_opt *r2, const o_opt *abij, double f)
{ return o_vv2v_444(abij, r2, W, r2->d.iop[0] == 0 ? f : 0.5 * f, "efmn", "efij", "mnij", 0); }

const i64 *o_zorb(void) { return ZORB; }

/* ---- kernels of the second-order ground state (src/grCPSd.SF/calL1_VTT.f90,
 * calL2_VTT.f90) ---- */

/* Wkbij_r1iabj.f90:1-16: W(ij,kb) -= f*P(ij){V(ck,bj)*r(c,i)} */
int o_Wkbij_r1iabj(o_opt *W, const o_opt *r1, const o_opt *iabj, double f)
{ return o_vv2v_424(iabj, r1, W, -f, "ckbj", "ci", "ijkb", 1); }

/* Wabdj_r1abcd.f90:1-18 (incore branch): W(ab,dj) += f*V(ab,dc)*r(c,j) */
int o_Wabdj_r1abcd(o_opt *W, const o_opt *r1, const o_opt *abcd, double f)
{ return o_vv2v_424(abcd, r1, W, f, "abdc", "cj", "abdj", 0); }

/* Wkbij_r1Uklij.f90:1-16: W(ij,kb) -= f*U(kl,ij)*r(b,l) */
int o_Wkbij_r1Uklij(o_opt *W, const o_opt *r1, const o_opt *U, double f)
{ return o_vv2v_424(U, r1, W, -f, "klij", "bl", "ijkb", 0); }

/* Fme_r1abij.f90:1-16: F(e,m) += f*r(f,n)*V(ef,mn) */
int o_Fme_r1abij(o_opt *F, const o_opt *r1, const o_opt *abij, double f)
{ return o_vv2v_422(abij, r1, F, f, "efmn", "fn", "em"); }

/* c1_r2Fme.f90:1-16: c(a,i) += f*r(ae,im)*F(e,m) */
int o_c1_r2Fme(o_opt *c1, const o_opt *r2, const o_opt *F, double f)
{ return o_vv2v_422(r2, F, c1, f, "aeim", "em", "ai"); }

/* p_effectT2 (effectT2.f90:47-140) types 1 and 2 on an antisymmetric
 * t(ab,ij): type 1 t += f [x(a,i) x(b,j) - x(a,j) x(b,i)] (x = y),
 * type 2 t += f P(ab) P(ij) {x(a,i) y(b,j)}.  Both are the outer product
 * antisymmetrised in both pairs (vv2v_224 with anti 3); for x = y the
 * double antisymmetrisation counts each term twice, hence f / 2. */
int o_effectT2(o_opt *t2, const o_opt *x, const o_opt *y, double f, int type)
{
    if (type != 1 && type != 2) return O_EARG;
    return o_vv2v_224(x, y, t2, type == 1 ? 0.5 * f : f, "ai", "bj", "abij", 3);
}

/* ---- kernels of the excited-state grCPS(D) (src/EE-grCPSd.SF: the left
 * vector of calEigenCISDoo.f90, calJ.f90, calC_VTTR.f90) ---- */

/* c1d_l1Wibaj.f90:1-16: c(a,i) += W(ai,bj) l(b,j) */
int o_c1d_l1Wibaj(o_opt *c1, const o_opt *l1, const o_opt *W, double f)
{ return o_vv2v_422(W, l1, c1, f, "aibj", "bj", "ai"); }

/* c1d_l1fab.f90:1-16: c(a,i) -= f(b,a) l(b,i) */
int o_c1d_l1fab(o_opt *c1, const o_opt *l1, const o_opt *F, double f)
{ return o_vv2v_222(F, l1, c1, -f, "ba", "bi", "ai"); }

/* c1d_l1fij.f90:1-16: c(a,i) += f(i,j) l(a,j) */
int o_c1d_l1fij(o_opt *c1, const o_opt *l1, const o_opt *F, double f)
{ return o_vv2v_222(l1, F, c1, f, "aj", "ij", "ai"); }

/* Fae_r1fia.f90:1-16: F(a,e) -= f(e,l) r(a,l) */
int o_Fae_r1fia(o_opt *c1, const o_opt *r1, const o_opt *F, double f)
{ return o_vv2v_222(r1, F, c1, -f, "al", "el", "ae"); }

/* Fmi_r1fia.f90:1-16: F(m,i) += r(d,i) f(d,m) */
int o_Fmi_r1fia(o_opt *c1, const o_opt *r1, const o_opt *F, double f)
{ return o_vv2v_222(F, r1, c1, f, "dm", "di", "mi"); }

/* Wkbij_r2Fkc.f90:1-16: W(ij,kb) -= F(c,k) r(cb,ij) */
int o_Wkbij_r2Fkc(o_opt *c1, const o_opt *r2, const o_opt *F, double f)
{ return o_vv2v_424(r2, F, c1, -f, "cbij", "ck", "ijkb", 0); }

/* Wlkjd_r1abij.f90:1-16: W(lk,jd) += r(c,j) V(cd,lk) */
int o_Wlkjd_r1abij(o_opt *c1, const o_opt *r1, const o_opt *V, double f)
{ return o_vv2v_424(V, r1, c1, f, "cdlk", "cj", "lkjd", 0); }
