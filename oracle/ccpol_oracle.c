/*
 * ccpol_oracle.c -- CPU FP64 oracle (TEST INFRASTRUCTURE ONLY; see ccpol_oracle.h).
 *
 * Restates, in C, the reference Fortran routines of ommair/CCpol23_plus_2025_MBMD that form
 * the force-evaluation hot path.  Loop nesting, cut-off tests, minimum-image arithmetic and
 * per-term formulas follow the cited reference lines; MPI reductions collapse to the
 * single-process case.  OpenMP splits the outermost molecule loop statically and reduces
 * per-thread partial arrays in thread order, as the reference's (inactive) !$omp regions
 * do with private arrays, so results are deterministic for a given thread count.
 */
#include "ccpol_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* common_arrays.f90:28-36, 189-190 */
static const double PI = 3.14159265358979323846264338327950288;
static const double R4PIE0 = 138935.4835;
static const double BOHR2A = 0.529177249;
static const double H2KCAL = 627.510;
#define TWOSQPI (2.0 / sqrt(PI))
#define DELTA2 (1.65 / BOHR2A)
#define DELTA3 (1.55 / BOHR2A)

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
static int nthreads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* Fortran nint: round half away from zero. */
static inline double fnint(double v) { return round(v); }
static inline double minimg(double d, double box) { return d - box * fnint(d / box); }

/* ---------------------------------------------------------------- utility.f90:89-125 */
double orc_tt(int n, double delta, double r) {
    double deltar = delta * r, term = 1.0, ssum = 1.0;
    for (int i = 1; i <= n; i++) {
        term = term * deltar / (double)i;
        ssum = ssum + term;
    }
    return 1.0 - exp(-deltar) * ssum;
}

double orc_dtt(int n, double delta, double r) {
    double ffact = 1.0;
    for (int i = 1; i <= n; i++) ffact = ffact * (double)i;
    double delr = delta * r;
    return delta * exp(-delr) * pow(delr, (double)n) / ffact;
}

/* ------------------------------------------- threebody_potential.f90:909-946, 2064-2131 */
static const int FS3_NTYPE[17] = {1, 2, 2, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 6, 6, 6, 6};

/* linear position of ntab(kp,jp,ip,k,j,i) in a 0-based array (k,j,i 1-based). */
static inline int tab_pos(int kp, int jp, int ip, int k, int j, int i) {
    return kp + 2 * jp + 4 * ip + 8 * (k - 1) + 136 * (j - 1) + 2312 * (i - 1);
}

static void type_block(int site, int *first, int *last) {
    int t = FS3_NTYPE[site - 1];
    *first = 0;
    *last = 0;
    for (int s = 1; s <= 17; s++) {
        if (FS3_NTYPE[s - 1] == t) {
            if (*first == 0) *first = s;
            *last = s;
        }
    }
}

static void fill_class(int *ntab, int iat, int jat, int kat, int ip, int jp, int kp, int nr) {
    int i0, i1, j0, j1, k0, k1;
    type_block(iat, &i0, &i1);
    type_block(jat, &j0, &j1);
    type_block(kat, &k0, &k1);
    for (int ii = i0; ii <= i1; ii++)
        for (int jj = j0; jj <= j1; jj++)
            for (int kk = k0; kk <= k1; kk++) {
                ntab[tab_pos(kp, jp, ip, kk, jj, ii)] = nr;
                ntab[tab_pos(jp, kp, ip, jj, kk, ii)] = nr;
                ntab[tab_pos(ip, kp, jp, ii, kk, jj)] = nr;
                ntab[tab_pos(kp, ip, jp, kk, ii, jj)] = nr;
                ntab[tab_pos(ip, jp, kp, ii, jj, kk)] = nr;
                ntab[tab_pos(jp, ip, kp, jj, ii, kk)] = nr;
            }
}

int orc_fill_index(int *ind) {
    memset(ind, 0, sizeof(int) * ORC_NTAB);
    int nnew = 0;
    for (int iat = 1; iat <= 17; iat++)
        for (int jat = 1; jat <= 17; jat++)
            for (int kat = 1; kat <= 17; kat++)
                for (int ip = 0; ip <= 1; ip++)
                    for (int jp = 0; jp <= 1; jp++)
                        for (int kp = 0; kp <= 1; kp++) {
                            int idx = tab_pos(kp, jp, ip, kat, jat, iat);
                            if (ind[idx] == 0) {
                                nnew++;
                                fill_class(ind, iat, jat, kat, ip, jp, kp, nnew);
                            }
                        }
    return nnew;
}

/* ---------------------------------------------------------------- ewald.f90:17-43 */
void orc_ewald_setup(double ewps, double rcut, double box, double *alp, int *k1, int *k2,
                     int *k3) {
    double eprec = fmin(fabs(ewps), 0.5);
    double tol = sqrt(fabs(log(eprec * rcut)));
    double a = sqrt(fabs(log(eprec * rcut * tol))) / rcut;
    double t2 = 2.0 * tol * a;
    double tol1 = sqrt(-log(eprec * rcut * (t2 * t2)));
    double fac = 1.0;
    int k = (int)fnint(0.25 + fac * box * a * tol1 / PI);
    *alp = a;
    *k1 = k;
    *k2 = k;
    *k3 = k;
}

/* ------------------------------------------------------- per-thread accumulation helper */
typedef struct {
    double *fx, *fy, *fz; /* site arrays [nm*ns] */
    double *cx, *cy, *cz; /* COM arrays [nm] */
    double e, v;
} acc_t;

static acc_t *acc_alloc(int nt, int nm, int ns) {
    acc_t *a = (acc_t *)calloc((size_t)nt, sizeof(acc_t));
    for (int t = 0; t < nt; t++) {
        a[t].fx = (double *)calloc((size_t)nm * ns, sizeof(double));
        a[t].fy = (double *)calloc((size_t)nm * ns, sizeof(double));
        a[t].fz = (double *)calloc((size_t)nm * ns, sizeof(double));
        a[t].cx = (double *)calloc((size_t)nm, sizeof(double));
        a[t].cy = (double *)calloc((size_t)nm, sizeof(double));
        a[t].cz = (double *)calloc((size_t)nm, sizeof(double));
    }
    return a;
}

static void acc_free(acc_t *a, int nt) {
    for (int t = 0; t < nt; t++) {
        free(a[t].fx); free(a[t].fy); free(a[t].fz);
        free(a[t].cx); free(a[t].cy); free(a[t].cz);
    }
    free(a);
}

/* --------------------------------------------------- threebody_potential.f90:101-674 */
void orc_fs2_term_bohr(const orc_model *m, const double *xx, const double *yy,
                       const double *zz, const double *xxs, const double *yys,
                       const double *zzs, int ld, double boxi, double *qfs2, double *fxs,
                       double *fys, double *fzs, double *fxfs2, double *fyfs2, double *fzfs2,
                       double *vir) {
    const int nm = m->nm, ns = m->ns;
    const double eta3 = 0.48056977605478400, beta3 = 0.85836606579445000, g3 = 0.4;
    const double alp3 = m->alpha3 * BOHR2A;
    const double rc2 = m->rcutsd3 * pow(BOHR2A, -2.0);
    const double r0dmp = 7.40446 / BOHR2A;
    const double delta33 = m->delta33;
    double charge3b[ORC_NSITE_MAX];
    for (int s = 0; s < ns; s++) charge3b[s] = 0.0;
    charge3b[0] = 0.258504607653328389;
    charge3b[1] = 0.564050362569283648;
    charge3b[2] = 0.564050362569283648;
    charge3b[3] = -0.693302666395947953;
    charge3b[4] = -0.693302666395947953;
#define XS(a, s, i) a[(size_t)(i) * ld + (s)]

    const int nt = nthreads();
    acc_t *acc = acc_alloc(nt, nm, ns);
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        acc_t *A = &acc[omp_get_thread_num()];
#else
        acc_t *A = &acc[0];
#endif
#pragma omp for schedule(static, 1)
        for (int k = 0; k < nm; k++) {
            for (int i = 0; i < nm - 1; i++) {
                if (k == i) continue;
                for (int j = i + 1; j < nm; j++) {
                    if (j == k) continue;
                    double dxij = xx[i] - xx[j], dyij = yy[i] - yy[j], dzij = zz[i] - zz[j];
                    double dxki = xx[k] - xx[i], dyki = yy[k] - yy[i], dzki = zz[k] - zz[i];
                    double xij = minimg(dxij, boxi), yij = minimg(dyij, boxi),
                           zij = minimg(dzij, boxi);
                    double xki = minimg(dxki, boxi), yki = minimg(dyki, boxi),
                           zki = minimg(dzki, boxi);
                    double xkj = xki + xij, ykj = yki + yij, zkj = zki + zij;
                    double dij2 = xij * xij + yij * yij + zij * zij;
                    double dki2 = xki * xki + yki * yki + zki * zki;
                    double dkj2 = xkj * xkj + ykj * ykj + zkj * zkj;
                    if (!(dij2 < rc2 && dki2 < rc2 && dkj2 < rc2)) continue;

                    double pom = exp(alp3 * (sqrt(dki2) - r0dmp));
                    double pomki = 1.0 / (1.0 + pom);
                    double flrki = pow(pomki, delta33);
                    double dflrki = -alp3 * delta33 * pom * pomki * flrki;
                    double dflrkiv = -alp3 * delta33 * pom * pomki * sqrt(dki2);
                    pom = exp(alp3 * (sqrt(dkj2) - r0dmp));
                    double pomkj = 1.0 / (1.0 + pom);
                    double flrkj = pow(pomkj, delta33);
                    double dflrkj = -alp3 * delta33 * pom * pomkj * flrkj;
                    double dflrkjv = -alp3 * delta33 * pom * pomkj * sqrt(dkj2);

                    for (int ks = 0; ks < 5; ks++) {
                        double qks = charge3b[ks];
                        for (int is = 0; is < 3; is++) {
                            for (int js = 0; js < 3; js++) {
                                double xsij = xij + (XS(xxs, is, i) - XS(xxs, js, j));
                                double ysij = yij + (XS(yys, is, i) - XS(yys, js, j));
                                double zsij = zij + (XS(zzs, is, i) - XS(zzs, js, j));
                                double dsij2 = xsij * xsij + ysij * ysij + zsij * zsij;
                                double dsij = sqrt(dsij2);
                                double dsij1i = 1.0 / dsij;
                                double eqij = eta3 * exp(-beta3 * dsij);
                                double dij = sqrt(dij2), dij1i = 1.0 / dij,
                                       dij3i = dij1i * dij1i * dij1i;
                                double dki = sqrt(dki2), dki1i = 1.0 / dki;
                                double dkj = sqrt(dkj2), dkj1i = 1.0 / dkj;
                                (void)dki1i;
                                (void)dkj1i;
                                double sk_x = XS(xxs, ks, k), sk_y = XS(yys, ks, k),
                                       sk_z = XS(zzs, ks, k);
                                double dxkqi = xki + sk_x - g3 * xij * dij1i;
                                double dykqi = yki + sk_y - g3 * yij * dij1i;
                                double dzkqi = zki + sk_z - g3 * zij * dij1i;
                                double dkqi = sqrt(dxkqi * dxkqi + dykqi * dykqi + dzkqi * dzkqi);
                                double dkqi1i = 1.0 / dkqi;
                                double dkqi3i = dkqi1i * dkqi1i * dkqi1i;
                                double dxkqj = xkj + sk_x + g3 * xij * dij1i;
                                double dykqj = ykj + sk_y + g3 * yij * dij1i;
                                double dzkqj = zkj + sk_z + g3 * zij * dij1i;
                                double dkqj = sqrt(dxkqj * dxkqj + dykqj * dykqj + dzkqj * dzkqj);
                                double dkqj1i = 1.0 / dkqj;
                                double dkqj3i = dkqj1i * dkqj1i * dkqj1i;
                                double dxkci = xki + sk_x, dykci = yki + sk_y, dzkci = zki + sk_z;
                                double dkci = sqrt(dxkci * dxkci + dykci * dykci + dzkci * dzkci);
                                double dkci1i = 1.0 / dkci;
                                double dkci3i = dkci1i * dkci1i * dkci1i;
                                double dxkcj = xkj + sk_x, dykcj = ykj + sk_y, dzkcj = zkj + sk_z;
                                double dkcj = sqrt(dxkcj * dxkcj + dykcj * dykcj + dzkcj * dzkcj);
                                double dkcj1i = 1.0 / dkcj;
                                double dkcj3i = dkcj1i * dkcj1i * dkcj1i;

                                double fl = flrki * flrkj;
                                double term0 = (dkci1i + dkcj1i - dkqi1i - dkqj1i);
                                A->e += qks * eqij * term0 * flrki * flrkj;
                                double termxy1 =
                                    (dxkqi * xij + dykqi * yij + dzkqi * zij) * g3 * dij1i * dkqi3i;
                                double termxy2 =
                                    (dxkqj * xij + dykqj * yij + dzkqj * zij) * g3 * dij1i * dkqj3i;
                                A->v += ((-beta3 * dsij - 1.0) + dflrkiv + dflrkjv) * qks * eqij *
                                            term0 * flrki * flrkj +
                                        qks * eqij * (termxy1 - termxy2) * flrki * flrkj;

                                double dotkqi = xij * dxkqi + yij * dykqi + zij * dzkqi;
                                double dotkqj = xij * dxkqj + yij * dykqj + zij * dzkqj;
                                double qe = qks * eqij;
                                double fxk = qe * (-dxkci * dkci3i - dxkcj * dkcj3i +
                                                   dxkqi * dkqi3i + dxkqj * dkqj3i);
                                double fyk = qe * (-dykci * dkci3i - dykcj * dkcj3i +
                                                   dykqi * dkqi3i + dykqj * dkqj3i);
                                double fzk = qe * (-dzkci * dkci3i - dzkcj * dkcj3i +
                                                   dzkqi * dkqi3i + dzkqj * dkqj3i);
                                double sdki = sqrt(dki2), sdkj = sqrt(dkj2);
                                A->cx[k] += -qe * term0 * dflrki * xki * flrkj / sdki -
                                            qe * term0 * dflrkj * xkj * flrki / sdkj;
                                A->cy[k] += -qe * term0 * dflrki * yki * flrkj / sdki -
                                            qe * term0 * dflrkj * ykj * flrki / sdkj;
                                A->cz[k] += -qe * term0 * dflrki * zki * flrkj / sdki -
                                            qe * term0 * dflrkj * zkj * flrki / sdkj;

                                double fxi1 = qe * (-beta3) * term0 * xsij * dsij1i;
                                double fyi1 = qe * (-beta3) * term0 * ysij * dsij1i;
                                double fzi1 = qe * (-beta3) * term0 * zsij * dsij1i;
                                double fxi2 = qe * (dxkci * dkci3i), fyi2 = qe * (dykci * dkci3i),
                                       fzi2 = qe * (dzkci * dkci3i);
                                double gi = 1.0 + g3 * dij1i;
                                double fxi3 = qe * dkqi3i * (-gi * dxkqi + g3 * dotkqi * xij * dij3i);
                                double fyi3 = qe * dkqi3i * (-gi * dykqi + g3 * dotkqi * yij * dij3i);
                                double fzi3 = qe * dkqi3i * (-gi * dzkqi + g3 * dotkqi * zij * dij3i);
                                double fxi4 = qe * dkqj3i * (g3 * dxkqj * dij1i - g3 * dotkqj * xij * dij3i);
                                double fyi4 = qe * dkqj3i * (g3 * dykqj * dij1i - g3 * dotkqj * yij * dij3i);
                                double fzi4 = qe * dkqj3i * (g3 * dzkqj * dij1i - g3 * dotkqj * zij * dij3i);
                                double fxj1 = qe * beta3 * term0 * xsij * dsij1i;
                                double fyj1 = qe * beta3 * term0 * ysij * dsij1i;
                                double fzj1 = qe * beta3 * term0 * zsij * dsij1i;
                                double fxj2 = qe * (dxkcj * dkcj3i), fyj2 = qe * (dykcj * dkcj3i),
                                       fzj2 = qe * (dzkcj * dkcj3i);
                                double fxj3 = qe * dkqi3i * (g3 * dxkqi * dij1i - g3 * dotkqi * xij * dij3i);
                                double fyj3 = qe * dkqi3i * (g3 * dykqi * dij1i - g3 * dotkqi * yij * dij3i);
                                double fzj3 = qe * dkqi3i * (g3 * dzkqi * dij1i - g3 * dotkqi * zij * dij3i);
                                double fxj4 = qe * dkqj3i * (-gi * dxkqj + g3 * dotkqj * xij * dij3i);
                                double fyj4 = qe * dkqj3i * (-gi * dykqj + g3 * dotkqj * yij * dij3i);
                                double fzj4 = qe * dkqj3i * (-gi * dzkqj + g3 * dotkqj * zij * dij3i);

                                size_t sk = (size_t)k * ns + ks, si = (size_t)i * ns + is,
                                       sj = (size_t)j * ns + js;
                                A->fx[sk] -= fxk * fl;
                                A->fy[sk] -= fyk * fl;
                                A->fz[sk] -= fzk * fl;
                                A->fx[si] -= fxi1 * fl;
                                A->fy[si] -= fyi1 * fl;
                                A->fz[si] -= fzi1 * fl;
                                A->fx[sj] -= fxj1 * fl;
                                A->fy[sj] -= fyj1 * fl;
                                A->fz[sj] -= fzj1 * fl;
                                A->cx[i] += -(fxi2 + fxi3 + fxi4) * fl +
                                            qe * term0 * dflrki * xki * flrkj / sdki;
                                A->cy[i] += -(fyi2 + fyi3 + fyi4) * fl +
                                            qe * term0 * dflrki * yki * flrkj / sdki;
                                A->cz[i] += -(fzi2 + fzi3 + fzi4) * fl +
                                            qe * term0 * dflrki * zki * flrkj / sdki;
                                A->cx[j] += -(fxj2 + fxj3 + fxj4) * fl +
                                            qe * term0 * flrki * dflrkj * xkj / sdkj;
                                A->cy[j] += -(fyj2 + fyj3 + fyj4) * fl +
                                            qe * term0 * flrki * dflrkj * ykj / sdkj;
                                A->cz[j] += -(fzj2 + fzj3 + fzj4) * fl +
                                            qe * term0 * flrki * dflrkj * zkj / sdkj;
                                (void)dij;
                                (void)dki;
                                (void)dkj;
                            }
                        }
                    }
                }
            }
        }
    }
    /* threebody_potential.f90:575-671: unit conversion, reduction, overwrite COM forces */
    const double cf = H2KCAL * 418.4 / BOHR2A;
    double e = 0.0, v = 0.0;
    for (int i = 0; i < nm; i++) {
        fxfs2[i] = 0.0;
        fyfs2[i] = 0.0;
        fzfs2[i] = 0.0;
    }
    for (int t = 0; t < nt; t++) {
        for (int i = 0; i < nm; i++) {
            fxfs2[i] += acc[t].cx[i] * cf;
            fyfs2[i] += acc[t].cy[i] * cf;
            fzfs2[i] += acc[t].cz[i] * cf;
            for (int s = 0; s < ns; s++) {
                fxs[(size_t)i * ld + s] += acc[t].fx[(size_t)i * ns + s] * cf;
                fys[(size_t)i * ld + s] += acc[t].fy[(size_t)i * ns + s] * cf;
                fzs[(size_t)i * ld + s] += acc[t].fz[(size_t)i * ns + s] * cf;
            }
        }
        e += acc[t].e;
        v += acc[t].v;
    }
    acc_free(acc, nt);
    *qfs2 = e * H2KCAL;
    *vir += v * H2KCAL * 418.4;
}

/* --------------------------------------------------- threebody_potential.f90:676-2062 */
typedef struct {
    const double *b, *g, *r0, *cs;
} fs3_tab;

/* One SR or LR sweep over the 17^3 site triples and 2^3 powers of a molecular triple,
   restating the inner loops of threebody_potential.f90:956-1170 (SR), 1183-1405 (LR) and
   1418-1937 (blend).  wsw multiplies energy and site-force terms (1, smfun or 1-smfun);
   cfs adds the switch derivative to the COM coefficient (0, +cf or -cf). */
static void fs3_sweep(const orc_model *m, const fs3_tab *T, int ld, const double *xxs,
                      const double *yys, const double *zzs, int i, int j, int k, double xij,
                      double yij, double zij, double xik, double yik, double zik, double xjk,
                      double yjk, double zjk, double dij2, double dik2, double djk2,
                      double fdmp, double dfdmp, double wsw, double cfs, acc_t *A) {
    const int ns = m->ns;
    const double rij = sqrt(dij2), rik = sqrt(dik2), rjk = sqrt(djk2);
    const double comc = dfdmp * wsw + fdmp * cfs;
    int itab = 0;
    for (int is = 0; is < 17; is++) {
        for (int js = 0; js < 17; js++) {
            for (int ks = 0; ks < 17; ks++) {
                double bsij = T->b[is * 17 + js], gsij = T->g[is * 17 + js], r0sij = T->r0[is * 17 + js];
                double xsij = xij + (XS(xxs, is, i) - XS(xxs, js, j));
                double ysij = yij + (XS(yys, is, i) - XS(yys, js, j));
                double zsij = zij + (XS(zzs, is, i) - XS(zzs, js, j));
                double dsij2 = xsij * xsij + ysij * ysij + zsij * zsij;
                double dsij = sqrt(dsij2);
                double dampsij = 1.0 / (1.0 + exp(-gsij * (dsij - r0sij)));

                double bsik = T->b[is * 17 + ks], gsik = T->g[is * 17 + ks], r0sik = T->r0[is * 17 + ks];
                double xsik = xik + (XS(xxs, is, i) - XS(xxs, ks, k));
                double ysik = yik + (XS(yys, is, i) - XS(yys, ks, k));
                double zsik = zik + (XS(zzs, is, i) - XS(zzs, ks, k));
                double dsik2 = xsik * xsik + ysik * ysik + zsik * zsik;
                double dsik = sqrt(dsik2);
                double dampsik = 1.0 / (1.0 + exp(-gsik * (dsik - r0sik)));

                double bsjk = T->b[js * 17 + ks], gsjk = T->g[js * 17 + ks], r0sjk = T->r0[js * 17 + ks];
                double xsjk = xjk + (XS(xxs, js, j) - XS(xxs, ks, k));
                double ysjk = yjk + (XS(yys, js, j) - XS(yys, ks, k));
                double zsjk = zjk + (XS(zzs, js, j) - XS(zzs, ks, k));
                double dsjk2 = xsjk * xsjk + ysjk * ysjk + zsjk * zsjk;
                double dsjk = sqrt(dsjk2);
                double dampsjk = 1.0 / (1.0 + exp(-gsjk * (dsjk - r0sjk)));

                double eks = (exp(-bsij * dsij) * dampsij) * (exp(-bsik * dsik) * dampsik) *
                             (exp(-bsjk * dsjk) * dampsjk);
                double der_fij = -bsij + gsij * exp(-gsij * (dsij - r0sij)) * dampsij;
                double der_fik = -bsik + gsik * exp(-gsik * (dsik - r0sik)) * dampsik;
                double der_fjk = -bsjk + gsjk * exp(-gsjk * (dsjk - r0sjk)) * dampsjk;

                for (int ip = 0; ip <= 1; ip++) {
                    double term1 = eks * (ip ? dsjk : 1.0);
                    double fsjk = der_fjk / dsjk + (double)ip / (dsjk * dsjk);
                    for (int jp = 0; jp <= 1; jp++) {
                        double term2 = term1 * (jp ? dsik : 1.0);
                        double fsik = der_fik / dsik + (double)jp / (dsik * dsik);
                        for (int kp = 0; kp <= 1; kp++) {
                            int iind = m->ind_lin[itab++];
                            double term3 = term2 * (kp ? dsij : 1.0);
                            double fsij = der_fij / dsij + (double)kp / (dsij * dsij);
                            double c = T->cs[iind - 1];
                            double ct = c * term3;
                            A->e += wsw * (ct * fdmp);
                            /* add_pair_virial_trace (threebody_potential.f90:2133-2142) */
                            A->v += ct * fdmp * wsw * fsij * dsij2;
                            A->v += ct * fdmp * wsw * fsik * dsik2;
                            A->v += ct * fdmp * wsw * fsjk * dsjk2;
                            A->v += ct * comc / rij * dij2;
                            A->v += ct * comc / rik * dik2;
                            A->v += ct * comc / rjk * djk2;
                            double sf = ct * fdmp * wsw;
                            size_t si = (size_t)i * ns + is, sj = (size_t)j * ns + js,
                                   sk = (size_t)k * ns + ks;
                            A->fx[si] -= sf * (fsij * xsij + fsik * xsik);
                            A->fy[si] -= sf * (fsij * ysij + fsik * ysik);
                            A->fz[si] -= sf * (fsij * zsij + fsik * zsik);
                            A->fx[sj] -= sf * (-fsij * xsij + fsjk * xsjk);
                            A->fy[sj] -= sf * (-fsij * ysij + fsjk * ysjk);
                            A->fz[sj] -= sf * (-fsij * zsij + fsjk * zsjk);
                            A->fx[sk] -= sf * (-fsik * xsik - fsjk * xsjk);
                            A->fy[sk] -= sf * (-fsik * ysik - fsjk * ysjk);
                            A->fz[sk] -= sf * (-fsik * zsik - fsjk * zsjk);
                            A->cx[i] -= ct * comc * (xij / rij + xik / rik);
                            A->cy[i] -= ct * comc * (yij / rij + yik / rik);
                            A->cz[i] -= ct * comc * (zij / rij + zik / rik);
                            A->cx[j] -= ct * comc * (-xij / rij + xjk / rjk);
                            A->cy[j] -= ct * comc * (-yij / rij + yjk / rjk);
                            A->cz[j] -= ct * comc * (-zij / rij + zjk / rjk);
                            A->cx[k] -= ct * comc * (-xik / rik - xjk / rjk);
                            A->cy[k] -= ct * comc * (-yik / rik - yjk / rjk);
                            A->cz[k] -= ct * comc * (-zik / rik - zjk / rjk);
                        }
                    }
                }
            }
        }
    }
}

static void orc_fs3_term_bohr(const orc_model *m, const double *xx, const double *yy,
                              const double *zz, const double *xxs, const double *yys,
                              const double *zzs, int ld, double boxi, double *qfs3,
                              double *fxs, double *fys, double *fzs, double *fxfs3,
                              double *fyfs3, double *fzfs3, double *vir) {
    const int nm = m->nm, ns = m->ns;
    const double rc2 = pow(6.3, 2.0) * pow(BOHR2A, -2.0);
    const double alp3 = m->alpha3 * BOHR2A;
    const double r0dmp = 6.20446 / BOHR2A;
    const double rmin = 4.5 / BOHR2A, rmax = 5.5 / BOHR2A;
    const double delta33 = m->delta33;
    const fs3_tab TS = {m->bS3_s, m->gS3_s, m->r0S3_s, m->cs3_s};
    const fs3_tab TL = {m->bS3_l, m->gS3_l, m->r0S3_l, m->cs3_l};

    const int nt = nthreads();
    acc_t *acc = acc_alloc(nt, nm, ns);
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        acc_t *A = &acc[omp_get_thread_num()];
#else
        acc_t *A = &acc[0];
#endif
#pragma omp for schedule(static, 1)
        for (int i = 0; i < nm - 2; i++) {
            for (int j = i + 1; j < nm - 1; j++) {
                for (int k = j + 1; k < nm; k++) {
                    double dxij = xx[i] - xx[j], dyij = yy[i] - yy[j], dzij = zz[i] - zz[j];
                    double dxik = xx[i] - xx[k], dyik = yy[i] - yy[k], dzik = zz[i] - zz[k];
                    double dxjk = xx[j] - xx[k], dyjk = yy[j] - yy[k], dzjk = zz[j] - zz[k];
                    double xij = minimg(dxij, boxi), yij = minimg(dyij, boxi), zij = minimg(dzij, boxi);
                    double xik = minimg(dxik, boxi), yik = minimg(dyik, boxi), zik = minimg(dzik, boxi);
                    double xjk = dxjk + boxi * fnint(dxij / boxi) - boxi * fnint(dxik / boxi);
                    double yjk = dyjk + boxi * fnint(dyij / boxi) - boxi * fnint(dyik / boxi);
                    double zjk = dzjk + boxi * fnint(dzij / boxi) - boxi * fnint(dzik / boxi);
                    double dij2 = xij * xij + yij * yij + zij * zij;
                    double dik2 = xik * xik + yik * yik + zik * zik;
                    double djk2 = xjk * xjk + yjk * yjk + zjk * zjk;
                    if (!(dij2 < rc2 && dik2 < rc2 && djk2 < rc2)) continue;
                    double ravg = (sqrt(dij2) + sqrt(djk2) + sqrt(dik2)) / 3.0;
                    double pomij = exp(alp3 * (ravg - r0dmp));
                    double ppomij = 1.0 / (1.0 + pomij);
                    double fdmp = pow(ppomij, delta33);
                    double dfdmp = -alp3 * delta33 * pomij * ppomij * fdmp * (1.0 / 3.0);
                    if (ravg <= rmin) {
                        fs3_sweep(m, &TS, ld, xxs, yys, zzs, i, j, k, xij, yij, zij, xik, yik, zik,
                                  xjk, yjk, zjk, dij2, dik2, djk2, fdmp, dfdmp, 1.0, 0.0, A);
                    } else if (ravg >= rmax) {
                        fs3_sweep(m, &TL, ld, xxs, yys, zzs, i, j, k, xij, yij, zij, xik, yik, zik,
                                  xjk, yjk, zjk, dij2, dik2, djk2, fdmp, dfdmp, 1.0, 0.0, A);
                    } else {
                        double cfact = (ravg - rmin) / (rmax - rmin);
                        double smfun = 1.0 + 2.0 * pow(cfact, 3.0) - 3.0 * pow(cfact, 2.0);
                        double smfun2 = 1.0 - smfun;
                        double cf = 2.0 / (rmax - rmin) * (pow(cfact, 2.0) - cfact);
                        fs3_sweep(m, &TS, ld, xxs, yys, zzs, i, j, k, xij, yij, zij, xik, yik, zik,
                                  xjk, yjk, zjk, dij2, dik2, djk2, fdmp, dfdmp, smfun, cf, A);
                        fs3_sweep(m, &TL, ld, xxs, yys, zzs, i, j, k, xij, yij, zij, xik, yik, zik,
                                  xjk, yjk, zjk, dij2, dik2, djk2, fdmp, dfdmp, smfun2, -cf, A);
                    }
                }
            }
        }
    }
    const double cf = H2KCAL * 418.4 / BOHR2A;
    double e = 0.0, v = 0.0;
    for (int i = 0; i < nm; i++) {
        fxfs3[i] = 0.0;
        fyfs3[i] = 0.0;
        fzfs3[i] = 0.0;
    }
    for (int t = 0; t < nt; t++) {
        for (int i = 0; i < nm; i++) {
            fxfs3[i] += acc[t].cx[i] * cf;
            fyfs3[i] += acc[t].cy[i] * cf;
            fzfs3[i] += acc[t].cz[i] * cf;
            for (int s = 0; s < ns; s++) {
                fxs[(size_t)i * ld + s] += acc[t].fx[(size_t)i * ns + s] * cf;
                fys[(size_t)i * ld + s] += acc[t].fy[(size_t)i * ns + s] * cf;
                fzs[(size_t)i * ld + s] += acc[t].fz[(size_t)i * ns + s] * cf;
            }
        }
        e += acc[t].e;
        v += acc[t].v;
    }
    acc_free(acc, nt);
    *qfs3 = H2KCAL * e;
    *vir += v * H2KCAL * 418.4;
}

/* ---------------------------------------------------- threebody_potential.f90:17-99 */
void orc_threebody_term(const orc_model *m, const double *x, const double *y,
                        const double *z, const double *xs, const double *ys,
                        const double *zs, int ld, double box, double *qfs2, double *qfs3,
                        double *fxs, double *fys, double *fzs, double *fxfs2, double *fyfs2,
                        double *fzfs2, double *fxfs3, double *fyfs3, double *fzfs3,
                        double *vir) {
    const int nm = m->nm, ns = m->ns;
    double *xx = (double *)malloc(sizeof(double) * nm), *yy = (double *)malloc(sizeof(double) * nm),
           *zz = (double *)malloc(sizeof(double) * nm);
    double *xxs = (double *)calloc((size_t)nm * ld, sizeof(double)),
           *yys = (double *)calloc((size_t)nm * ld, sizeof(double)),
           *zzs = (double *)calloc((size_t)nm * ld, sizeof(double));
    for (int i = 0; i < nm; i++) {
        xx[i] = x[i] / BOHR2A;
        yy[i] = y[i] / BOHR2A;
        zz[i] = z[i] / BOHR2A;
        for (int s = 0; s < ns; s++) {
            xxs[(size_t)i * ld + s] = xs[(size_t)i * ld + s] / BOHR2A;
            yys[(size_t)i * ld + s] = ys[(size_t)i * ld + s] / BOHR2A;
            zzs[(size_t)i * ld + s] = zs[(size_t)i * ld + s] / BOHR2A;
        }
    }
    double boxi = box / BOHR2A;
    if (m->s2_term)
        orc_fs2_term_bohr(m, xx, yy, zz, xxs, yys, zzs, ld, boxi, qfs2, fxs, fys, fzs, fxfs2,
                          fyfs2, fzfs2, vir);
    if (m->s3_term)
        orc_fs3_term_bohr(m, xx, yy, zz, xxs, yys, zzs, ld, boxi, qfs3, fxs, fys, fzs, fxfs3,
                          fyfs3, fzfs3, vir);
    free(xx); free(yy); free(zz);
    free(xxs); free(yys); free(zzs);
}

/* ---------------------------------------------------------------- ewald.f90:45-174 */
void orc_ewald_self_correction(const orc_model *m, double alp, double box, const double *x,
                               const double *y, const double *z, const double *xs,
                               const double *ys, const double *zs, int ld, double *qscpe,
                               double *fxs, double *fys, double *fzs, double *vir) {
    const int nm = m->nm, ns = m->ns;
    double volmi = box * box * box;
    double sumq = 0.0, sumq2 = 0.0;
    for (int i = 0; i < nm; i++)
        for (int is = 0; is < ns; is++) {
            sumq = sumq + m->charge[is];
            sumq2 = sumq2 + m->charge[is] * m->charge[is];
        }
    double t = sumq / alp;
    double e_selfp = -PI * (t * t) / (2.0 * volmi);
    e_selfp = e_selfp - alp * sumq2 / sqrt(PI);
    double sumff = 0.0, qv = 0.0;
    for (int i = 0; i < nm; i++) {
        for (int is = 0; is < ns - 1; is++) {
            for (int js = is + 1; js < ns; js++) {
                double chgprd = m->charge[is] * m->charge[js];
                if (chgprd == 0.0) continue;
                double drx = (x[i] + XS(xs, is, i)) - (x[i] + XS(xs, js, i));
                double dry = (y[i] + XS(ys, is, i)) - (y[i] + XS(ys, js, i));
                double drz = (z[i] + XS(zs, is, i)) - (z[i] + XS(zs, js, i));
                double drr = sqrt(drx * drx + dry * dry + drz * drz);
                sumff = sumff + erf(alp * drr) * chgprd / drr;
                double ad = alp * drr;
                double fs = -R4PIE0 * chgprd *
                            (erf(alp * drr) / (drr * drr * drr) -
                             TWOSQPI * alp * exp(-(ad * ad)) / (drr * drr));
                double fxsij = drx * fs, fysij = dry * fs, fzsij = drz * fs;
                XS(fxs, is, i) += fxsij;
                XS(fys, is, i) += fysij;
                XS(fzs, is, i) += fzsij;
                XS(fxs, js, i) -= fxsij;
                XS(fys, js, i) -= fysij;
                XS(fzs, js, i) -= fzsij;
                qv = qv - (drx * fxsij + dry * fysij + drz * fzsij);
            }
        }
    }
    double e_selfi = -sumff;
    *qscpe = R4PIE0 * (e_selfp + e_selfi) / 418.4;
    *vir += qv;
}

/* ---------------------------------------------------------------- ewald.f90:177-405 */
/* vdw_ccpol23plus.f90:174-477 */
void orc_ccpol23plus(const orc_model *m, const double *xx, const double *yy, const double *zz,
                     const double *xxs, const double *yys, const double *zzs, int ld,
                     double boxi, double *qvdwe, double *fxs, double *fys, double *fzs,
                     double *vir) {
    const int nm = m->nm, ns = m->ns;
    const double gamma = 20.0 / BOHR2A, sqr0 = 1.4 * BOHR2A;
    for (int j = 0; j < nm; j++)
        for (int js = 0; js < ns; js++) {
            fxs[(size_t)j * ld + js] = 0.0;
            fys[(size_t)j * ld + js] = 0.0;
            fzs[(size_t)j * ld + js] = 0.0;
        }
    const int nt = nthreads();
    acc_t *acc = acc_alloc(nt, nm, ns);
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        acc_t *A = &acc[omp_get_thread_num()];
#else
        acc_t *A = &acc[0];
#endif
#pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < nm - 1; i++) {
            for (int j = i + 1; j < nm; j++) {
                double xcc = minimg(xx[i] - xx[j], boxi), ycc = minimg(yy[i] - yy[j], boxi),
                       zcc = minimg(zz[i] - zz[j], boxi);
                double rccsq = xcc * xcc + ycc * ycc + zcc * zcc;
                if (!(rccsq < m->rcutsd)) continue;
                for (int is = 0; is < ns; is++) {
                    for (int js = 0; js < ns; js++) {
                        const int k = m->vdw_row[is * ORC_NSITE_MAX + js];
                        if (k < 0) continue;
                        const double *p = m->vdw[k];
                        const double beta = p[0], c0 = p[1], c1 = p[2], c2 = p[3], c3 = p[4];
                        const double c6 = p[5], c8 = p[6], c10 = p[7];
                        const double d1 = p[8], d6 = p[9], d8 = p[10], d10 = p[11];
                        double rsx = xcc + XS(xxs, is, i) - XS(xxs, js, j);
                        double rsy = ycc + XS(yys, is, i) - XS(yys, js, j);
                        double rsz = zcc + XS(zzs, is, i) - XS(zzs, js, j);
                        double qis = m->charge[is], qjs = m->charge[js];
                        double rssq = rsx * rsx + rsy * rsy + rsz * rsz;
                        double sqr = sqrt(rssq);
                        double eks = exp(-beta * sqr);
                        double u_exp = eks * (c0 + c1 * sqr + c2 * pow(sqr, 2.0) + c3 * pow(sqr, 3.0));
                        double fdamp = 1.0 / (1.0 + exp(-gamma * (sqr - sqr0)));
                        u_exp = u_exp * fdamp;
                        double f1 = orc_tt(1, d1, sqr);
                        double u_ele = R4PIE0 * (f1 - 1.0) * qis * qjs / sqr;
                        double f6 = orc_tt(6, d6, sqr), f8 = orc_tt(8, d8, sqr),
                               f10 = orc_tt(10, d10, sqr);
                        double r6 = rssq * rssq * rssq, r8 = rssq * r6, r10 = rssq * r8;
                        double u_ind = -f6 * c6 / r6 - f8 * c8 / r8 - f10 * c10 / r10;
                        A->e += u_exp + u_ele + u_ind;
                        double du_exp = -beta * u_exp * fdamp +
                                        eks * fdamp * (c1 + 2.0 * c2 * sqr + 3.0 * c3 * pow(sqr, 2.0)) +
                                        gamma * exp(-gamma * (sqr - sqr0)) * pow(fdamp, 2.0) * u_exp;
                        double df1 = orc_dtt(1, d1, sqr);
                        double du_ele = -R4PIE0 * qis * qjs * ((f1 - 1.0) / pow(sqr, 2.0) - df1 / sqr);
                        double df6 = orc_dtt(6, d6, sqr), df8 = orc_dtt(8, d8, sqr),
                               df10 = orc_dtt(10, d10, sqr);
                        double du_ind = -df6 * c6 / r6 + 6.0 * f6 * c6 / pow(sqr, 7.0) -
                                        df8 * c8 / r8 + 8.0 * f8 * c8 / pow(sqr, 9.0) -
                                        df10 * c10 / r10 + 10.0 * f10 * c10 / pow(sqr, 11.0);
                        double wij = du_exp + du_ele + du_ind;
                        double vfij = -wij / sqr;
                        double fxsij = rsx * vfij, fysij = rsy * vfij, fzsij = rsz * vfij;
                        size_t si = (size_t)i * ns + is, sj = (size_t)j * ns + js;
                        A->fx[si] += fxsij;
                        A->fy[si] += fysij;
                        A->fz[si] += fzsij;
                        A->fx[sj] -= fxsij;
                        A->fy[sj] -= fysij;
                        A->fz[sj] -= fzsij;
                        A->v -= (rsx * fxsij + rsy * fysij + rsz * fzsij);
                    }
                }
            }
        }
    }
    double e = 0.0, v = 0.0;
    for (int t = 0; t < nt; t++) {
        for (int i = 0; i < nm; i++)
            for (int s = 0; s < ns; s++) {
                fxs[(size_t)i * ld + s] += acc[t].fx[(size_t)i * ns + s];
                fys[(size_t)i * ld + s] += acc[t].fy[(size_t)i * ns + s];
                fzs[(size_t)i * ld + s] += acc[t].fz[(size_t)i * ns + s];
            }
        e += acc[t].e;
        v += acc[t].v;
    }
    acc_free(acc, nt);
    *qvdwe = e / 418.4;
    *vir = v;
}

void orc_rspace_ewald(const orc_model *m, const double *xx, const double *yy,
                      const double *zz, const double *xxs, const double *yys,
                      const double *zzs, int ld, double boxi, double alp, double *qrcpe,
                      double *fxs, double *fys, double *fzs, double *vir) {
    const int nm = m->nm, ns = m->ns;
    const int nt = nthreads();
    acc_t *acc = acc_alloc(nt, nm, ns);
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        acc_t *A = &acc[omp_get_thread_num()];
#else
        acc_t *A = &acc[0];
#endif
#pragma omp for schedule(static, 1)
        for (int i = 0; i < nm - 1; i++) {
            for (int j = i + 1; j < nm; j++) {
                double xcc = minimg(xx[i] - xx[j], boxi), ycc = minimg(yy[i] - yy[j], boxi),
                       zcc = minimg(zz[i] - zz[j], boxi);
                double rccsq = xcc * xcc + ycc * ycc + zcc * zcc;
                if (!(rccsq < m->rcutsd)) continue;
                for (int is = 0; is < ns; is++) {
                    for (int js = 0; js < ns; js++) {
                        double qis = m->charge[is], qjs = m->charge[js];
                        double rsx = xcc + XS(xxs, is, i) - XS(xxs, js, j);
                        double rsy = ycc + XS(yys, is, i) - XS(yys, js, j);
                        double rsz = zcc + XS(zzs, is, i) - XS(zzs, js, j);
                        double rssq = rsx * rsx + rsy * rsy + rsz * rsz;
                        double drr = sqrt(rssq);
                        double ec = erfc(alp * drr);
                        A->e += R4PIE0 * qis * qjs * ec / drr;
                        double ad = alp * drr;
                        double fc = R4PIE0 * qis * qjs * (ec / drr + TWOSQPI * alp * exp(-(ad * ad)));
                        double cfij = fc / rssq;
                        double fxsij = rsx * cfij, fysij = rsy * cfij, fzsij = rsz * cfij;
                        size_t si = (size_t)i * ns + is, sj = (size_t)j * ns + js;
                        A->fx[si] += fxsij;
                        A->fy[si] += fysij;
                        A->fz[si] += fzsij;
                        A->fx[sj] -= fxsij;
                        A->fy[sj] -= fysij;
                        A->fz[sj] -= fzsij;
                        A->v -= (rsx * fxsij + rsy * fysij + rsz * fzsij);
                    }
                }
            }
        }
    }
    double e = 0.0, v = 0.0;
    for (int t = 0; t < nt; t++) {
        for (int i = 0; i < nm; i++)
            for (int s = 0; s < ns; s++) {
                fxs[(size_t)i * ld + s] += acc[t].fx[(size_t)i * ns + s];
                fys[(size_t)i * ld + s] += acc[t].fy[(size_t)i * ns + s];
                fzs[(size_t)i * ld + s] += acc[t].fz[(size_t)i * ns + s];
            }
        e += acc[t].e;
        v += acc[t].v;
    }
    acc_free(acc, nt);
    *qrcpe = e / 418.4;
    *vir += v;
}

/* ------------------------------------------------ shared reciprocal-space machinery */
/* Per-site cos/sin tables built by the reference's angle-addition recurrence
   (ewald.f90:882-917; nb_induction_model.f90:729-763 and the other k-space routines). */
typedef struct {
    int n, lim[3];
    double *c[3], *s[3]; /* [ii*(lim+1) + l] */
} ktab_t;

static void ktab_build(ktab_t *T, int n, const double *px, const double *py, const double *pz,
                       int l1, int l2, int l3, double box) {
    const double twopi = 2.0 * PI;
    const double *p[3] = {px, py, pz};
    T->n = n;
    T->lim[0] = l1;
    T->lim[1] = l2;
    T->lim[2] = l3;
    for (int a = 0; a < 3; a++) {
        int L = T->lim[a] + 1;
        T->c[a] = (double *)malloc(sizeof(double) * (size_t)n * (L > 2 ? L : 2));
        T->s[a] = (double *)malloc(sizeof(double) * (size_t)n * (L > 2 ? L : 2));
        int W = (L > 2 ? L : 2);
        for (int ii = 0; ii < n; ii++) {
            T->c[a][ii * W + 0] = 1.0;
            T->s[a][ii * W + 0] = 0.0;
            T->c[a][ii * W + 1] = cos(twopi * p[a][ii] / box);
            T->s[a][ii * W + 1] = sin(twopi * p[a][ii] / box);
        }
        for (int l = 2; l <= T->lim[a]; l++)
            for (int ii = 0; ii < n; ii++) {
                double cp = T->c[a][ii * W + l - 1], sp = T->s[a][ii * W + l - 1];
                double c1 = T->c[a][ii * W + 1], s1 = T->s[a][ii * W + 1];
                T->c[a][ii * W + l] = cp * c1 - sp * s1;
                T->s[a][ii * W + l] = sp * c1 + cp * s1;
            }
    }
}

static inline int ktab_w(const ktab_t *T, int a) {
    int L = T->lim[a] + 1;
    return L > 2 ? L : 2;
}

static void ktab_free(ktab_t *T) {
    for (int a = 0; a < 3; a++) {
        free(T->c[a]);
        free(T->s[a]);
    }
}

/* Iterates the half-space k-vectors with the spherical cut-off in the reference's order
   (ll outer, mm, nn inner; ewald.f90:933-1082) and, for each, fills ckr/skr for all
   table sites and calls visit(). */
typedef void (*kvisit_fn)(void *ctx, double rl, double rm, double rn, double ak, double rksq,
                          const double *ckr, const double *skr);

static void kspace_walk(const ktab_t *T, int lmax, int mmax, int nmax, double alp, double box,
                        kvisit_fn visit, void *ctx) {
    const double twopi = 2.0 * PI;
    int klmmax = lmax < mmax ? lmax : mmax;
    klmmax = klmmax < nmax ? klmmax : nmax;
    int klmmaxsq = klmmax * klmmax;
    double volmi = box * box * box;
    int n = T->n;
    double *clm = (double *)malloc(sizeof(double) * n), *slm = (double *)malloc(sizeof(double) * n);
    double *ckr = (double *)malloc(sizeof(double) * n), *skr = (double *)malloc(sizeof(double) * n);
    int wl = ktab_w(T, 0), wm = ktab_w(T, 1), wn = ktab_w(T, 2);
    int mmin = 0, nmin = 1;
    for (int ll = 0; ll <= lmax; ll++) {
        double rl = twopi * ll / box;
        int li = ll;
        if (ll > 0) mmin = -mmax;
        for (int mm = mmin; mm <= mmax; mm++) {
            int mi = abs(mm);
            double rm = twopi * mm / box;
            if (mm >= 0) {
                for (int ii = 0; ii < n; ii++) {
                    clm[ii] = T->c[0][ii * wl + li] * T->c[1][ii * wm + mi] -
                              T->s[0][ii * wl + li] * T->s[1][ii * wm + mi];
                    slm[ii] = T->s[0][ii * wl + li] * T->c[1][ii * wm + mi] +
                              T->s[1][ii * wm + mi] * T->c[0][ii * wl + li];
                }
            } else {
                for (int ii = 0; ii < n; ii++) {
                    clm[ii] = T->c[0][ii * wl + li] * T->c[1][ii * wm + mi] +
                              T->s[0][ii * wl + li] * T->s[1][ii * wm + mi];
                    slm[ii] = T->s[0][ii * wl + li] * T->c[1][ii * wm + mi] -
                              T->s[1][ii * wm + mi] * T->c[0][ii * wl + li];
                }
            }
            for (int nn = nmin; nn <= nmax; nn++) {
                int ni = abs(nn);
                double rn = twopi * nn / box;
                int kk = ll * ll + mm * mm + nn * nn;
                if (kk <= klmmaxsq) {
                    double rksq = rl * rl + rm * rm + rn * rn;
                    double ak = twopi / volmi * exp(-0.25 * rksq / (alp * alp)) / rksq;
                    if (nn >= 0) {
                        for (int ii = 0; ii < n; ii++) {
                            ckr[ii] = clm[ii] * T->c[2][ii * wn + ni] - slm[ii] * T->s[2][ii * wn + ni];
                            skr[ii] = slm[ii] * T->c[2][ii * wn + ni] + clm[ii] * T->s[2][ii * wn + ni];
                        }
                    } else {
                        for (int ii = 0; ii < n; ii++) {
                            ckr[ii] = clm[ii] * T->c[2][ii * wn + ni] + slm[ii] * T->s[2][ii * wn + ni];
                            skr[ii] = slm[ii] * T->c[2][ii * wn + ni] - clm[ii] * T->s[2][ii * wn + ni];
                        }
                    }
                    visit(ctx, rl, rm, rn, ak, rksq, ckr, skr);
                }
            }
            nmin = -nmax;
        }
    }
    free(clm); free(slm); free(ckr); free(skr);
}

/* ---------------------------------------------------------------- ewald.f90:754-1173 */
typedef struct {
    int noq;
    const double *qi;
    double alp;
    double *fx, *fy, *fz; /* per table site */
    double qpe, qvir;
} kew_ctx;

static void kew_visit(void *c, double rl, double rm, double rn, double ak, double rksq,
                      const double *ckr, const double *skr) {
    kew_ctx *K = (kew_ctx *)c;
    double ckcs = 0.0, ckss = 0.0;
    for (int ii = 0; ii < K->noq; ii++) {
        ckcs = ckcs + K->qi[ii] * ckr[ii];
        ckss = ckss + K->qi[ii] * skr[ii];
    }
    double s2 = ckcs * ckcs + ckss * ckss;
    K->qpe += ak * s2;
    K->qvir -= (1.0 - 0.5 * rksq / (K->alp * K->alp)) * ak * s2;
    for (int ii = 0; ii < K->noq; ii++) {
        double qforce = 4.0 * R4PIE0 * ak * ((K->qi[ii] * skr[ii]) * ckcs - (K->qi[ii] * ckr[ii]) * ckss);
        K->fx[ii] += rl * qforce;
        K->fy[ii] += rm * qforce;
        K->fz[ii] += rn * qforce;
    }
}

void orc_kspace_ewald(const orc_model *m, const double *xx, const double *yy,
                      const double *zz, const double *xxs, const double *yys,
                      const double *zzs, int ld, int lmax, int mmax, int nmax, double alp,
                      double boxi, double *qkcpe, double *fxs, double *fys, double *fzs,
                      double *vir) {
    const int nm = m->nm, ns = m->ns;
    int nq = 0;
    double *qi = (double *)malloc(sizeof(double) * nm * ns), *pxi = (double *)malloc(sizeof(double) * nm * ns),
           *pyi = (double *)malloc(sizeof(double) * nm * ns), *pzi = (double *)malloc(sizeof(double) * nm * ns);
    int *owner = (int *)malloc(sizeof(int) * nm * ns);
    for (int j = 0; j < nm; j++)
        for (int js = 0; js < ns; js++)
            if (m->charge[js] != 0.0) {
                qi[nq] = m->charge[js];
                pxi[nq] = xx[j] + XS(xxs, js, j);
                pyi[nq] = yy[j] + XS(yys, js, j);
                pzi[nq] = zz[j] + XS(zzs, js, j);
                owner[nq] = j * ld + js;
                nq++;
            }
    ktab_t T;
    ktab_build(&T, nq, pxi, pyi, pzi, lmax, mmax, nmax, boxi);
    kew_ctx K = {nq, qi, alp, (double *)calloc(nq, sizeof(double)), (double *)calloc(nq, sizeof(double)),
                 (double *)calloc(nq, sizeof(double)), 0.0, 0.0};
    kspace_walk(&T, lmax, mmax, nmax, alp, boxi, kew_visit, &K);
    for (int ii = 0; ii < nq; ii++) {
        fxs[owner[ii]] += K.fx[ii];
        fys[owner[ii]] += K.fy[ii];
        fzs[owner[ii]] += K.fz[ii];
    }
    *qkcpe = 2.0 * R4PIE0 * K.qpe / 418.4;
    *vir += 2.0 * R4PIE0 * K.qvir;
    ktab_free(&T);
    free(K.fx); free(K.fy); free(K.fz);
    free(qi); free(pxi); free(pyi); free(pzi); free(owner);
}

/* ============================================================ nb_induction_model.f90 */
typedef struct {
    const orc_model *m;
    int nm, ns, npol, ld;
    const double *xx, *yy, *zz, *xxs, *yys, *zzs;
    double box, alp;
    /* [i*ns + is] work arrays */
    double *rE0[3], *kE0[3], *slfE0[3], *shtE0[3];
    double *rEi[3], *kEi[3], *slfEi[3], *shtEi[3];
    double *idm[3];
    ktab_t T;      /* all nm*ns sites, table built once per call */
    double *px, *py, *pz;
} ind_t;

#define W3(arr, i, s) arr[(size_t)(i) * I->ns + (s)]

/* nb_induction_model.f90:128-293 */
static void rspace_efield_stat(ind_t *I) {
    const int ld = I->ld;
    const int nm = I->nm, ns = I->ns, p0 = ns - I->npol;
    const double alp = I->alp, box = I->box;
#pragma omp parallel for schedule(static, 1) num_threads(nthreads())
    for (int i = 0; i < nm; i++) {
        for (int s = 0; s < ns; s++) W3(I->rE0[0], i, s) = W3(I->rE0[1], i, s) = W3(I->rE0[2], i, s) = 0.0;
        for (int j = 0; j < nm; j++) {
            if (j == i) continue;
            double xcc = minimg(I->xx[i] - I->xx[j], box), ycc = minimg(I->yy[i] - I->yy[j], box),
                   zcc = minimg(I->zz[i] - I->zz[j], box);
            double rccsq = xcc * xcc + ycc * ycc + zcc * zcc;
            if (!(rccsq < I->m->rcutsd)) continue;
            for (int is = p0; is < ns; is++)
                for (int js = 0; js < ns; js++) {
                    double qjs = I->m->charge[js];
                    double ddx = xcc + (XS(I->xxs, is, i) - XS(I->xxs, js, j));
                    double ddy = ycc + (XS(I->yys, is, i) - XS(I->yys, js, j));
                    double ddz = zcc + (XS(I->zzs, is, i) - XS(I->zzs, js, j));
                    double dist2 = ddx * ddx + ddy * ddy + ddz * ddz;
                    double dist = sqrt(dist2);
                    double ad = alp * dist;
                    double expar2 = exp(-(ad * ad));
                    double d1i = erfc(alp * dist) / dist;
                    double d2i = 1.0 / dist2;
                    double d3i = d2i * (d1i + TWOSQPI * alp * expar2);
                    W3(I->rE0[0], i, is) += qjs * ddx * d3i;
                    W3(I->rE0[1], i, is) += qjs * ddy * d3i;
                    W3(I->rE0[2], i, is) += qjs * ddz * d3i;
                }
        }
    }
}

/* nb_induction_model.f90:597-975 */
typedef struct {
    ind_t *I;
    double *ex, *ey, *ez;
    int mode; /* 0: static charges; 1: dipoles */
} kfield_ctx;

static void kfield_visit(void *c, double rl, double rm, double rn, double ak, double rksq,
                         const double *ckr, const double *skr) {
    (void)rksq;
    kfield_ctx *K = (kfield_ctx *)c;
    ind_t *I = K->I;
    int n = I->nm * I->ns;
    double ckcs = 0.0, ckss = 0.0;
    if (K->mode == 0) {
        for (int mx = 0; mx < n; mx++) {
            double q = I->m->charge[mx % I->ns];
            ckcs = ckcs + q * ckr[mx];
            ckss = ckss + q * skr[mx];
        }
        for (int ii = 0; ii < n; ii++) {
            double qefld = 4.0 * ak * (skr[ii] * ckcs - ckr[ii] * ckss);
            K->ex[ii] += rl * qefld;
            K->ey[ii] += rm * qefld;
            K->ez[ii] += rn * qefld;
        }
    } else {
        for (int mx = 0; mx < n; mx++) {
            double dk = rl * I->idm[0][mx] + rm * I->idm[1][mx] + rn * I->idm[2][mx];
            ckcs = ckcs + dk * ckr[mx];
            ckss = ckss + dk * skr[mx];
        }
        for (int ii = 0; ii < n; ii++) {
            double muefld = -4.0 * ak * (ckr[ii] * ckcs + skr[ii] * ckss);
            K->ex[ii] += rl * muefld;
            K->ey[ii] += rm * muefld;
            K->ez[ii] += rn * muefld;
        }
    }
}

static void kspace_field(ind_t *I, int mode, double **out) {
    const int ld = I->ld;
    int n = I->nm * I->ns;
    for (int a = 0; a < 3; a++) memset(out[a], 0, sizeof(double) * n);
    kfield_ctx K = {I, out[0], out[1], out[2], mode};
    kspace_walk(&I->T, I->m->kmax1, I->m->kmax2, I->m->kmax3, I->alp, I->box, kfield_visit, &K);
}

/* nb_induction_model.f90:977-1115 (intramolecular uses x + xs as the reference does) */
static void self_efield_stat(ind_t *I) {
    const int ld = I->ld;
    const int nm = I->nm, ns = I->ns, p0 = ns - I->npol;
    const double alp = I->alp;
    for (int i = 0; i < nm; i++) {
        for (int s = 0; s < ns; s++) W3(I->slfE0[0], i, s) = W3(I->slfE0[1], i, s) = W3(I->slfE0[2], i, s) = 0.0;
        for (int is = p0; is < ns; is++)
            for (int js = 0; js < ns - I->npol; js++) {
                double qjs = I->m->charge[js];
                double ddx = (I->xx[i] + XS(I->xxs, is, i)) - (I->xx[i] + XS(I->xxs, js, i));
                double ddy = (I->yy[i] + XS(I->yys, is, i)) - (I->yy[i] + XS(I->yys, js, i));
                double ddz = (I->zz[i] + XS(I->zzs, is, i)) - (I->zz[i] + XS(I->zzs, js, i));
                double dist2 = ddx * ddx + ddy * ddy + ddz * ddz;
                if (dist2 == 0.0) continue;
                double drr = sqrt(dist2);
                double d1i = 1.0 / drr, d2i = d1i * d1i, d3i = d2i * d1i;
                double ad = alp * drr;
                double expar2 = exp(-(ad * ad));
                double f = erf(alp * drr) * d3i - TWOSQPI * alp * expar2 * d2i;
                W3(I->slfE0[0], i, is) -= qjs * ddx * f;
                W3(I->slfE0[1], i, is) -= qjs * ddy * f;
                W3(I->slfE0[2], i, is) -= qjs * ddz * f;
            }
    }
}

/* nb_induction_model.f90:5454-5629 */
static void shortrange_efield_stat(ind_t *I) {
    const int ld = I->ld;
    const int nm = I->nm, ns = I->ns, p0 = ns - I->npol;
    const double box = I->box;
#pragma omp parallel for schedule(static, 1) num_threads(nthreads())
    for (int i = 0; i < nm; i++) {
        for (int s = 0; s < ns; s++) W3(I->shtE0[0], i, s) = W3(I->shtE0[1], i, s) = W3(I->shtE0[2], i, s) = 0.0;
        for (int j = 0; j < nm; j++) {
            if (j == i) continue;
            double xcc = minimg(I->xx[i] - I->xx[j], box), ycc = minimg(I->yy[i] - I->yy[j], box),
                   zcc = minimg(I->zz[i] - I->zz[j], box);
            double rccsq = xcc * xcc + ycc * ycc + zcc * zcc;
            if (!(rccsq < I->m->rcutsd)) continue;
            for (int is = p0; is < ns; is++)
                for (int js = 0; js < ns; js++) {
                    double qjs = I->m->charge[js];
                    double ddx = xcc + (XS(I->xxs, is, i) - XS(I->xxs, js, j));
                    double ddy = ycc + (XS(I->yys, is, i) - XS(I->yys, js, j));
                    double ddz = zcc + (XS(I->zzs, is, i) - XS(I->zzs, js, j));
                    double dist2 = ddx * ddx + ddy * ddy + ddz * ddz;
                    double dist = sqrt(dist2);
                    double d1i = 1.0 / dist, d2i = d1i * d1i, d3i = d2i * d1i;
                    double f2 = orc_tt(2, DELTA2, dist);
                    W3(I->shtE0[0], i, is) += (f2 - 1.0) * qjs * ddx * d3i;
                    W3(I->shtE0[1], i, is) += (f2 - 1.0) * qjs * ddy * d3i;
                    W3(I->shtE0[2], i, is) += (f2 - 1.0) * qjs * ddz * d3i;
                }
        }
    }
}

/* nb_induction_model.f90:1409-1569 */
static void rspace_efield_idm(ind_t *I) {
    const int ld = I->ld;
    const int nm = I->nm, ns = I->ns, p0 = ns - I->npol;
    const double alp = I->alp, box = I->box, alp3 = alp * alp * alp;
#pragma omp parallel for schedule(static, 1) num_threads(nthreads())
    for (int i = 0; i < nm; i++) {
        for (int s = 0; s < ns; s++) W3(I->rEi[0], i, s) = W3(I->rEi[1], i, s) = W3(I->rEi[2], i, s) = 0.0;
        for (int j = 0; j < nm; j++) {
            if (j == i) continue;
            double xcc = minimg(I->xx[i] - I->xx[j], box), ycc = minimg(I->yy[i] - I->yy[j], box),
                   zcc = minimg(I->zz[i] - I->zz[j], box);
            double rccsq = xcc * xcc + ycc * ycc + zcc * zcc;
            if (!(rccsq < I->m->rcutsd)) continue;
            for (int is = p0; is < ns; is++)
                for (int js = p0; js < ns; js++) {
                    double ddx = xcc + XS(I->xxs, is, i) - XS(I->xxs, js, j);
                    double ddy = ycc + XS(I->yys, is, i) - XS(I->yys, js, j);
                    double ddz = zcc + XS(I->zzs, is, i) - XS(I->zzs, js, j);
                    double dist2 = ddx * ddx + ddy * ddy + ddz * ddz;
                    double drr = sqrt(dist2);
                    double d1i = 1.0 / drr, d2i = d1i * d1i, d3i = d2i * d1i, d5i = d3i * d2i;
                    double mjx = W3(I->idm[0], j, js), mjy = W3(I->idm[1], j, js), mjz = W3(I->idm[2], j, js);
                    double dotj = mjx * ddx + mjy * ddy + mjz * ddz;
                    double ad = alp * drr;
                    double expar2 = exp(-(ad * ad));
                    double ec = erfc(alp * drr);
                    double d3ii = ec * d3i + TWOSQPI * alp * expar2 * d2i;
                    double d5ii = ec * d5i + TWOSQPI * alp * expar2 * d2i * d2i +
                                  2.0 * TWOSQPI * alp3 * expar2 * d2i / 3.0;
                    W3(I->rEi[0], i, is) += 3.0 * d5ii * dotj * ddx - mjx * d3ii;
                    W3(I->rEi[1], i, is) += 3.0 * d5ii * dotj * ddy - mjy * d3ii;
                    W3(I->rEi[2], i, is) += 3.0 * d5ii * dotj * ddz - mjz * d3ii;
                }
        }
    }
}

/* nb_induction_model.f90:2663-2829 */
static void self_efield_idm(ind_t *I) {
    const int ld = I->ld;
    const int nm = I->nm, ns = I->ns, p0 = ns - I->npol;
    const double alp = I->alp, alp3 = alp * alp * alp;
    double selffac = 4.0 * alp3 / (3.0 * sqrt(PI));
    for (int i = 0; i < nm; i++) {
        for (int s = 0; s < ns; s++) W3(I->slfEi[0], i, s) = W3(I->slfEi[1], i, s) = W3(I->slfEi[2], i, s) = 0.0;
        for (int is = p0; is < ns; is++)
            for (int a = 0; a < 3; a++) W3(I->slfEi[a], i, is) += selffac * W3(I->idm[a], i, is);
        double ll[3][ORC_NSITE_MAX];
        for (int s = 0; s < ns; s++) ll[0][s] = ll[1][s] = ll[2][s] = 0.0;
        for (int is = p0; is < ns; is++)
            for (int js = p0; js < ns; js++) {
                if (js == is) continue;
                double ddx = (I->xx[i] + XS(I->xxs, is, i)) - (I->xx[i] + XS(I->xxs, js, i));
                double ddy = (I->yy[i] + XS(I->yys, is, i)) - (I->yy[i] + XS(I->yys, js, i));
                double ddz = (I->zz[i] + XS(I->zzs, is, i)) - (I->zz[i] + XS(I->zzs, js, i));
                double dist2 = ddx * ddx + ddy * ddy + ddz * ddz;
                double drr = sqrt(dist2);
                double d1i = 1.0 / drr, d2i = d1i * d1i, d3i = d2i * d1i, d5i = d3i * d2i;
                double mjx = W3(I->idm[0], i, js), mjy = W3(I->idm[1], i, js), mjz = W3(I->idm[2], i, js);
                double dotj = mjx * ddx + mjy * ddy + mjz * ddz;
                double ad = alp * drr;
                double expar2 = exp(-(ad * ad));
                double ef = erf(alp * drr);
                double d3ii = ef * d3i - TWOSQPI * alp * expar2 * d2i;
                double d5ii = ef * d5i - TWOSQPI * alp * expar2 * d2i * d2i -
                              2.0 * TWOSQPI * alp3 * expar2 * d2i / 3.0;
                ll[0][is] -= (3.0 * d5ii * dotj * ddx - mjx * d3ii);
                ll[1][is] -= (3.0 * d5ii * dotj * ddy - mjy * d3ii);
                ll[2][is] -= (3.0 * d5ii * dotj * ddz - mjz * d3ii);
            }
        for (int s = 0; s < ns; s++)
            for (int a = 0; a < 3; a++) W3(I->slfEi[a], i, s) += ll[a][s];
    }
}

/* nb_induction_model.f90:5634-5789 */
static void shortrange_efield_idm(ind_t *I) {
    const int ld = I->ld;
    const int nm = I->nm, ns = I->ns, p0 = ns - I->npol;
    const double box = I->box;
#pragma omp parallel for schedule(static, 1) num_threads(nthreads())
    for (int i = 0; i < nm; i++) {
        for (int s = 0; s < ns; s++) W3(I->shtEi[0], i, s) = W3(I->shtEi[1], i, s) = W3(I->shtEi[2], i, s) = 0.0;
        for (int j = 0; j < nm; j++) {
            if (j == i) continue;
            double xcc = minimg(I->xx[i] - I->xx[j], box), ycc = minimg(I->yy[i] - I->yy[j], box),
                   zcc = minimg(I->zz[i] - I->zz[j], box);
            double rccsq = xcc * xcc + ycc * ycc + zcc * zcc;
            if (!(rccsq < I->m->rcutsd)) continue;
            for (int is = p0; is < ns; is++)
                for (int js = p0; js < ns; js++) {
                    double ddx = xcc + XS(I->xxs, is, i) - XS(I->xxs, js, j);
                    double ddy = ycc + XS(I->yys, is, i) - XS(I->yys, js, j);
                    double ddz = zcc + XS(I->zzs, is, i) - XS(I->zzs, js, j);
                    double dist2 = ddx * ddx + ddy * ddy + ddz * ddz;
                    double dist = sqrt(dist2);
                    double d1i = 1.0 / dist, d2i = d1i * d1i, d3i = d2i * d1i, d5i = d3i * d2i;
                    double f3 = orc_tt(3, DELTA3, dist);
                    double mjx = W3(I->idm[0], j, js), mjy = W3(I->idm[1], j, js), mjz = W3(I->idm[2], j, js);
                    double dotj = mjx * ddx + mjy * ddy + mjz * ddz;
                    W3(I->shtEi[0], i, is) += (f3 - 1.0) * (3.0 * d5i * dotj * ddx - mjx * d3i);
                    W3(I->shtEi[1], i, is) += (f3 - 1.0) * (3.0 * d5i * dotj * ddy - mjy * d3i);
                    W3(I->shtEi[2], i, is) += (f3 - 1.0) * (3.0 * d5i * dotj * ddz - mjz * d3i);
                }
        }
    }
}

/* --------------------------------------------------------- induction forces */
/* Per-site field (from dipoles) and 3x3 field-gradient accumulators, combined as
   F = r4pie0 * (q E + mu . grad E) by each force routine. */
typedef struct {
    double *E[3];   /* [i*ns+s] */
    double *G[9];   /* gxx gyy gzz gxy gyx gxz gzx gyz gzy */
} fg_t;

enum { GXX = 0, GYY, GZZ, GXY, GYX, GXZ, GZX, GYZ, GZY };

static void fg_alloc(fg_t *f, size_t n) {
    for (int a = 0; a < 3; a++) f->E[a] = (double *)calloc(n, sizeof(double));
    for (int a = 0; a < 9; a++) f->G[a] = (double *)calloc(n, sizeof(double));
}
static void fg_free(fg_t *f) {
    for (int a = 0; a < 3; a++) free(f->E[a]);
    for (int a = 0; a < 9; a++) free(f->G[a]);
}

/* nb_induction_model.f90:3069-3631 */
static void real_forces(ind_t *I, double *fxs, double *fys, double *fzs, double *vir) {
    const int ld = I->ld;
    const int nm = I->nm, ns = I->ns;
    const double alp = I->alp, box = I->box;
    const double alp3 = alp * alp * alp, alp5 = alp3 * alp * alp;
    const int nt = nthreads();
    size_t n = (size_t)nm * ns;
    fg_t *fg = (fg_t *)malloc(sizeof(fg_t) * nt);
    double *vt = (double *)calloc(nt, sizeof(double));
    for (int t = 0; t < nt; t++) fg_alloc(&fg[t], n);
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        int tid = omp_get_thread_num();
#else
        int tid = 0;
#endif
        fg_t *F = &fg[tid];
        double lv = 0.0;
#pragma omp for schedule(static, 1)
        for (int i = 0; i < nm - 1; i++) {
            for (int j = i + 1; j < nm; j++) {
                double xcc = minimg(I->xx[i] - I->xx[j], box), ycc = minimg(I->yy[i] - I->yy[j], box),
                       zcc = minimg(I->zz[i] - I->zz[j], box);
                double rccsq = xcc * xcc + ycc * ycc + zcc * zcc;
                if (!(rccsq < I->m->rcutsd)) continue;
                for (int is = 0; is < ns; is++)
                    for (int js = 0; js < ns; js++) {
                        double qis = I->m->charge[is], qjs = I->m->charge[js];
                        double ddx = xcc + (XS(I->xxs, is, i) - XS(I->xxs, js, j));
                        double ddy = ycc + (XS(I->yys, is, i) - XS(I->yys, js, j));
                        double ddz = zcc + (XS(I->zzs, is, i) - XS(I->zzs, js, j));
                        double dist2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        double dist = sqrt(dist2);
                        double d1i = 1.0 / dist, d2i = d1i * d1i, d3i = d2i * d1i, d4i = d2i * d2i;
                        double d5i = d3i * d2i, d6i = d3i * d3i, d7i = d5i * d2i;
                        double ad = alp * dist;
                        double expar2 = exp(-(ad * ad));
                        double mix = W3(I->idm[0], i, is), miy = W3(I->idm[1], i, is), miz = W3(I->idm[2], i, is);
                        double mjx = W3(I->idm[0], j, js), mjy = W3(I->idm[1], j, js), mjz = W3(I->idm[2], j, js);
                        double doti = mix * ddx + miy * ddy + miz * ddz;
                        double dotj = mjx * ddx + mjy * ddy + mjz * ddz;
                        double ec = erfc(alp * dist);
                        double d3ii = ec * d3i + TWOSQPI * alp * expar2 * d2i;
                        double d5ii = ec * d5i + TWOSQPI * alp * expar2 * d4i + 2.0 * TWOSQPI * alp3 * expar2 * d2i / 3.0;
                        double d7ii = ec * d7i + TWOSQPI * alp * expar2 * d6i + 2.0 * TWOSQPI * alp3 * expar2 * d4i / 3.0 +
                                      4.0 * TWOSQPI * alp5 * expar2 * d2i / 15.0;
                        double d[3] = {ddx, ddy, ddz};
                        double mj[3] = {mjx, mjy, mjz}, mi[3] = {mix, miy, miz};
                        size_t si = (size_t)i * ns + is, sj = (size_t)j * ns + js;
                        /* field and gradient at (is,i) from (js,j) */
                        double efi[3];
                        for (int a = 0; a < 3; a++) efi[a] = 3.0 * d5ii * dotj * d[a] - mj[a] * d3ii;
                        for (int a = 0; a < 3; a++) F->E[a][si] += efi[a];
                        lv -= qis * (efi[0] * ddx + efi[1] * ddy + efi[2] * ddz);
                        /* gradient components: g_ab, ordering as the reference's names */
                        static const int ga[9] = {0, 1, 2, 0, 1, 0, 2, 1, 2};
                        static const int gb[9] = {0, 1, 2, 1, 0, 2, 0, 2, 1};
                        double tot[9];
                        for (int c = 0; c < 9; c++) {
                            int a = ga[c], b = gb[c];
                            double ef0 = qjs * (-3.0 * d5ii * d[a] * d[b] + (a == b ? d3ii : 0.0));
                            double efi_g = -15.0 * d7ii * d[a] * d[b] * dotj +
                                           3.0 * d5ii * (a == b ? (dotj + 2.0 * d[a] * mj[a])
                                                                : (mj[a] * d[b] + mj[b] * d[a]));
                            tot[c] = ef0 + efi_g;
                            F->G[c][si] += tot[c];
                        }
                        lv -= ((mix * tot[GXX] + miy * tot[GYX] + miz * tot[GZX]) * ddx +
                               (mix * tot[GXY] + miy * tot[GYY] + miz * tot[GZY]) * ddy +
                               (mix * tot[GXZ] + miy * tot[GYZ] + miz * tot[GZZ]) * ddz);
                        /* field and gradient at (js,j) from (is,i) */
                        for (int a = 0; a < 3; a++) F->E[a][sj] += 3.0 * d5ii * doti * d[a] - mi[a] * d3ii;
                        for (int c = 0; c < 9; c++) {
                            int a = ga[c], b = gb[c];
                            double ef0 = qis * (-3.0 * d5ii * d[a] * d[b] + (a == b ? d3ii : 0.0));
                            double efi_g = 15.0 * d7ii * d[a] * d[b] * doti +
                                           3.0 * d5ii * (a == b ? (-doti - 2.0 * d[a] * mi[a])
                                                                : (-mi[a] * d[b] - mi[b] * d[a]));
                            F->G[c][sj] += ef0 + efi_g;
                        }
                    }
            }
        }
        vt[tid] = lv;
    }
    double qv = 0.0;
    for (int t = 0; t < nt; t++) qv += vt[t];
    for (int i = 0; i < nm; i++)
        for (int is = 0; is < ns; is++) {
            size_t si = (size_t)i * ns + is;
            double E[3] = {0, 0, 0}, G[9] = {0};
            for (int t = 0; t < nt; t++) {
                for (int a = 0; a < 3; a++) E[a] += fg[t].E[a][si];
                for (int c = 0; c < 9; c++) G[c] += fg[t].G[c][si];
            }
            double q = I->m->charge[is];
            double mx = W3(I->idm[0], i, is), my = W3(I->idm[1], i, is), mz = W3(I->idm[2], i, is);
            double fx = q * E[0] + mx * G[GXX] + my * G[GYX] + mz * G[GZX];
            double fy = q * E[1] + mx * G[GXY] + my * G[GYY] + mz * G[GZY];
            double fz = q * E[2] + mx * G[GXZ] + my * G[GYZ] + mz * G[GZZ];
            XS(fxs, is, i) += fx * R4PIE0;
            XS(fys, is, i) += fy * R4PIE0;
            XS(fzs, is, i) += fz * R4PIE0;
        }
    *vir += R4PIE0 * qv;
    for (int t = 0; t < nt; t++) fg_free(&fg[t]);
    free(fg);
    free(vt);
}

/* nb_induction_model.f90:4171-4839 */
typedef struct {
    ind_t *I;
    fg_t *F;
    double qvir;
} kforce_ctx;

static void kforce_visit(void *c, double rl, double rm, double rn, double ak, double rksq,
                         const double *ckr, const double *skr) {
    kforce_ctx *K = (kforce_ctx *)c;
    ind_t *I = K->I;
    int n = I->nm * I->ns;
    double ckcqs = 0.0, cksqs = 0.0, ckcds = 0.0, cksds = 0.0;
    for (int mx = 0; mx < n; mx++) {
        double dk = rl * I->idm[0][mx] + rm * I->idm[1][mx] + rn * I->idm[2][mx];
        double q = I->m->charge[mx % I->ns];
        ckcqs = ckcqs + q * ckr[mx];
        cksqs = cksqs + q * skr[mx];
        ckcds = ckcds + dk * ckr[mx];
        cksds = cksds + dk * skr[mx];
    }
    double alp = I->alp;
    K->qvir -= 2.0 * ak *
               ((ckcds * cksqs - cksds * ckcqs) + (ckcds * ckcds + cksds * cksds) +
                0.5 * (2.0 * (ckcds * cksqs - cksds * ckcqs) + (ckcds * ckcds + cksds * cksds)) *
                    (1.0 - 0.5 * rksq / (alp * alp)));
    double r[3] = {rl, rm, rn};
    static const int ga[9] = {0, 1, 2, 0, 1, 0, 2, 1, 2};
    static const int gb[9] = {0, 1, 2, 1, 0, 2, 0, 2, 1};
    for (int ii = 0; ii < n; ii++) {
        double mufac = -4.0 * ak * (ckr[ii] * ckcds + skr[ii] * cksds);
        K->F->E[0][ii] += rl * mufac;
        K->F->E[1][ii] += rm * mufac;
        K->F->E[2][ii] += rn * mufac;
        double qfac = -4.0 * ak * (-ckr[ii] * ckcqs - skr[ii] * cksqs);
        double mufaci = -4.0 * ak * (ckr[ii] * cksds - skr[ii] * ckcds);
        for (int cc = 0; cc < 9; cc++) {
            double rr = r[ga[cc]] * r[gb[cc]];
            K->F->G[cc][ii] += rr * qfac + rr * mufaci;
        }
    }
}

static void kspace_forces(ind_t *I, double *fxs, double *fys, double *fzs, double *vir) {
    const int ld = I->ld;
    const int nm = I->nm, ns = I->ns;
    fg_t F;
    fg_alloc(&F, (size_t)nm * ns);
    kforce_ctx K = {I, &F, 0.0};
    kspace_walk(&I->T, I->m->kmax1, I->m->kmax2, I->m->kmax3, I->alp, I->box, kforce_visit, &K);
    for (int i = 0; i < nm; i++)
        for (int is = 0; is < ns; is++) {
            size_t si = (size_t)i * ns + is;
            double q = I->m->charge[is];
            double mx = I->idm[0][si], my = I->idm[1][si], mz = I->idm[2][si];
            double fx = q * F.E[0][si] + mx * F.G[GXX][si] + my * F.G[GYX][si] + mz * F.G[GZX][si];
            double fy = q * F.E[1][si] + mx * F.G[GXY][si] + my * F.G[GYY][si] + mz * F.G[GZY][si];
            double fz = q * F.E[2][si] + mx * F.G[GXZ][si] + my * F.G[GYZ][si] + mz * F.G[GZZ][si];
            XS(fxs, is, i) += fx * R4PIE0;
            XS(fys, is, i) += fy * R4PIE0;
            XS(fzs, is, i) += fz * R4PIE0;
        }
    *vir += 2.0 * R4PIE0 * K.qvir;
    fg_free(&F);
}

/* nb_induction_model.f90:4841-5360 */
static void self_forces(ind_t *I, double *fxs, double *fys, double *fzs, double *vir) {
    const int ld = I->ld;
    const int nm = I->nm, ns = I->ns;
    const double alp = I->alp, alp3 = alp * alp * alp, alp5 = alp3 * alp * alp;
    const double selffac = 4.0 * alp3 / (3.0 * sqrt(PI));
    static const int ga[9] = {0, 1, 2, 0, 1, 0, 2, 1, 2};
    static const int gb[9] = {0, 1, 2, 1, 0, 2, 0, 2, 1};
    double qv = 0.0;
    double E[3][ORC_NSITE_MAX], G[9][ORC_NSITE_MAX];
    for (int i = 0; i < nm; i++) {
        for (int s = 0; s < ns; s++) {
            double q = I->m->charge[s];
            for (int a = 0; a < 3; a++) E[a][s] = selffac * W3(I->idm[a], i, s);
            for (int c = 0; c < 9; c++) G[c][s] = 0.0;
            G[GXX][s] -= selffac * q;
            G[GYY][s] -= selffac * q;
            G[GZZ][s] -= selffac * q;
        }
        for (int is = 0; is < ns - 1; is++)
            for (int js = is + 1; js < ns; js++) {
                double qis = I->m->charge[is], qjs = I->m->charge[js];
                double ddx = (I->xx[i] + XS(I->xxs, is, i)) - (I->xx[i] + XS(I->xxs, js, i));
                double ddy = (I->yy[i] + XS(I->yys, is, i)) - (I->yy[i] + XS(I->yys, js, i));
                double ddz = (I->zz[i] + XS(I->zzs, is, i)) - (I->zz[i] + XS(I->zzs, js, i));
                double dist2 = ddx * ddx + ddy * ddy + ddz * ddz;
                if (dist2 == 0.0) continue;
                double drr = sqrt(dist2);
                double d1i = 1.0 / drr, d2i = d1i * d1i, d3i = d2i * d1i, d4i = d2i * d2i;
                double d5i = d3i * d2i, d6i = d3i * d3i, d7i = d6i * d1i;
                double ad = alp * drr;
                double expar2 = exp(-(ad * ad));
                double mi[3] = {W3(I->idm[0], i, is), W3(I->idm[1], i, is), W3(I->idm[2], i, is)};
                double mj[3] = {W3(I->idm[0], i, js), W3(I->idm[1], i, js), W3(I->idm[2], i, js)};
                double d[3] = {ddx, ddy, ddz};
                double dotis = mi[0] * ddx + mi[1] * ddy + mi[2] * ddz;
                double dotjs = mj[0] * ddx + mj[1] * ddy + mj[2] * ddz;
                double ef = erf(alp * drr);
                double d3ii = ef * d3i - TWOSQPI * alp * expar2 * d2i;
                double d5ii = ef * d5i - TWOSQPI * alp * expar2 * d4i - (2.0 / 3.0) * TWOSQPI * alp3 * expar2 * d2i;
                double d7ii = ef * d7i - TWOSQPI * alp * expar2 * d6i - (2.0 / 3.0) * TWOSQPI * alp3 * expar2 * d4i -
                              (4.0 / 15.0) * TWOSQPI * alp5 * expar2 * d2i;
                double efl[3];
                for (int a = 0; a < 3; a++) efl[a] = -(3.0 * d5ii * dotjs * d[a] - mj[a] * d3ii);
                for (int a = 0; a < 3; a++) E[a][is] += efl[a];
                qv -= qis * (efl[0] * ddx + efl[1] * ddy + efl[2] * ddz);
                double tot[9];
                for (int c = 0; c < 9; c++) {
                    int a = ga[c], b = gb[c];
                    double ef0 = -qjs * (-3.0 * d5ii * d[a] * d[b] + (a == b ? d3ii : 0.0));
                    double efi_g = -(-15.0 * d7ii * d[a] * d[b] * dotjs +
                                     3.0 * d5ii * (a == b ? (dotjs + 2.0 * d[a] * mj[a])
                                                          : (mj[a] * d[b] + mj[b] * d[a])));
                    tot[c] = ef0 + efi_g;
                    G[c][is] += tot[c];
                }
                qv -= ((mi[0] * tot[GXX] + mi[1] * tot[GYX] + mi[2] * tot[GZX]) * ddx +
                       (mi[0] * tot[GXY] + mi[1] * tot[GYY] + mi[2] * tot[GZY]) * ddy +
                       (mi[0] * tot[GXZ] + mi[1] * tot[GYZ] + mi[2] * tot[GZZ]) * ddz);
                for (int a = 0; a < 3; a++) E[a][js] += -(3.0 * d5ii * dotis * d[a] - mi[a] * d3ii);
                for (int c = 0; c < 9; c++) {
                    int a = ga[c], b = gb[c];
                    double ef0 = -qis * (-3.0 * d5ii * d[a] * d[b] + (a == b ? d3ii : 0.0));
                    double efi_g = -(15.0 * d7ii * d[a] * d[b] * dotis +
                                     3.0 * d5ii * (a == b ? (-dotis - 2.0 * d[a] * mi[a])
                                                          : (-mi[a] * d[b] - mi[b] * d[a])));
                    G[c][js] += ef0 + efi_g;
                }
            }
        for (int is = 0; is < ns; is++) {
            double q = I->m->charge[is];
            double mx = W3(I->idm[0], i, is), my = W3(I->idm[1], i, is), mz = W3(I->idm[2], i, is);
            double fx = q * E[0][is] + mx * G[GXX][is] + my * G[GYX][is] + mz * G[GZX][is];
            double fy = q * E[1][is] + mx * G[GXY][is] + my * G[GYY][is] + mz * G[GZY][is];
            double fz = q * E[2][is] + mx * G[GXZ][is] + my * G[GYZ][is] + mz * G[GZZ][is];
            XS(fxs, is, i) += fx * R4PIE0;
            XS(fys, is, i) += fy * R4PIE0;
            XS(fzs, is, i) += fz * R4PIE0;
        }
    }
    *vir += R4PIE0 * qv;
}

/* nb_induction_model.f90:5975-6557.  The gradient here is stored as g_ab = dE_b/dx_a
   and contracted as F_a = q E_a + sum_b mu_b g_ab, exactly as the reference does. */
static void shortrange_forces(ind_t *I, double *fxs, double *fys, double *fzs, double *vir) {
    const int ld = I->ld;
    const int nm = I->nm, ns = I->ns;
    const double box = I->box, cst = 1.0;
    const int nt = nthreads();
    size_t n = (size_t)nm * ns;
    fg_t *fg = (fg_t *)malloc(sizeof(fg_t) * nt);
    double *vt = (double *)calloc(nt, sizeof(double));
    for (int t = 0; t < nt; t++) fg_alloc(&fg[t], n);
    /* component c -> (field component b, derivative direction a), names g<b><a> */
    static const int gE[9] = {0, 1, 2, 0, 1, 0, 2, 1, 2}; /* first letter */
    static const int gD[9] = {0, 1, 2, 1, 0, 2, 0, 2, 1}; /* second letter */
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        int tid = omp_get_thread_num();
#else
        int tid = 0;
#endif
        fg_t *F = &fg[tid];
        double lv = 0.0;
#pragma omp for schedule(static, 1)
        for (int i = 0; i < nm - 1; i++) {
            for (int j = i + 1; j < nm; j++) {
                double xcc = minimg(I->xx[i] - I->xx[j], box), ycc = minimg(I->yy[i] - I->yy[j], box),
                       zcc = minimg(I->zz[i] - I->zz[j], box);
                double rccsq = xcc * xcc + ycc * ycc + zcc * zcc;
                if (!(rccsq < I->m->rcutsd)) continue;
                for (int is = 0; is < ns; is++)
                    for (int js = 0; js < ns; js++) {
                        double qis = I->m->charge[is], qjs = I->m->charge[js];
                        double ddx = xcc + (XS(I->xxs, is, i) - XS(I->xxs, js, j));
                        double ddy = ycc + (XS(I->yys, is, i) - XS(I->yys, js, j));
                        double ddz = zcc + (XS(I->zzs, is, i) - XS(I->zzs, js, j));
                        double dist2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        double dist = sqrt(dist2);
                        double d1i = 1.0 / dist, d2i = d1i * d1i, d3i = d2i * d1i;
                        double d5i = d3i * d2i, d7i = d5i * d2i;
                        double f2 = orc_tt(2, DELTA2, dist), f3 = orc_tt(3, DELTA3, dist);
                        double df2 = orc_dtt(2, DELTA2, dist), df3 = orc_dtt(3, DELTA3, dist);
                        double d[3] = {ddx, ddy, ddz};
                        double mi[3] = {W3(I->idm[0], i, is), W3(I->idm[1], i, is), W3(I->idm[2], i, is)};
                        double mj[3] = {W3(I->idm[0], j, js), W3(I->idm[1], j, js), W3(I->idm[2], j, js)};
                        double doti = mi[0] * ddx + mi[1] * ddy + mi[2] * ddz;
                        double dotj = mj[0] * ddx + mj[1] * ddy + mj[2] * ddz;
                        size_t si = (size_t)i * ns + is, sj = (size_t)j * ns + js;
                        double efl[3];
                        for (int a = 0; a < 3; a++)
                            efl[a] = (f2 - 1.0) * (3.0 * d5i * dotj * d[a] - mj[a] * d3i) - dotj * d3i * df2 * d1i * d[a];
                        for (int a = 0; a < 3; a++) F->E[a][si] += efl[a];
                        lv -= qis * (efl[0] * ddx + efl[1] * ddy + efl[2] * ddz);
                        double tot[9];
                        for (int c = 0; c < 9; c++) {
                            int b = gE[c], a = gD[c]; /* g_{b a}: component b, direction a */
                            double ef0 = (f2 - 1.0) * qjs * (-3.0 * d5i * d[b] * d[a] + (a == b ? d3i : 0.0)) +
                                         qjs * d[a] * d3i * df2 * d[b] * d1i;
                            double efi_g;
                            if (a == b)
                                efi_g = (f3 - 1.0) * (-15.0 * dotj * d7i * d[a] * d[a] + 3.0 * dotj * d5i +
                                                      2.0 * 3.0 * d5i * mj[a] * d[a]) +
                                        cst * (3.0 * d[a] * dotj * d5i - mj[a] * d3i) * df3 * d[a] * d1i;
                            else
                                efi_g = (f3 - 1.0) * (-15.0 * dotj * d7i * d[b] * d[a] + 3.0 * d5i * mj[b] * d[a] +
                                                      3.0 * d5i * mj[a] * d[b]) +
                                        cst * (3.0 * d[a] * dotj * d5i - mj[a] * d3i) * df3 * d[b] * d1i;
                            tot[c] = ef0 + efi_g;
                            F->G[c][si] += tot[c];
                        }
                        lv -= (mi[0] * tot[GXX] * ddx + mi[1] * tot[GXY] * ddx + mi[2] * tot[GXZ] * ddx +
                               mi[0] * tot[GYX] * ddy + mi[1] * tot[GYY] * ddy + mi[2] * tot[GYZ] * ddy +
                               mi[0] * tot[GZX] * ddz + mi[1] * tot[GZY] * ddz + mi[2] * tot[GZZ] * ddz);
                        for (int a = 0; a < 3; a++)
                            F->E[a][sj] += (f2 - 1.0) * (3.0 * d5i * doti * d[a] - mi[a] * d3i) - doti * d3i * df2 * d1i * d[a];
                        for (int c = 0; c < 9; c++) {
                            int b = gE[c], a = gD[c];
                            double ef0 = (f2 - 1.0) * qis * (-3.0 * d5i * d[b] * d[a] + (a == b ? d3i : 0.0)) +
                                         qis * d[a] * d3i * df2 * d[b] * d1i;
                            double efi_g;
                            if (a == b)
                                efi_g = -(f3 - 1.0) * (-15.0 * doti * d7i * d[a] * d[a] + 3.0 * doti * d5i +
                                                       2.0 * 3.0 * d5i * mi[a] * d[a]) -
                                        cst * (3.0 * d[a] * doti * d5i - mi[a] * d3i) * df3 * d[a] * d1i;
                            else
                                efi_g = -(f3 - 1.0) * (-15.0 * doti * d7i * d[b] * d[a] + 3.0 * d5i * mi[b] * d[a] +
                                                       3.0 * d5i * mi[a] * d[b]) -
                                        cst * (3.0 * d[a] * doti * d5i - mi[a] * d3i) * df3 * d[b] * d1i;
                            F->G[c][sj] += ef0 + efi_g;
                        }
                    }
            }
        }
        vt[tid] = lv;
    }
    double qv = 0.0;
    for (int t = 0; t < nt; t++) qv += vt[t];
    for (int i = 0; i < nm; i++)
        for (int is = 0; is < ns; is++) {
            size_t si = (size_t)i * ns + is;
            double E[3] = {0, 0, 0}, G[9] = {0};
            for (int t = 0; t < nt; t++) {
                for (int a = 0; a < 3; a++) E[a] += fg[t].E[a][si];
                for (int c = 0; c < 9; c++) G[c] += fg[t].G[c][si];
            }
            double q = I->m->charge[is];
            double mx = W3(I->idm[0], i, is), my = W3(I->idm[1], i, is), mz = W3(I->idm[2], i, is);
            double fx = q * E[0] + mx * G[GXX] + my * G[GXY] + mz * G[GXZ];
            double fy = q * E[1] + mx * G[GYX] + my * G[GYY] + mz * G[GYZ];
            double fz = q * E[2] + mx * G[GZX] + my * G[GZY] + mz * G[GZZ];
            XS(fxs, is, i) += fx * R4PIE0;
            XS(fys, is, i) += fy * R4PIE0;
            XS(fzs, is, i) += fz * R4PIE0;
        }
    *vir += R4PIE0 * qv;
    for (int t = 0; t < nt; t++) fg_free(&fg[t]);
    free(fg);
    free(vt);
}

/* nb_induction_model.f90:25-126 with iteridm (1193-1407) */
int orc_nb_induction(const orc_model *m, const double *x, const double *y, const double *z,
                     const double *xs, const double *ys, const double *zs, int ld, double box,
                     int maxit, double *qindpe, double *idmx, double *idmy, double *idmz,
                     double *fxs, double *fys, double *fzs, double *vir, int *iters) {
    ind_t I;
    memset(&I, 0, sizeof(I));
    I.m = m;
    I.nm = m->nm;
    I.ns = m->ns;
    I.npol = m->npol;
    I.ld = ld;
    I.xx = x; I.yy = y; I.zz = z;
    I.xxs = xs; I.yys = ys; I.zzs = zs;
    I.box = box;
    I.alp = m->alpha;
    size_t n = (size_t)m->nm * m->ns;
    for (int a = 0; a < 3; a++) {
        I.rE0[a] = (double *)calloc(n, sizeof(double));
        I.kE0[a] = (double *)calloc(n, sizeof(double));
        I.slfE0[a] = (double *)calloc(n, sizeof(double));
        I.shtE0[a] = (double *)calloc(n, sizeof(double));
        I.rEi[a] = (double *)calloc(n, sizeof(double));
        I.kEi[a] = (double *)calloc(n, sizeof(double));
        I.slfEi[a] = (double *)calloc(n, sizeof(double));
        I.shtEi[a] = (double *)calloc(n, sizeof(double));
        I.idm[a] = (double *)calloc(n, sizeof(double));
    }
    I.px = (double *)malloc(sizeof(double) * n);
    I.py = (double *)malloc(sizeof(double) * n);
    I.pz = (double *)malloc(sizeof(double) * n);
    for (int j = 0; j < m->nm; j++)
        for (int js = 0; js < m->ns; js++) {
            size_t ii = (size_t)j * m->ns + js;
            I.px[ii] = x[j] + xs[(size_t)j * ld + js];
            I.py[ii] = y[j] + ys[(size_t)j * ld + js];
            I.pz[ii] = z[j] + zs[(size_t)j * ld + js];
        }
    ktab_build(&I.T, (int)n, I.px, I.py, I.pz, m->kmax1, m->kmax2, m->kmax3, box);

    rspace_efield_stat(&I);
    kspace_field(&I, 0, I.kE0);
    self_efield_stat(&I);
    if (m->damped) shortrange_efield_stat(&I);

    /* iteridm (nb_induction_model.f90:1193-1407) */
    const int nm = m->nm, ns = m->ns, p0 = ns - m->npol;
    double change = 10.0, energy = 0.0;
    int isteps = 0;
    const double thr_iter = 1.0e-20;
    while (change > thr_iter && isteps < maxit) {
        rspace_efield_idm(&I);
        kspace_field(&I, 1, I.kEi);
        self_efield_idm(&I);
        if (m->damped) shortrange_efield_idm(&I);
        double lchange = 0.0, lenergy = 0.0;
        for (int i = 0; i < nm; i++)
            for (int is = p0; is < ns; is++) {
                size_t si = (size_t)i * ns + is;
                double E0[3], Et[3];
                for (int a = 0; a < 3; a++) {
                    E0[a] = I.rE0[a][si] + I.kE0[a][si] + I.slfE0[a][si] + I.shtE0[a][si];
                    double Ei = I.rEi[a][si] + I.kEi[a][si] + I.slfEi[a][si] + I.shtEi[a][si];
                    Et[a] = Ei + E0[a];
                }
                double polr = m->polarizability[is] * pow(BOHR2A, 3.0);
                double p[3] = {polr * Et[0], polr * Et[1], polr * Et[2]};
                double dx = I.idm[0][si] - p[0], dy = I.idm[1][si] - p[1], dz = I.idm[2][si] - p[2];
                lchange = dx * dx + dy * dy + dz * dz + lchange;
                for (int a = 0; a < 3; a++) I.idm[a][si] = p[a];
                lenergy = -0.5 * polr * (Et[0] * E0[0] + Et[1] * E0[1] + Et[2] * E0[2]) + lenergy;
            }
        change = lchange;
        energy = lenergy;
        isteps++;
    }
    int status = (isteps >= maxit) ? 1 : 0;
    *qindpe = R4PIE0 * energy / 418.4;
    *iters = isteps;

    /* forces with the converged dipoles (nb_induction_model.f90:90-113) */
    real_forces(&I, fxs, fys, fzs, vir);
    kspace_forces(&I, fxs, fys, fzs, vir);
    self_forces(&I, fxs, fys, fzs, vir);
    if (m->damped) shortrange_forces(&I, fxs, fys, fzs, vir);

    for (int i = 0; i < nm; i++)
        for (int s = 0; s < ns; s++) {
            size_t si = (size_t)i * ns + s;
            idmx[(size_t)i * ld + s] = I.idm[0][si];
            idmy[(size_t)i * ld + s] = I.idm[1][si];
            idmz[(size_t)i * ld + s] = I.idm[2][si];
        }
    for (int a = 0; a < 3; a++) {
        free(I.rE0[a]); free(I.kE0[a]); free(I.slfE0[a]); free(I.shtE0[a]);
        free(I.rEi[a]); free(I.kEi[a]); free(I.slfEi[a]); free(I.shtEi[a]);
        free(I.idm[a]);
    }
    free(I.px); free(I.py); free(I.pz);
    ktab_free(&I.T);
    return status;
}
