/*
 * ccpol_oracle.h -- CPU FP64 oracle for the CCpol23+(2025) force-evaluation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference Fortran
 * routines (ommair/CCpol23_plus_2025_MBMD), written to be used as the parity checker
 * by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  It is never
 * linked into, loaded by, or called from the product library.
 *
 * Each routine follows the loop nesting, cut-off tests and arithmetic of the reference
 * routine it names (file:line cited at each definition), with the MPI master/worker
 * dispatch reduced to its single-process (MPIcomm_size == 1) semantics.
 *
 * Pinning: the reference ships no golden energies or forces.  The oracle is pinned by
 * the reference's own FS2 known-answer test (source/tests/check_fs2_periodic.py:
 * periodic invariance + central finite differences of forces and rigid virial, same
 * fixture and tolerances), ported into tests/test_oracle_fs2_kat.py, and by the same
 * finite-difference/periodicity properties applied to FS3, Ewald and induction.
 * FS2 is pinned by that test.  FS3, induction and Ewald are "parity unpinned": they are
 * checked by properties (finite differences, periodicity, virial identity), not against
 * reference-produced numbers, because no Fortran compiler exists here to run the
 * reference and it ships no golden values for them.
 *
 * Units follow the reference: positions in Angstrom, energies returned in kcal/mol,
 * forces in internal units (10 J/mol/Angstrom), virial in internal units.
 * Array layout follows the reference's Fortran arrays: COM arrays x[nm]; site arrays
 * xs[i*ld + is] (site index fastest, leading dimension ld >= ns, nsite=50 in the
 * reference).
 */
#ifndef CCPOL_ORACLE_H
#define CCPOL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NSITE_MAX 50
#define ORC_NS3 17            /* FS3 sites per molecule */
#define ORC_NTAB (17 * 17 * 17 * 8)
#define ORC_VDW_MAX 64

typedef struct orc_model {
    int nm, ns, npol;
    double charge[ORC_NSITE_MAX];         /* e; chgs(is,i) = charge(is) */
    double polarizability[ORC_NSITE_MAX]; /* bohr^3; apol = polarizability*bohr2a**3 */
    double alpha;                         /* Ewald alpha (1/A) */
    int kmax1, kmax2, kmax3;
    double rcut, rcutsd;                  /* COM cut-off for pair terms (A, A^2) */
    double rcut3, rcutsd3;                /* FS2 COM cut-off (A, A^2) */
    double alpha3, delta33;               /* 3-body damping parameters (CONTROL line 15) */
    int s2_term, s3_term, damped;         /* CONTROL flags */
    /* FS3 short-range (data3b_full) and long-range (data3b_full_LR_4p5) tables,
       stored [is*17 + js] with is, js 0-based. */
    double bS3_s[289], gS3_s[289], r0S3_s[289];
    double bS3_l[289], gS3_l[289], r0S3_l[289];
    double cs3_s[5000], cs3_l[5000];      /* linear coefficients, 0-based (file index - 1) */
    int nlin;                             /* number of linear coefficients in the files */
    int ind_lin[ORC_NTAB];                /* 1-based coefficient index per (is,js,ks,ip,jp,kp) */
    int nclass;                           /* number of classes produced by the index fill */
    /* ccpol23plus 2-body parameters (FIELD "vdw parameters", initialization.f90:612-628):
       row k holds beta, c0, c1, c2, c3, c6, c8, c10, d1, d6, d8, d10 with c0..c10 already
       in internal energy units (x 418.4); vdw_row[is*ORC_NSITE_MAX + js] is the row whose
       site-name pair matches (is, js) in either order, or -1. */
    int nvdw;
    double vdw[ORC_VDW_MAX][12];
    int vdw_row[ORC_NSITE_MAX * ORC_NSITE_MAX];
} orc_model;

/* ccpol23plus (vdw_ccpol23plus.f90:174-477): the 2-body CCpol23+ site-site energy
   (damped exponential + short-range Coulomb correction + damped C6/C8/C10), forces and
   virial over molecule pairs with COM distance below rcut.  As the reference, it ZEROES the
   site forces of the first ns sites and SETS *vir before accumulating; energy in kcal/mol.
   The long-range correction, which the reference computes but does not add, is omitted. */
void orc_ccpol23plus(const orc_model *m, const double *x, const double *y, const double *z,
                     const double *xs, const double *ys, const double *zs, int ld, double box,
                     double *qvdwe, double *fxs, double *fys, double *fzs, double *vir);

/* Tang-Toennies damping f_n(delta r) and its derivative (utility.f90:89-125). */
double orc_tt(int n, double delta, double r);
double orc_dtt(int n, double delta, double r);

/* FS3 symmetric coefficient index (threebody_potential.f90:909-946, 2064-2131).
   Writes ind[ORC_NTAB] and returns the number of classes. */
int orc_fill_index(int *ind);

/* Ewald alpha and k-max from the precision and cut-off (ewald.f90:17-43). */
void orc_ewald_setup(double ewps, double rcut, double box, double *alp,
                     int *k1, int *k2, int *k3);

/* threebody_term (threebody_potential.f90:17-99): FS2 (if s2_term) then FS3 (if s3_term).
   Site forces and vir accumulate; fxfs2/fxfs3 are overwritten (zeroed when the term is
   off is NOT done, matching the reference, which leaves them untouched). */
void orc_threebody_term(const orc_model *m,
                        const double *x, const double *y, const double *z,
                        const double *xs, const double *ys, const double *zs, int ld,
                        double box, double *qfs2, double *qfs3,
                        double *fxs, double *fys, double *fzs,
                        double *fxfs2, double *fyfs2, double *fzfs2,
                        double *fxfs3, double *fyfs3, double *fzfs3, double *vir);

/* Same, but the FS2 part alone on coordinates already in bohr (threebody_potential.f90:
   101-674); used by the port of the reference's FS2 test. */
void orc_fs2_term_bohr(const orc_model *m,
                       const double *xx, const double *yy, const double *zz,
                       const double *xxs, const double *yys, const double *zzs, int ld,
                       double boxi, double *qfs2,
                       double *fxs, double *fys, double *fzs,
                       double *fxfs2, double *fyfs2, double *fzfs2, double *vir);

/* Ewald charge-charge terms (ewald.f90:45-174, 177-405, 754-1173). */
void orc_ewald_self_correction(const orc_model *m, double alp, double box,
                               const double *x, const double *y, const double *z,
                               const double *xs, const double *ys, const double *zs, int ld,
                               double *qscpe, double *fxs, double *fys, double *fzs,
                               double *vir);
void orc_rspace_ewald(const orc_model *m,
                      const double *x, const double *y, const double *z,
                      const double *xs, const double *ys, const double *zs, int ld,
                      double box, double alp, double *qrcpe,
                      double *fxs, double *fys, double *fzs, double *vir);
void orc_kspace_ewald(const orc_model *m,
                      const double *x, const double *y, const double *z,
                      const double *xs, const double *ys, const double *zs, int ld,
                      int lmax, int mmax, int nmax, double alp, double box, double *qkcpe,
                      double *fxs, double *fys, double *fzs, double *vir);

/* nb_induction (nb_induction_model.f90:25-126): static field, Jacobi dipole iteration,
   induction forces.  Returns 0 on convergence, 1 when the iteration hit maxit (the
   reference calls `stop` there).  *iters receives the number of iterations taken. */
int orc_nb_induction(const orc_model *m,
                     const double *x, const double *y, const double *z,
                     const double *xs, const double *ys, const double *zs, int ld,
                     double box, int maxit, double *qindpe,
                     double *idmx, double *idmy, double *idmz,
                     double *fxs, double *fys, double *fzs, double *vir, int *iters);

/* Thread count used by the OpenMP regions (0 = library default). */
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
