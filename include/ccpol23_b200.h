/*
 * ccpol23_b200.h -- C ABI of the B200-native CCpol23+(2025) force-evaluation hot path.
 *
 * The entry points below replace, one for one, the Fortran module procedures that
 * md.f90/evolve.f90 call on the hot path of ommair/CCpol23_plus_2025_MBMD.  Each keeps
 * the reference's argument meaning and units:
 *   positions in Angstrom; COM arrays x[nm]; site arrays xs[i*ld + is] (site index
 *   fastest, leading dimension ld >= ns; the reference passes its nsite=50 arrays);
 *   energies returned in kcal/mol; site forces ACCUMULATE into fxs/fys/fzs in internal
 *   units (10 J/mol/Angstrom); the 3-body COM forces fxfs2/fxfs3 are OVERWRITTEN;
 *   the virial ACCUMULATES into *vir (internal units); induced dipoles are overwritten.
 * Every entry point returns an int status (CCP_OK == 0) instead of the reference's
 * `stop`.  All buffers in these signatures are host memory unless the name ends in
 * _device, in which case they are device pointers on the context's GPU.
 *
 * Parameters that the reference reads from module globals (charges, polarisabilities,
 * cut-offs, Ewald alpha/k-max, FS3 tables, CONTROL flags) live in a ccp_model loaded
 * from the reference's own input files, and are copied into the context.
 */
#ifndef CCPOL23_B200_H
#define CCPOL23_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define CCP_OK 0
#define CCP_ERR_BAD_INPUT 1      /* null pointer, nm/ld out of range, bad file contents;
                                    from a context's evaluations also a NaN or infinite
                                    coordinate or site offset (found on the device as the
                                    inputs are read, reported at the evaluation's end; the
                                    outputs of that call are then undefined) */
#define CCP_ERR_NOT_CONVERGED 2  /* dipole iteration hit maxit (reference: `stop`,
                                    nb_induction_model.f90:1374-1379) */
#define CCP_ERR_CUDA 3           /* a CUDA runtime call failed; see ccp_last_error() */
#define CCP_ERR_NO_DEVICE 4      /* no CUDA device / library built without one */
#define CCP_ERR_IO 5             /* an input file could not be opened */
#define CCP_ERR_CAPACITY 6       /* an internal list overflowed twice (not expected) */

/* precision forms of a context */
#define CCP_FP64 0   /* plain FP64 everywhere */
#define CCP_MIXED 1  /* FP32 for FS2's spectator terms (and, with option
                        "fs3_fp32_passes", for two of the three FS3 gradient passes); the
                        induced dipoles by preconditioned conjugate gradients in FP64 to
                        1e-8 D RMS (option "dipole_solver"); FP64 for FS3, Ewald, the
                        induction fields and forces, and all sums */

typedef struct ccp_model ccp_model;
typedef struct ccp_context ccp_context;

/* Per-term energies (kcal/mol) and bookkeeping of one hot-path evaluation. */
typedef struct ccp_energies {
    double scpe;      /* Ewald self + intramolecular correction */
    double rcpe;      /* Ewald real space */
    double kcpe;      /* Ewald reciprocal space */
    double indpe;     /* induction */
    double fs2pe;     /* FS2 three-body */
    double fs3pe;     /* FS3 three-body */
    double vir;       /* virial added by these terms (internal units) */
    int ind_iters;    /* dipole-solve steps taken (Jacobi iterations, or PCG steps) */
    int n_fs3_triples;    /* molecular triples inside the FS3 cut-off */
    int n_fs3_blend;      /* of which in the SR/LR switching region */
    int n_fs2_triples;    /* (spectator, pair) combinations inside the FS2 cut-off */
    double vdwpe;     /* ccpol23plus 2-body (only when that term is evaluated) */
} ccp_energies;

/* Last error message of the calling thread (never NULL). */
const char *ccp_last_error(void);

/* ------------------------------------------------------------------- parameters */
/* Reads CONTROL, FIELD, data3b_full and data3b_full_LR_4p5 from `dir`
   (replaces control_parameters + molecule, initialization.f90:463-720), then builds the
   principal-axis site frame (shift_to_com + principle_moment_inertia,
   initialization.f90:728-845) and the FS3 coefficient index
   (threebody_potential.f90:909-946, 2064-2131). */
int ccp_model_load(const char *dir, ccp_model **out);
void ccp_model_free(ccp_model *m);

/* Scalar accessors/overrides (the reference reads these from common_arrays). */
int ccp_model_get_int(const ccp_model *m, const char *name, int *value);
int ccp_model_get_double(const ccp_model *m, const char *name, double *value);
int ccp_model_set_int(ccp_model *m, const char *name, int value);
int ccp_model_set_double(ccp_model *m, const char *name, double value);
/* Per-site arrays: "charge", "polarizability", "mass" (ns values),
   "pcoord" (ns*3, site-major), "pmi" (3). */
int ccp_model_get_array(const ccp_model *m, const char *name, double *out, int n);

/* sites (molecular_sites.f90:14-47): site offsets from the COM of every molecule from
   its quaternion q[i*4 + 0..3]; writes xs/ys/zs[i*ld + is]. */
int ccp_sites(const ccp_model *m, int nm, const double *q, int ld, double *xs, double *ys,
              double *zs);

/* ewald_setup (ewald.f90:17-43). */
int ccp_ewald_setup(double ewps, double rcut, double box, double *alp, int *k1, int *k2,
                    int *k3);

/* --------------------------------------------------------------------- context */
/* Allocates device-resident state for boxes of nm >= 1 molecules on `device` (ordinal),
   precision CCP_FP64 or CCP_MIXED.  Ewald alpha/k-max default to
   ccp_ewald_setup(1e-6, rcut, box0). */
int ccp_context_create(const ccp_model *m, int nm, double box0, int device, int precision,
                       ccp_context **out);
int ccp_context_destroy(ccp_context *ctx);
/* Override alpha and kmax1..3 (the reference's module globals alpha, kmax1-3). */
int ccp_context_set_ewald(ccp_context *ctx, double alpha, int k1, int k2, int k3);
/* Cap on dipole iterations (reference: maxit = 500, nb_induction_model.f90:1221). */
int ccp_context_set_maxit(ccp_context *ctx, int maxit);
/* Run subsequent device work on this cudaStream_t (NULL = the context's own stream; the
   legacy default stream is named by cudaStreamLegacy).  An evaluation then starts after the
   work already queued on that stream, which is how a caller orders it after its own input
   copies. */
int ccp_context_set_stream(ccp_context *ctx, void *stream);

/* ------------------------------------------- reference entry points (host buffers) */
/* ewald_self_correction(alp, boxi, qscpe) -- ewald.f90:45-174 (the reference reads the
   global x, xs; here they are arguments). */
int ccp_ewald_self_correction(ccp_context *ctx, double alp, double box, const double *x,
                              const double *y, const double *z, const double *xs,
                              const double *ys, const double *zs, int ld, double *qscpe,
                              double *fxs, double *fys, double *fzs, double *vir);

/* rspace_ewald(xx,yy,zz,xxs,yys,zzs,boxi,alp,qrcpe) -- ewald.f90:177-405. */
int ccp_rspace_ewald(ccp_context *ctx, const double *x, const double *y, const double *z,
                     const double *xs, const double *ys, const double *zs, int ld,
                     double box, double alp, double *qrcpe, double *fxs, double *fys,
                     double *fzs, double *vir);

/* kspace_ewald(xx,..,lmax,mmax,nmax,alp,boxi,qkcpe) -- ewald.f90:754-1173. */
int ccp_kspace_ewald(ccp_context *ctx, const double *x, const double *y, const double *z,
                     const double *xs, const double *ys, const double *zs, int ld, int lmax,
                     int mmax, int nmax, double alp, double box, double *qkcpe, double *fxs,
                     double *fys, double *fzs, double *vir);

/* ccpol23plus(xx,..,boxi,qqvdwe) -- vdw_ccpol23plus.f90:174-477, the 2-body term.  As the
   reference, it OVERWRITES the site forces (fxs = 2-body forces of the first ns sites) and
   SETS *vir to the 2-body virial: the MD step calls it first and the other terms add on.
   The long-range correction, computed but not added by the reference, is not computed. */
int ccp_ccpol23plus(ccp_context *ctx, const double *x, const double *y, const double *z,
                    const double *xs, const double *ys, const double *zs, int ld, double box,
                    double *qvdwe, double *fxs, double *fys, double *fzs, double *vir);

/* nb_induction(xx,..,boxi,qindpe) -- nb_induction_model.f90:25-126: static field, Jacobi
   dipole iteration (iteridm, :1193-1407), induction forces.  idm* receive the induced
   dipoles at every site (non-polarisable sites 0).  *iters may be NULL. */
int ccp_nb_induction(ccp_context *ctx, const double *x, const double *y, const double *z,
                     const double *xs, const double *ys, const double *zs, int ld,
                     double box, double *qindpe, double *idmx, double *idmy, double *idmz,
                     double *fxs, double *fys, double *fzs, double *vir, int *iters);

/* threebody_term(xxx,..,boxii,qfs2,qfs3) -- threebody_potential.f90:17-99: FS2 (if the
   model's S2_term) and FS3 (if S3_term).  fxfs2/fxfs3 are overwritten only for the terms
   that run, as in the reference. */
int ccp_threebody_term(ccp_context *ctx, const double *x, const double *y, const double *z,
                       const double *xs, const double *ys, const double *zs, int ld,
                       double box, double *qfs2, double *qfs3, double *fxs, double *fys,
                       double *fzs, double *fxfs2, double *fyfs2, double *fzfs2,
                       double *fxfs3, double *fyfs3, double *fzfs3, double *vir);

/* The whole sequence evolve.f90:842-877 runs after the 2-body term: Ewald self, real and
   reciprocal, nb_induction (if the model's induction flag), threebody_term (if
   nonadditive_3B), in one call with one upload and one download.  Any output pointer may
   be NULL to skip that download. */
int ccp_hot_path(ccp_context *ctx, const double *x, const double *y, const double *z,
                 const double *xs, const double *ys, const double *zs, int ld, double box,
                 ccp_energies *e, double *fxs, double *fys, double *fzs, double *fxfs2,
                 double *fyfs2, double *fzfs2, double *fxfs3, double *fyfs3,
                 double *fzfs3, double *idmx, double *idmy, double *idmz);

/* ------------------------------------------------ device-resident form */
/* Same as ccp_hot_path with every array already on the device (same layouts).  Nothing
   is copied between host and device except the ccp_energies scalars. */
int ccp_hot_path_device(ccp_context *ctx, const double *x_device, const double *y_device,
                        const double *z_device, const double *xs_device,
                        const double *ys_device, const double *zs_device, int ld, double box,
                        ccp_energies *e, double *fxs_device, double *fys_device,
                        double *fzs_device, double *fxfs2_device, double *fyfs2_device,
                        double *fzfs2_device, double *fxfs3_device, double *fyfs3_device,
                        double *fzfs3_device, double *idmx_device, double *idmy_device,
                        double *idmz_device);

/* ------------------------------------------ reciprocal-space Ewald, fixed scratch */
/* No counterpart in the reference.  kspace_ewald (ewald.f90:754-1173) for callers that
   cannot let the library allocate device memory: an MD driver that hands all device memory
   to its own pool or caching allocator up front, or that cannot afford cudaMalloc/cudaFree
   (cudaFree synchronises the whole device) inside its per-step loop.  Every temporary lives
   in one fixed 16 MiB device array per device (CCP_KSPACE_FIXED_SCRATCH_BYTES): with the 5
   charged sites of the water model that covers 2048 molecules at k-max 15; a call that would
   need more returns CCP_ERR_CAPACITY with the byte count in ccp_last_error() and launches
   nothing.  No context is needed; `m` only supplies the site charges.
   - All arrays are DEVICE pointers on the calling thread's current device, in the layouts of
     ccp_kspace_ewald; forces and *vir are added to, *qkcpe is overwritten.
   - Work is enqueued on `stream` (a cudaStream_t; NULL = the legacy default stream) and the
     call returns without synchronising; results are ready when the stream reaches them.
   - The first call on each device looks the scratch array up (cudaGetSymbolAddress, which
     also loads the module) and keeps its address for the life of the process; a caller
     that captures streams makes one call before capturing.  The kept address belongs to the
     device's primary context (the one the CUDA runtime API uses): calls from a different
     driver context, or after cudaDeviceReset, are not supported.
   - The scratch is shared by all calls on a device: calls whose execution overlaps (other
     streams, other host threads) race on it and give wrong results.  Order them on one
     stream or with events.
   - Allocates no device memory and, on success, no host memory.  The library clears what it
     accumulates into (forces of its own, energy sums) inside the launch sequence.
   Refusals, all returned before anything is launched:
   - CCP_ERR_BAD_INPUT: a NULL pointer; nm < 1; ld below the model's sites per molecule;
     lmax, mmax or nmax below 1; box or alp not positive; a model with no charged sites or
     with more charged sites per molecule than the library's compact site set holds (8);
     a device ordinal above 63;
   - CCP_ERR_CAPACITY: lmax, mmax or nmax above 64, or scratch needs above 16 MiB (the byte
     count is in ccp_last_error());
   - CCP_ERR_CUDA: a CUDA error of earlier work still pending on the calling thread (it is
     left pending), or cudaGetDevice / cudaGetSymbolAddress failing. */
#define CCP_KSPACE_FIXED_SCRATCH_BYTES (16u << 20)
int ccp_kspace_ewald_fixed(const ccp_model *m, int nm, const double *x_device,
                           const double *y_device, const double *z_device,
                           const double *xs_device, const double *ys_device,
                           const double *zs_device, int ld, int lmax, int mmax, int nmax,
                           double alp, double box, double *qkcpe_device, double *fxs_device,
                           double *fys_device, double *fzs_device, double *vir_device,
                           void *stream);

/* Any subset of the hot path's terms on device arrays (layouts of ccp_hot_path_device).
   Terms the model switches off are skipped; energies of terms not run are 0.  This is how
   a caller evaluates, e.g., the three-body plus induction energy alone. */
#define CCP_TERM_SELF 1u       /* ewald_self_correction */
#define CCP_TERM_RSPACE 2u     /* rspace_ewald */
#define CCP_TERM_KSPACE 4u     /* kspace_ewald */
#define CCP_TERM_INDUCTION 8u  /* nb_induction */
#define CCP_TERM_FS2 16u       /* threebody_term, FS2 part */
#define CCP_TERM_FS3 32u       /* threebody_term, FS3 part */
#define CCP_TERM_VDW 64u       /* ccpol23plus 2-body term (vdw_ccpol23plus.f90:174-477) */
#define CCP_TERM_HOT 63u       /* the hot path: every term but the 2-body one */
#define CCP_TERM_ALL 127u
int ccp_terms_device(ccp_context *ctx, unsigned terms, const double *x_device,
                     const double *y_device, const double *z_device, const double *xs_device,
                     const double *ys_device, const double *zs_device, int ld, double box,
                     ccp_energies *e, double *fxs_device, double *fys_device,
                     double *fzs_device, double *fxfs2_device, double *fyfs2_device,
                     double *fzfs2_device, double *fxfs3_device, double *fyfs3_device,
                     double *fzfs3_device, double *idmx_device, double *idmy_device,
                     double *idmz_device);

/* ------------------------------------------- FS3 parameters and their gradient */
/* The FS3 fit of a context, initially the model's data3b_full (SR) and data3b_full_LR_4p5
   (LR): ncoef linear coefficients per fit (ccp_model_get_int "nclass", the cs3 array of
   threebody_potential.f90) and the site-pair nonlinear parameters as three arrays of 289,
   b, g and r0 of site pair (is, js) at is*17 + js (bohr units, as in the files).  Setting
   them re-uploads the tables.  With the context option "fs3_param_grad" on, every
   evaluation that includes FS3 also accumulates the FS3 energy's gradient with respect to
   all of them (kcal/mol per parameter unit), read with ccp_context_fs3_param_grad.  These
   have no counterpart in the reference, which has no derivatives with respect to its fit. */
int ccp_context_get_fs3_params(const ccp_context *ctx, double *cs_sr, double *cs_lr, int ncoef,
                               double *bgr_sr, double *bgr_lr);
int ccp_context_set_fs3_params(ccp_context *ctx, const double *cs_sr, const double *cs_lr,
                               int ncoef, const double *bgr_sr, const double *bgr_lr);
int ccp_context_fs3_param_grad(ccp_context *ctx, double *dcs_sr, double *dcs_lr, int ncoef,
                               double *dbgr_sr, double *dbgr_lr);

/* ------------------------------------------------------ batches of independent frames */
/* No counterpart in the reference, which evaluates one configuration per call.  A batch
   owns `slots` contexts of nm molecules (own device buffers and CUDA streams each).
   ccp_batch_terms_device evaluates nframes independent frames: frame f runs on slot
   f % slots, with one host worker thread per slot, so up to `slots` frames are in flight on
   the GPU at once.  Results equal those of ccp_terms_device called frame by frame.  Device
   arrays hold the frames one after another: x[f*nm + i], xs[(f*nm + i)*ld + s] (and the
   same for every output), box[f] and e[f] on the host.  With pgrad non-null (the option
   "fs3_param_grad" on, set with ccp_batch_set_option) frame f's FS3 parameter gradient goes
   to pgrad[f*pgrad_len ...]: dcs_sr, dcs_lr (ncoef each), dbgr_sr, dbgr_lr (867 each),
   pgrad_len = 2 ncoef + 1734.  The first failing frame's status is returned, with its index
   in ccp_last_error(); a slot stops at its first failure.  Calls on one batch must not
   overlap. */
typedef struct ccp_batch ccp_batch;
int ccp_batch_create(const ccp_model *m, int nm, double box0, int slots, int device,
                     int precision, ccp_batch **out);
int ccp_batch_destroy(ccp_batch *b);
int ccp_batch_slots(const ccp_batch *b, int *slots);
/* the context of one slot (options, FS3 parameters, diagnostics of its last frame) */
int ccp_batch_context(ccp_batch *b, int slot, ccp_context **ctx);
/* Sets a context option (ccp_context_set_option) on every slot, or the batch's own option
     "fuse_fs3" 0 (default): each frame's FS3 runs in its own evaluation; 1: when the frames
                share one box length, FS3 runs once for all frames (one neighbour search,
                triple list and FS3 launch on the batch's own stream) while the slots
                evaluate the other terms.  The results are the same; fused was 7 % slower at
                32 frames of 256 waters. */
int ccp_batch_set_option(ccp_batch *b, const char *name, int value);
int ccp_batch_set_fs3_params(ccp_batch *b, const double *cs_sr, const double *cs_lr, int ncoef,
                             const double *bgr_sr, const double *bgr_lr);
int ccp_batch_terms_device(ccp_batch *b, unsigned terms, int nframes, const double *box,
                           const double *x_device, const double *y_device,
                           const double *z_device, const double *xs_device,
                           const double *ys_device, const double *zs_device, int ld,
                           ccp_energies *e, double *fxs_device, double *fys_device,
                           double *fzs_device, double *fxfs2_device, double *fyfs2_device,
                           double *fzfs2_device, double *fxfs3_device, double *fyfs3_device,
                           double *fzfs3_device, double *idmx_device, double *idmy_device,
                           double *idmz_device, double *pgrad, int pgrad_len);

/* --------------------------------------------------- NVE molecular dynamics (device) */
/* The reference's rigid-molecule NVE integrator, nve_1 with the nosquish rotation
   (evolve.f90:621-1061, 8107-8203), with the state resident on the device: centres x, y, z
   (A), COM velocities v[3*i+a] (A/ps), unit quaternions q[4*i+a], principal-frame angular
   momenta j[3*i+a] (amu A^2/ps).  Forces are the 2-body term (when the model is
   ccpol23plus) plus the hot path.  ccp_md_set_state uploads a state and evaluates its forces
   (initialization.f90:357-381); ccp_md_nve advances nsteps steps of dt ps in a fixed cubic box
   and, when stats is not NULL, fills stats[0..nsteps-1] with each step's energies (kcal/mol),
   temperature (K), virial (kcal/mol) and pressure (katm), as md.f90 writes them to OUTPUT.
   Only these scalars cross PCIe per step. */
typedef struct ccp_md_stats {
    double vdwpe, cpe, indpe, pe3b, pe;  /* 2-body, Coulomb (self+real+reciprocal), induction,
                                            three-body, total potential */
    double tke, rke, te;                 /* translational, rotational, total energy */
    double sys_temp, vir, pres;
    int ind_iters;
    double box, volm;                    /* box length (A) and volume (A^3) of the step */
    double chit, chip;                   /* thermostat and barostat variables after the step
                                            (REVCON's chit, chip) */
    double consv;                        /* nvt_h: 0.5 qmass chit^2 + ceng cint; npt_h adds
                                            0.5 pmass chip^2 + pres0 V; else 0 */
} ccp_md_stats;
int ccp_md_set_state(ccp_context *ctx, double box, const double *x, const double *y,
                     const double *z, const double *v, const double *q, const double *j);
int ccp_md_get_state(ccp_context *ctx, double *x, double *y, double *z, double *v, double *q,
                     double *j);
int ccp_md_nve(ccp_context *ctx, int nsteps, double dt, ccp_md_stats *stats);
/* Ensembles of ccp_md_run, with CONTROL's temp0 (K), taut (ps), pres0 (katm) and taup (ps):
     CCP_MD_NVE    nve_1, as ccp_md_nve (default);
     CCP_MD_NVT_B  nvt_b (evolve.f90:1063-1644): after each step, COM velocities and angular
                   momenta times sqrt(1 + dt/taut (temp0/T - 1)), T the system temperature;
                   the centres are not wrapped; the statistics follow the scaling;
     CCP_MD_NPT_B  npt_b_1 (evolve.f90:7485-8104): before each step the Berendsen barostat
                   chip = 1 + 0.007372 dt (P - pres0)/taup scales the volume by chip, the box
                   and the centres (in the drift) by chip^(1/3), with k-max reset for the new
                   box; after it the system's COM velocity is removed, the nvt_b thermostat
                   applied and the centres wrapped into the new box;
     CCP_MD_NVT_H  nvt_hov_3 (evolve.f90:3316-3834): nve_1's step, then the Nose-Hoover
                   thermostat of nptqscl_t_dl4 (:8305-8369) with its step dt/4 on the
                   thermostat variable chit (ccp_md_set_thermostat; 0 for a fresh run);
     CCP_MD_NPT_H  npt_hov_2 (evolve.f90:5567-6155): before and after each step the
                   Nose-Hoover thermostat (dt/4), barostat nptqscl_p_dl4 (dt/2, :8435-8495),
                   thermostat sequence; volume times exp(3 dt chip), centres scaled by
                   exp(dt chip) about the system's centre in the drift; the step's forces use
                   the old box, the new box applies after the step, then the COM velocity is
                   removed and the centres wrapped;
     CCP_MD_NPT_MTK npt_mtk (evolve.f90:6158-6745): npt_h with the MTK barostat
                   nptqscl_p_dl4_mtk (:8497-8558) and the centres scaled about the origin. */
#define CCP_MD_NVE 0
#define CCP_MD_NVT_B 1
#define CCP_MD_NPT_B 2
#define CCP_MD_NVT_H 3
#define CCP_MD_NPT_H 4
#define CCP_MD_NPT_MTK 5
int ccp_md_set_ensemble(ccp_context *ctx, int ensemble, double temp0, double taut,
                        double pres0_katm, double taup);
int ccp_md_run(ccp_context *ctx, int nsteps, double dt, ccp_md_stats *stats);
/* Thermostat and barostat variables, as REVCON carries them (initialization.f90:62); the
   thermostat's integral (cint) restarts at 0 (initialization.f90:172). */
int ccp_md_set_thermostat(ccp_context *ctx, double chit, double chip);
/* Induced dipoles of the current MD state (its last evaluation), idm*[i*ld + is], for
   HISTORY output; non-polarisable sites get 0. */
int ccp_md_get_dipoles(ccp_context *ctx, int ld, double *idmx, double *idmy, double *idmz);
/* The next nsteps steps of ccp_md_nve are equilibration steps (md.f90:187-193, `step <=
   nequil` with the nve ensemble): after each, COM velocities and angular momenta are scaled
   to temp0 by sqrt(temp0 / T_trans) and sqrt(temp0 / T_rot) (equilibrationGRU,
   utility.f90:353-368).  The step's statistics are those before the scaling, as the
   reference's OUTPUT row. */
int ccp_md_set_equilibration(ccp_context *ctx, double temp0, int nsteps);
/* Statistics of the current MD state without a step (the step-0 row that md.f90:148-152
   writes for a run starting at t = 0; initialization.f90:76-89, 386-399). */
int ccp_md_get_stats(ccp_context *ctx, ccp_md_stats *stats);

/* ---------------------------------------------------------------- diagnostics */
/* These have no counterpart in the reference; they serve benchmarking and profiling. */

/* Launch statistics of the last evaluation: number of kernels this library launched. */
int ccp_context_last_launches(const ccp_context *ctx, int *launches);

/* When on, every evaluation records CUDA events on the launching stream between its
   phases; ccp_context_phase_ms then returns the durations (ms) of the last evaluation:
   [0] input packing + neighbour list, [1] Ewald real space + static field (real) +
   intramolecular terms, [2] Ewald reciprocal space, [3] induction set-up (static reciprocal
   field, dipole tensors, phase factors), [4] dipole iteration, [5] induction forces,
   [6] FS2, [7] FS3 triple list, [8] FS3 kernel, [9] 2-body term. */
#define CCP_NPHASE 10
int ccp_context_set_timing(ccp_context *ctx, int on);
int ccp_context_phase_ms(const ccp_context *ctx, double *ms, int n);

/* Execution options of the induced-dipole solve (results do not depend on them beyond
   round-off):
     "graph_loop"    1 (default): the Jacobi loop runs as one CUDA graph with a conditional
                     WHILE node, no host round trip per iteration; 0: the host launches each
                     iteration and reads the convergence state (profilers that cannot see
                     kernels inside conditional graphs need this);
     "overlap"       1 (default): FS2 and FS3 run on low-priority side streams concurrently
                     with the Ewald and induction kernels (on a high-priority stream);
     "fs3_triples_per_block"  8 (default): FS3 triples per block when overlapping, so that
                     blocks retire often (0: one persistent wave of blocks);
     "fs3_blocks_per_sm"  0 (default, no cap): when overlapping, at most this many FS3
                     blocks per SM (a persistent grid on that many slots), leaving the rest
                     of each SM to the Ewald and induction kernels;
     "fs3_param_grad" 0 (default): see ccp_context_fs3_param_grad;
     "phase_matrix"  1 (default): the polarisable sites' phases are tabulated once per
                     evaluation as exp(i(l x + m y)) and exp(i n z) factors (when they take at
                     most 1 GiB), so a (site, k) phase is one complex product; 0: never (the
                     tiled on-the-fly reciprocal kernels run every iteration);
     "phase_matrix_full" 1 (default): with the factor tables, the full (site, k-vector)
                     phase matrix is formed once per evaluation when it fits in half of the L2
                     (38 MB at 512 waters), and the dipole steps read one phase per pair;
                     0: never.  Query "phase_matrix_full_active" tells whether it was used;
     "dipole_row_form" 1 (default): without the full phase matrix, the dipole steps take the
                     reciprocal sums row by row of the k-vector list (one (l, m), a run of n),
                     so each loaded factor serves many products; 0: one phase per (site,
                     k-vector) product from the factor tables.  The same sums to rounding.
                     Query "dipole_row_form_active" tells whether it was used;
     "dipole_sum_sites" 1..128 (default 32): polarisable sites per structure-factor block of
                     a dipole step (a tuning option; results unchanged);
     "dipole_gather_sites" 2, 3, 4 (default), 6 or 8: polarisable sites per reciprocal-field
                     block of a dipole step (a tuning option; results unchanged);
     "dipole_solver" 0 (CCP_FP64 default): the reference's Jacobi iteration and criterion
                     (sum |dmu|^2 < 1e-20 e^2 A^2); 1: preconditioned conjugate gradients
                     (preconditioner diag(alpha), so the convergence quantity is the Jacobi
                     update at the iterate) to the same criterion; 2 (CCP_MIXED default): PCG
                     to an RMS update of 1e-8 D per polarisable site.  PCG needs the phase
                     table; without it the solve is Jacobi.  ind_iters then counts PCG steps;
     "fs3_fp32_passes" 0 (default): FS3 in FP64 in both forms; 1: in the CCP_MIXED form FS3's
                     ik and jk gradient passes run in FP32 (about 3 % faster FS3; site forces
                     within 2e-6 of FP64, but per-molecule forces 1.45e-5 off at 2048
                     waters, above the mixed form's 1e-5 bar);
     "fs3_high_priority" 0 (default): FS3's side stream at the low priority (1: at the
                     Ewald/induction chain's high priority);
     "pdl"           1 (default): the two kernels of a dipole step are launched with
                     programmatic dependent launch (each starts while its predecessor drains);
     "cell_list"     1 (default): the neighbour lists come from a cell list when the box holds
                     six or more cells of half the list radius per axis (the same lists as the
                     all-pairs scan); 0: always the all-pairs scan.
   ccp_context_get_option also reports "phase_matrix_active" (whether the last evaluation
   used the table), "dipole_solver_pcg_active" (whether its dipole solve was PCG) and
   "cell_list_active" (whether its neighbour lists came from the cell list). */
int ccp_context_set_option(ccp_context *ctx, const char *name, int value);
int ccp_context_get_option(const ccp_context *ctx, const char *name, int *value);

/* Measured peak of the FP64 (precision CCP_FP64) or FP32 (CCP_MIXED) fused multiply-add
   pipe of `device`, in TFLOP/s (2 flops per FMA), from a register-resident FMA chain. */
int ccp_device_fma_peak(int device, int precision, double *tflops);
/* Measured peak of the special-function pipe (MUFU): single-precision hardware
   exponentials per second (Tops/s), from 8 independent exp chains per thread. */
int ccp_device_mufu_peak(int device, double *tops);

#ifdef __cplusplus
}
#endif
#endif
