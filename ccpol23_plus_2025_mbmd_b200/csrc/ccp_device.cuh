// ccp_device.cuh -- device-side helpers and the kernel interface of the hot path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ccpd {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kR4pie0 = 138935.4835;
constexpr double kBohr2a = 0.529177249;
constexpr double kH2kcal = 627.510;
constexpr int kNs3 = 17;
constexpr int kMaxQ = 8;   // charged sites per molecule
constexpr int kMaxP = 4;   // polarisable sites per molecule
constexpr int kMaxA = 12;  // charged or polarisable ("active") sites per molecule

// ---- exact IEEE arithmetic for the decisions that must match the reference bit for bit
// (minimum image, COM cut-offs, R_avg branch).  __d*_rn never fuse into FMA.
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
// d - box*nint(d/box), Fortran nint rounds half away from zero like round().
__device__ __forceinline__ double minimg(double d, double box) {
  return xsub(d, xmul(box, round(__ddiv_rn(d, box))));
}
__device__ __forceinline__ double norm2x(double x, double y, double z) {
  return xadd(xadd(xmul(x, x), xmul(y, y)), xmul(z, z));
}

// Compensated FP64 accumulator (Neumaier's variant of Kahan summation: the rounding error of
// every addition is carried in c, whichever operand is larger).  Used for the per-thread and
// per-block energy and virial sums of the three-body kernels, whose terms come in with both
// signs and magnitudes far above their sum.
struct CompSum {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double x) {
    const double t = __dadd_rn(s, x);
    c = __dadd_rn(c, fabs(s) >= fabs(x) ? __dadd_rn(__dsub_rn(s, t), x)
                                        : __dadd_rn(__dsub_rn(x, t), s));
    s = t;
  }
  __device__ __forceinline__ double value() const { return __dadd_rn(s, c); }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Tang-Toennies f_n(delta r) and derivative (utility.f90:89-125), n small and fixed.
template <int N>
__device__ __forceinline__ double tt(double delta, double r) {
  double dr = delta * r, term = 1.0, sum = 1.0;
#pragma unroll
  for (int i = 1; i <= N; i++) {
    term = term * dr * (1.0 / (double)i);
    sum += term;
  }
  return 1.0 - exp(-dr) * sum;
}
template <int N>
__device__ __forceinline__ double dtt(double delta, double r) {
  constexpr double kInvFact = N == 2 ? 1.0 / 2.0 : (N == 3 ? 1.0 / 6.0 : 1.0 / 24.0);
  static_assert(N >= 2 && N <= 4, "Tang-Toennies order");
  double dr = delta * r, p = 1.0;
#pragma unroll
  for (int i = 1; i <= N; i++) p *= dr;
  return delta * exp(-dr) * p * kInvFact;
}

}  // namespace ccpd

// Scalar accumulator slots (doubles) in ctx->d_scal.
enum ScalSlot {
  S_SELF_SUMFF = 0,  // ewald intramolecular sum erf(a r) q q / r
  S_SELF_VIR,
  S_RC_E,
  S_RC_VIR,
  S_KC_E,
  S_KC_VIR,
  S_IND_CHANGE,
  S_IND_ENERGY,
  S_IND_VIR_R,
  S_IND_VIR_K,
  S_IND_VIR_S,
  S_IND_VIR_SHT,
  S_FS2_E,
  S_FS2_VIR,
  S_FS3_E,
  S_FS3_VIR,
  S_VDW_E,
  S_VDW_VIR,
  S_COUNT
};

// Integer counters in ctx->d_icnt.
enum CountSlot {
  C_NPAIR_FS2 = 0,
  C_NTRI_FS3,
  C_NBLEND_FS3,
  C_NTRI_FS2,
  C_OVERFLOW,
  C_COUNT
};
// One more slot past those k_prep clears: set by k_prep when an input coordinate is not
// finite, read back with the counters and cleared by the host when it reports the error.
enum { C_NONFINITE = C_COUNT, C_ALLOC };

// Model constants the kernels need, passed by value.
struct SiteSets {
  int ns, nq, np, na;
  int qsite[ccpd::kMaxQ];    // site index of each charged site
  int psite[ccpd::kMaxP];    // site index of each polarisable site (last npol sites)
  int asite[ccpd::kMaxA];    // site index of each active site
  int a_of_q[ccpd::kMaxQ];   // active slot of each charged site
  int a_of_p[ccpd::kMaxP];   // active slot of each polarisable site
  int p_of_a[ccpd::kMaxA];   // polarisable slot of each active site (-1 if none)
  double q[ccpd::kMaxA];     // charge of each active site
  double apol[ccpd::kMaxP];  // polarizability*bohr2a^3 of each polarisable site (A^3)
  int nself_q;               // charged sites outside the last npol (self field sources)
  int self_q[ccpd::kMaxQ];   // their charged-slot indices
};

struct EwaldParams {
  double alpha, rcutsd, box, twosqpi, delta2, delta3;
  int damped;
};

struct Fs3Params {
  double boxb, rc2, alp3, r0dmp, delta33, rmin, rmax;
};

struct Fs2Params {
  double boxb, rc2, alp3, r0dmp, delta33;
};

struct KVec {
  double rl, rm, rn, ak;  // 2*pi*(l,m,n)/L and a(k)
  int l, m, n, pad;
};

// The reciprocal gather's view of a k-vector: its components and its rows in the phase
// tables, lmni = (l (2 mmax + 1) + m + mmax) << 8 | (n + nmax); 32 bytes, one L2 sector.
struct KGather {
  double rl, rm, rn;
  int lmni, pad;
};

// One row of the k-vector list: the k-vectors of one (l, m), n = nlo .. nlo + len - 1 at list
// positions kbeg .. kbeg + len - 1 (the list runs over n innermost, ewald.f90:933-1082), with
// their 2 pi l / L, 2 pi m / L and the row of (l, m) in the XY factor table.  The row kernels
// of the dipole step take the rows in decreasing length (32 bytes, one L2 sector).
struct KRow {
  double rl, rm;
  int kbeg, len, nlo, lm;
};
constexpr int kRowTile = 32;  // rows per structure-factor block of the row form

// Arguments of one step of the dipole solve with the phase matrix (k_iter.cu): a Jacobi step,
// or with cu.. set a preconditioned-conjugate-gradient step.
struct IterArgs {
  const int *nbr, *ncnt;
  int cap, nw, np;  // nw = polarisable sites = nm * np
  const double4 *T4;
  const double *TB;
  const double4 *S4;
  const double *SB;
  double *mu, *eim;
  const double *e0;
  const KVec *kv;
  const KGather *kg;
  int nk;
  const double2 *XY;  // [nw][nlm] exp(i(l x + m y)), lm = l (2 mmax + 1) + m + mmax
  const double2 *Z;   // [nw][nz] exp(i n z) (conjugated for n < 0), nz = 2 nmax + 1
  int nlm, nz, mmax, nmax;
  // [nw][nk] the phase of every (polarisable site, k-vector) pair, XY[lm] * Z[n] formed once
  // per evaluation (launch_phase_matrix), or null: the step kernels then form each phase
  // from the factor rows
  const double2 *PM;
  // the row form (PM null, rows set): the k-vector rows by decreasing length, the factor
  // tables XYr[r][w] = exp(i(l x + m y)) of row r and site w, Z[w][n] as above and its
  // transpose ZT[n][w], and rn[n + nmax] = 2 pi n / L
  const KRow *rows;
  int nrow;
  int row_span;  // the largest n range of a tile of kRowTile consecutive rows
  const double2 *XYr, *ZT;
  const double *rn;
  // sk[k] holds two S(k) buffers, (re, im) of steps of parity 0 and 1: a step accumulates
  // into its own and clears the other, which the previous step's gather has finished with
  double *sk, *scal, *state;  // state: see IterStateSlot
  int par;                    // parity of this step
  unsigned *ticket;
  double thr;
  int maxit, use_graph;
  cudaGraphConditionalHandle handle;
  SiteSets S;
  // preconditioned conjugate gradients (k_iter.cu): the vectors u (preconditioned residual),
  // w = A u, s = A p and p of every polarisable site component; mu holds the iterate x
  double *cu, *cw, *cs, *cp;
  // launch the two kernels of a step with programmatic dependent launch: each lets the next
  // kernel's blocks launch early and waits for its predecessor's results itself
  int pdl;
  // block shapes: polarisable sites per structure-factor block (1..128) and per gather and
  // update block (2, 3, 4, 6 or 8)
  int sum_sites, gather_sites;
};

// Slots of the dipole solve's state array (doubles).
enum IterStateSlot {
  kIterIters = 0,    // steps taken
  kIterChange,       // sum |dmu|^2 of the last step (Jacobi) or sum |u|^2 at the iterate (PCG)
  kIterEnergy,       // induction energy sum of the last step
  kIterFinished,     // 1 once the solve has converged (or hit maxit)
  kIterAlpha,        // PCG: step length of the next update
  kIterBeta,         // PCG: direction weight of the next update
  kIterGamma,        // PCG: (r, u) of the current iterate
  kIterAcc,          // PCG: 4 accumulators (gamma, delta, change, energy) of a step
  kIterStateLen = kIterAcc + 4
};

// ccpol23plus 2-body parameters (vdw_ccpol23plus.f90): rows of beta, c0, c1, c2, c3, c6, c8,
// c10 (internal energy units), d1, d6, d8, d10; row[is * ns + js] = row index or -1 and
// qq[is * ns + js] = charge product of the site pair.
constexpr int kVdwPar = 12;
constexpr int kVdwMaxRows = 64;

// ------------------------------------------------------------------ launchers
// All launchers enqueue on `st` and return cudaGetLastError().
// FS3 parameter-gradient buffer (launch_fs3's gfs3): [2][216][8] coefficient-table entries,
// then [2][3][289] (b, g, r0) of each site pair, SR then LR; energy-sum units (hartree).
constexpr int kFs3GradLen = 2 * 216 * 8 + 2 * 3 * 289;
// b[0..n) += a[0..n)
cudaError_t launch_add(int n, const double *a, double *b, cudaStream_t st);
// NVE integrator (k_md.cu); state arrays are structures of arrays [component][nm].
cudaError_t launch_md_stage1(int nm, int ns, const double *f, const double *fc2,
                             const double *fc3, const double *xs, const double *ys,
                             const double *zs, double *x, double *y, double *z, double *v,
                             double *q, double *j, const double pmi[3], double totm, double dt,
                             double scale, const double centre[3], cudaStream_t st);
cudaError_t launch_md_sites(int nm, int ns, const double *q, const double *pcoord, double *xs,
                            double *ys, double *zs, cudaStream_t st);
cudaError_t launch_md_stage2(int nm, int ns, const double *f, const double *fc2,
                             const double *fc3, const double *xs, const double *ys,
                             const double *zs, double *x, double *y, double *z, double *v,
                             const double *q, double *j, const double pmi[3], double totm,
                             double dt, double box, int wrap, double *red, cudaStream_t st);
// launch_md_stage2's red (6 doubles): {sum v^2, sum J^2 / I, sum f . xs, sum v (3)}.
// Sums of the current state into red (9 doubles) = {sum v^2, sum J^2 / I, sum f . xs,
// sum v (3), sum of the centres x (3)}.
cudaError_t launch_md_sums(int nm, int ns, const double *f, const double *fc2, const double *fc3,
                           const double *xs, const double *ys, const double *zs, const double *v,
                           const double *j, const double *x, const double pmi[3], double *red,
                           cudaStream_t st);
// v = fv (v - c) per axis, j *= fj (3 nm each); x, y, z into [-box/2, box/2).
cudaError_t launch_md_scale(int nm, double *v, const double c[3], double fv, double *j, double fj,
                            cudaStream_t st);
cudaError_t launch_md_wrap(int nm, double *x, double *y, double *z, double box, cudaStream_t st);
// ccpol23plus 2-body term (k_vdw.cu): site forces added to f (atomics), energy and virial
// into scal[S_VDW_E], scal[S_VDW_VIR] (internal units).
cudaError_t launch_vdw(const double *xs, const double *ys, const double *zs, int ld,
                       const int *nbr, const double4 *nbrv, const int *ncnt, int cap, int nm,
                       int ns, double rcutsd, const int *row, const double *qq,
                       const double *par, int nrows, const int *vsite, int nv, double *f,
                       double *scal, cudaStream_t st);
cudaError_t launch_prep(const double *x, const double *y, const double *z, const double *xs,
                        const double *ys, const double *zs, int nm, int ld, SiteSets S,
                        double4 *com, double4 *act, double4 *comb, double4 *s17, int ns3,
                        double *f, int nf, double *fc2, double *fc3, double *scal,
                        int *icnt, cudaStream_t st);
cudaError_t launch_neighbors(const double4 *com, int nm, double box, double rlist2, int cap,
                             int *nbr, double4 *nbrv, int *ncnt, int *icnt, cudaStream_t st,
                             int frame_nm = 0);
// Cell-list form of launch_neighbors (same lists): cells per axis for a box and list radius
// (0 when the box holds fewer than six cells of side >= rlist/2 per axis, or more than
// kMaxCellsPerAxis), the int scratch it needs, and the launcher.
constexpr int kMaxCellsPerAxis = 64;
int cell_grid(double box, double rlist);
size_t cell_scratch_ints(int nc, int nm);
cudaError_t launch_neighbors_cells(const double4 *com, int nm, double box, double rlist2,
                                   int nc, int cap, int *scratch, int *nbr, double4 *nbrv,
                                   int *ncnt, int *icnt, cudaStream_t st);
cudaError_t launch_pair_static(const double *x, const double *y, const double *z,
                               const double *xs, const double *ys, const double *zs, int ld,
                               const double4 *act, const int *nbr, const double4 *nbrv,
                               const int *ncnt, int cap, int nm, SiteSets S, EwaldParams P,
                               double *f, double *e0r, double *e0s, int with_self, double *fself,
                               double *e0slf, double *scal, cudaStream_t st);
cudaError_t launch_self_static(const double *x, const double *y, const double *z,
                               const double *xs, const double *ys, const double *zs, int nm,
                               int ld, SiteSets S, EwaldParams P, double *f, double *e0slf,
                               double *scal, cudaStream_t st);
cudaError_t launch_dip_tensor(const double *x, const double *y, const double *z,
                              const double *xs, const double *ys, const double *zs, int ld,
                              const double4 *act, const int *nbr, const double4 *nbrv,
                              const int *ncnt, int cap, int nm, SiteSets S, EwaldParams P,
                              double4 *T4, double *TB, double4 *S4, double *SB, cudaStream_t st);
cudaError_t launch_static_total(int n, const double *a, const double *b, const double *c,
                                const double *d, double *out, cudaStream_t st);
// Convergence node of the Jacobi loop; state = {iterations, change, energy}.  Sets the WHILE
// node's condition only when use_graph is non-zero.
cudaError_t launch_dip_cond(cudaGraphConditionalHandle h, int use_graph, double *scal,
                            double *state, double thr, int maxit, cudaStream_t st);
// k_iter.cu
cudaError_t launch_phase_factors(const double2 *tab, int nm, SiteSets S, int kl, int km, int kn,
                                 double2 *XY, double2 *Z, cudaStream_t st);
cudaError_t launch_tmu(const int *nbr, const int *ncnt, int cap, int nm, int np, const double4 *T4,
                       const double *TB, const double4 *S4, const double *SB, const double *mu,
                       double *eim, cudaStream_t st);
size_t iter_rows_smem_a(int sum_sites, int row_span);
size_t iter_rows_smem_b(int nz, int row_span);
bool iter_rows_fit(int sum_sites, int nz, int row_span);
cudaError_t launch_phase_rows(const double2 *tab, int nm, SiteSets S, int kl, int km, int kn,
                              const KRow *rows, int nrow, double2 *XYr, double2 *Z,
                              double2 *ZT, cudaStream_t st);
cudaError_t launch_phase_matrix(const KGather *kg, int nk, int nw, int nlm, int nz,
                                const double2 *XY, const double2 *Z, double2 *PM,
                                cudaStream_t st);
cudaError_t launch_dip_first(const IterArgs &A, cudaStream_t st);
// Start of the PCG form of the solve (A.cu.. set): x = 0, u = alpha E0, state cleared.
cudaError_t launch_pcg_first(const IterArgs &A, cudaStream_t st);
cudaError_t launch_iter_a(const IterArgs &A, cudaStream_t st);
cudaError_t launch_iter_b(const IterArgs &A, cudaStream_t st);
cudaError_t launch_pair_indforce(const double *x, const double *y, const double *z,
                                 const double *xs, const double *ys, const double *zs,
                                 int ld, const double4 *act, const int *nbr,
                                 const double4 *nbrv, const int *ncnt, int cap, int nm,
                                 SiteSets S, EwaldParams P, const double *mu, double *f,
                                 double *scal, cudaStream_t st);

// reciprocal space
cudaError_t launch_ktab(const double4 *com, const double4 *act, int nm, SiteSets S,
                        double box, int kmax_l, int kmax_m, int kmax_n, double2 *tab,
                        cudaStream_t st);
// mode: 0 Ewald (charged sites: energy, virial, forces)
//       1 static field at polarisable sites from charges
//       2 dipole field at polarisable sites
//       3 induction forces at active sites
// sums: structure factors into sk (4 doubles per k, zeroed by the launcher);
// energy: per-k energy/virial of modes 0 and 3 into scal;
// gather: MODES 1, 2 write the field into out (zeroed by the launcher), 0 and 3 add forces
// into f.
cudaError_t launch_kspace_sums(int mode, const KVec *kv, int nk, const double2 *tab, int nm,
                               SiteSets S, int kl, int km, int kn, const double *mu,
                               double *sk, cudaStream_t st);
cudaError_t launch_kspace_energy(int mode, const KVec *kv, int nk, const double *sk,
                                 double alpha, double *scal, cudaStream_t st);
cudaError_t launch_kspace_gather(int mode, const KVec *kv, int nk, const double2 *tab, int nm,
                                 SiteSets S, int kl, int km, int kn, const double *mu,
                                 const double *sk, double *out, double *f, cudaStream_t st);
// Jacobi update: mu_out = alpha (e0 + eim + ek), change and energy into scal.
cudaError_t launch_dip_update(int nm, SiteSets S, const double *e0, const double *eim,
                              const double *ek, const double *mu, double *mu_out, double *scal,
                              cudaStream_t st);

// three-body.  FS3 triples are kept as records of fs3_record_bytes() bytes each.
size_t fs3_record_bytes();
cudaError_t launch_fs3_enum(const double4 *comb, const int *nbr, const int *ncnt, int cap,
                            int nm, Fs3Params P, void *rec, int tri_cap, int *icnt,
                            cudaStream_t st);
// With frame_nm > 0 the molecules come in frames of frame_nm (one list of triples for the
// independent boxes of a batch): frame f's energy and virial go to scal + f * scal_stride and
// its parameter gradient to gfs3 + f * kFs3GradLen.
cudaError_t launch_fs3(int precision, const void *rec, const int *icnt, int tri_cap,
                       const double4 *s17, const double *coef, const double *bgr, int nm, int ns,
                       double *f, double *fc3, double *scal, int nsm, int triples_per_block,
                       int blocks_per_sm, double *gfs3, cudaStream_t st, int frame_nm = 0,
                       int scal_stride = 0);
// Triples and blend-region triples per frame into counts[2 f], counts[2 f + 1] (cleared by
// the caller).
cudaError_t launch_fs3_frame_counts(const void *rec, const int *icnt, int tri_cap, int frame_nm,
                                    int *counts, cudaStream_t st);
cudaError_t launch_fs2_enum(const double4 *comb, const int *nbr, const int *ncnt, int cap,
                            int nm, Fs2Params P, int2 *pairs, int pair_cap, int *icnt,
                            cudaStream_t st);
cudaError_t launch_fs2(int precision, const int2 *pairs, const int *icnt, int pair_cap,
                       const double4 *comb, const double4 *s17, const int *nbr,
                       const int *ncnt, int cap, Fs2Params P, int nm, int ns, double *f,
                       double *fc2, double *scal, cudaStream_t st);
