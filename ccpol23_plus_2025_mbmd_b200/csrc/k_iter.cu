// k_iter.cu -- one Jacobi step of the induced-dipole solve as two kernels (sm_100a, FP64).
//
// iteridm (nb_induction_model.f90:1193-1407) updates every polarisable dipole from the field
//   E = T.mu (real space + short-range + intramolecular)  +  E_k(mu) (reciprocal)  +  E0.
// The geometry is fixed during the solve, so besides the dipole tensors (k_induction.cu) the
// phases exp(i k.r_s) of the polarisable sites are prepared once per evaluation, factored as
// exp(i(l x + m y)) for every (l, m) and exp(i n z) for every n of each site (the product
// order of the reference's recurrence, ewald.f90:960-1010): a (site, k-vector) phase is then
// one complex product of two table entries, and the tables (nlm + nz per site) stay in L2
// where the full (site, k) matrix would not.  Each iteration then is
//   A  blocks [0, nA):  T.mu, one warp per polarisable site, lanes over its (neighbour, site)
//                       tensor entries (contiguous, so the loads coalesce); these blocks also
//                       clear the S(k) buffer of the other step parity;
//      blocks [nA, ..): dipole structure factors -4 a(k) S(k), S(k) = sum_s (k.mu_s)
//                       e^{ik.r_s}, one thread per k over a chunk of sites, merged with FP64
//                       atomics into this step's buffer;
//   B  one warp per polarisable site: reciprocal field sum_k k g(k, s) (lanes over k), the
//      update mu' = alpha (E_real + E_k + E0) in place, the |mu - mu'|^2 and energy sums;
//      the last block to finish (atomic ticket) closes the iteration: it records the
//      iteration count, change and energy, clears the accumulators for the next iteration,
//      marks the solve finished when it has converged (state[3]: a later B in the same pass
//      of a graph body that unrolls several steps then returns at once) and, inside the
//      graph, sets the WHILE node's condition.  S(k) alternates between two buffers by step
//      parity, so no block has to clear it after the gather.
// When the full phase matrix [site][k] fits in L2 both passes read one phase per pair from
// it; otherwise the row form (k_iter_a_rows, k_iter_b_rows below) takes the sums row by row
// of the k-vector list from factors staged in shared memory.  The same step can also run on
// the factor tables alone (k_iter_a/k_iter_b without the matrix).
#include <climits>

#include "ccp_device.cuh"

using namespace ccpd;

namespace {

constexpr int kThreads = 128;  // small blocks fit beside two FS3 blocks on an SM (see the step kernels)

// Programmatic dependent launch (sm_90+): `launch_dependents` lets the next kernel in the
// stream (launched with programmatic stream serialization) start its blocks once every block
// of this one has executed it; `wait` blocks until the preceding kernel has completed and its
// writes are visible.  Both are no-ops in a kernel launched without the attribute.
__device__ __forceinline__ void pdl_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
constexpr int kWarps = kThreads / 32;
// threads of a gather/update block (k_iter_b): they split the k-vectors, so the block's
// serial chain of dependent loads is nk / kGatherThreads iterations long
#ifndef CCP_GATHER_THREADS
#define CCP_GATHER_THREADS 128
#endif
constexpr int kGatherThreads = CCP_GATHER_THREADS;
constexpr int kGatherWarps = kGatherThreads / 32;
constexpr int kSumSitesMax = 128;  // polarisable sites per structure-factor block (A.sum_sites)
// polarisable sites per gather/update block: a template argument, 2, 3, 4, 6 or 8 (A.gather_sites)

// Phase factors of polarisable site w from the per-axis tables tab[axis][l][site] (ewald.f90:
// 960-1010): XY[w][l][m] = exp(i l x) exp(+-i |m| y) in the reference's product order, and
// Z[w][n] = exp(i |n| z), conjugated for n < 0, so that the phase of k = (l, m, n) is
// XY[l][m] * Z[n] exactly as the reference's final product.
__global__ void k_phase_factors(const double2 *__restrict__ tab, int nm, SiteSets S, int k1,
                                int lmax, int mmax, int nmax, double2 *XY, double2 *Z) {
  const int nw = nm * S.np;
  const int M = 2 * mmax + 1, nlm = (lmax + 1) * M, nz = 2 * nmax + 1;
  const size_t N = (size_t)nm * S.na;
  const size_t total = (size_t)nw * (nlm + nz);
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int w = (int)(t / (nlm + nz)), u = (int)(t - (size_t)w * (nlm + nz));
    const int i = w / S.np, p = w % S.np;
    const size_t st = (size_t)i * S.na + S.a_of_p[p];
    if (u < nlm) {
      const int l = u / M, m = u % M - mmax;
      const double2 el = tab[(size_t)(0 * k1 + l) * N + st];
      const double2 em = tab[(size_t)(1 * k1 + (m < 0 ? -m : m)) * N + st];
      double clm, slm;
      if (m >= 0) {
        clm = el.x * em.x - el.y * em.y;
        slm = el.y * em.x + em.y * el.x;
      } else {
        clm = el.x * em.x + el.y * em.y;
        slm = el.y * em.x - em.y * el.x;
      }
      XY[(size_t)w * nlm + u] = make_double2(clm, slm);
    } else {
      const int n = u - nlm - nmax;
      const double2 en = tab[(size_t)(2 * k1 + (n < 0 ? -n : n)) * N + st];
      Z[(size_t)w * nz + (u - nlm)] = make_double2(en.x, n < 0 ? -en.y : en.y);
    }
  }
}

// The factor tables of the row form: XYr[r][w] for the k-vector rows (KRow, lm = l (2 mmax +
// 1) + m + mmax), formed as k_phase_factors forms XY, and Z both as Z[w][n] and as its
// transpose ZT[n][w].  Site-fastest order, so the row-major writes and the per-axis table
// reads coalesce.
__global__ void k_phase_rows(const double2 *__restrict__ tab, int nm, SiteSets S, int k1,
                             int mmax, int nmax, const KRow *__restrict__ rows, int nrow,
                             double2 *XYr, double2 *Z, double2 *ZT) {
  const int nw = nm * S.np;
  const int M = 2 * mmax + 1, nz = 2 * nmax + 1;
  const size_t N = (size_t)nm * S.na;
  const size_t nxy = (size_t)nrow * nw, total = nxy + (size_t)nz * nw;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    if (t < nxy) {
      const int r = (int)(t / nw), w = (int)(t - (size_t)r * nw);
      const int i = w / S.np, p = w % S.np;
      const size_t st = (size_t)i * S.na + S.a_of_p[p];
      const int lm = rows[r].lm, l = lm / M, m = lm % M - mmax;
      const double2 el = tab[(size_t)(0 * k1 + l) * N + st];
      const double2 em = tab[(size_t)(1 * k1 + (m < 0 ? -m : m)) * N + st];
      double clm, slm;
      if (m >= 0) {
        clm = el.x * em.x - el.y * em.y;
        slm = el.y * em.x + em.y * el.x;
      } else {
        clm = el.x * em.x + el.y * em.y;
        slm = el.y * em.x - em.y * el.x;
      }
      XYr[t] = make_double2(clm, slm);
    } else {
      const size_t u = t - nxy;
      const int ni = (int)(u / nw), w = (int)(u - (size_t)ni * nw);
      const int i = w / S.np, p = w % S.np;
      const size_t st = (size_t)i * S.na + S.a_of_p[p];
      const int n = ni - nmax;
      const double2 en = tab[(size_t)(2 * k1 + (n < 0 ? -n : n)) * N + st];
      const double2 z = make_double2(en.x, n < 0 ? -en.y : en.y);
      ZT[u] = z;
      Z[(size_t)w * nz + ni] = z;
    }
  }
}

// phase of k = (l, m, n) at site w from its factor rows
__device__ __forceinline__ double2 kphase(const double2 *__restrict__ xyw,
                                          const double2 *__restrict__ zw, int lm, int ni) {
  const double2 a = xyw[lm], b = zw[ni];
  return make_double2(a.x * b.x - a.y * b.y, a.y * b.x + a.x * b.y);
}

// Phase of k-vector k (rows lm, ni of the factor tables) at polarisable site w: with the
// phase matrix one coalesced load of row w, else the product of the two factor entries.
template <bool PM>
__device__ __forceinline__ double2 site_phase(const IterArgs &A, int w, int k, int lm, int ni) {
  if constexpr (PM) return A.PM[(size_t)w * A.nk + k];
  return kphase(A.XY + (size_t)w * A.nlm, A.Z + (size_t)w * A.nz, lm, ni);
}

// The phase matrix PM[w][k] = XY[w][lm(k)] * Z[w][n(k)] (kphase, the same product the step
// kernels form without it), one coalesced row of nk phases per polarisable site.
__global__ void k_phase_matrix(const KGather *__restrict__ kg, int nk, int nw, int nlm, int nz,
                               const double2 *__restrict__ XY, const double2 *__restrict__ Z,
                               double2 *PM) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nk) return;
  const int lmni = kg[k].lmni, lm = lmni >> 8, ni = lmni & 255;
  for (int w = blockIdx.y; w < nw; w += gridDim.y)
    PM[(size_t)w * nk + k] = kphase(XY + (size_t)w * nlm, Z + (size_t)w * nz, lm, ni);
}

// The vector a T.mu product reads: the dipoles themselves (Jacobi).
struct MuIn {
  const double *__restrict__ mu;
  __device__ __forceinline__ double3 operator()(size_t site, int) const {
    const double *m = mu + site * 3;
    return make_double3(m[0], m[1], m[2]);
  }
};

// Preconditioned conjugate gradients (the mixed form's dipole solve) for the same linear
// system as the Jacobi step: A mu = E0 with A mu = mu / alpha - F(mu), F(mu) the field of the
// dipoles (T.mu real space + reciprocal + intramolecular corrections, which is symmetric), and
// the preconditioner M^-1 = diag(alpha), so that the preconditioned residual u = alpha (E0 -
// A x) = alpha (E0 + F(x)) - x is exactly the Jacobi update at the iterate x.  The recurrences
// are Chronopoulos and Gear's one-reduction form (Chronopoulos & Gear, J. Comput. Appl. Math.
// 25 (1989) 153-168): with w = A u and s = A p,
//   p = u + beta p,  s = w + beta s,  x += alpha p,  u -= alpha M^-1 s,  w = A u,
//   gamma = (u, M u), delta = (w, u), beta' = gamma' / gamma,
//   alpha' = gamma' / (delta' - beta' gamma' / alpha),
// so one step is one product A u and one merged reduction, as a Jacobi step is.  The new u
// of a site is needed by every reader of the product before the update kernel can store it,
// so readers form it where they read it (pcg_s, pcg_u) from the stored u, w and s and the two
// scalars of the step; the update kernel forms the same values with the same operations
// (explicit roundings, no contraction), so all of them see the same u.
__device__ __forceinline__ double pcg_s(double w, double s, double beta) {
  return __fma_rn(beta, s, w);
}
__device__ __forceinline__ double pcg_u(double u, double s_new, double apol, double alpha) {
  return __fma_rn(-alpha, __dmul_rn(apol, s_new), u);
}
struct PcgIn {
  const double *__restrict__ u;
  const double *__restrict__ w;
  const double *__restrict__ s;
  double alpha, beta, a0, a1, a2, a3;  // step scalars; polarisabilities of sites 0..3
  __device__ __forceinline__ double apol(int q) const {
    return q == 0 ? a0 : (q == 1 ? a1 : (q == 2 ? a2 : a3));
  }
  __device__ __forceinline__ double comp(size_t o, double ap) const {
    return pcg_u(u[o], pcg_s(w[o], s[o], beta), ap, alpha);
  }
  __device__ __forceinline__ double3 operator()(size_t site, int q) const {
    const double ap = apol(q);
    const size_t o = site * 3;
    return make_double3(comp(o, ap), comp(o + 1, ap), comp(o + 2, ap));
  }
};

__device__ __forceinline__ PcgIn pcg_in(const IterArgs &A) {
  PcgIn in;
  in.u = A.cu;
  in.w = A.cw;
  in.s = A.cs;
  in.alpha = A.state[kIterAlpha];
  in.beta = A.state[kIterBeta];
  in.a0 = A.S.apol[0];
  in.a1 = A.np > 1 ? A.S.apol[1] : 0.0;
  in.a2 = A.np > 2 ? A.S.apol[2] : 0.0;
  in.a3 = A.np > 3 ? A.S.apol[3] : 0.0;
  return in;
}

// T.mu of polarisable site w = (i, p): entries T4/TB[i][p][n][q] for the neighbours n of i and
// the polarisable sites q of each, plus the intramolecular entries S4/SB[i][p][q].  Called by
// whole warps; the sum is returned to every lane.  `in` gives the vector multiplied.
template <typename In>
__device__ __forceinline__ void tmu_warp(int w, int lane, const int *__restrict__ nbr,
                                         const int *__restrict__ ncnt, int cap, int np,
                                         const double4 *__restrict__ T4,
                                         const double *__restrict__ TB,
                                         const double4 *__restrict__ S4,
                                         const double *__restrict__ SB, const In &in,
                                         double &ex, double &ey, double &ez) {
  const int i = w / np;
  const int cnt = ncnt[i];
  const size_t base = (size_t)w * cap * np;
  ex = ey = ez = 0.0;
  const int n_ent = cnt * np;
#pragma unroll 4
  for (int e = lane; e < n_ent; e += 32) {
    const int n = e / np, q = e - n * np;
    const int j = nbr[(size_t)i * cap + n];
    const double4 t = T4[base + e];
    const double b = TB[base + e];
    const double3 m = in((size_t)j * np + q, q);
    const double mx = m.x, my = m.y, mz = m.z;
    const double dm = t.w * (t.x * mx + t.y * my + t.z * mz);
    ex += dm * t.x - b * mx;
    ey += dm * t.y - b * my;
    ez += dm * t.z - b * mz;
  }
  if (lane < np) {
    const size_t o = (size_t)w * np + lane;
    const double4 t = S4[o];
    const double b = SB[o];
    const double3 m = in((size_t)i * np + lane, lane);
    const double mx = m.x, my = m.y, mz = m.z;
    const double dm = t.w * (t.x * mx + t.y * my + t.z * mz);
    ex += dm * t.x - b * mx;
    ey += dm * t.y - b * my;
    ez += dm * t.z - b * mz;
  }
  ex = warp_sum(ex);
  ey = warp_sum(ey);
  ez = warp_sum(ez);
}

// One warp per polarisable site (the fallback path's real-space part).
__global__ void __launch_bounds__(kThreads)
    k_tmu(const int *__restrict__ nbr, const int *__restrict__ ncnt, int cap, int nw, int np,
          const double4 *__restrict__ T4, const double *__restrict__ TB,
          const double4 *__restrict__ S4, const double *__restrict__ SB,
          const double *__restrict__ mu, double *eim) {
  const int w = blockIdx.x * kWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= nw) return;
  double ex, ey, ez;
  tmu_warp(w, lane, nbr, ncnt, cap, np, T4, TB, S4, SB, MuIn{mu}, ex, ey, ez);
  if (lane == 0) {
    eim[(size_t)w * 3 + 0] = ex;
    eim[(size_t)w * 3 + 1] = ey;
    eim[(size_t)w * 3 + 2] = ez;
  }
}

// Blocks [0, nA) of a step's first kernel: T.mu, one warp per polarisable site; they also
// clear the S(k) buffer of the other step parity, whose last reader, the previous step's
// gather, has finished.
template <bool PCG>
__device__ __forceinline__ void iter_a_tmu(const IterArgs &A, const PcgIn &pin, int nA) {
  double2 *other = reinterpret_cast<double2 *>(A.sk) + (A.par ^ 1);
  for (int k = blockIdx.x * kThreads + threadIdx.x; k < A.nk; k += nA * kThreads)
    other[2 * (size_t)k] = make_double2(0.0, 0.0);
  const int w = blockIdx.x * kWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= A.nw) return;
  double ex, ey, ez;
  if constexpr (PCG)
    tmu_warp(w, lane, A.nbr, A.ncnt, A.cap, A.np, A.T4, A.TB, A.S4, A.SB, pin, ex, ey, ez);
  else
    tmu_warp(w, lane, A.nbr, A.ncnt, A.cap, A.np, A.T4, A.TB, A.S4, A.SB, MuIn{A.mu}, ex, ey,
             ez);
  // the next kernel may launch once every block is this far: late enough that its blocks
  // do not hold SM slots (which concurrent kernels could use) for long while they wait
  pdl_launch_dependents();
  if (lane == 0) {
    A.eim[(size_t)w * 3 + 0] = ex;
    A.eim[(size_t)w * 3 + 1] = ey;
    A.eim[(size_t)w * 3 + 2] = ez;
  }
}

template <bool PCG, bool PM>
__global__ void __launch_bounds__(kThreads)
    k_iter_a(IterArgs A) {
  // no test of the finished flag here: a step after the finish only rewrites the T.mu
  // scratch and S(k), which the next use clears, and it saves a dependent load per step
  pdl_wait();  // the previous step's dipoles (and its gather's last use of the S(k) buffer)
  const int nA = (A.nw + kWarps - 1) / kWarps;
  PcgIn pin;
  if constexpr (PCG) pin = pcg_in(A);
  if ((int)blockIdx.x < nA) {
    iter_a_tmu<PCG>(A, pin, nA);
    return;
  }
  // structure factors: block b covers k-vectors [kt*256, kt*256+256) and sites of chunk sc
  extern __shared__ double smu[];  // A.sum_sites x 3 dipole components
  const int b = blockIdx.x - nA;
  const int nkt = (A.nk + kThreads - 1) / kThreads;
  const int kt = b % nkt, sc = b / nkt;
  const int s0 = sc * A.sum_sites, cnt = min(A.sum_sites, A.nw - s0);
  for (int u = threadIdx.x; u < cnt * 3; u += kThreads) {
    if constexpr (PCG) {
      const int site = s0 + u / 3;
      smu[u] = pin.comp((size_t)s0 * 3 + u, pin.apol(site % A.np));
    } else {
      smu[u] = A.mu[(size_t)s0 * 3 + u];
    }
  }
  __syncthreads();
  const int k = kt * kThreads + threadIdx.x;
  if (k >= A.nk) return;
  const KVec K = A.kv[k];
  const int lm = K.l * (2 * A.mmax + 1) + K.m + A.mmax, ni = K.n + A.nmax;
  double a0 = 0.0, a1 = 0.0;
#pragma unroll 4
  for (int s = 0; s < cnt; s++) {
    const double2 ph = site_phase<PM>(A, s0 + s, k, lm, ni);
    const double dk = K.rl * smu[3 * s] + K.rm * smu[3 * s + 1] + K.rn * smu[3 * s + 2];
    a0 += dk * ph.x;
    a1 += dk * ph.y;
  }
  pdl_launch_dependents();
  // kspace_efield_idm's weight (nb_induction_model.f90:2560-2600), applied before the merge
  const double g = -4.0 * K.ak;
  atomicAdd(&A.sk[(size_t)k * 4 + 2 * A.par], g * a0);
  atomicAdd(&A.sk[(size_t)k * 4 + 2 * A.par + 1], g * a1);
}

// The PCG step's update for the GS sites of a block, after the reciprocal field of
// u is in `part`: the vectors of the step (s, p, x, u, w = A u) in place, the partial sums
// of (u, M u), (w, u), |u|^2 and the energy -1/2 x.E0 (the reference's energy expression at
// the iterate), and in the last block to finish the step's scalars and the convergence test
// on sum |u|^2, the Jacobi update's norm at the iterate.
// ek(g, c) gives component c of the reciprocal field at the block's site g; the updating
// threads (one per site) are all in warp 0.
template <typename EK>
__device__ __forceinline__ void pcg_update(const IterArgs &A, int w0, int ns_blk, const EK &ekf) {
  double gam = 0.0, del = 0.0, ch = 0.0, en = 0.0;
  if ((int)threadIdx.x < ns_blk) {
    const int g = threadIdx.x, w = w0 + g;
    double ek[3];
    for (int c = 0; c < 3; c++) ek[c] = ekf(g, c);
    const double ap = A.S.apol[w % A.np];
    const double ca = A.state[kIterAlpha], cb = A.state[kIterBeta];
    for (int c = 0; c < 3; c++) {
      const size_t o = (size_t)w * 3 + c;
      const double u0 = A.cu[o];
      const double s = pcg_s(A.cw[o], A.cs[o], cb);
      const double p = __fma_rn(cb, A.cp[o], u0);
      const double x = __fma_rn(ca, p, A.mu[o]);
      const double u = pcg_u(u0, s, ap, ca);
      const double wv = u / ap - (A.eim[o] + ek[c]);
      A.cs[o] = s;
      A.cp[o] = p;
      A.mu[o] = x;
      A.cu[o] = u;
      A.cw[o] = wv;
      gam += u * u / ap;
      del += wv * u;
      ch += u * u;
      en += -0.5 * x * A.e0[o];
    }
  }
  gam = warp_sum(gam);  // the updating threads are all in warp 0
  del = warp_sum(del);
  ch = warp_sum(ch);
  en = warp_sum(en);
  __shared__ bool last;
  double *acc = A.state + kIterAcc;
  if (threadIdx.x == 0) {
    atomicAdd(acc + 0, gam);
    atomicAdd(acc + 1, del);
    atomicAdd(acc + 2, ch);
    atomicAdd(acc + 3, en);
    __threadfence();
    last = atomicAdd(A.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    const double g1 = atomicAdd(acc + 0, 0.0), d1 = atomicAdd(acc + 1, 0.0);
    const double chg = atomicAdd(acc + 2, 0.0), ene = atomicAdd(acc + 3, 0.0);
    for (int k = 0; k < 4; k++) acc[k] = 0.0;
    *A.ticket = 0u;
    int it = (int)A.state[kIterIters] + 1;
    A.state[kIterChange] = chg;
    A.state[kIterEnergy] = ene;
    bool more = chg > A.thr && it < A.maxit;
    if (more) {
      const double beta = it == 1 ? 0.0 : g1 / A.state[kIterGamma];
      const double alpha = it == 1 ? g1 / d1 : g1 / (d1 - beta * g1 / A.state[kIterAlpha]);
      if (alpha > 0.0 && alpha < 1e300) {
        A.state[kIterAlpha] = alpha;
        A.state[kIterBeta] = beta;
        A.state[kIterGamma] = g1;
      } else {  // breakdown (not positive definite): reported as no convergence
        it = A.maxit;
        more = false;
      }
    }
    A.state[kIterIters] = (double)it;
    if (!more) A.state[kIterFinished] = 1.0;
    if (A.use_graph) cudaGraphSetConditional(A.handle, more ? 1u : 0u);
  }
}

// The Jacobi update of the block's sites (nb_induction_model.f90:1317-1359) from their
// reciprocal field ek(g, c), the change and energy sums, and in the last block to finish the
// step's close (iteration count, convergence test, the graph's condition).  The updating
// threads (one per site) are all in warp 0.
template <typename EK>
__device__ __forceinline__ void jacobi_update(const IterArgs &A, int w0, int ns_blk,
                                              const EK &ekf) {
  double ch = 0.0, en = 0.0;
  if ((int)threadIdx.x < ns_blk) {
    const int g = threadIdx.x, w = w0 + g;
    double ek[3];
    for (int c = 0; c < 3; c++) ek[c] = ekf(g, c);
    const double polr = A.S.apol[w % A.np];
    double Et[3], E0[3];
    for (int c = 0; c < 3; c++) {
      const size_t o = (size_t)w * 3 + c;
      E0[c] = A.e0[o];
      Et[c] = (A.eim[o] + ek[c]) + E0[c];
      const double m = polr * Et[c];
      const double d = A.mu[o] - m;
      ch += d * d;
      A.mu[o] = m;
    }
    en = -0.5 * polr * (Et[0] * E0[0] + Et[1] * E0[1] + Et[2] * E0[2]);
  }
  ch = warp_sum(ch);  // the updating threads are all in warp 0
  en = warp_sum(en);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    atomicAdd(&A.scal[S_IND_CHANGE], ch);
    atomicAdd(&A.scal[S_IND_ENERGY], en);
    __threadfence();
    last = atomicAdd(A.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  // every other block has added its sums
  __threadfence();
  if (threadIdx.x == 0) {
    const double chg = atomicAdd(&A.scal[S_IND_CHANGE], 0.0);
    const double ene = atomicAdd(&A.scal[S_IND_ENERGY], 0.0);
    const int it = (int)A.state[kIterIters] + 1;
    A.state[kIterIters] = (double)it;
    A.state[kIterChange] = chg;
    A.state[kIterEnergy] = ene;
    A.scal[S_IND_CHANGE] = 0.0;
    A.scal[S_IND_ENERGY] = 0.0;
    *A.ticket = 0u;
    const bool more = chg > A.thr && it < A.maxit;
    if (!more) A.state[kIterFinished] = 1.0;
    if (A.use_graph) cudaGraphSetConditional(A.handle, more ? 1u : 0u);
  }
}

template <bool PCG, bool PM, int GS>
__global__ void __launch_bounds__(kGatherThreads)
    k_iter_b(IterArgs A) {
  // GS polarisable sites per block; the warps split the k-vectors, so every
  // k-vector's weights are loaded once per block and reused for all its sites
  pdl_wait();  // T.mu, S(k) and the step scalars of this step's first kernel
  if (A.state[kIterFinished] != 0.0) return;  // finished in an earlier step of this pass
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int w0 = blockIdx.x * GS;
  const int ns_blk = min(GS, A.nw - w0);
  double acc[GS][3];
#pragma unroll
  for (int g = 0; g < GS; g++) acc[g][0] = acc[g][1] = acc[g][2] = 0.0;
  const double2 *skp = reinterpret_cast<const double2 *>(A.sk) + A.par;
  // the next k-vector's record and S(k) are loaded one iteration ahead, so that an iteration
  // waits for its phase loads only, not for the record that indexes them first
  KGather Kn{};
  double2 fn = make_double2(0.0, 0.0);
  if ((int)threadIdx.x < A.nk) {
    Kn = A.kg[threadIdx.x];
    fn = skp[2 * (size_t)threadIdx.x];
  }
#pragma unroll 2
  for (int k = threadIdx.x; k < A.nk; k += kGatherThreads) {
    const KGather K = Kn;
    const double2 f = fn;
    if (k + kGatherThreads < A.nk) {
      Kn = A.kg[k + kGatherThreads];
      fn = skp[2 * (size_t)(k + kGatherThreads)];
    }
    const int lm = K.lmni >> 8, ni = K.lmni & 255;
    // kspace_efield_idm gather (nb_induction_model.f90:2560-2600): g = -4 a_k (c S_re + s S_im)
    const double f0 = f.x, f1 = f.y;
#pragma unroll
    for (int g = 0; g < GS; g++) {
      if (g < ns_blk) {
        const double2 ph = site_phase<PM>(A, w0 + g, k, lm, ni);
        const double t = ph.x * f0 + ph.y * f1;
        acc[g][0] += K.rl * t;
        acc[g][1] += K.rm * t;
        acc[g][2] += K.rn * t;
      }
    }
  }
  pdl_launch_dependents();  // the gather, the bulk of the kernel, is done
  __shared__ double part[kGatherWarps][GS * 3];
#pragma unroll
  for (int g = 0; g < GS; g++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double v = warp_sum(acc[g][c]);
      if (lane == 0) part[wid][g * 3 + c] = v;
    }
  __syncthreads();
  const auto ek = [&](int g, int c) {
    double v = 0.0;
    for (int u = 0; u < kGatherWarps; u++) v += part[u][g * 3 + c];
    return v;
  };
  if constexpr (PCG)
    pcg_update(A, w0, ns_blk, ek);
  else
    jacobi_update(A, w0, ns_blk, ek);
}

// ------------------------------------------------------------------ the row form
// For boxes whose phase matrix does not fit in L2 the step kernels above form each (site,
// k-vector) phase from two factor-table loads, and both passes then run at the L1 load rate,
// far below the FP64 rate.  The row form regroups the same sums by the rows of the k-vector
// list (one (l, m), a run of n), so that every loaded value serves many products:
//   structure factors  S(k) = sum_w Z(w, n) (B(w, r) + k_n C(w, r)),
//                      B = XY(w, r) (k_l mu_x + k_m mu_y),  C = XY(w, r) mu_z;
//   gather             E(w) = sum_r Re[XY(w, r) (k_l Q, k_m Q, Q_z)],
//                      Q = sum_n Z(w, n) conj F(k),  Q_z = sum_n k_n Z(w, n) conj F(k),
// F(k) the weighted S(k) of the step.  These are k_iter_a's and k_iter_b's sums with the
// products reassociated (equal to rounding).
constexpr int kRowLanes = 8;  // n lanes per row of a structure-factor block: n = nb + lane + 8 j
// gather blocks: sites per block (8, 16 or 32), rows per thread, warps per block
#ifndef CCP_ROW_SITES
#define CCP_ROW_SITES 16
#endif
#ifndef CCP_ROW_R
#define CCP_ROW_R 4
#endif
#ifndef CCP_ROW_WARPS
#define CCP_ROW_WARPS 8
#endif
// structure-factor blocks resident per SM that the register allocation targets
#ifndef CCP_ROW_SUM_BLOCKS
#define CCP_ROW_SUM_BLOCKS 1
#endif
constexpr int kRowSites = CCP_ROW_SITES, kRowR = CCP_ROW_R, kRowWarps = CCP_ROW_WARPS;
constexpr int kRowSumBlocks = CCP_ROW_SUM_BLOCKS;
static_assert(kRowSites == 8 || kRowSites == 16 || kRowSites == 32, "sites per gather block");
static_assert(kThreads / kRowLanes * 2 == kRowTile, "a structure-factor block takes two rows per thread");

// Structure factors of the row form: block b (after the T.mu blocks) covers tile b % ntile
// (kRowTile consecutive rows of the length-sorted list, n in [nb, ne) of their union) and the
// sites of chunk b / ntile.  A thread takes two adjacent rows of the tile and the n = nb +
// lane + 8 j (j < J) of them, so that each Z factor it loads serves both; the partial sums are
// merged with FP64 atomics as in k_iter_a.  The chunk's XY factors of the tile's rows and its
// Z factors of the tile's n range are staged in shared memory before the wait for the
// previous step (the tables are fixed during the solve), so the site loop reads only shared
// memory.
template <bool PCG, int J>
__global__ void __launch_bounds__(kThreads, kRowSumBlocks) k_iter_a_rows(IterArgs A) {
  const int nA = (A.nw + kWarps - 1) / kWarps;
  if ((int)blockIdx.x < nA) {
    pdl_wait();  // the previous step's dipoles (and its gather's last use of the S(k) buffer)
    PcgIn pin;
    if constexpr (PCG) pin = pcg_in(A);
    iter_a_tmu<PCG>(A, pin, nA);
    return;
  }
  // the chunk's dipoles [site] (x, y, z, 0), the XY factors [site][row] of the tile's rows and
  // the Z factors [site][n - nb] of its n range (row stride row_span)
  extern __shared__ double4 smu4[];
  constexpr int kXs = kRowTile + 1;  // site stride of the staged XY: no bank conflicts
  double2 *bxy = reinterpret_cast<double2 *>(smu4 + A.sum_sites);
  double2 *zs = bxy + (size_t)A.sum_sites * kXs;
  __shared__ int s_nb, s_ne;
  const int b = blockIdx.x - nA;
  const int ntile = (A.nrow + kRowTile - 1) / kRowTile;
  const int rt = b % ntile, sc = b / ntile;
  const int s0 = sc * A.sum_sites, cnt = min(A.sum_sites, A.nw - s0);
  const int r0 = rt * kRowTile, nr = min(kRowTile, A.nrow - r0);
  if (threadIdx.x == 0) {
    int nb = A.rows[r0].nlo, ne = nb + A.rows[r0].len;
    for (int r = 1; r < nr; r++) {
      const int lo = A.rows[r0 + r].nlo;
      nb = min(nb, lo);
      ne = max(ne, lo + A.rows[r0 + r].len);
    }
    s_nb = nb;
    s_ne = ne;
  }
  for (int u = threadIdx.x; u < nr * cnt; u += kThreads) {
    const int r = u / cnt, s = u - r * cnt;
    bxy[s * kXs + r] = A.XYr[(size_t)(r0 + r) * A.nw + s0 + s];
  }
  __syncthreads();
  const int nb = s_nb, nn = s_ne - nb;  // nn <= row_span
  for (int u = threadIdx.x; u < cnt * nn; u += kThreads) {
    const int s = u / nn, j = u - s * nn;
    zs[s * A.row_span + j] = A.Z[(size_t)(s0 + s) * A.nz + nb + j + A.nmax];
  }
  pdl_wait();  // the previous step's dipoles (and its gather's last use of the S(k) buffer)
  PcgIn pin;
  if constexpr (PCG) pin = pcg_in(A);
  for (int u = threadIdx.x; u < cnt; u += kThreads) {
    const size_t o = (size_t)(s0 + u) * 3;
    if constexpr (PCG) {
      const double ap = pin.apol((s0 + u) % A.np);
      smu4[u] = make_double4(pin.comp(o, ap), pin.comp(o + 1, ap), pin.comp(o + 2, ap), 0.0);
    } else {
      smu4[u] = make_double4(A.mu[o], A.mu[o + 1], A.mu[o + 2], 0.0);
    }
  }
  __syncthreads();
  const int ra = 2 * (threadIdx.x / kRowLanes), c = threadIdx.x % kRowLanes;
  if (ra >= nr) return;
  // this thread's rows ra and ra + 1 of the tile (the second empty past the tile's end)
  const KRow R0 = A.rows[r0 + ra];
  KRow R1 = R0;
  if (ra + 1 < nr)
    R1 = A.rows[r0 + ra + 1];
  else
    R1.len = 0;
  const int rb1 = ra + 1 < nr ? ra + 1 : ra;
  const int jt = (nn + kRowLanes - 1) / kRowLanes;  // jt <= J: row_span
  // per n = nb + c + 8 j: the staged Z column (clamped to the range, so idle lanes read a
  // column another lane reads), k_n, and the k-vector of each row that holds that n
  int col[J], k0[J], k1[J];
  double rnj[J];
#pragma unroll
  for (int j = 0; j < J; j++) {
    const int d = c + kRowLanes * j, n = nb + d;
    col[j] = min(d, nn - 1);
    rnj[j] = d < nn ? A.rn[n + A.nmax] : 0.0;
    k0[j] = j < jt && n >= R0.nlo && n < R0.nlo + R0.len ? R0.kbeg + (n - R0.nlo) : -1;
    k1[j] = j < jt && n >= R1.nlo && n < R1.nlo + R1.len ? R1.kbeg + (n - R1.nlo) : -1;
  }
  double ax[J], ay[J], bx_[J], by_[J];
#pragma unroll
  for (int j = 0; j < J; j++) ax[j] = ay[j] = bx_[j] = by_[j] = 0.0;
#pragma unroll 2
  for (int s = 0; s < cnt; s++) {
    const double4 m = smu4[s];
    const double2 xy0 = bxy[s * kXs + ra], xy1 = bxy[s * kXs + rb1];
    const double a0 = R0.rl * m.x + R0.rm * m.y, a1 = R1.rl * m.x + R1.rm * m.y;
    const double b0x = xy0.x * a0, b0y = xy0.y * a0, c0x = xy0.x * m.z, c0y = xy0.y * m.z;
    const double b1x = xy1.x * a1, b1y = xy1.y * a1, c1x = xy1.x * m.z, c1y = xy1.y * m.z;
    const double2 *zw = zs + s * A.row_span;
#pragma unroll
    for (int j = 0; j < J; j++) {
      if (j < jt) {
        const double2 z = zw[col[j]];
        const double t0x = rnj[j] * c0x + b0x, t0y = rnj[j] * c0y + b0y;
        const double t1x = rnj[j] * c1x + b1x, t1y = rnj[j] * c1y + b1y;
        ax[j] += z.x * t0x - z.y * t0y;
        ay[j] += z.x * t0y + z.y * t0x;
        bx_[j] += z.x * t1x - z.y * t1y;
        by_[j] += z.x * t1y + z.y * t1x;
      }
    }
  }
  pdl_launch_dependents();
#pragma unroll
  for (int j = 0; j < J; j++) {
    // kspace_efield_idm's weight (nb_induction_model.f90:2560-2600), applied before the merge
    if (k0[j] >= 0) {
      const double g = -4.0 * A.kv[k0[j]].ak;
      atomicAdd(&A.sk[(size_t)k0[j] * 4 + 2 * A.par], g * ax[j]);
      atomicAdd(&A.sk[(size_t)k0[j] * 4 + 2 * A.par + 1], g * ay[j]);
    }
    if (k1[j] >= 0) {
      const double g = -4.0 * A.kv[k1[j]].ak;
      atomicAdd(&A.sk[(size_t)k1[j] * 4 + 2 * A.par], g * bx_[j]);
      atomicAdd(&A.sk[(size_t)k1[j] * 4 + 2 * A.par + 1], g * by_[j]);
    }
  }
}

// Gather and update of the row form: a block takes kRowSites sites and its warps take the
// groups of rows in turn (kRowR rows per thread, 32 / kRowSites threads per site, so a warp
// covers 32 / kRowSites x kRowR consecutive rows of the length-sorted list, whose n ranges are
// close).  The block's Z factors are staged in shared memory before the wait for the step's
// first kernel (they are fixed during the solve), and each warp stages the F(k) of a group's
// rows before running over its n range, so that the loop reads only shared memory.  The
// update is k_iter_b's.
template <bool PCG>
__global__ void __launch_bounds__(kRowWarps * 32, 768 / (kRowWarps * 32)) k_iter_b_rows(IterArgs A) {
  constexpr int kSB = kRowSites, kRL = 32 / kRowSites, kG = kRL * kRowR;
  // Z [n][site] of the block's sites (nz rows), then per warp the F(k) [row][n - nlo] of its
  // group's kG rows (row stride row_span)
  extern __shared__ double2 zsh[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int si = lane % kSB, h = lane / kSB;
  const int w0 = blockIdx.x * kSB;
  const int ns_blk = min(kSB, A.nw - w0);
  for (int u = threadIdx.x; u < A.nz * kSB; u += kRowWarps * 32) {
    const int ni = u / kSB, s = u - ni * kSB;
    zsh[u] = s < ns_blk ? A.ZT[(size_t)ni * A.nw + w0 + s] : make_double2(0.0, 0.0);
  }
  double *rns = reinterpret_cast<double *>(zsh + (size_t)A.nz * kSB);  // k_n by n + nmax
  for (int u = threadIdx.x; u < A.nz; u += kRowWarps * 32) rns[u] = A.rn[u];
  double2 *fsh = zsh + (size_t)A.nz * kSB + (A.nz + 1) / 2 + (size_t)wid * kG * A.row_span;
  pdl_wait();  // T.mu, S(k) and the step scalars of this step's first kernel
  __syncthreads();  // the staged Z
  if (A.state[kIterFinished] != 0.0) return;  // finished in an earlier step of this pass
  const int wc = w0 + (si < ns_blk ? si : 0);  // the site whose XY this lane reads
  const double2 *skp = reinterpret_cast<const double2 *>(A.sk) + A.par;
  const double2 *xyr = A.XYr + wc;
  const double2 *zl = zsh + si + A.nmax * kSB;  // Z of n at zl[n * kSB]
  double ex = 0.0, ey = 0.0, ez = 0.0;
  const int ng = (A.nrow + kG - 1) / kG;
  for (int g = wid; g < ng; g += kRowWarps) {
    // the warp's rows g kG .. g kG + kG - 1: stage their F(k), then this lane's kRowR of them
    const int gb = g * kG, gn = min(kG, A.nrow - gb);
    __syncwarp();  // the previous group's reads of the staging buffer are done
    for (int u = lane; u < gn * A.row_span; u += 32) {
      const int r = u / A.row_span, j = u - r * A.row_span;
      const KRow &K = A.rows[gb + r];
      if (j < K.len) fsh[u] = skp[2 * (size_t)(K.kbeg + j)];
    }
    __syncwarp();
    const int rb = gb + h * kRowR;  // this lane's rows rb .. rb + kRowR - 1
    int nlo[kRowR], len[kRowR];
    int nb = INT_MAX, ne = INT_MIN;
#pragma unroll
    for (int r = 0; r < kRowR; r++) {
      nlo[r] = len[r] = 0;
      if (rb + r < A.nrow) {
        const KRow &K = A.rows[rb + r];
        nlo[r] = K.nlo;
        len[r] = K.len;
        nb = min(nb, nlo[r]);
        ne = max(ne, nlo[r] + len[r]);
      }
    }
    // the warp runs the n range of all its rows
#pragma unroll
    for (int o = kSB; o < 32; o <<= 1) {
      nb = min(nb, __shfl_xor_sync(0xffffffffu, nb, o));
      ne = max(ne, __shfl_xor_sync(0xffffffffu, ne, o));
    }
    const double2 *fl = fsh + (size_t)h * kRowR * A.row_span;
    // this lane's XY factors of its rows, loaded now so that their latency overlaps the sums
    double2 xy[kRowR];
#pragma unroll
    for (int r = 0; r < kRowR; r++)
      xy[r] = len[r] > 0 ? xyr[(size_t)(rb + r) * A.nw] : make_double2(0.0, 0.0);
    double qx[kRowR], qy[kRowR], zx[kRowR], zy[kRowR];
#pragma unroll
    for (int r = 0; r < kRowR; r++) qx[r] = qy[r] = zx[r] = zy[r] = 0.0;
#pragma unroll 2
    for (int n = nb; n < ne; n++) {
      const double2 z = zl[n * kSB];
      const double rn = rns[n + A.nmax];
#pragma unroll
      for (int r = 0; r < kRowR; r++) {
        if ((unsigned)(n - nlo[r]) < (unsigned)len[r]) {
          // kspace_efield_idm gather (nb_induction_model.f90:2560-2600): the phase times the
          // conjugate of the weighted S(k), summed over the row
          const double2 f = fl[r * A.row_span + (n - nlo[r])];
          const double px = z.x * f.x + z.y * f.y, py = z.y * f.x - z.x * f.y;
          qx[r] += px;
          qy[r] += py;
          zx[r] += rn * px;
          zy[r] += rn * py;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kRowR; r++) {
      if (len[r] > 0) {
        const KRow &K = A.rows[rb + r];
        const double a = xy[r].x * qx[r] - xy[r].y * qy[r];
        ex += K.rl * a;
        ey += K.rm * a;
        ez += xy[r].x * zx[r] - xy[r].y * zy[r];
      }
    }
  }
  pdl_launch_dependents();  // the gather, the bulk of the kernel, is done
#pragma unroll
  for (int o = kSB; o < 32; o <<= 1) {
    ex += __shfl_xor_sync(0xffffffffu, ex, o);
    ey += __shfl_xor_sync(0xffffffffu, ey, o);
    ez += __shfl_xor_sync(0xffffffffu, ez, o);
  }
  __shared__ double part[kRowWarps][3][kSB];
  if (h == 0) {
    part[wid][0][si] = ex;
    part[wid][1][si] = ey;
    part[wid][2][si] = ez;
  }
  __syncthreads();
  const auto ek = [&](int g, int c) {
    double v = 0.0;
    for (int u = 0; u < kRowWarps; u++) v += part[u][c][g];
    return v;
  };
  if constexpr (PCG)
    pcg_update(A, w0, ns_blk, ek);
  else
    jacobi_update(A, w0, ns_blk, ek);
}

// The first Jacobi step from mu = 0 (nb_induction_model.f90:1317-1359), where T.mu and the
// reciprocal field are zero: mu = alpha E0, with the change and energy sums the full step
// forms, in one block.  It records iteration 1 in the state and, inside the graph, sets the
// WHILE node's condition, so the loop starts at the second step.
constexpr int kFirstThreads = 1024;
__global__ void __launch_bounds__(kFirstThreads) k_dip_first(IterArgs A) {
  double ch = 0.0, en = 0.0;
  for (int w = threadIdx.x; w < A.nw; w += kFirstThreads) {
    const double polr = A.S.apol[w % A.np];
    double Et[3], E0[3];
    for (int c = 0; c < 3; c++) {
      const size_t o = (size_t)w * 3 + c;
      E0[c] = A.e0[o];
      Et[c] = (0.0 + 0.0) + E0[c];
      const double m = polr * Et[c];
      const double d = 0.0 - m;
      ch += d * d;
      A.mu[o] = m;
    }
    en += -0.5 * polr * (Et[0] * E0[0] + Et[1] * E0[1] + Et[2] * E0[2]);
  }
  __shared__ double red[2][kFirstThreads / 32];
  ch = warp_sum(ch);
  en = warp_sum(en);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = ch;
    red[1][threadIdx.x >> 5] = en;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double chg = 0.0, ene = 0.0;
    for (int u = 0; u < kFirstThreads / 32; u++) {
      chg += red[0][u];
      ene += red[1][u];
    }
    A.state[kIterIters] = 1.0;
    A.state[kIterChange] = chg;
    A.state[kIterEnergy] = ene;
    const bool more = chg > A.thr && 1 < A.maxit;
    A.state[kIterFinished] = more ? 0.0 : 1.0;
    if (A.use_graph) cudaGraphSetConditional(A.handle, more ? 1u : 0u);
  }
}

// The start of the PCG solve: x = 0, u = alpha E0 (the Jacobi first step's dipoles), w, s
// and p zero and the step scalars zero, so that the first step forms w = A u and its scalars
// from them (k_iter_a/k_iter_b with PCG); inside the graph it lets the WHILE node run.
__global__ void __launch_bounds__(kFirstThreads) k_pcg_first(IterArgs A) {
  for (int o = threadIdx.x; o < A.nw * 3; o += kFirstThreads) {
    A.mu[o] = 0.0;
    A.cu[o] = A.S.apol[(o / 3) % A.np] * A.e0[o];
    A.cw[o] = 0.0;
    A.cs[o] = 0.0;
    A.cp[o] = 0.0;
  }
  if (threadIdx.x == 0) {
    for (int k = 0; k < kIterStateLen; k++) A.state[k] = 0.0;
    if (A.maxit < 1) A.state[kIterFinished] = 1.0;
    if (A.use_graph) cudaGraphSetConditional(A.handle, A.maxit >= 1 ? 1u : 0u);
  }
}

}  // namespace

cudaError_t launch_dip_first(const IterArgs &A, cudaStream_t st) {
  k_dip_first<<<1, kFirstThreads, 0, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_pcg_first(const IterArgs &A, cudaStream_t st) {
  k_pcg_first<<<1, kFirstThreads, 0, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_phase_factors(const double2 *tab, int nm, SiteSets S, int kl, int km, int kn,
                                 double2 *XY, double2 *Z, cudaStream_t st) {
  int k1 = kl > km ? kl : km;
  k1 = (k1 > kn ? k1 : kn) + 1;
  if (k1 < 2) k1 = 2;
  const size_t total = (size_t)nm * S.np * ((size_t)(kl + 1) * (2 * km + 1) + 2 * kn + 1);
  if (total == 0) return cudaSuccess;
  size_t blocks = (total + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_phase_factors<<<(unsigned)blocks, 256, 0, st>>>(tab, nm, S, k1, kl, km, kn, XY, Z);
  return cudaGetLastError();
}

cudaError_t launch_tmu(const int *nbr, const int *ncnt, int cap, int nm, int np, const double4 *T4,
                       const double *TB, const double4 *S4, const double *SB, const double *mu,
                       double *eim, cudaStream_t st) {
  const int nw = nm * np;
  k_tmu<<<(nw + kWarps - 1) / kWarps, kThreads, 0, st>>>(nbr, ncnt, cap, nw, np, T4, TB, S4, SB,
                                                         mu, eim);
  return cudaGetLastError();
}

// Launches a step kernel, with programmatic stream serialization when A.pdl is set.
template <typename Kernel>
cudaError_t launch_step(Kernel kernel, int blocks, const IterArgs &A, cudaStream_t st,
                        size_t smem = 0, int threads = kThreads) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = A.pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, A);
}

// Dynamic shared memory of the row form's two kernels; the row form runs only where both fit
// the default 48 KB per block (less the static arrays).
size_t iter_rows_smem_a(int sum_sites, int row_span) {
  return sizeof(double4) * (size_t)sum_sites +
         sizeof(double2) * (size_t)sum_sites * (kRowTile + 1 + row_span);
}
size_t iter_rows_smem_b(int nz, int row_span) {
  return sizeof(double2) * ((size_t)nz * kRowSites + (nz + 1) / 2 +
                            (size_t)kRowWarps * 32 / kRowSites * kRowR * row_span);
}
bool iter_rows_fit(int sum_sites, int nz, int row_span) {
  constexpr size_t kDefault = 48 * 1024 - 2048;  // room for the static shared arrays
  return iter_rows_smem_a(sum_sites, row_span) <= kDefault &&
         iter_rows_smem_b(nz, row_span) <= kDefault;
}

template <int J>
cudaError_t launch_iter_a_rows(const IterArgs &A, int nb, size_t smem, cudaStream_t st) {
  return A.cu ? launch_step(k_iter_a_rows<true, J>, nb, A, st, smem)
              : launch_step(k_iter_a_rows<false, J>, nb, A, st, smem);
}

cudaError_t launch_iter_a(const IterArgs &A, cudaStream_t st) {
  if (A.sum_sites < 1 || A.sum_sites > kSumSitesMax) return cudaErrorInvalidValue;
  const int nA = (A.nw + kWarps - 1) / kWarps;
  const int nsc = (A.nw + A.sum_sites - 1) / A.sum_sites;
  if (A.rows) {
    if (!iter_rows_fit(A.sum_sites, A.nz, A.row_span)) return cudaErrorInvalidValue;
    const int ntile = (A.nrow + kRowTile - 1) / kRowTile;
    const size_t smem = iter_rows_smem_a(A.sum_sites, A.row_span);
    const int nb = nA + ntile * nsc;
    const int j = (A.row_span + kRowLanes - 1) / kRowLanes;
    if (j <= 2) return launch_iter_a_rows<2>(A, nb, smem, st);
    if (j <= 4) return launch_iter_a_rows<4>(A, nb, smem, st);
    if (j <= 8) return launch_iter_a_rows<8>(A, nb, smem, st);
    return cudaErrorInvalidValue;
  }
  const size_t smem = sizeof(double) * 3 * A.sum_sites;
  const int nkt = (A.nk + kThreads - 1) / kThreads;
  const int nb = nA + nkt * nsc;
  if (A.PM)
    return A.cu ? launch_step(k_iter_a<true, true>, nb, A, st, smem)
                : launch_step(k_iter_a<false, true>, nb, A, st, smem);
  return A.cu ? launch_step(k_iter_a<true, false>, nb, A, st, smem)
              : launch_step(k_iter_a<false, false>, nb, A, st, smem);
}

template <int GS>
cudaError_t launch_iter_b_gs(const IterArgs &A, cudaStream_t st) {
  const int nb = (A.nw + GS - 1) / GS;
  constexpr int T = kGatherThreads;
  if (A.PM)
    return A.cu ? launch_step(k_iter_b<true, true, GS>, nb, A, st, 0, T)
                : launch_step(k_iter_b<false, true, GS>, nb, A, st, 0, T);
  return A.cu ? launch_step(k_iter_b<true, false, GS>, nb, A, st, 0, T)
              : launch_step(k_iter_b<false, false, GS>, nb, A, st, 0, T);
}

cudaError_t launch_iter_b(const IterArgs &A, cudaStream_t st) {
  if (A.rows) {
    if (!iter_rows_fit(A.sum_sites, A.nz, A.row_span)) return cudaErrorInvalidValue;
    const int nb = (A.nw + kRowSites - 1) / kRowSites;
    const size_t smem = iter_rows_smem_b(A.nz, A.row_span);
    return A.cu ? launch_step(k_iter_b_rows<true>, nb, A, st, smem, kRowWarps * 32)
                : launch_step(k_iter_b_rows<false>, nb, A, st, smem, kRowWarps * 32);
  }
  switch (A.gather_sites) {
    case 2: return launch_iter_b_gs<2>(A, st);
    case 3: return launch_iter_b_gs<3>(A, st);
    case 4: return launch_iter_b_gs<4>(A, st);
    case 6: return launch_iter_b_gs<6>(A, st);
    case 8: return launch_iter_b_gs<8>(A, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_phase_rows(const double2 *tab, int nm, SiteSets S, int kl, int km, int kn,
                              const KRow *rows, int nrow, double2 *XYr, double2 *Z,
                              double2 *ZT, cudaStream_t st) {
  int k1 = kl > km ? kl : km;
  k1 = (k1 > kn ? k1 : kn) + 1;
  if (k1 < 2) k1 = 2;
  const size_t total = (size_t)nm * S.np * ((size_t)nrow + 2 * kn + 1);
  if (total == 0) return cudaSuccess;
  size_t blocks = (total + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_phase_rows<<<(unsigned)blocks, 256, 0, st>>>(tab, nm, S, k1, km, kn, rows, nrow, XYr, Z, ZT);
  return cudaGetLastError();
}

cudaError_t launch_phase_matrix(const KGather *kg, int nk, int nw, int nlm, int nz,
                                const double2 *XY, const double2 *Z, double2 *PM,
                                cudaStream_t st) {
  if (nk <= 0 || nw <= 0) return cudaSuccess;
  const dim3 grid((nk + 127) / 128, nw < 1024 ? nw : 1024);
  k_phase_matrix<<<grid, 128, 0, st>>>(kg, nk, nw, nlm, nz, XY, Z, PM);
  return cudaGetLastError();
}
