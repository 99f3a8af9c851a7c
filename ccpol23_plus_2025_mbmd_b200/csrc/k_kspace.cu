// k_kspace.cu -- reciprocal-space Ewald sums of the hot path (sm_100a, FP64).
//
// Per-site phase tables exp(i 2 pi l x / L), l = 0..kmax, per axis, are built with the
// reference's angle-addition recurrence (ewald.f90:882-917).  A structure-factor kernel
// then reduces, per block, the sums over all source sites for a tile of k-vectors; a gather
// kernel gives every target site its field / field gradient / force from all k-vectors
// staged through shared memory.  Modes:
//   0  kspace_ewald               (ewald.f90:754-1173)              charges -> charges
//   1  kspace_efield_stat          (nb_induction_model.f90:597-975)  charges -> pol. sites
//   2  kspace_efield_idm           (nb_induction_model.f90:2263-2660) dipoles -> pol. sites
//   3  kspace_forces               (nb_induction_model.f90:4171-4839) q + mu -> active sites
#include "ccp_device.cuh"

using namespace ccpd;

namespace {

constexpr int kKB = 8;       // k-vectors per structure-factor block
constexpr int kSumThreads = 256;

__global__ void k_ktab(const double4 *__restrict__ com, const double4 *__restrict__ act, int nm,
                       int na, double box, int kl, int km, int kn, int k1, double2 *tab) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = nm * na;
  if (t >= N) return;
  const int i = t / na;
  const double4 c = com[i];
  const double4 s = act[t];
  const double twopi = 2.0 * kPi;
  const double p[3] = {c.x + s.x, c.y + s.y, c.z + s.z};
  const int lim[3] = {kl, km, kn};
  for (int a = 0; a < 3; a++) {
    double2 *T = tab + (size_t)a * k1 * N;
    double c1, s1;
    sincos(twopi * p[a] / box, &s1, &c1);
    T[t] = make_double2(1.0, 0.0);
    T[(size_t)N + t] = make_double2(c1, s1);
    double cp = c1, sp = s1;
    for (int l = 2; l <= lim[a]; l++) {
      const double cn = cp * c1 - sp * s1;
      const double sn = sp * c1 + cp * s1;
      T[(size_t)l * N + t] = make_double2(cn, sn);
      cp = cn;
      sp = sn;
    }
  }
}

// exp(i k.r) of table site st from the per-axis tables, in the reference's product order.
__device__ __forceinline__ void expikr(const double2 *__restrict__ tab, int N, int k1, int st,
                                       int l, int m, int n, double &c, double &s) {
  const double2 el = __ldg(&tab[(size_t)l * N + st]);
  const double2 em = __ldg(&tab[((size_t)k1 + (m < 0 ? -m : m)) * N + st]);
  const double2 en = __ldg(&tab[((size_t)2 * k1 + (n < 0 ? -n : n)) * N + st]);
  double clm, slm;
  if (m >= 0) {
    clm = el.x * em.x - el.y * em.y;
    slm = el.y * em.x + em.y * el.x;
  } else {
    clm = el.x * em.x + el.y * em.y;
    slm = el.y * em.x - em.y * el.x;
  }
  if (n >= 0) {
    c = clm * en.x - slm * en.y;
    s = slm * en.x + clm * en.y;
  } else {
    c = clm * en.x + slm * en.y;
    s = slm * en.x - clm * en.y;
  }
}

// number and identity of the source / target sites of a mode
__device__ __forceinline__ int mode_count(int mode, const SiteSets &S) {
  return mode <= 1 ? S.nq : (mode == 2 ? S.np : S.na);
}
__device__ __forceinline__ int mode_slot(int mode, const SiteSets &S, int r) {
  return mode <= 1 ? S.a_of_q[r] : (mode == 2 ? S.a_of_p[r] : r);
}
// targets: charged sites (0), polarisable sites (1, 2), active sites (3)
__device__ __forceinline__ int target_count(int mode, const SiteSets &S) {
  return mode == 0 ? S.nq : (mode == 3 ? S.na : S.np);
}
__device__ __forceinline__ int target_slot(int mode, const SiteSets &S, int r) {
  return mode == 0 ? S.a_of_q[r] : (mode == 3 ? r : S.a_of_p[r]);
}

template <int MODE>
__global__ void __launch_bounds__(kSumThreads)
    k_ksums(const KVec *__restrict__ kv, int nk, const double2 *__restrict__ tab, int nm,
            SiteSets S, int k1, const double *__restrict__ mu, double *sk, double *scal,
            double alpha) {
  constexpr int NC = MODE == 3 ? 4 : 2;
  __shared__ KVec kk[kKB];
  __shared__ double red[kSumThreads / 32][kKB][NC];
  const int k0 = blockIdx.x * kKB;
  if (threadIdx.x < kKB && k0 + (int)threadIdx.x < nk) kk[threadIdx.x] = kv[k0 + threadIdx.x];
  __syncthreads();
  const int nkb = min(kKB, nk - k0);
  double acc[kKB][NC];
#pragma unroll
  for (int q = 0; q < kKB; q++)
#pragma unroll
    for (int c = 0; c < NC; c++) acc[q][c] = 0.0;
  const int per = mode_count(MODE, S);
  const int nsrc = nm * per;
  const int N = nm * S.na;
  for (int t = threadIdx.x; t < nsrc; t += blockDim.x) {
    const int i = t / per, r = t % per;
    const int a = mode_slot(MODE, S, r);
    const int st = i * S.na + a;
    const double q = S.q[a];
    double mx = 0.0, my = 0.0, mz = 0.0;
    if (MODE >= 2) {
      const int p = S.p_of_a[a];
      if (p >= 0) {
        mx = mu[((size_t)i * S.np + p) * 3 + 0];
        my = mu[((size_t)i * S.np + p) * 3 + 1];
        mz = mu[((size_t)i * S.np + p) * 3 + 2];
      }
    }
#pragma unroll
    for (int u = 0; u < kKB; u++) {
      if (u >= nkb) break;
      const KVec K = kk[u];
      double c, s;
      expikr(tab, N, k1, st, K.l, K.m, K.n, c, s);
      if (MODE <= 1) {
        acc[u][0] += q * c;
        acc[u][1] += q * s;
      } else {
        const double dk = K.rl * mx + K.rm * my + K.rn * mz;
        if (MODE == 2) {
          acc[u][0] += dk * c;
          acc[u][1] += dk * s;
        } else {
          acc[u][0] += q * c;
          acc[u][1] += q * s;
          acc[u][2] += dk * c;
          acc[u][3] += dk * s;
        }
      }
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int u = 0; u < kKB; u++)
#pragma unroll
    for (int c = 0; c < NC; c++) {
      const double v = warp_sum(acc[u][c]);
      if (lane == 0) red[wid][u][c] = v;
    }
  __syncthreads();
  if (threadIdx.x < kKB * NC) {
    const int u = threadIdx.x / NC, c = threadIdx.x % NC;
    double v = 0.0;
    for (int w = 0; w < kSumThreads / 32; w++) v += red[w][u][c];
    if (u < nkb) sk[(size_t)(k0 + u) * 4 + c] = v;
    red[0][u][c] = v;  // warp 0's slot is no longer read by anyone else
  }
  __syncthreads();
  if (threadIdx.x == 0 && (MODE == 0 || MODE == 3)) {
    double e = 0.0, vir = 0.0;
    for (int u = 0; u < nkb; u++) {
      const KVec K = kk[u];
      const double rksq = K.rl * K.rl + K.rm * K.rm + K.rn * K.rn;
      const double fac = 1.0 - 0.5 * rksq / (alpha * alpha);
      if (MODE == 0) {
        const double s2 = red[0][u][0] * red[0][u][0] + red[0][u][1] * red[0][u][1];
        e += K.ak * s2;
        vir -= fac * K.ak * s2;
      } else {
        const double cq = red[0][u][0], sq = red[0][u][1], cd = red[0][u][2], sd = red[0][u][3];
        const double x1 = cd * sq - sd * cq, x2 = cd * cd + sd * sd;
        vir -= 2.0 * K.ak * (x1 + x2 + 0.5 * (2.0 * x1 + x2) * fac);
      }
    }
    if (MODE == 0) {
      atomicAdd(&scal[S_KC_E], e);
      atomicAdd(&scal[S_KC_VIR], vir);
    } else {
      atomicAdd(&scal[S_IND_VIR_K], vir);
    }
  }
}

// One warp per target site: the site's phase tables (3 axes x k1 entries) are staged in
// shared memory, lanes stride over the k-vectors, and the warp reduces at the end.
// MODE 2 also performs the Jacobi update of that site (nb_induction_model.f90:1317-1359):
// E0 = r + k + self + short-range static fields, Eidm = real/short-range/self part (from the
// T.mu matvec) + this reciprocal part, mu <- alpha (E0 + Eidm), with the squared change
// and the energy -1/2 alpha (E0 + Eidm).E0 reduced into scal.
constexpr int kGatherWarps = 8;

template <int MODE>
__global__ void __launch_bounds__(kGatherWarps * 32)
    k_kgather(const KVec *__restrict__ kv, int nk, const double2 *__restrict__ tab, int nm,
              SiteSets S, int k1, const double *__restrict__ mu, const double *__restrict__ sk,
              double *out, double *f, const double *__restrict__ e0, const double *__restrict__ eim,
              double *mu_out, double *scal) {
  extern __shared__ double2 stab[];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int per = target_count(MODE, S);
  const int t = blockIdx.x * kGatherWarps + wl;
  const bool live = t < nm * per;
  double ch = 0.0, en = 0.0;
  if (live) {
    const int i = t / per, r = t % per;
    const int a = target_slot(MODE, S, r);
    const int st = i * S.na + a;
    const int N = nm * S.na;
    double2 *my = stab + (size_t)wl * 3 * k1;
    for (int u = lane; u < 3 * k1; u += 32) my[u] = tab[(size_t)u * N + st];
    __syncwarp();
    const double q = S.q[a];
    double mx = 0.0, my_ = 0.0, mz = 0.0;
    const int p = S.p_of_a[a];
    if (MODE == 3 && p >= 0) {
      mx = mu[((size_t)i * S.np + p) * 3 + 0];
      my_ = mu[((size_t)i * S.np + p) * 3 + 1];
      mz = mu[((size_t)i * S.np + p) * 3 + 2];
    }
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int k = lane; k < nk; k += 32) {
      const KVec K = kv[k];
      const double4 A = *reinterpret_cast<const double4 *>(sk + (size_t)k * 4);
      const double2 el = my[K.l];
      const double2 em = my[k1 + (K.m < 0 ? -K.m : K.m)];
      const double2 en = my[2 * k1 + (K.n < 0 ? -K.n : K.n)];
      double clm, slm, c, s;
      if (K.m >= 0) {
        clm = el.x * em.x - el.y * em.y;
        slm = el.y * em.x + em.y * el.x;
      } else {
        clm = el.x * em.x + el.y * em.y;
        slm = el.y * em.x - em.y * el.x;
      }
      if (K.n >= 0) {
        c = clm * en.x - slm * en.y;
        s = slm * en.x + clm * en.y;
      } else {
        c = clm * en.x + slm * en.y;
        s = slm * en.x - clm * en.y;
      }
      double g;
      if (MODE == 0) {
        g = 4.0 * kR4pie0 * K.ak * ((q * s) * A.x - (q * c) * A.y);
      } else if (MODE == 1) {
        g = 4.0 * K.ak * (s * A.x - c * A.y);
      } else if (MODE == 2) {
        g = -4.0 * K.ak * (c * A.x + s * A.y);
      } else {
        const double mufac = -4.0 * K.ak * (c * A.z + s * A.w);
        const double qfac = -4.0 * K.ak * (-c * A.x - s * A.y);
        const double mufaci = -4.0 * K.ak * (c * A.w - s * A.z);
        const double mk = mx * K.rl + my_ * K.rm + mz * K.rn;
        g = q * mufac + mk * (qfac + mufaci);
      }
      ax += K.rl * g;
      ay += K.rm * g;
      az += K.rn * g;
    }
    ax = warp_sum(ax);
    ay = warp_sum(ay);
    az = warp_sum(az);
    if (lane == 0) {
      if (MODE == 0 || MODE == 3) {
        const double sc = MODE == 3 ? kR4pie0 : 1.0;
        const size_t nfs = (size_t)nm * S.ns;
        const size_t o = (size_t)i * S.ns + S.asite[a];
        f[o] += sc * ax;
        f[nfs + o] += sc * ay;
        f[2 * nfs + o] += sc * az;
      } else if (MODE == 1) {
        const size_t o = ((size_t)i * S.np + r) * 3;
        out[o] = ax;
        out[o + 1] = ay;
        out[o + 2] = az;
      } else {
        const size_t o = ((size_t)i * S.np + r) * 3;
        const double kE[3] = {ax, ay, az};
        const double polr = S.apol[r];
        double Et[3], E0[3];
        for (int c3 = 0; c3 < 3; c3++) {
          E0[c3] = e0[o + c3];
          Et[c3] = (eim[o + c3] + kE[c3]) + E0[c3];
          const double m = polr * Et[c3];
          const double d = mu[o + c3] - m;
          ch += d * d;
          mu_out[o + c3] = m;
        }
        en = -0.5 * polr * (Et[0] * E0[0] + Et[1] * E0[1] + Et[2] * E0[2]);
      }
    }
  }
  if (MODE == 2) {
    __shared__ double red[2][kGatherWarps];
    if (lane == 0) {
      red[0][wl] = ch;
      red[1][wl] = en;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double c2 = 0.0, e2 = 0.0;
      for (int w = 0; w < kGatherWarps; w++) {
        c2 += red[0][w];
        e2 += red[1][w];
      }
      atomicAdd(&scal[S_IND_CHANGE], c2);
      atomicAdd(&scal[S_IND_ENERGY], e2);
    }
  }
}

}  // namespace

cudaError_t launch_ktab(const double4 *com, const double4 *act, int nm, SiteSets S,
                        double box, int kl, int km, int kn, double2 *tab, cudaStream_t st) {
  int k1 = kl > km ? kl : km;
  k1 = (k1 > kn ? k1 : kn) + 1;
  if (k1 < 2) k1 = 2;
  const int N = nm * S.na;
  k_ktab<<<(N + 127) / 128, 128, 0, st>>>(com, act, nm, S.na, box, kl, km, kn, k1, tab);
  return cudaGetLastError();
}

static inline int k1_of(int kl, int km, int kn) {
  int k1 = kl > km ? kl : km;
  k1 = (k1 > kn ? k1 : kn) + 1;
  return k1 < 2 ? 2 : k1;
}

cudaError_t launch_kspace_sums(int mode, const KVec *kv, int nk, const double2 *tab, int nm,
                                SiteSets S, int kl, int km, int kn, const double *mu,
                                double *sk, double *scal, double alpha, cudaStream_t st) {
  if (nk <= 0) return cudaSuccess;
  const int k1 = k1_of(kl, km, kn);
  const int blocks = (nk + kKB - 1) / kKB;
  switch (mode) {
    case 0: k_ksums<0><<<blocks, kSumThreads, 0, st>>>(kv, nk, tab, nm, S, k1, mu, sk, scal, alpha); break;
    case 1: k_ksums<1><<<blocks, kSumThreads, 0, st>>>(kv, nk, tab, nm, S, k1, mu, sk, scal, alpha); break;
    case 2: k_ksums<2><<<blocks, kSumThreads, 0, st>>>(kv, nk, tab, nm, S, k1, mu, sk, scal, alpha); break;
    default: k_ksums<3><<<blocks, kSumThreads, 0, st>>>(kv, nk, tab, nm, S, k1, mu, sk, scal, alpha); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_kspace_gather(int mode, const KVec *kv, int nk, const double2 *tab, int nm,
                                 SiteSets S, int kl, int km, int kn, const double *mu,
                                 const double *sk, double *out, double *f, const double *e0,
                                 const double *eim, double *mu_out, double *scal, cudaStream_t st) {
  const int k1 = k1_of(kl, km, kn);
  const int per_t = mode == 0 ? S.nq : (mode == 3 ? S.na : S.np);
  const int n = nm * per_t;
  const int blocks = (n + kGatherWarps - 1) / kGatherWarps;
  const size_t smem = sizeof(double2) * 3 * (size_t)k1 * kGatherWarps;
  const int th = kGatherWarps * 32;
  switch (mode) {
    case 0: k_kgather<0><<<blocks, th, smem, st>>>(kv, nk, tab, nm, S, k1, mu, sk, out, f, e0, eim, mu_out, scal); break;
    case 1: k_kgather<1><<<blocks, th, smem, st>>>(kv, nk, tab, nm, S, k1, mu, sk, out, f, e0, eim, mu_out, scal); break;
    case 2: k_kgather<2><<<blocks, th, smem, st>>>(kv, nk, tab, nm, S, k1, mu, sk, out, f, e0, eim, mu_out, scal); break;
    default: k_kgather<3><<<blocks, th, smem, st>>>(kv, nk, tab, nm, S, k1, mu, sk, out, f, e0, eim, mu_out, scal); break;
  }
  return cudaGetLastError();
}
