// k_kspace.cu -- reciprocal-space Ewald sums of the hot path (sm_100a, FP64).
//
// Per-site phase tables exp(i 2 pi l x / L), l = 0..kmax, per axis, are built with the
// reference's angle-addition recurrence (ewald.f90:882-917).  Both reciprocal-space passes
// are tiled over (64 k-vectors) x (64 sites) per block, with the sites' tables and the
// k-vectors staged in shared memory, so every launch has ~(nk/64)(nsites/64) blocks:
//   structure factors  S(k) = sum_s w_s(k) exp(i k.r_s)       (atomic merge over site tiles)
//   gathers            X(s) = sum_k g(k, s) k                   (atomic merge over k tiles)
// Modes (the weights w and gather g of each reference routine):
//   0  kspace_ewald         (ewald.f90:754-1173)               charges -> charge forces
//   1  kspace_efield_stat   (nb_induction_model.f90:597-975)   charges -> field at pol. sites
//   2  kspace_efield_idm    (nb_induction_model.f90:2263-2660) dipoles -> field at pol. sites
//   3  kspace_forces        (nb_induction_model.f90:4171-4839) q + mu  -> forces, active sites
#include "ccp_device.cuh"

using namespace ccpd;

namespace {

constexpr int kKT = 64;     // k-vectors per tile
constexpr int kST = 64;     // sites per tile
constexpr int kThreads = 256;
constexpr int kParts = kThreads / kST;  // gathers: warps over a site tile, each a k quarter
constexpr int kSumLanes = 2 * kThreads / kKT;  // sums: lanes over the sites of one k-vector
static_assert(kSumLanes == 8 && kParts * kST == kThreads, "tile shapes");

__global__ void k_ktab(const double4 *__restrict__ com, const double4 *__restrict__ act, int nm,
                       int na, double box, int k1, double2 *tab) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = nm * na;
  if (t >= N) return;
  const int i = t / na;
  const double4 c = com[i];
  const double4 s = act[t];
  const double twopi = 2.0 * kPi;
  const double p[3] = {c.x + s.x, c.y + s.y, c.z + s.z};
  for (int a = 0; a < 3; a++) {
    double2 *T = tab + (size_t)a * k1 * N;
    double c1, s1;
    sincos(twopi * p[a] / box, &s1, &c1);
    T[t] = make_double2(1.0, 0.0);
    T[(size_t)N + t] = make_double2(c1, s1);
    double cp = c1, sp = s1;
    for (int l = 2; l < k1; l++) {
      const double cn = cp * c1 - sp * s1;
      const double sn = sp * c1 + cp * s1;
      T[(size_t)l * N + t] = make_double2(cn, sn);
      cp = cn;
      sp = sn;
    }
  }
}

// source / target sites of a mode, as slots of the active-site list
__device__ __forceinline__ int src_count(int mode, const SiteSets &S) {
  return mode <= 1 ? S.nq : (mode == 2 ? S.np : S.na);
}
__device__ __forceinline__ int src_slot(int mode, const SiteSets &S, int r) {
  return mode <= 1 ? S.a_of_q[r] : (mode == 2 ? S.a_of_p[r] : r);
}
__device__ __forceinline__ int tgt_count(int mode, const SiteSets &S) {
  return mode == 0 ? S.nq : (mode == 3 ? S.na : S.np);
}
__device__ __forceinline__ int tgt_slot(int mode, const SiteSets &S, int r) {
  return mode == 0 ? S.a_of_q[r] : (mode == 3 ? r : S.a_of_p[r]);
}

// exp(i k.r) of the staged site `ls` (tables [axis][l][site] in shared memory), in the
// reference's product order: exp(i(l x + m y)) first (phase_lm), then times exp(i n z)
// (phase_n), so that k-vectors of one (l, m) can share the first product.
__device__ __forceinline__ double2 phase_lm(const double2 *__restrict__ T, int k1, int ls, int l,
                                            int m) {
  const double2 el = T[(0 * k1 + l) * kST + ls];
  const double2 em = T[(1 * k1 + (m < 0 ? -m : m)) * kST + ls];
  if (m >= 0) return make_double2(el.x * em.x - el.y * em.y, el.y * em.x + em.y * el.x);
  return make_double2(el.x * em.x + el.y * em.y, el.y * em.x - em.y * el.x);
}
__device__ __forceinline__ void phase_n(const double2 *__restrict__ T, int k1, int ls,
                                        double2 lm, int n, double &c, double &s) {
  const double2 en = T[(2 * k1 + (n < 0 ? -n : n)) * kST + ls];
  const double clm = lm.x, slm = lm.y;
  if (n >= 0) {
    c = clm * en.x - slm * en.y;
    s = slm * en.x + clm * en.y;
  } else {
    c = clm * en.x + slm * en.y;
    s = slm * en.x - clm * en.y;
  }
}

// Stage the tables and (mu, q) of a tile of sites; returns the tile's site count.
template <bool WANT_MU>
__device__ __forceinline__ int stage_sites(int mode, bool source, const double2 *__restrict__ tab,
                                           int nm, const SiteSets &S, int k1,
                                           const double *__restrict__ mu, int s0, double2 *T,
                                           double4 *W) {
  const int per = source ? src_count(mode, S) : tgt_count(mode, S);
  const int total = nm * per;
  const int cnt = min(kST, total - s0);
  const int N = nm * S.na;
  for (int u = threadIdx.x; u < 3 * k1 * kST; u += blockDim.x) {
    const int row = u / kST, ls = u % kST;
    if (ls < cnt) {
      const int g = s0 + ls, i = g / per, r = g % per;
      const int a = source ? src_slot(mode, S, r) : tgt_slot(mode, S, r);
      T[u] = tab[(size_t)row * N + i * S.na + a];
    }
  }
  for (int ls = threadIdx.x; ls < kST; ls += blockDim.x) {
    double4 w = make_double4(0.0, 0.0, 0.0, 0.0);
    if (ls < cnt) {
      const int g = s0 + ls, i = g / per, r = g % per;
      const int a = source ? src_slot(mode, S, r) : tgt_slot(mode, S, r);
      w.w = S.q[a];
      const int p = S.p_of_a[a];
      if (WANT_MU && p >= 0) {
        w.x = mu[((size_t)i * S.np + p) * 3 + 0];
        w.y = mu[((size_t)i * S.np + p) * 3 + 1];
        w.z = mu[((size_t)i * S.np + p) * 3 + 2];
      }
    }
    W[ls] = w;
  }
  return cnt;
}

template <int MODE>
__global__ void __launch_bounds__(kThreads)
    k_ksums(const KVec *__restrict__ kv, int nk, const double2 *__restrict__ tab, int nm,
            SiteSets S, int k1, const double *__restrict__ mu, double *sk) {
  extern __shared__ __align__(16) unsigned char raw[];
  double2 *T = reinterpret_cast<double2 *>(raw);
  double4 *W = reinterpret_cast<double4 *>(T + 3 * k1 * kST);
  KVec *K = reinterpret_cast<KVec *>(W + kST);
  const int k0 = blockIdx.x * kKT, s0 = blockIdx.y * kST;
  const int cnt = stage_sites<MODE >= 2>(MODE, true, tab, nm, S, k1, mu, s0, T, W);
  for (int u = threadIdx.x; u < kKT; u += blockDim.x)
    if (k0 + u < nk) K[u] = kv[k0 + u];
  __syncthreads();
  // kSumLanes lanes per k-vector over the sites, each thread two k-vectors (kk and kk +
  // kKT / 2): a quarter-warp reads one table row at consecutive sites, and the site weights
  // are loaded once for both k-vectors.  (Adjacent k-vectors sharing exp(i(l x + m y)) here
  // cost registers and occupancy: k_ksums<3> took 548 against 443 us at 2048 waters.)
  const int kk = threadIdx.x / kSumLanes, part = threadIdx.x % kSumLanes;
  double a[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
  const bool on0 = k0 + kk < nk, on1 = k0 + kk + kKT / 2 < nk;
  if (on0) {
    const KVec ka = K[kk], kb = on1 ? K[kk + kKT / 2] : K[kk];
    for (int ls = part; ls < cnt; ls += kSumLanes) {
      const double4 w = W[ls];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const KVec &k = h == 0 ? ka : kb;
        double c, s;
        phase_n(T, k1, ls, phase_lm(T, k1, ls, k.l, k.m), k.n, c, s);
        if (MODE <= 1) {
          a[h][0] += w.w * c;
          a[h][1] += w.w * s;
        } else {
          const double dk = k.rl * w.x + k.rm * w.y + k.rn * w.z;
          if (MODE == 2) {
            a[h][0] += dk * c;
            a[h][1] += dk * s;
          } else {
            a[h][0] += w.w * c;
            a[h][1] += w.w * s;
            a[h][2] += dk * c;
            a[h][3] += dk * s;
          }
        }
      }
    }
  }
#pragma unroll
  for (int h = 0; h < 2; h++)
#pragma unroll
    for (int off = 1; off < kSumLanes; off <<= 1)
#pragma unroll
      for (int c = 0; c < (MODE == 3 ? 4 : 2); c++)
        a[h][c] += __shfl_xor_sync(0xffffffffu, a[h][c], off);
  if (part == 0) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (h == 0 ? !on0 : !on1) continue;
      double *o = sk + (size_t)(k0 + kk + h * (kKT / 2)) * 4;
      atomicAdd(o, a[h][0]);
      atomicAdd(o + 1, a[h][1]);
      if (MODE == 3) {
        atomicAdd(o + 2, a[h][2]);
        atomicAdd(o + 3, a[h][3]);
      }
    }
  }
}

// Energy and virial of the Ewald (MODE 0) or induction-force (MODE 3) reciprocal sums,
// per k (ewald.f90:1043-1045; nb_induction_model.f90:4579-4581).
template <int MODE>
__global__ void k_kenergy(const KVec *__restrict__ kv, int nk, const double *__restrict__ sk,
                          double alpha, double *scal) {
  double e = 0.0, vir = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += gridDim.x * blockDim.x) {
    const KVec K = kv[k];
    const double *A = sk + (size_t)k * 4;
    const double rksq = K.rl * K.rl + K.rm * K.rm + K.rn * K.rn;
    const double fac = 1.0 - 0.5 * rksq / (alpha * alpha);
    if (MODE == 0) {
      const double s2 = A[0] * A[0] + A[1] * A[1];
      e += K.ak * s2;
      vir -= fac * K.ak * s2;
    } else {
      const double x1 = A[2] * A[1] - A[3] * A[0], x2 = A[2] * A[2] + A[3] * A[3];
      vir -= 2.0 * K.ak * (x1 + x2 + 0.5 * (2.0 * x1 + x2) * fac);
    }
  }
  e = warp_sum(e);
  vir = warp_sum(vir);
  if ((threadIdx.x & 31) == 0) {
    if (MODE == 0) {
      atomicAdd(&scal[S_KC_E], e);
      atomicAdd(&scal[S_KC_VIR], vir);
    } else {
      atomicAdd(&scal[S_IND_VIR_K], vir);
    }
  }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads)
    k_kgather(const KVec *__restrict__ kv, int nk, const double2 *__restrict__ tab, int nm,
              SiteSets S, int k1, const double *__restrict__ mu, const double *__restrict__ sk,
              double *out, double *f) {
  extern __shared__ __align__(16) unsigned char raw[];
  double2 *T = reinterpret_cast<double2 *>(raw);
  double4 *W = reinterpret_cast<double4 *>(T + 3 * k1 * kST);
  KVec *K = reinterpret_cast<KVec *>(W + kST);
  double4 *A = reinterpret_cast<double4 *>(K + kKT);
  const int k0 = blockIdx.x * kKT, s0 = blockIdx.y * kST;
  const int cnt = stage_sites<MODE == 3>(MODE, false, tab, nm, S, k1, mu, s0, T, W);
  const int nkt = min(kKT, nk - k0);
  // each k-vector's gather weights, the mode's factor times its sums, so that a (site, k)
  // pair's weight g is two or four products of the phase (cos, sin):
  //   0: g = q (s W0 + c W1), W = 4 r4pie0 a(k) (S_re, -S_im)
  //   1: g = s W0 + c W1,     W = 4 a(k) (S_re, -S_im)
  //   2: g = c W0 + s W1,     W = -4 a(k) (S_re, S_im)
  //   3: g = q (c W0 + s W1) + (mu.k)(c W2 + s W3), with f = -4 a(k) and the charge and dipole
  //      sums (S, D): W = (f D_re, f D_im, f (D_im - S_re), -f (S_im + D_re))
  // (nb_induction_model.f90:4171-4839 for mode 3: mufac, qfac and mufaci regrouped)
  for (int u = threadIdx.x; u < nkt; u += blockDim.x) {
    const KVec kq = kv[k0 + u];
    K[u] = kq;
    const double *s = sk + (size_t)(k0 + u) * 4;
    if (MODE == 0) {
      const double f = 4.0 * kR4pie0 * kq.ak;
      A[u] = make_double4(f * s[0], -f * s[1], 0.0, 0.0);
    } else if (MODE == 1) {
      const double f = 4.0 * kq.ak;
      A[u] = make_double4(f * s[0], -f * s[1], 0.0, 0.0);
    } else if (MODE == 2) {
      const double f = -4.0 * kq.ak;
      A[u] = make_double4(f * s[0], f * s[1], 0.0, 0.0);
    } else {
      const double f = -4.0 * kq.ak;
      A[u] = make_double4(f * s[2], f * s[3], f * (s[3] - s[0]), -f * (s[1] + s[2]));
    }
  }
  __syncthreads();
  // site-major lanes: a warp takes 32 consecutive sites of the tile and one contiguous
  // quarter of its k-vectors, so its table loads are contiguous rows, its k-vector loads
  // broadcasts, and consecutive k-vectors of one (l, m) share exp(i(l x + m y))
  const int ls = threadIdx.x % kST, part = threadIdx.x / kST;
  double ax = 0.0, ay = 0.0, az = 0.0;
  if (ls < cnt) {
    const double4 w = W[ls];
    const double q = w.w;
    const int ub = part * (kKT / kParts), ue = min(ub + kKT / kParts, nkt);
    int pl = -1, pm = 0;
    double2 lm = make_double2(0.0, 0.0);
    for (int u = ub; u < ue; u++) {
      const KVec k = K[u];
      const double4 a = A[u];
      if (k.l != pl || k.m != pm) {  // warp-uniform: the warp's lanes share u
        lm = phase_lm(T, k1, ls, k.l, k.m);
        pl = k.l;
        pm = k.m;
      }
      double c, s;
      phase_n(T, k1, ls, lm, k.n, c, s);
      double g;
      if (MODE == 0) {
        g = q * (s * a.x + c * a.y);
      } else if (MODE == 1) {
        g = s * a.x + c * a.y;
      } else if (MODE == 2) {
        g = c * a.x + s * a.y;
      } else {
        const double mk = w.x * k.rl + w.y * k.rm + w.z * k.rn;
        g = q * (c * a.x + s * a.y) + mk * (c * a.z + s * a.w);
      }
      ax += k.rl * g;
      ay += k.rm * g;
      az += k.rn * g;
    }
  }
  // the quarters' partial sums of each site, added in shared memory
  double *red = reinterpret_cast<double *>(A + kKT);
  red[(part * 3 + 0) * kST + ls] = ax;
  red[(part * 3 + 1) * kST + ls] = ay;
  red[(part * 3 + 2) * kST + ls] = az;
  __syncthreads();
  if (part == 0) {
    for (int p = 1; p < kParts; p++) {
      ax += red[(p * 3 + 0) * kST + ls];
      ay += red[(p * 3 + 1) * kST + ls];
      az += red[(p * 3 + 2) * kST + ls];
    }
  }
  if (part == 0 && ls < cnt) {
    const int per = tgt_count(MODE, S);
    const int g = s0 + ls, i = g / per, r = g % per;
    if (MODE == 0 || MODE == 3) {
      const double sc = MODE == 3 ? kR4pie0 : 1.0;
      const int a = tgt_slot(MODE, S, r);
      const size_t nfs = (size_t)nm * S.ns;
      const size_t o = (size_t)i * S.ns + S.asite[a];
      atomicAdd(&f[o], sc * ax);
      atomicAdd(&f[nfs + o], sc * ay);
      atomicAdd(&f[2 * nfs + o], sc * az);
    } else {
      const size_t o = ((size_t)i * S.np + r) * 3;
      atomicAdd(&out[o], ax);
      atomicAdd(&out[o + 1], ay);
      atomicAdd(&out[o + 2], az);
    }
  }
}

// Jacobi update of every polarisable site (nb_induction_model.f90:1317-1359):
//   Eidm = (real + short-range + self part) + reciprocal part,  Et = Eidm + E0,
//   mu' = alpha Et,  change += |mu - mu'|^2,  energy += -1/2 alpha Et.E0.
__global__ void k_dip_update(int n, SiteSets S, const double *__restrict__ e0,
                             const double *__restrict__ eim, const double *__restrict__ ek,
                             const double *__restrict__ mu, double *mu_out, double *scal) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double ch = 0.0, en = 0.0;
  if (t < n) {
    const double polr = S.apol[t % S.np];
    double Et[3], E0[3];
    for (int c = 0; c < 3; c++) {
      const size_t o = (size_t)t * 3 + c;
      E0[c] = e0[o];
      Et[c] = (eim[o] + ek[o]) + E0[c];
      const double m = polr * Et[c];
      const double d = mu[o] - m;
      ch += d * d;
      mu_out[o] = m;
    }
    en = -0.5 * polr * (Et[0] * E0[0] + Et[1] * E0[1] + Et[2] * E0[2]);
  }
  __shared__ double red[2][8];
  ch = warp_sum(ch);
  en = warp_sum(en);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][wid] = ch;
    red[1][wid] = en;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double c2 = 0.0, e2 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      c2 += red[0][w];
      e2 += red[1][w];
    }
    atomicAdd(&scal[S_IND_CHANGE], c2);
    atomicAdd(&scal[S_IND_ENERGY], e2);
  }
}

inline int k1_of(int kl, int km, int kn) {
  int k1 = kl > km ? kl : km;
  k1 = (k1 > kn ? k1 : kn) + 1;
  return k1 < 2 ? 2 : k1;
}

inline size_t tile_smem(int k1, bool gather) {
  return sizeof(double2) * 3 * (size_t)k1 * kST + sizeof(double4) * kST + sizeof(KVec) * kKT +
         (gather ? sizeof(double4) * kKT + sizeof(double) * 3 * kParts * kST : 0);
}

template <typename F>
cudaError_t set_smem(F kern, size_t smem) {
  if (smem > 48 * 1024)
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return cudaSuccess;
}

}  // namespace

cudaError_t launch_ktab(const double4 *com, const double4 *act, int nm, SiteSets S,
                        double box, int kl, int km, int kn, double2 *tab, cudaStream_t st) {
  const int k1 = k1_of(kl, km, kn);
  const int N = nm * S.na;
  k_ktab<<<(N + 127) / 128, 128, 0, st>>>(com, act, nm, S.na, box, k1, tab);
  return cudaGetLastError();
}

cudaError_t launch_kspace_sums(int mode, const KVec *kv, int nk, const double2 *tab, int nm,
                               SiteSets S, int kl, int km, int kn, const double *mu,
                               double *sk, cudaStream_t st) {
  if (nk <= 0) return cudaSuccess;
  const int k1 = k1_of(kl, km, kn);
  const int per = mode <= 1 ? S.nq : (mode == 2 ? S.np : S.na);
  const dim3 grid((nk + kKT - 1) / kKT, (nm * per + kST - 1) / kST);
  const size_t smem = tile_smem(k1, false);
  cudaError_t e = cudaMemsetAsync(sk, 0, sizeof(double) * 4 * (size_t)nk, st);
  if (e != cudaSuccess) return e;
  switch (mode) {
    case 0:
      if ((e = set_smem(k_ksums<0>, smem)) != cudaSuccess) return e;
      k_ksums<0><<<grid, kThreads, smem, st>>>(kv, nk, tab, nm, S, k1, mu, sk);
      break;
    case 1:
      if ((e = set_smem(k_ksums<1>, smem)) != cudaSuccess) return e;
      k_ksums<1><<<grid, kThreads, smem, st>>>(kv, nk, tab, nm, S, k1, mu, sk);
      break;
    case 2:
      if ((e = set_smem(k_ksums<2>, smem)) != cudaSuccess) return e;
      k_ksums<2><<<grid, kThreads, smem, st>>>(kv, nk, tab, nm, S, k1, mu, sk);
      break;
    default:
      if ((e = set_smem(k_ksums<3>, smem)) != cudaSuccess) return e;
      k_ksums<3><<<grid, kThreads, smem, st>>>(kv, nk, tab, nm, S, k1, mu, sk);
      break;
  }
  return cudaGetLastError();
}

cudaError_t launch_kspace_energy(int mode, const KVec *kv, int nk, const double *sk,
                                 double alpha, double *scal, cudaStream_t st) {
  if (nk <= 0) return cudaSuccess;
  const int blocks = (nk + 255) / 256 < 64 ? (nk + 255) / 256 : 64;
  if (mode == 0)
    k_kenergy<0><<<blocks, 256, 0, st>>>(kv, nk, sk, alpha, scal);
  else
    k_kenergy<3><<<blocks, 256, 0, st>>>(kv, nk, sk, alpha, scal);
  return cudaGetLastError();
}

cudaError_t launch_kspace_gather(int mode, const KVec *kv, int nk, const double2 *tab, int nm,
                                 SiteSets S, int kl, int km, int kn, const double *mu,
                                 const double *sk, double *out, double *f, cudaStream_t st) {
  if (nk <= 0) return cudaSuccess;
  const int k1 = k1_of(kl, km, kn);
  const int per_t = mode == 0 ? S.nq : (mode == 3 ? S.na : S.np);
  const dim3 grid((nk + kKT - 1) / kKT, (nm * per_t + kST - 1) / kST);
  const size_t smem = tile_smem(k1, true);
  cudaError_t e;
  if (mode == 1 || mode == 2) {
    e = cudaMemsetAsync(out, 0, sizeof(double) * 3 * (size_t)nm * S.np, st);
    if (e != cudaSuccess) return e;
  }
  switch (mode) {
    case 0:
      if ((e = set_smem(k_kgather<0>, smem)) != cudaSuccess) return e;
      k_kgather<0><<<grid, kThreads, smem, st>>>(kv, nk, tab, nm, S, k1, mu, sk, out, f);
      break;
    case 1:
      if ((e = set_smem(k_kgather<1>, smem)) != cudaSuccess) return e;
      k_kgather<1><<<grid, kThreads, smem, st>>>(kv, nk, tab, nm, S, k1, mu, sk, out, f);
      break;
    case 2:
      if ((e = set_smem(k_kgather<2>, smem)) != cudaSuccess) return e;
      k_kgather<2><<<grid, kThreads, smem, st>>>(kv, nk, tab, nm, S, k1, mu, sk, out, f);
      break;
    default:
      if ((e = set_smem(k_kgather<3>, smem)) != cudaSuccess) return e;
      k_kgather<3><<<grid, kThreads, smem, st>>>(kv, nk, tab, nm, S, k1, mu, sk, out, f);
      break;
  }
  return cudaGetLastError();
}

cudaError_t launch_dip_update(int nm, SiteSets S, const double *e0, const double *eim,
                              const double *ek, const double *mu, double *mu_out, double *scal,
                              cudaStream_t st) {
  const int n = nm * S.np;
  k_dip_update<<<(n + 255) / 256, 256, 0, st>>>(n, S, e0, eim, ek, mu, mu_out, scal);
  return cudaGetLastError();
}
