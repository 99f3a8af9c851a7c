// k_vdw.cu -- the ccpol23plus 2-body term (vdw_ccpol23plus.f90:174-477) on sm_100a, FP64.
//
// For every molecule pair with COM distance below rcut (the reference's exact minimum-image
// test, from the neighbour list) and every pair of sites whose names have a parameter row:
//   u = e^{-beta r} (c0 + c1 r + c2 r^2 + c3 r^3) / (1 + e^{-gamma (r - r0)})
//     + r4pie0 (f1(d1 r) - 1) q_a q_b / r
//     - f6(d6 r) c6 / r^6 - f8(d8 r) c8 / r^8 - f10(d10 r) c10 / r^10,
// f_n the Tang-Toennies damping, gamma = 20/bohr2a, r0 = 1.4 bohr2a.  Molecule i handles half
// of its neighbour pairs: the pair (i, j) goes to i when i < j and i + j is odd or i > j and
// i + j is even, so that every molecule has about half its neighbours (with j > i alone the
// low-numbered molecules carried twice the average and the launch ran in two waves); kSplit
// blocks share a molecule's pairs.  Warp w takes the sites js = w, w + 4, ... of j, lane = site is of i, so j's site
// forces are warp reductions (3 atomics per site) and i's accumulate in registers.  Each
// exponential is evaluated once and serves the damping and its derivative.
#include "ccp_device.cuh"

using namespace ccpd;

namespace {

constexpr int kThreads = 128;
// blocks per molecule: each takes every kSplit-th pair of the molecule's share, so that more
// warps are in flight (a molecule's pairs are independent; its site forces are added
// atomically)
#ifndef CCP_VDW_SPLIT
#define CCP_VDW_SPLIT 4
#endif
constexpr int kSplit = CCP_VDW_SPLIT;
constexpr int kWarps = kThreads / 32;

// Tang-Toennies f_N(delta r) and its derivative (utility.f90:89-125) from one exponential.
// The series' divisions by i are products with the reciprocals 1/i (compile-time constants):
// FP64 divisions would dominate the kernel.
template <int N>
__device__ __forceinline__ void tt_both(double delta, double r, double &f, double &df) {
  const double dr = delta * r, ex = exp(-dr);
  double term = 1.0, sum = 1.0;
#pragma unroll
  for (int i = 1; i <= N; i++) {
    term = term * dr * (1.0 / (double)i);
    sum += term;
  }
  f = 1.0 - ex * sum;
  df = delta * ex * term;  // term = (delta r)^N / N!
}

__global__ void __launch_bounds__(kThreads)
    k_vdw(const double *__restrict__ xs, const double *__restrict__ ys,
          const double *__restrict__ zs, int ld, const int *__restrict__ nbr,
          const double4 *__restrict__ nbrv, const int *__restrict__ ncnt, int cap, int ns,
          double rcutsd, const int *__restrict__ row, const double *__restrict__ qq,
          const double *__restrict__ par, int nrows, const int *__restrict__ vsite, int nv,
          double *f, double *scal, int nm) {
  __shared__ double P[kVdwMaxRows * kVdwPar];
  __shared__ double fi[kWarps][32][3];
  __shared__ double red[2][kWarps];
  const int i = blockIdx.x / kSplit, part = blockIdx.x % kSplit;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int u = threadIdx.x; u < nrows * kVdwPar; u += kThreads) P[u] = par[u];
  __syncthreads();
  const double gamma = 20.0 / kBohr2a, sqr0 = 1.4 * kBohr2a;
  const bool lact = lane < nv;
  const int is = lact ? vsite[lane] : 0;
  const size_t oi = (size_t)i * ld + is;
  const double sxi = lact ? xs[oi] : 0.0, syi = lact ? ys[oi] : 0.0, szi = lact ? zs[oi] : 0.0;
  double fx = 0.0, fy = 0.0, fz = 0.0, e = 0.0, v = 0.0;
  const int cnt = ncnt[i];
  const size_t nfs = (size_t)nm * ns;
  for (int n = part; n < cnt; n += kSplit) {
    const int j = nbr[(size_t)i * cap + n];
    if (j == i || (j > i) != (((i + j) & 1) != 0)) continue;  // the pair is j's
    const double4 c = nbrv[(size_t)i * cap + n];
    if (!(c.w < rcutsd)) continue;
    for (int jv = wid; jv < nv; jv += kWarps) {
      const int js = vsite[jv];
      const size_t oj = (size_t)j * ld + js;
      const double sxj = xs[oj], syj = ys[oj], szj = zs[oj];
      double gx = 0.0, gy = 0.0, gz = 0.0;
      const int k = lact ? row[is * ns + js] : -1;
      if (k >= 0) {
        const double *p = P + k * kVdwPar;
        const double beta = p[0], c0 = p[1], c1 = p[2], c2 = p[3], c3 = p[4];
        const double c6 = p[5], c8 = p[6], c10 = p[7], d1 = p[8], d6 = p[9], d8 = p[10],
                     d10 = p[11];
        const double rsx = c.x + sxi - sxj, rsy = c.y + syi - syj, rsz = c.z + szi - szj;
        const double rssq = rsx * rsx + rsy * rsy + rsz * rsz;
        const double sqr = sqrt(rssq);
        const double ir = 1.0 / sqr, ir2 = ir * ir;  // one division serves every 1/r^n
        // exchange-repulsion with the short-range damping
        const double eks = exp(-beta * sqr);
        const double poly = c0 + c1 * sqr + c2 * sqr * sqr + c3 * sqr * sqr * sqr;
        const double eg = exp(-gamma * (sqr - sqr0));
        const double fdamp = 1.0 / (1.0 + eg);
        const double u_exp = eks * poly * fdamp;
        const double du_exp = -beta * u_exp * fdamp +
                              eks * fdamp * (c1 + 2.0 * c2 * sqr + 3.0 * c3 * sqr * sqr) +
                              gamma * eg * fdamp * fdamp * u_exp;
        double u = u_exp, du = du_exp;
        // short-range Coulomb correction; q_a q_b of the site pair
        const double qab = qq[is * ns + js];
        if (qab != 0.0) {
          double f1, df1;
          tt_both<1>(d1, sqr, f1, df1);
          u += kR4pie0 * (f1 - 1.0) * qab * ir;
          du += -kR4pie0 * qab * ((f1 - 1.0) * ir2 - df1 * ir);
        }
        const double ir6 = ir2 * ir2 * ir2, ir8 = ir2 * ir6, ir10 = ir2 * ir8;
        if (c6 != 0.0) {
          double f6, df6;
          tt_both<6>(d6, sqr, f6, df6);
          u += -f6 * c6 * ir6;
          du += -df6 * c6 * ir6 + 6.0 * f6 * c6 * ir6 * ir;
        }
        if (c8 != 0.0) {
          double f8, df8;
          tt_both<8>(d8, sqr, f8, df8);
          u += -f8 * c8 * ir8;
          du += -df8 * c8 * ir8 + 8.0 * f8 * c8 * ir8 * ir;
        }
        if (c10 != 0.0) {
          double f10, df10;
          tt_both<10>(d10, sqr, f10, df10);
          u += -f10 * c10 * ir10;
          du += -df10 * c10 * ir10 + 10.0 * f10 * c10 * ir10 * ir;
        }
        e += u;
        const double vf = -du * ir;
        gx = rsx * vf;
        gy = rsy * vf;
        gz = rsz * vf;
        fx += gx;
        fy += gy;
        fz += gz;
        v -= rsx * gx + rsy * gy + rsz * gz;
      }
      gx = warp_sum(gx);
      gy = warp_sum(gy);
      gz = warp_sum(gz);
      if (lane == 0 && (gx != 0.0 || gy != 0.0 || gz != 0.0)) {
        const size_t o = (size_t)j * ns + js;
        atomicAdd(&f[o], -gx);
        atomicAdd(&f[nfs + o], -gy);
        atomicAdd(&f[2 * nfs + o], -gz);
      }
    }
  }
  fi[wid][lane][0] = fx;
  fi[wid][lane][1] = fy;
  fi[wid][lane][2] = fz;
  e = warp_sum(e);
  v = warp_sum(v);
  if (lane == 0) {
    red[0][wid] = e;
    red[1][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32 && lact) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int w = 0; w < kWarps; w++) {
      sx += fi[w][lane][0];
      sy += fi[w][lane][1];
      sz += fi[w][lane][2];
    }
    const size_t o = (size_t)i * ns + is;
    atomicAdd(&f[o], sx);
    atomicAdd(&f[nfs + o], sy);
    atomicAdd(&f[2 * nfs + o], sz);
  }
  if (threadIdx.x == 0) {
    double se = 0.0, sv = 0.0;
    for (int w = 0; w < kWarps; w++) {
      se += red[0][w];
      sv += red[1][w];
    }
    atomicAdd(&scal[S_VDW_E], se);
    atomicAdd(&scal[S_VDW_VIR], sv);
  }
}

}  // namespace

cudaError_t launch_vdw(const double *xs, const double *ys, const double *zs, int ld,
                       const int *nbr, const double4 *nbrv, const int *ncnt, int cap, int nm,
                       int ns, double rcutsd, const int *row, const double *qq,
                       const double *par, int nrows, const int *vsite, int nv, double *f,
                       double *scal, cudaStream_t st) {
  if (nv < 1 || nv > 32 || nrows < 1 || nrows > kVdwMaxRows) return cudaErrorInvalidValue;
  k_vdw<<<nm * kSplit, kThreads, 0, st>>>(xs, ys, zs, ld, nbr, nbrv, ncnt, cap, ns, rcutsd, row, qq, par,
                                 nrows, vsite, nv, f, scal, nm);
  return cudaGetLastError();
}
