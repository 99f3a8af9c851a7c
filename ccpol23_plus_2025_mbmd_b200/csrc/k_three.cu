// k_three.cu -- FS3 and FS2 nonadditive three-body kernels (sm_100a).
//
// FS3 (threebody_potential.f90:676-2062).  For a molecular triple (i,j,k) the reference
// sums, over 17^3 site triples and 2^3 powers,
//     c(types, ip,jp,kp) * e_ij e_ik e_jk * d_jk^ip d_ik^jp d_ij^kp,
// with e_ab = exp(-b r) / (1 + exp(-g (r - r0))) of the site pair.  Every exponential
// belongs to a site PAIR, so a block first tabulates e, r and d ln(e)/dr for the 3 x 289
// site pairs of the triple, then sweeps the 4913 site triples with multiply-adds only.
// The gradient of the triple sum with respect to a site-pair distance,
//     G_ab = sum_third e_ij e_ik e_jk (dln e_ab/dr P + dP/dr_ab) / r_ab,
// is accumulated per site pair (three passes, one per pair family, each thread owning one
// site pair and looping over the third site); site forces are then sums of G_ab times
// the pair vectors, which is the reference's per-term force sum regrouped.  The
// coefficients depend only on the site types (6 types: 6^3 x 8 table).
//
// FS2 (threebody_potential.f90:101-674).  For a pair (i<j) the nine O/H-O/H exchange
// terms eta exp(-beta r) do not depend on the spectator, so one warp per pair computes
// them once and its lanes then walk the spectators k (5 spectator sites each).
#include "ccp_device.cuh"

// FS3 blocks resident per SM the register allocation targets (2: <= 96 registers).
#ifndef CCP_FS3_MINBLOCKS
#define CCP_FS3_MINBLOCKS 2
#endif

using namespace ccpd;

namespace {

constexpr int kPairs = 289;
constexpr int kItems = 3 * kPairs;
constexpr int kNt = 6;            // FS3 site types
constexpr int kCoef = kNt * kNt * kNt * 8;

// ------------------------------------------------------------------ FS3 triples
// One block per molecule i: the candidates j > i from i's neighbour list that pass the
// reference's exact bohr cut-off test are staged in shared memory, then every pair
// (j < k) of them is tested with the reference's consistent-image j-k vector.
__global__ void k_fs3_enum(const double4 *__restrict__ comb, const int *__restrict__ nbr,
                           const int *__restrict__ ncnt, int cap, int nm, Fs3Params P,
                           int4 *tri, int tri_cap, int *icnt) {
  extern __shared__ unsigned char smem_raw[];
  int *lj = reinterpret_cast<int *>(smem_raw);
  double *lx = reinterpret_cast<double *>(lj + ((cap + 1) & ~1));
  double *ly = lx + cap, *lz = ly + cap;
  __shared__ int nl;
  const int i = blockIdx.x;
  if (threadIdx.x == 0) nl = 0;
  __syncthreads();
  const double4 ci = comb[i];
  const int cnt = ncnt[i];
  // the neighbour list is in increasing j; keep the order with a ballot scan per warp
  for (int n0 = 0; n0 < cnt; n0 += blockDim.x) {
    const int n = n0 + threadIdx.x;
    bool keep = false;
    int j = 0;
    double xij = 0, yij = 0, zij = 0;
    if (n < cnt) {
      j = nbr[(size_t)i * cap + n];
      if (j > i) {
        const double4 cj = comb[j];
        xij = minimg(xsub(ci.x, cj.x), P.boxb);
        yij = minimg(xsub(ci.y, cj.y), P.boxb);
        zij = minimg(xsub(ci.z, cj.z), P.boxb);
        keep = norm2x(xij, yij, zij) < P.rc2;
      }
    }
    __shared__ int wcount[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) wcount[wid] = __popc(bal);
    __syncthreads();
    int off = nl;
    for (int w = 0; w < wid; w++) off += wcount[w];
    if (keep) {
      const int pos = off + __popc(bal & ((1u << lane) - 1u));
      lj[pos] = j;
      lx[pos] = xij;
      ly[pos] = yij;
      lz[pos] = zij;
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) nl += wcount[w];
    __syncthreads();
  }
  const int L = nl;
  for (int t = threadIdx.x; t < L * L; t += blockDim.x) {
    const int a = t / L, b = t % L;
    if (b <= a) continue;
    const int j = lj[a], k = lj[b];
    const double4 cj = comb[j], ck = comb[k];
    // xik exactly as the reference: dxik - box*nint(dxik/box)
    const double dxik = xsub(ci.x, ck.x), dyik = xsub(ci.y, ck.y), dzik = xsub(ci.z, ck.z);
    const double xik = minimg(dxik, P.boxb), yik = minimg(dyik, P.boxb), zik = minimg(dzik, P.boxb);
    if (!(norm2x(xik, yik, zik) < P.rc2)) continue;
    // xjk = dxjk + box*nint(dxij/box) - box*nint(dxik/box)  (threebody_potential.f90:883-885)
    const double dxij = xsub(ci.x, cj.x), dyij = xsub(ci.y, cj.y), dzij = xsub(ci.z, cj.z);
    const double b_ = P.boxb;
    const double xjk = xsub(xadd(xsub(cj.x, ck.x), xmul(b_, round(__ddiv_rn(dxij, b_)))),
                            xmul(b_, round(__ddiv_rn(dxik, b_))));
    const double yjk = xsub(xadd(xsub(cj.y, ck.y), xmul(b_, round(__ddiv_rn(dyij, b_)))),
                            xmul(b_, round(__ddiv_rn(dyik, b_))));
    const double zjk = xsub(xadd(xsub(cj.z, ck.z), xmul(b_, round(__ddiv_rn(dzij, b_)))),
                            xmul(b_, round(__ddiv_rn(dzik, b_))));
    const double djk2 = norm2x(xjk, yjk, zjk);
    if (!(djk2 < P.rc2)) continue;
    const double ravg = (sqrt(norm2x(lx[a], ly[a], lz[a])) + sqrt(djk2) +
                         sqrt(norm2x(xik, yik, zik))) / 3.0;
    const int branch = ravg <= P.rmin ? 0 : (ravg >= P.rmax ? 1 : 2);
    if (branch == 2) atomicAdd(&icnt[C_NBLEND_FS3], 1);
    const int slot = atomicAdd(&icnt[C_NTRI_FS3], 1);
    if (slot < tri_cap) tri[slot] = make_int4(i, j, k, branch);
  }
}

// Recompute the reference's COM vectors of a triple (bohr), exactly.
struct TripleGeom {
  double xij, yij, zij, xik, yik, zik, xjk, yjk, zjk;
  double dij2, dik2, djk2;
};

__device__ __forceinline__ void triple_geom(double4 ci, double4 cj, double4 ck, double b,
                                            TripleGeom &g) {
  const double dxij = xsub(ci.x, cj.x), dyij = xsub(ci.y, cj.y), dzij = xsub(ci.z, cj.z);
  const double dxik = xsub(ci.x, ck.x), dyik = xsub(ci.y, ck.y), dzik = xsub(ci.z, ck.z);
  g.xij = minimg(dxij, b);
  g.yij = minimg(dyij, b);
  g.zij = minimg(dzij, b);
  g.xik = minimg(dxik, b);
  g.yik = minimg(dyik, b);
  g.zik = minimg(dzik, b);
  g.xjk = xsub(xadd(xsub(cj.x, ck.x), xmul(b, round(__ddiv_rn(dxij, b)))), xmul(b, round(__ddiv_rn(dxik, b))));
  g.yjk = xsub(xadd(xsub(cj.y, ck.y), xmul(b, round(__ddiv_rn(dyij, b)))), xmul(b, round(__ddiv_rn(dyik, b))));
  g.zjk = xsub(xadd(xsub(cj.z, ck.z), xmul(b, round(__ddiv_rn(dzij, b)))), xmul(b, round(__ddiv_rn(dzik, b))));
  g.dij2 = norm2x(g.xij, g.yij, g.zij);
  g.dik2 = norm2x(g.xik, g.yik, g.zik);
  g.djk2 = norm2x(g.xjk, g.yjk, g.zjk);
}

// ---- FS3 sweep, register-blocked form --------------------------------------------
// Sites are padded from 17 to 18 (a dummy with zero weight after site 0) so that the six
// type blocks [0,d], [1,2], [3,4], [5..8], [9..12], [13..16] start at even padded indices.
// With U0 = e and U1 = e d for every site pair, each gradient pass is, per type block of
// the summed (third) site, four small matrix products
//     M_xy(a, b) = sum_{c in block} U_x(a, c) V_y(b, c),
// contracted with that type triple's 8 coefficients; a thread owns a 2x2 tile of outputs
// (both rows and both columns of one type) and keeps M in registers.
constexpr int kP = 18;       // padded sites
constexpr int kRS = 19;      // row stride (conflict-free for 8 distinct rows of 16 B)
constexpr int kTile = 9;     // 2x2 tiles per dimension
constexpr int kPassThreads = 96;
constexpr int kFs3Block = 3 * kPassThreads;

__device__ __forceinline__ int pidx(int s) { return s == 0 ? 0 : s + 1; }
__constant__ int kPType[kP] = {0, 0, 1, 1, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5};

template <typename T>
struct Vec2;
template <>
struct Vec2<double> {
  using type = double2;
};
template <>
struct Vec2<float> {
  using type = float2;
};

template <typename T>
struct Fs3Smem {
  using V2 = typename Vec2<T>::type;
  double coef[2][kCoef];         // SR, LR coefficient by type triple
  double bgr[2][3][kPairs];      // SR, LR b, g, r0 of each site pair
  double site[3][kNs3][3];       // site offsets (bohr) of i, j, k
  V2 uu[3][kP][kRS];             // (e, e d) of each site pair, families ij, ik, jk
  V2 dl[3][kP][kRS];             // (d, d ln e / dr)
  double G[3][kP][kRS];          // accumulated site-force weights
  double red[kFs3Block / 32];
  double cv[3][3];               // COM vectors ij, ik, jk of the current triple (bohr)
  double rr[3];                  // their lengths
  double sc[6];                  // fdmp, dfdmp, smfun, cf, energy, comc
  int mol[3];
  int branch;
};

template <typename T>
__device__ __forceinline__ T t_exp(T v);
template <>
__device__ __forceinline__ double t_exp<double>(double v) { return exp(v); }
template <>
__device__ __forceinline__ float t_exp<float>(float v) { return __expf(v); }

template <typename T>
__device__ __forceinline__ T t_sqrt(T v);
template <>
__device__ __forceinline__ double t_sqrt<double>(double v) { return sqrt(v); }
template <>
__device__ __forceinline__ float t_sqrt<float>(float v) { return sqrtf(v); }

template <typename T>
__device__ __forceinline__ T t_rcp(T v);
template <>
__device__ __forceinline__ double t_rcp<double>(double v) { return 1.0 / v; }
template <>
__device__ __forceinline__ float t_rcp<float>(float v) { return __frcp_rn(v); }

// Pair family p: 0 = (i,j), 1 = (i,k), 2 = (j,k).
__device__ __forceinline__ void family(int p, int &m1, int &m2) {
  m1 = p == 2 ? 1 : 0;
  m2 = p == 0 ? 1 : 2;
}

// One gradient pass for the 2x2 output tile (r0, r0+1) x (c0, c0+1) of family `fam`:
//   fam 0: outputs (is, js), sums over ks: X = U_ik(is, ks), Y = U_jk(js, ks)
//   fam 1: outputs (is, ks), sums over js: X = U_ij(is, js), Y = U_jk(js, ks)
//   fam 2: outputs (js, ks), sums over is: X = U_ij(is, js), Y = U_ik(is, ks)
// q0/q1 receive the two coefficient-contracted sums; P = q0 + d q1 and dP/dd = q1 for the
// output pair's own distance d.
template <typename T, int fam>
__device__ __forceinline__ void fs3_pass(const Fs3Smem<T> &S, const double *__restrict__ C,
                                         int r0, int c0, T q0[4], T q1[4]) {
  using V2 = typename Vec2<T>::type;
  const int tr = kPType[r0], tc = kPType[c0];
#pragma unroll
  for (int o = 0; o < 4; o++) q0[o] = q1[o] = (T)0;
  constexpr int kStart[7] = {0, 2, 4, 6, 10, 14, 18};
#pragma unroll
  for (int tb = 0; tb < 6; tb++) {
    T M[4][4];
#pragma unroll
    for (int o = 0; o < 4; o++)
#pragma unroll
      for (int u = 0; u < 4; u++) M[o][u] = (T)0;
#pragma unroll
    for (int c = kStart[tb]; c < kStart[tb + 1]; c++) {
      V2 xa, xb, ya, yb;
      if (fam == 0) {
        xa = S.uu[1][r0][c];
        xb = S.uu[1][r0 + 1][c];
        ya = S.uu[2][c0][c];
        yb = S.uu[2][c0 + 1][c];
      } else if (fam == 1) {
        xa = S.uu[0][r0][c];
        xb = S.uu[0][r0 + 1][c];
        ya = S.uu[2][c][c0];
        yb = S.uu[2][c][c0 + 1];
      } else {
        xa = S.uu[0][c][r0];
        xb = S.uu[0][c][r0 + 1];
        ya = S.uu[1][c][c0];
        yb = S.uu[1][c][c0 + 1];
      }
      const V2 X[2] = {xa, xb}, Y[2] = {ya, yb};
#pragma unroll
      for (int rr = 0; rr < 2; rr++)
#pragma unroll
        for (int cc = 0; cc < 2; cc++) {
          const int o = rr * 2 + cc;
          M[o][0] += X[rr].x * Y[cc].x;
          M[o][1] += X[rr].x * Y[cc].y;
          M[o][2] += X[rr].y * Y[cc].x;
          M[o][3] += X[rr].y * Y[cc].y;
        }
    }
    // coefficient c[ip*4 + jp*2 + kp] of the type triple (ti, tj, tk)
    int ti, tj, tk;
    if (fam == 0) {
      ti = tr; tj = tc; tk = tb;
    } else if (fam == 1) {
      ti = tr; tj = tb; tk = tc;
    } else {
      ti = tb; tj = tr; tk = tc;
    }
    const double *cp = C + ((ti * kNt + tj) * kNt + tk) * 8;
    T c[8];
#pragma unroll
    for (int u = 0; u < 8; u++) c[u] = (T)cp[u];
#pragma unroll
    for (int o = 0; o < 4; o++) {
      // M[o][x*2 + y] = sum X_x Y_y with x, y the powers carried by X and Y:
      //  fam 0: X -> jp (d_ik), Y -> ip (d_jk); outputs carry kp (d_ij)
      //  fam 1: X -> kp (d_ij), Y -> ip (d_jk); outputs carry jp (d_ik)
      //  fam 2: X -> kp (d_ij), Y -> jp (d_ik); outputs carry ip (d_jk)
      if (fam == 0) {
        q0[o] += c[0] * M[o][0] + c[4] * M[o][1] + c[2] * M[o][2] + c[6] * M[o][3];
        q1[o] += c[1] * M[o][0] + c[5] * M[o][1] + c[3] * M[o][2] + c[7] * M[o][3];
      } else if (fam == 1) {
        q0[o] += c[0] * M[o][0] + c[4] * M[o][1] + c[1] * M[o][2] + c[5] * M[o][3];
        q1[o] += c[2] * M[o][0] + c[6] * M[o][1] + c[3] * M[o][2] + c[7] * M[o][3];
      } else {
        q0[o] += c[0] * M[o][0] + c[2] * M[o][1] + c[1] * M[o][2] + c[3] * M[o][3];
        q1[o] += c[4] * M[o][0] + c[6] * M[o][1] + c[5] * M[o][2] + c[7] * M[o][3];
      }
    }
  }
}

template <typename T>
__device__ double fs3_variant(Fs3Smem<T> &S, int v, double wsite) {
  using V2 = typename Vec2<T>::type;
  const int tid = threadIdx.x;
  // ---- pair phase: e, r and d ln e / dr of the 867 site pairs (padded layout)
#pragma unroll
  for (int rnd = 0; rnd < (kItems + kFs3Block - 1) / kFs3Block; rnd++) {
    const int it = tid + rnd * kFs3Block;
    if (it >= kItems) break;
    const int p = it / kPairs, ab = it % kPairs, a = ab / kNs3, b = ab % kNs3;
    int m1, m2;
    family(p, m1, m2);
    const double vx = S.cv[p][0] + (S.site[m1][a][0] - S.site[m2][b][0]);
    const double vy = S.cv[p][1] + (S.site[m1][a][1] - S.site[m2][b][1]);
    const double vz = S.cv[p][2] + (S.site[m1][a][2] - S.site[m2][b][2]);
    const T r2 = (T)(vx * vx + vy * vy + vz * vz);
    const T r = t_sqrt<T>(r2);
    const T bb = (T)S.bgr[v][0][ab], gg = (T)S.bgr[v][1][ab], r0 = (T)S.bgr[v][2][ab];
    const T ex = t_exp<T>(-gg * (r - r0));
    const T damp = t_rcp<T>((T)1 + ex);
    const T e = t_exp<T>(-bb * r) * damp;
    V2 u, w;
    u.x = e;
    u.y = e * r;
    w.x = r;
    w.y = -bb + gg * ex * damp;
    S.uu[p][pidx(a)][pidx(b)] = u;
    S.dl[p][pidx(a)][pidx(b)] = w;
  }
  __syncthreads();
  // ---- gradient passes: warps 0-2 family ij, 3-5 ik, 6-8 jk
  const int fam = tid / kPassThreads, lt = tid % kPassThreads;
  double esum = 0.0;
  if (lt < kTile * kTile) {
    const int r0 = 2 * (lt / kTile), c0 = 2 * (lt % kTile);
    T q0[4], q1[4];
    if (fam == 0)
      fs3_pass<T, 0>(S, S.coef[v], r0, c0, q0, q1);
    else if (fam == 1)
      fs3_pass<T, 1>(S, S.coef[v], r0, c0, q0, q1);
    else
      fs3_pass<T, 2>(S, S.coef[v], r0, c0, q0, q1);
#pragma unroll
    for (int o = 0; o < 4; o++) {
      const int r = r0 + (o >> 1), c = c0 + (o & 1);
      const V2 u = S.uu[fam][r][c], w = S.dl[fam][r][c];
      const T P = q0[o] + w.x * q1[o];
      if (fam == 0) esum += (double)u.x * (double)P;
      S.G[fam][r][c] += wsite * (double)(u.x * (w.y * P + q1[o]) / w.x);
    }
  }
  esum = warp_sum(esum);
  if ((tid & 31) == 0) S.red[tid >> 5] = esum;
  __syncthreads();
  double tot = 0.0;
#pragma unroll
  for (int w = 0; w < kFs3Block / 32; w++) tot += S.red[w];
  __syncthreads();
  return tot;
}

template <typename T>
__global__ void __launch_bounds__(kFs3Block, CCP_FS3_MINBLOCKS)
    k_fs3(const int4 *__restrict__ tri, const int *__restrict__ icnt, int tri_cap,
          const double4 *__restrict__ comb, const double4 *__restrict__ s17, Fs3Params P,
          const double *__restrict__ coef, const double *__restrict__ bgr,
          const int *__restrict__ types, int nm, int ns, double *f, double *fc3, double *scal) {
  using V2 = typename Vec2<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Fs3Smem<T> &S = *reinterpret_cast<Fs3Smem<T> *>(smem_raw);
  const int tid = threadIdx.x;
  (void)types;
  for (int t = tid; t < 2 * kCoef; t += kFs3Block) (&S.coef[0][0])[t] = coef[t];
  for (int t = tid; t < 2 * 3 * kPairs; t += kFs3Block) (&S.bgr[0][0][0])[t] = bgr[t];
  // padded dummy site: zero weight, unit distance (keeps e / d finite)
  for (int t = tid; t < 3 * kP; t += kFs3Block) {
    const int p = t / kP, q = t % kP;
    V2 z, one;
    z.x = z.y = (T)0;
    one.x = (T)1;
    one.y = (T)0;
    S.uu[p][1][q] = z;
    S.uu[p][q][1] = z;
    S.dl[p][1][q] = one;
    S.dl[p][q][1] = one;
  }
  __syncthreads();
  const int ntri = min(icnt[C_NTRI_FS3], tri_cap);
  const double conv = kH2kcal * 418.4 / kBohr2a;
  const size_t nfs = (size_t)nm * ns;
  double e_tot = 0.0, v_tot = 0.0;
  for (int t = blockIdx.x; t < ntri; t += gridDim.x) {
    if (tid == 0) {
      const int4 T4 = tri[t];
      S.mol[0] = T4.x;
      S.mol[1] = T4.y;
      S.mol[2] = T4.z;
      TripleGeom g;
      triple_geom(comb[T4.x], comb[T4.y], comb[T4.z], P.boxb, g);
      const double rij = sqrt(g.dij2), rik = sqrt(g.dik2), rjk = sqrt(g.djk2);
      const double ravg = (rij + rjk + rik) / 3.0;
      const double pom = exp(P.alp3 * (ravg - P.r0dmp));
      const double ppom = 1.0 / (1.0 + pom);
      const double fdmp = pow(ppom, P.delta33);
      S.cv[0][0] = g.xij; S.cv[0][1] = g.yij; S.cv[0][2] = g.zij;
      S.cv[1][0] = g.xik; S.cv[1][1] = g.yik; S.cv[1][2] = g.zik;
      S.cv[2][0] = g.xjk; S.cv[2][1] = g.yjk; S.cv[2][2] = g.zjk;
      S.rr[0] = rij; S.rr[1] = rik; S.rr[2] = rjk;
      S.sc[0] = fdmp;
      S.sc[1] = -P.alp3 * P.delta33 * pom * ppom * fdmp * (1.0 / 3.0);
      S.branch = ravg <= P.rmin ? 0 : (ravg >= P.rmax ? 1 : 2);
      const double cfact = (ravg - P.rmin) / (P.rmax - P.rmin);
      S.sc[2] = 1.0 + 2.0 * cfact * cfact * cfact - 3.0 * cfact * cfact;
      S.sc[3] = 2.0 / (P.rmax - P.rmin) * (cfact * cfact - cfact);
    }
    __syncthreads();
    for (int u = tid; u < 3 * kNs3; u += kFs3Block) {
      const int m = u / kNs3, s = u % kNs3;
      const double4 o = s17[(size_t)S.mol[m] * kNs3 + s];
      S.site[m][s][0] = o.x;
      S.site[m][s][1] = o.y;
      S.site[m][s][2] = o.z;
    }
    for (int u = tid; u < 3 * kP * kRS; u += kFs3Block) (&S.G[0][0][0])[u] = 0.0;
    __syncthreads();
    {
      const double fdmp = S.sc[0], dfdmp = S.sc[1];
      const int br = S.branch;
      double energy, comc;
      if (br != 2) {
        const double Sv = fs3_variant<T>(S, br, fdmp);
        energy = fdmp * Sv;
        comc = dfdmp * Sv;
      } else {
        const double smfun = S.sc[2], smfun2 = 1.0 - smfun, cf = S.sc[3];
        const double Ssr = fs3_variant<T>(S, 0, fdmp * smfun);
        const double Slr = fs3_variant<T>(S, 1, fdmp * smfun2);
        energy = fdmp * (smfun * Ssr + smfun2 * Slr);
        comc = Ssr * (dfdmp * smfun + fdmp * cf) + Slr * (dfdmp * smfun2 - fdmp * cf);
      }
      if (tid == 0) {
        S.sc[4] = energy;
        S.sc[5] = comc;
      }
    }
    // ---- site forces: F = -sum_partner G * (pair vector); 4 lanes per (molecule, site),
    // each summing a quarter of the 17 partners, reduced with shuffles.
    double vsite = 0.0;
    {
      const int item = tid >> 2, part = tid & 3;
      const bool act = item < 3 * kNs3;
      const int m = act ? item / kNs3 : 0, s = act ? item % kNs3 : 0, ps = pidx(s);
      double fx = 0.0, fy = 0.0, fz = 0.0;
      if (act) {
        for (int o = part; o < kNs3; o += 4) {
          const int po = pidx(o);
          if (m == 0) {
            const double g0 = S.G[0][ps][po], g1 = S.G[1][ps][po];
            const double a0 = S.cv[0][0] + (S.site[0][s][0] - S.site[1][o][0]);
            const double a1 = S.cv[0][1] + (S.site[0][s][1] - S.site[1][o][1]);
            const double a2 = S.cv[0][2] + (S.site[0][s][2] - S.site[1][o][2]);
            const double b0 = S.cv[1][0] + (S.site[0][s][0] - S.site[2][o][0]);
            const double b1 = S.cv[1][1] + (S.site[0][s][1] - S.site[2][o][1]);
            const double b2 = S.cv[1][2] + (S.site[0][s][2] - S.site[2][o][2]);
            fx -= g0 * a0 + g1 * b0;
            fy -= g0 * a1 + g1 * b1;
            fz -= g0 * a2 + g1 * b2;
            vsite += g0 * (a0 * a0 + a1 * a1 + a2 * a2) + g1 * (b0 * b0 + b1 * b1 + b2 * b2);
          } else if (m == 1) {
            const double g0 = S.G[0][po][ps], g2 = S.G[2][ps][po];
            const double a0 = S.cv[0][0] + (S.site[0][o][0] - S.site[1][s][0]);
            const double a1 = S.cv[0][1] + (S.site[0][o][1] - S.site[1][s][1]);
            const double a2 = S.cv[0][2] + (S.site[0][o][2] - S.site[1][s][2]);
            const double c0 = S.cv[2][0] + (S.site[1][s][0] - S.site[2][o][0]);
            const double c1 = S.cv[2][1] + (S.site[1][s][1] - S.site[2][o][1]);
            const double c2 = S.cv[2][2] + (S.site[1][s][2] - S.site[2][o][2]);
            fx -= -g0 * a0 + g2 * c0;
            fy -= -g0 * a1 + g2 * c1;
            fz -= -g0 * a2 + g2 * c2;
            vsite += g2 * (c0 * c0 + c1 * c1 + c2 * c2);
          } else {
            const double g1 = S.G[1][po][ps], g2 = S.G[2][po][ps];
            const double b0 = S.cv[1][0] + (S.site[0][o][0] - S.site[2][s][0]);
            const double b1 = S.cv[1][1] + (S.site[0][o][1] - S.site[2][s][1]);
            const double b2 = S.cv[1][2] + (S.site[0][o][2] - S.site[2][s][2]);
            const double c0 = S.cv[2][0] + (S.site[1][o][0] - S.site[2][s][0]);
            const double c1 = S.cv[2][1] + (S.site[1][o][1] - S.site[2][s][1]);
            const double c2 = S.cv[2][2] + (S.site[1][o][2] - S.site[2][s][2]);
            fx -= -g1 * b0 - g2 * c0;
            fy -= -g1 * b1 - g2 * c1;
            fz -= -g1 * b2 - g2 * c2;
          }
        }
      }
#pragma unroll
      for (int off = 1; off < 4; off <<= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, off);
        fy += __shfl_xor_sync(0xffffffffu, fy, off);
        fz += __shfl_xor_sync(0xffffffffu, fz, off);
      }
      if (act && part == 0) {
        const size_t o = (size_t)S.mol[m] * ns + s;
        atomicAdd(&f[o], fx * conv);
        atomicAdd(&f[nfs + o], fy * conv);
        atomicAdd(&f[2 * nfs + o], fz * conv);
      }
    }
    if (tid == 0) {
      // COM forces from the R_avg damping and switch (threebody_potential.f90:1092-1120)
      const double comc = S.sc[5];
      const double rij = S.rr[0], rik = S.rr[1], rjk = S.rr[2];
      const double ux = S.cv[0][0] / rij, uy = S.cv[0][1] / rij, uz = S.cv[0][2] / rij;
      const double wx = S.cv[1][0] / rik, wy = S.cv[1][1] / rik, wz = S.cv[1][2] / rik;
      const double sx = S.cv[2][0] / rjk, sy = S.cv[2][1] / rjk, sz = S.cv[2][2] / rjk;
      const int m0 = S.mol[0], m1 = S.mol[1], m2 = S.mol[2];
      atomicAdd(&fc3[m0], -comc * (ux + wx) * conv);
      atomicAdd(&fc3[nm + m0], -comc * (uy + wy) * conv);
      atomicAdd(&fc3[2 * nm + m0], -comc * (uz + wz) * conv);
      atomicAdd(&fc3[m1], -comc * (-ux + sx) * conv);
      atomicAdd(&fc3[nm + m1], -comc * (-uy + sy) * conv);
      atomicAdd(&fc3[2 * nm + m1], -comc * (-uz + sz) * conv);
      atomicAdd(&fc3[m2], -comc * (-wx - sx) * conv);
      atomicAdd(&fc3[nm + m2], -comc * (-wy - sy) * conv);
      atomicAdd(&fc3[2 * nm + m2], -comc * (-wz - sz) * conv);
      e_tot += S.sc[4];
      v_tot += comc * (rij + rik + rjk);
    }
    v_tot += vsite;
    __syncthreads();
  }
  v_tot = warp_sum(v_tot);
  if ((tid & 31) == 0) {
    atomicAdd(&scal[S_FS3_VIR], v_tot);
    if (tid == 0) atomicAdd(&scal[S_FS3_E], e_tot);
  }
}

// ------------------------------------------------------------------------ FS2
__global__ void k_fs2_enum(const double4 *__restrict__ comb, const int *__restrict__ nbr,
                           const int *__restrict__ ncnt, int cap, int nm, Fs2Params P,
                           int2 *pairs, int pair_cap, int *icnt) {
  const int i = blockIdx.x;
  const double4 ci = comb[i];
  const int cnt = ncnt[i];
  for (int n = threadIdx.x; n < cnt; n += blockDim.x) {
    const int j = nbr[(size_t)i * cap + n];
    if (j <= i) continue;
    const double4 cj = comb[j];
    const double xij = minimg(xsub(ci.x, cj.x), P.boxb);
    const double yij = minimg(xsub(ci.y, cj.y), P.boxb);
    const double zij = minimg(xsub(ci.z, cj.z), P.boxb);
    if (!(norm2x(xij, yij, zij) < P.rc2)) continue;
    const int slot = atomicAdd(&icnt[C_NPAIR_FS2], 1);
    if (slot < pair_cap) pairs[slot] = make_int2(i, j);
  }
}

__constant__ double kCharge3b[5] = {0.258504607653328389, 0.564050362569283648,
                                    0.564050362569283648, -0.693302666395947953,
                                    -0.693302666395947953};

__global__ void __launch_bounds__(128)
    k_fs2(const int2 *__restrict__ pairs, const int *__restrict__ icnt, int pair_cap,
          const double4 *__restrict__ comb, const double4 *__restrict__ s17,
          const int *__restrict__ nbr, const int *__restrict__ ncnt, int cap, Fs2Params P,
          int nm, int ns, double *f, double *fc2, double *scal, int *ncomb) {
  const double eta3 = 0.48056977605478400, beta3 = 0.85836606579445000, g3 = 0.4;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int npair = min(icnt[C_NPAIR_FS2], pair_cap);
  if (w >= npair) return;
  const int i = pairs[w].x, j = pairs[w].y;
  const double4 ci = comb[i], cj = comb[j];
  const double xij = minimg(xsub(ci.x, cj.x), P.boxb);
  const double yij = minimg(xsub(ci.y, cj.y), P.boxb);
  const double zij = minimg(xsub(ci.z, cj.z), P.boxb);
  const double dij2 = norm2x(xij, yij, zij);
  const double dij = sqrt(dij2), dij1i = 1.0 / dij, dij3i = dij1i * dij1i * dij1i;
  // spectator-independent exchange sums over the 3x3 O/H site pairs (lanes 0..8)
  double eq = 0.0, evq = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
  if (lane < 9) {
    const int is = lane / 3, js = lane % 3;
    const double4 si = s17[(size_t)i * kNs3 + is], sj = s17[(size_t)j * kNs3 + js];
    const double xs_ = xij + (si.x - sj.x), ys_ = yij + (si.y - sj.y), zs_ = zij + (si.z - sj.z);
    const double ds = sqrt(xs_ * xs_ + ys_ * ys_ + zs_ * zs_);
    eq = eta3 * exp(-beta3 * ds);
    evq = eq * (-beta3 * ds - 1.0);
    const double c = eq * beta3 / ds;
    ux = c * xs_;
    uy = c * ys_;
    uz = c * zs_;
  }
  // U_i(is) = -sum_js eq beta r/|r| ; U_j(js) = +sum_is eq beta r/|r|
  double Ui[3][3], Uj[3][3];
#pragma unroll
  for (int s = 0; s < 3; s++) {
#pragma unroll
    for (int c = 0; c < 3; c++) Ui[s][c] = Uj[s][c] = 0.0;
  }
#pragma unroll
  for (int l = 0; l < 9; l++) {
    const double vx = __shfl_sync(0xffffffffu, ux, l), vy = __shfl_sync(0xffffffffu, uy, l),
                 vz = __shfl_sync(0xffffffffu, uz, l);
    Ui[l / 3][0] -= vx;
    Ui[l / 3][1] -= vy;
    Ui[l / 3][2] -= vz;
    Uj[l % 3][0] += vx;
    Uj[l % 3][1] += vy;
    Uj[l % 3][2] += vz;
  }
  const double E = warp_sum(eq), Ev = warp_sum(evq);
  const double conv = kH2kcal * 418.4 / kBohr2a;
  const size_t nfs = (size_t)nm * ns;
  double e_loc = 0.0, v_loc = 0.0, A_loc = 0.0;
  double Ci[3] = {0, 0, 0}, Cj[3] = {0, 0, 0};
  int nspec = 0;
  const int cnt = ncnt[i];
  for (int n = lane; n < cnt; n += 32) {
    const int k = nbr[(size_t)i * cap + n];
    if (k == j) continue;
    const double4 ck = comb[k];
    const double xki = minimg(xsub(ck.x, ci.x), P.boxb);
    const double yki = minimg(xsub(ck.y, ci.y), P.boxb);
    const double zki = minimg(xsub(ck.z, ci.z), P.boxb);
    const double xkj = xadd(xki, xij), ykj = xadd(yki, yij), zkj = xadd(zki, zij);
    const double dki2 = norm2x(xki, yki, zki), dkj2 = norm2x(xkj, ykj, zkj);
    if (!(dki2 < P.rc2 && dkj2 < P.rc2)) continue;
    const double sdki = sqrt(dki2), sdkj = sqrt(dkj2);
    double pom = exp(P.alp3 * (sdki - P.r0dmp));
    const double pomki = 1.0 / (1.0 + pom);
    const double flrki = pow(pomki, P.delta33);
    const double dflrki = -P.alp3 * P.delta33 * pom * pomki * flrki;
    const double dflrkiv = -P.alp3 * P.delta33 * pom * pomki * sdki;
    pom = exp(P.alp3 * (sdkj - P.r0dmp));
    const double pomkj = 1.0 / (1.0 + pom);
    const double flrkj = pow(pomkj, P.delta33);
    const double dflrkj = -P.alp3 * P.delta33 * pom * pomkj * flrkj;
    const double dflrkjv = -P.alp3 * P.delta33 * pom * pomkj * sdkj;
    const double fl = flrki * flrkj;
    nspec++;
    double ck_x = 0, ck_y = 0, ck_z = 0;  // COM force on k
    for (int ks = 0; ks < 5; ks++) {
      const double qks = kCharge3b[ks];
      const double4 sk = s17[(size_t)k * kNs3 + ks];
      const double dxkqi = xki + sk.x - g3 * xij * dij1i;
      const double dykqi = yki + sk.y - g3 * yij * dij1i;
      const double dzkqi = zki + sk.z - g3 * zij * dij1i;
      const double dkqi1i = 1.0 / sqrt(dxkqi * dxkqi + dykqi * dykqi + dzkqi * dzkqi);
      const double dkqi3i = dkqi1i * dkqi1i * dkqi1i;
      const double dxkqj = xkj + sk.x + g3 * xij * dij1i;
      const double dykqj = ykj + sk.y + g3 * yij * dij1i;
      const double dzkqj = zkj + sk.z + g3 * zij * dij1i;
      const double dkqj1i = 1.0 / sqrt(dxkqj * dxkqj + dykqj * dykqj + dzkqj * dzkqj);
      const double dkqj3i = dkqj1i * dkqj1i * dkqj1i;
      const double dxkci = xki + sk.x, dykci = yki + sk.y, dzkci = zki + sk.z;
      const double dkci1i = 1.0 / sqrt(dxkci * dxkci + dykci * dykci + dzkci * dzkci);
      const double dkci3i = dkci1i * dkci1i * dkci1i;
      const double dxkcj = xkj + sk.x, dykcj = ykj + sk.y, dzkcj = zkj + sk.z;
      const double dkcj1i = 1.0 / sqrt(dxkcj * dxkcj + dykcj * dykcj + dzkcj * dzkcj);
      const double dkcj3i = dkcj1i * dkcj1i * dkcj1i;
      const double term0 = dkci1i + dkcj1i - dkqi1i - dkqj1i;
      const double qE = qks * E;
      e_loc += qE * term0 * fl;
      const double termxy1 = (dxkqi * xij + dykqi * yij + dzkqi * zij) * g3 * dij1i * dkqi3i;
      const double termxy2 = (dxkqj * xij + dykqj * yij + dzkqj * zij) * g3 * dij1i * dkqj3i;
      v_loc += (qks * Ev + (dflrkiv + dflrkjv) * qE) * term0 * fl + qE * (termxy1 - termxy2) * fl;
      A_loc += qks * term0 * fl;
      const double dotkqi = xij * dxkqi + yij * dykqi + zij * dzkqi;
      const double dotkqj = xij * dxkqj + yij * dykqj + zij * dzkqj;
      // spectator site force
      const double fkx = qE * (-dxkci * dkci3i - dxkcj * dkcj3i + dxkqi * dkqi3i + dxkqj * dkqj3i);
      const double fky = qE * (-dykci * dkci3i - dykcj * dkcj3i + dykqi * dkqi3i + dykqj * dkqj3i);
      const double fkz = qE * (-dzkci * dkci3i - dzkcj * dkcj3i + dzkqi * dkqi3i + dzkqj * dkqj3i);
      const size_t so = (size_t)k * ns + ks;
      atomicAdd(&f[so], -fkx * fl * conv);
      atomicAdd(&f[nfs + so], -fky * fl * conv);
      atomicAdd(&f[2 * nfs + so], -fkz * fl * conv);
      // COM forces from the long-range damping and the exchange-charge positions
      const double tki = qE * term0 * dflrki * flrkj / sdki;
      const double tkj = qE * term0 * dflrkj * flrki / sdkj;
      ck_x += -tki * xki - tkj * xkj;
      ck_y += -tki * yki - tkj * ykj;
      ck_z += -tki * zki - tkj * zkj;
      const double gi = 1.0 + g3 * dij1i;
      const double fxi = qE * (dxkci * dkci3i) +
                         qE * dkqi3i * (-gi * dxkqi + g3 * dotkqi * xij * dij3i) +
                         qE * dkqj3i * (g3 * dxkqj * dij1i - g3 * dotkqj * xij * dij3i);
      const double fyi = qE * (dykci * dkci3i) +
                         qE * dkqi3i * (-gi * dykqi + g3 * dotkqi * yij * dij3i) +
                         qE * dkqj3i * (g3 * dykqj * dij1i - g3 * dotkqj * yij * dij3i);
      const double fzi = qE * (dzkci * dkci3i) +
                         qE * dkqi3i * (-gi * dzkqi + g3 * dotkqi * zij * dij3i) +
                         qE * dkqj3i * (g3 * dzkqj * dij1i - g3 * dotkqj * zij * dij3i);
      const double fxj = qE * (dxkcj * dkcj3i) +
                         qE * dkqi3i * (g3 * dxkqi * dij1i - g3 * dotkqi * xij * dij3i) +
                         qE * dkqj3i * (-gi * dxkqj + g3 * dotkqj * xij * dij3i);
      const double fyj = qE * (dykcj * dkcj3i) +
                         qE * dkqi3i * (g3 * dykqi * dij1i - g3 * dotkqi * yij * dij3i) +
                         qE * dkqj3i * (-gi * dykqj + g3 * dotkqj * yij * dij3i);
      const double fzj = qE * (dzkcj * dkcj3i) +
                         qE * dkqi3i * (g3 * dzkqi * dij1i - g3 * dotkqi * zij * dij3i) +
                         qE * dkqj3i * (-gi * dzkqj + g3 * dotkqj * zij * dij3i);
      Ci[0] += -fxi * fl + tki * xki;
      Ci[1] += -fyi * fl + tki * yki;
      Ci[2] += -fzi * fl + tki * zki;
      Cj[0] += -fxj * fl + tkj * xkj;
      Cj[1] += -fyj * fl + tkj * ykj;
      Cj[2] += -fzj * fl + tkj * zkj;
    }
    atomicAdd(&fc2[k], ck_x * conv);
    atomicAdd(&fc2[nm + k], ck_y * conv);
    atomicAdd(&fc2[2 * nm + k], ck_z * conv);
  }
  e_loc = warp_sum(e_loc);
  v_loc = warp_sum(v_loc);
  A_loc = warp_sum(A_loc);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    Ci[c] = warp_sum(Ci[c]);
    Cj[c] = warp_sum(Cj[c]);
  }
  if (lane < 3) {
    // site forces on i's and j's O/H sites: -A U
    const int s = lane;
    const size_t oi = (size_t)i * ns + s, oj = (size_t)j * ns + s;
    atomicAdd(&f[oi], -A_loc * Ui[s][0] * conv);
    atomicAdd(&f[nfs + oi], -A_loc * Ui[s][1] * conv);
    atomicAdd(&f[2 * nfs + oi], -A_loc * Ui[s][2] * conv);
    atomicAdd(&f[oj], -A_loc * Uj[s][0] * conv);
    atomicAdd(&f[nfs + oj], -A_loc * Uj[s][1] * conv);
    atomicAdd(&f[2 * nfs + oj], -A_loc * Uj[s][2] * conv);
  }
  if (lane == 0) {
    for (int c = 0; c < 3; c++) {
      atomicAdd(&fc2[c * nm + i], Ci[c] * conv);
      atomicAdd(&fc2[c * nm + j], Cj[c] * conv);
    }
    atomicAdd(&scal[S_FS2_E], e_loc);
    atomicAdd(&scal[S_FS2_VIR], v_loc);
  }
  for (int o = 16; o > 0; o >>= 1) nspec += __shfl_xor_sync(0xffffffffu, nspec, o);
  if (lane == 0 && nspec) atomicAdd(ncomb, nspec);
}

}  // namespace

cudaError_t launch_fs3_enum(const double4 *comb, const int *nbr, const int *ncnt, int cap,
                            int nm, Fs3Params P, int4 *tri, int tri_cap, int *icnt,
                            cudaStream_t st) {
  const size_t smem = sizeof(int) * (size_t)((cap + 1) & ~1) + 3 * sizeof(double) * (size_t)cap;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_fs3_enum, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_fs3_enum<<<nm, 128, smem, st>>>(comb, nbr, ncnt, cap, nm, P, tri, tri_cap, icnt);
  return cudaGetLastError();
}

cudaError_t launch_fs3(int precision, const int4 *tri, const int *icnt, int tri_cap,
                       const double4 *comb, const double4 *s17, Fs3Params P,
                       const double *coef, const double *bgr, const int *types, int nm, int ns,
                       double *f, double *fc3, double *scal, int nsm, cudaStream_t st) {
  cudaError_t e;
  if (precision == 0) {
    const size_t smem = sizeof(Fs3Smem<double>);
    e = cudaFuncSetAttribute(k_fs3<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fs3<double>, kFs3Block, smem);
    if (per_sm < 1) per_sm = 1;
    k_fs3<double><<<nsm * per_sm, kFs3Block, smem, st>>>(tri, icnt, tri_cap, comb, s17, P, coef,
                                                           bgr, types, nm, ns, f, fc3, scal);
  } else {
    const size_t smem = sizeof(Fs3Smem<float>);
    e = cudaFuncSetAttribute(k_fs3<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fs3<float>, kFs3Block, smem);
    if (per_sm < 1) per_sm = 1;
    k_fs3<float><<<nsm * per_sm, kFs3Block, smem, st>>>(tri, icnt, tri_cap, comb, s17, P, coef,
                                                          bgr, types, nm, ns, f, fc3, scal);
  }
  return cudaGetLastError();
}

cudaError_t launch_fs2_enum(const double4 *comb, const int *nbr, const int *ncnt, int cap,
                            int nm, Fs2Params P, int2 *pairs, int pair_cap, int *icnt,
                            cudaStream_t st) {
  k_fs2_enum<<<nm, 64, 0, st>>>(comb, nbr, ncnt, cap, nm, P, pairs, pair_cap, icnt);
  return cudaGetLastError();
}

cudaError_t launch_fs2(int precision, const int2 *pairs, const int *icnt, int pair_cap,
                       const double4 *comb, const double4 *s17, const int *nbr,
                       const int *ncnt, int cap, Fs2Params P, int nm, int ns, double *f,
                       double *fc2, double *scal, cudaStream_t st) {
  (void)precision;
  // one warp per pair; the pair count is on the device, so launch for the capacity and
  // let surplus warps exit at once.
  const int warps = pair_cap;
  const int threads = 128;
  const int blocks = (warps * 32 + threads - 1) / threads;
  k_fs2<<<blocks, threads, 0, st>>>(pairs, icnt, pair_cap, comb, s17, nbr, ncnt, cap, P, nm, ns,
                                    f, fc2, scal, const_cast<int *>(icnt) + C_NTRI_FS2);
  return cudaGetLastError();
}
