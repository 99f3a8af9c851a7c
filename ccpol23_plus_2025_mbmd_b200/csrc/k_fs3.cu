// k_fs3.cu -- FS3 nonadditive three-body kernels (sm_100a).
//
// FS3 (threebody_potential.f90:676-2062).  For a molecular triple (i,j,k) with all three COM
// distances below 6.3 A the reference sums, over 17^3 site triples and 2^3 powers,
//     c(types, ip,jp,kp) * e_ij e_ik e_jk * d_jk^ip d_ik^jp d_ij^kp,
// e_ab = exp(-b r)/(1 + exp(-g (r - r0))) of the site pair, times the R_avg damping f_dmp
// and, between 4.5 and 5.5 A, the SR/LR switch.  Every exponential belongs to a site PAIR,
// so a block first tabulates e, e d and the force-weight factors for the 3 x 289 site pairs
// of the triple; the energy and the gradient with respect to every site-pair distance,
//     G_ab = sum_third e_ij e_ik e_jk (dln e_ab/dr P + dP/dr_ab) / r_ab,
// then come from three passes (one per pair family) of small matrix products: with sites
// padded from 17 to 18 (a zero-weight dummy after site 0) the six site-type blocks
//     [0,dummy] [1,2] [3,4] [5..8] [9..12] [13..16]
// start at even indices, and per type block of the summed site each pass accumulates
//     M_xy(a, b) = sum_c U_x(a, c) V_y(b, c),  U_0 = e, U_1 = e d,
// for a 2x2 tile of outputs in registers, then contracts M with that type triple's 8
// coefficients.  Site forces are sums of G_ab times the pair vectors: the reference's
// per-term force sum regrouped.
//
// A block takes a contiguous run of the triple list, one triple at a time (SR, LR or both
// sweeps), so that consecutive triples of one molecule pair (i, j) reuse its ij tables.
#include "ccp_device.cuh"

// FS3 blocks resident per SM that the register allocation targets.
#ifndef CCP_FS3_MINBLOCKS
#define CCP_FS3_MINBLOCKS 2
#endif

using namespace ccpd;

namespace {

constexpr int kPairs = 289;
constexpr int kNt = 6;                     // FS3 site types
constexpr int kCoef = kNt * kNt * kNt * 8;
constexpr int kP = 18;                     // padded sites
constexpr int kRS = 19;                    // row stride of the site-pair tables
constexpr int kPassThreads = 96;           // 81 tiles per pair family, warp aligned
constexpr int kFs3Block = 320;             // 3 x 96 pass threads + one warp; 289 pair threads
constexpr int kRecWords = 18;              // doubles per triple record

__device__ __forceinline__ int pidx(int s) { return s == 0 ? 0 : s + 1; }
// Storage order of a padded index in the site-pair tables: even indices first, then odd,
// so the two rows (or columns) of a 2x2 output tile sit 9 rows apart and neighbouring
// tiles hit different shared-memory banks.
__host__ __device__ constexpr int sp(int x) { return (x & 1) * 9 + (x >> 1); }
// Coefficients in shared memory: the 8 of type triple (ti, tj, tk) start at double
// ti * kSi + tj * kSj + tk * kSk.  The strides keep entries 8 doubles apart and were chosen
// by enumerating the half-warp phases of the passes' coefficient loads under the tile order
// below: no two distinct entries read in one phase share a bank, except one phase in 19.
constexpr int kSi = 45, kSj = 325, kSk = 54;
constexpr int kCoefT = 5 * (kSi + kSj + kSk) + 8;  // doubles per SR / LR table

// Per-triple record written by the enumeration: COM vectors ij, ik, jk (bohr, computed as
// the reference computes them), their lengths, f_dmp, d f_dmp / d r (with the 1/3 of
// R_avg), the switch value and its derivative, the molecules and the R_avg branch.
struct Fs3Rec {
  double cv[3][3];
  double rr[3];
  double fdmp, dfdmp, smfun, cf;
  int mol[3];
  int branch;  // 0 SR, 1 LR, 2 blend
};
static_assert(sizeof(Fs3Rec) == kRecWords * 8, "record layout");

// ------------------------------------------------------------------ FS3 triples
// One block per molecule i: the candidates j > i from i's neighbour list that pass the
// reference's exact bohr cut-off test are staged in shared memory, then every pair
// (j < k) of them is tested with the reference's consistent-image j-k vector
// (threebody_potential.f90:860-892).  Accepted triples get a full record.
__global__ void k_fs3_enum(const double4 *__restrict__ comb, const int *__restrict__ nbr,
                           const int *__restrict__ ncnt, int cap, int nm, Fs3Params P,
                           Fs3Rec *rec, int tri_cap, int *icnt) {
  extern __shared__ unsigned char smem_raw[];
  int *lj = reinterpret_cast<int *>(smem_raw);
  double *lx = reinterpret_cast<double *>(lj + ((cap + 1) & ~1));
  double *ly = lx + cap, *lz = ly + cap;
  __shared__ int nl;
  __shared__ int wcount[32];
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
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
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
  const double b = P.boxb;
  // the pairs a < c of the staged candidates, by their index in row-major upper-triangle
  // order: row a starts at a L - a (a + 1) / 2
  const int npairs = L * (L - 1) / 2;
  for (int t = threadIdx.x; t < npairs; t += blockDim.x) {
    const double h = 2.0 * L - 1.0;
    int a = (int)floor(0.5 * (h - sqrt(h * h - 8.0 * t)));
    while (a > 0 && a * L - a * (a + 1) / 2 > t) a--;
    while ((a + 1) * L - (a + 1) * (a + 2) / 2 <= t) a++;
    const int c = t - (a * L - a * (a + 1) / 2) + a + 1;
    const int j = lj[a], k = lj[c];
    const double4 cj = comb[j], ck = comb[k];
    const double dxik = xsub(ci.x, ck.x), dyik = xsub(ci.y, ck.y), dzik = xsub(ci.z, ck.z);
    const double xik = minimg(dxik, b), yik = minimg(dyik, b), zik = minimg(dzik, b);
    const double dik2 = norm2x(xik, yik, zik);
    if (!(dik2 < P.rc2)) continue;
    // xjk = dxjk + box*nint(dxij/box) - box*nint(dxik/box)  (threebody_potential.f90:883-885)
    const double dxij = xsub(ci.x, cj.x), dyij = xsub(ci.y, cj.y), dzij = xsub(ci.z, cj.z);
    const double xjk = xsub(xadd(xsub(cj.x, ck.x), xmul(b, round(__ddiv_rn(dxij, b)))),
                            xmul(b, round(__ddiv_rn(dxik, b))));
    const double yjk = xsub(xadd(xsub(cj.y, ck.y), xmul(b, round(__ddiv_rn(dyij, b)))),
                            xmul(b, round(__ddiv_rn(dyik, b))));
    const double zjk = xsub(xadd(xsub(cj.z, ck.z), xmul(b, round(__ddiv_rn(dzij, b)))),
                            xmul(b, round(__ddiv_rn(dzik, b))));
    const double djk2 = norm2x(xjk, yjk, zjk);
    if (!(djk2 < P.rc2)) continue;
    const double dij2 = norm2x(lx[a], ly[a], lz[a]);
    const double rij = sqrt(dij2), rik = sqrt(dik2), rjk = sqrt(djk2);
    const double ravg = (rij + rjk + rik) / 3.0;  // threebody_potential.f90:894-898
    const int branch = ravg <= P.rmin ? 0 : (ravg >= P.rmax ? 1 : 2);
    if (branch == 2) atomicAdd(&icnt[C_NBLEND_FS3], 1);
    const int slot = atomicAdd(&icnt[C_NTRI_FS3], 1);
    if (slot >= tri_cap) continue;
    // global damping and switch (threebody_potential.f90:898-904, 1418-1423)
    const double pom = exp(P.alp3 * (ravg - P.r0dmp));
    const double ppom = 1.0 / (1.0 + pom);
    const double fdmp = pow(ppom, P.delta33);
    const double cfact = (ravg - P.rmin) / (P.rmax - P.rmin);
    Fs3Rec R;
    R.cv[0][0] = lx[a];
    R.cv[0][1] = ly[a];
    R.cv[0][2] = lz[a];
    R.cv[1][0] = xik;
    R.cv[1][1] = yik;
    R.cv[1][2] = zik;
    R.cv[2][0] = xjk;
    R.cv[2][1] = yjk;
    R.cv[2][2] = zjk;
    R.rr[0] = rij;
    R.rr[1] = rik;
    R.rr[2] = rjk;
    R.fdmp = fdmp;
    R.dfdmp = -P.alp3 * P.delta33 * pom * ppom * fdmp * (1.0 / 3.0);
    R.smfun = 1.0 + 2.0 * cfact * cfact * cfact - 3.0 * cfact * cfact;
    R.cf = 2.0 / (P.rmax - P.rmin) * (cfact * cfact - cfact);
    R.mol[0] = i;
    R.mol[1] = j;
    R.mol[2] = k;
    R.branch = branch;
    rec[slot] = R;
  }
}

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

// FP32 copy of the (e, e d) tables, read by the family-1 and family-2 passes of the mixed
// form; the FP64 form reads the FP64 tables and keeps no copy.
template <typename T>
struct LowUU {
  float2 v[3][kP][kRS];
};
template <>
struct LowUU<double> {
  char v[8];
};

// T is the arithmetic of the family-1 and family-2 passes.  The site-pair tables, the
// family-0 pass (whose outputs carry the energy sum) and everything after the passes are
// FP64 in both forms: the FS3 sum cancels heavily (sum |terms| / |sum| up to ~1e5), so an
// energy formed from FP32 tables or terms would carry ~1e-4 relative error into the energy
// and the R_avg-damping COM forces.
template <typename T>
struct Fs3Smem {
  double coef[2][kCoefT];    // SR, LR coefficients, strided layout (kSi, kSj, kSk)
  double bgr[2][3][kPairs];  // SR, LR b, g, r0 of each site pair
  double site[3][3][kNs3][3];  // site offsets (bohr) of i, j, k, per staging slot
  double2 uu[3][kP][kRS];    // (e, e d) of each site pair, families ij, ik, jk
  // force weights of each site pair: with P = q0 + d q1 the passes' output and l = d ln e / dr,
  // the weight G = e (l P + q1) / d is (e l / d) q0 + (e l + e / d) q1, so the table holds
  // (e l / d, e l + e / d) and the passes' epilogue needs no division; the parameter-gradient
  // form keeps (d, l)
  double2 dl[3][kP][kRS];
  LowUU<T> uul;              // FP32 copy of uu (mixed form)
  double G[2][3][kP][kRS];   // accumulated site-force weights, two triples in flight
  double red[kFs3Block / 32];
  Fs3Rec rec[3];             // staging slots: previous, current and next triple
};

// Extra shared memory of the parameter-gradient form: this block's partial sums of
// dS/d(coefficient table entry) and dS/d(b, g, r0), weighted like the energy, and the
// damping factor exp(-g (r - r0)) / (1 + exp(-g (r - r0))) of each site pair.
template <typename T>
struct Fs3Grad {
  double gc[2][kCoef];
  double gb[2][3][kPairs];
  double exd[3][kP][kRS];
};

template <typename T>
__host__ __device__ constexpr size_t fs3_grad_offset() {
  return (sizeof(Fs3Smem<T>) + 15) & ~size_t(15);
}

// One gradient pass for the 2x2 output tile (r0, r0+1) x (c0, c0+1), generic over the three
// pair families (one code path keeps the instruction footprint small):
//   fam 0: outputs (is, js), sum over ks: X = uu[ik][is][ks], Y = uu[jk][js][ks]
//   fam 1: outputs (is, ks), sum over js: X = uu[ij][is][js], Y = uu[jk][js][ks]
//   fam 2: outputs (js, ks), sum over is: X = uu[ij][is][js], Y = uu[ik][is][ks]
// X carries the powers of one distance, Y of another; the output pair carries the third.
// Offsets are in table elements of uu (physical rows/columns, see sp()).  Per type block of
// the summed site, M_u (u = 2x + y for X_x Y_y) is contracted with the type triple's
// coefficients: q0 with c[pa[u]] (power 0 of the output distance) and q1 with c[pb[u]], so
// that P = q0 + d q1 and dP/dd = q1.  Coefficient offsets are in doubles of the padded table.
struct PassCfg {
  int xb, xr, xs, yb, yr, ys, mr, mc, mb;
  int pa[4], pb[4];
};

__device__ __forceinline__ PassCfg pass_cfg(int fam) {
  constexpr int F = kP * kRS;
  PassCfg c;
  if (fam == 0) {  // coefficient (ti, tj, tk) = (row, col, sum)
    c = {1 * F, kRS, 1, 2 * F, kRS, 1, kSi, kSj, kSk, {0, 4, 2, 6}, {1, 5, 3, 7}};
  } else if (fam == 1) {  // (row, sum, col)
    c = {0, kRS, 1, 2 * F, 1, kRS, kSi, kSk, kSj, {0, 4, 1, 5}, {2, 6, 3, 7}};
  } else {  // (sum, row, col)
    c = {0, 1, kRS, 1 * F, 1, kRS, kSj, kSk, kSi, {0, 2, 1, 3}, {4, 6, 5, 7}};
  }
  return c;
}

// With GRAD and a family-0 pass (outputs are the ij pairs), gcv also receives, for each type
// block and power combination, wsite * sum_tile U_z(ij) M_u: the derivative of the sweep's
// energy sum with respect to that coefficient-table entry, index 4y + 2x + z.
// U is the (e, e d) table (3 families of kP x kRS entries) in the pass's arithmetic T.
template <typename T, bool GRAD>
__device__ __forceinline__ void fs3_pass(const typename Vec2<T>::type *U,
                                         const double *__restrict__ C, const PassCfg &g, int r0,
                                         int c0, T q0[4], T q1[4], double *gcv, double wsite) {
  using V2 = typename Vec2<T>::type;
  // site types of the padded indices: [0,2) [2,4) [4,6) [6,10) [10,14) [14,18)
  const int tr = r0 < 6 ? r0 >> 1 : (r0 + 6) >> 2, tc = c0 < 6 ? c0 >> 1 : (c0 + 6) >> 2;
  V2 Ut[4];
  if (GRAD && gcv) {
#pragma unroll
    for (int o = 0; o < 4; o++) Ut[o] = U[sp(r0 + (o >> 1)) * kRS + sp(c0 + (o & 1))];
  }
  const double *cbase = C + tr * g.mr + tc * g.mc;
  // physical rows/columns of the tile (r0, c0 even): sp(r0) = r0/2, sp(r0+1) = 9 + r0/2
  const V2 *X0 = U + g.xb + (r0 >> 1) * g.xr, *X1 = X0 + 9 * g.xr;
  const V2 *Y0 = U + g.yb + (c0 >> 1) * g.yr, *Y1 = Y0 + 9 * g.yr;
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
      const int pc = sp(c);
      const V2 X[2] = {X0[pc * g.xs], X1[pc * g.xs]};
      const V2 Y[2] = {Y0[pc * g.ys], Y1[pc * g.ys]};
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
    if (GRAD && gcv) {
      double *gt = gcv + ((tr * 6 + tc) * 6 + tb) * 8;
#pragma unroll
      for (int u = 0; u < 4; u++) {
        T b0 = (T)0, b1 = (T)0;
#pragma unroll
        for (int o = 0; o < 4; o++) {
          b0 += Ut[o].x * M[o][u];
          b1 += Ut[o].y * M[o][u];
        }
        const int pz0 = 4 * (u & 1) + 2 * (u >> 1);
        atomicAdd(gt + pz0, wsite * (double)b0);
        atomicAdd(gt + pz0 + 1, wsite * (double)b1);
      }
    }
    const double *cp = cbase + tb * g.mb;
    T ca[4], cb[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      ca[u] = (T)cp[g.pa[u]];
      cb[u] = (T)cp[g.pb[u]];
    }
#pragma unroll
    for (int o = 0; o < 4; o++) {
      q0[o] += ca[0] * M[o][0] + ca[1] * M[o][1] + ca[2] * M[o][2] + ca[3] * M[o][3];
      q1[o] += cb[0] * M[o][0] + cb[1] * M[o][1] + cb[2] * M[o][2] + cb[3] * M[o][3];
    }
  }
}

// The pair phase of one SR (v = 0) or LR (v = 1) sweep of the triple in staging slot `sl`:
// tabulate (e, e d) and the force-weight factors of its site pairs.  With keep_ij the ij
// family's tables already hold this molecule pair and variant (the previous sweep of the
// block had them) and are not tabulated again.  No barrier: the caller adds it.
template <typename T, bool GRAD>
__device__ __forceinline__ void fs3_pairs(Fs3Smem<T> &S, Fs3Grad<T> *GS, int v, int sl,
                                          bool keep_ij) {
  constexpr bool kLow = sizeof(T) == 4;
  const int tid = threadIdx.x;
  if (tid >= kPairs) return;
  const Fs3Rec &R = S.rec[sl];
  const double(*site)[kNs3][3] = S.site[sl];
  const int a = tid / kNs3, b = tid % kNs3;
  const double bb = S.bgr[v][0][tid], gg = S.bgr[v][1][tid], r0 = S.bgr[v][2][tid];
#pragma unroll 1
  for (int p = keep_ij ? 1 : 0; p < 3; p++) {
    const int m1 = p == 2 ? 1 : 0, m2 = p == 0 ? 1 : 2;
    const double vx = R.cv[p][0] + (site[m1][a][0] - site[m2][b][0]);
    const double vy = R.cv[p][1] + (site[m1][a][1] - site[m2][b][1]);
    const double vz = R.cv[p][2] + (site[m1][a][2] - site[m2][b][2]);
    const double r = sqrt(vx * vx + vy * vy + vz * vz);
    const double ex = exp(-gg * (r - r0));
    double2 u;
    if constexpr (GRAD) {
      const double damp = 1.0 / (1.0 + ex);
      const double e = exp(-bb * r) * damp;
      u = make_double2(e, e * r);
      S.dl[p][sp(pidx(a))][sp(pidx(b))] = make_double2(r, -bb + gg * ex * damp);
      GS->exd[p][sp(pidx(a))][sp(pidx(b))] = ex * damp;
    } else {
      // one division gives both the damping 1/(1+x) and 1/r
      const double t = 1.0 / ((1.0 + ex) * r);
      const double eor = exp(-bb * r) * t;  // e / r
      const double e = eor * r;
      const double dln = -bb + gg * ex * (t * r);
      u = make_double2(e, e * r);
      S.dl[p][sp(pidx(a))][sp(pidx(b))] = make_double2(eor * dln, e * dln + eor);
    }
    S.uu[p][sp(pidx(a))][sp(pidx(b))] = u;
    if constexpr (kLow) S.uul.v[p][sp(pidx(a))][sp(pidx(b))] = make_float2((float)u.x, (float)u.y);
  }
}

// The three gradient passes of the sweep whose tables the pair phase wrote: store (first
// sweep of the triple) or add wsite * G into the force-weight buffer G, and return the
// sweep's energy sum to every thread.  Ends with a barrier.
template <typename T, bool GRAD>
__device__ __forceinline__ double fs3_passes(Fs3Smem<T> &S, Fs3Grad<T> *GS, int v,
                                             double wsite, bool first,
                                             double (*G)[kP][kRS]) {
  constexpr bool kLow = sizeof(T) == 4;
  const int tid = threadIdx.x;
  double esum = 0.0;
  const int fam = tid / kPassThreads, lt = tid % kPassThreads;
  // 2x2 output tiles (R, C) of the 9 x 9 grid by quarter-warp: quarters 0..8 take row R and
  // columns 0..7, quarter 9 takes column 8 of rows 0..7 and the first lane of quarter 10 takes
  // (8, 8).  A quarter then reads at most 8 distinct rows or columns of a table, which its
  // row stride spreads over distinct banks.
  const int q8 = lt >> 3, i8 = lt & 7;
  const int R = q8 < 9 ? q8 : (q8 == 9 ? i8 : 8), Ct = q8 < 9 ? i8 : 8;
  if (fam < 3 && (q8 < 10 || (q8 == 10 && i8 == 0))) {
    const int r0 = 2 * R, c0 = 2 * Ct;
    const PassCfg g = pass_cfg(fam);
    const double *C = S.coef[v];
    double q0[4], q1[4];
    bool done = false;
    if constexpr (kLow) {
      if (fam != 0) {  // warp-uniform: 96 pass threads per family
        float f0[4], f1[4];
        fs3_pass<float, false>(&S.uul.v[0][0][0], C, g, r0, c0, f0, f1, nullptr, wsite);
#pragma unroll
        for (int o = 0; o < 4; o++) {
          q0[o] = f0[o];
          q1[o] = f1[o];
        }
        done = true;
      }
    }
    if (!done)
      fs3_pass<double, GRAD>(&S.uu[0][0][0], C, g, r0, c0, q0, q1,
                             (GRAD && fam == 0) ? GS->gc[v] : nullptr, wsite);
#pragma unroll
    for (int o = 0; o < 4; o++) {
      const int r = sp(r0 + (o >> 1)), c = sp(c0 + (o & 1));
      const double2 w = S.dl[fam][r][c];
      if constexpr (!GRAD) {
        if (fam == 0) {  // warp-uniform: only the ij family's outputs carry the energy
          const double2 u = S.uu[0][r][c];
          esum += u.x * q0[o] + u.y * q1[o];
        }
        const double gw = wsite * (w.x * q0[o] + w.y * q1[o]);
        if (first)
          G[fam][r][c] = gw;
        else
          G[fam][r][c] += gw;
        continue;
      }
      const double2 u = S.uu[fam][r][c];
      const double P = q0[o] + w.x * q1[o];
      if (fam == 0) esum += u.x * P;
      const double gw = wsite * (u.x * (w.y * P + q1[o]) / w.x);
      G[fam][r][c] = first ? gw : G[fam][r][c] + gw;
      const int ra = r0 + (o >> 1), cb = c0 + (o & 1);
      if (GRAD && ra != 1 && cb != 1) {
        // dS/de_ab = P; de/db = -r e, de/dg = (r - r0) e x, de/dr0 = -g e x with
        // x = exp(-g (r - r0)) / (1 + exp(-g (r - r0)))
        const int q = (ra == 0 ? 0 : ra - 1) * kNs3 + (cb == 0 ? 0 : cb - 1);
        const double wPe = wsite * P * u.x;
        const double rr = w.x, xd = GS->exd[fam][r][c];
        atomicAdd(&GS->gb[v][0][q], -wPe * rr);
        atomicAdd(&GS->gb[v][1][q], wPe * (rr - S.bgr[v][2][q]) * xd);
        atomicAdd(&GS->gb[v][2][q], -wPe * S.bgr[v][1][q] * xd);
      }
    }
  }
  esum = warp_sum(esum);
  if ((tid & 31) == 0) S.red[tid >> 5] = esum;
  __syncthreads();
  double tot = 0.0;
#pragma unroll
  for (int w = 0; w < kFs3Block / 32; w++) tot += S.red[w];
  // S.red is rewritten only after the next sweep's pair-phase barrier, which every thread
  // reaches after this read, so no barrier is needed here
  return tot;
}

// Stages the record and site offsets of triple t into slot sl: threads [kPairs, kFs3Block),
// which the pair phase leaves idle, copy the record and the 3 x 17 site offsets.
template <typename T>
__device__ __forceinline__ void fs3_stage(Fs3Smem<T> &S, const Fs3Rec *__restrict__ recs,
                                          const double4 *__restrict__ s17, int t, int sl) {
  const int u = (int)threadIdx.x - kPairs;
  if (u < 0) return;
  constexpr int kStagers = kFs3Block - kPairs;
  if (u < kRecWords)
    reinterpret_cast<double *>(&S.rec[sl])[u] = reinterpret_cast<const double *>(recs + t)[u];
  for (int k = u; k < 3 * kNs3; k += kStagers) {
    const int m = k / kNs3, s = k % kNs3;
    const double4 o = s17[(size_t)recs[t].mol[m] * kNs3 + s];
    S.site[sl][m][s][0] = o.x;
    S.site[sl][m][s][1] = o.y;
    S.site[sl][m][s][2] = o.z;
  }
}

// Site forces of the triple in slot sl from its force weights G (F = -sum_partner G * pair
// vector; 4 lanes per (molecule, site), each summing a quarter of the 17 partners, reduced
// with shuffles), the R_avg damping/switch COM forces (threebody_potential.f90:1092-1120,
// weight comc, by the block's last thread) and the triple's virial; returns this thread's
// share of the virial.
template <typename T>
__device__ __forceinline__ double fs3_forces(const Fs3Smem<T> &S, int sl,
                                             const double (*G)[kP][kRS], double comc, int nm,
                                             int ns, double *f, double *fc3) {
  const int tid = threadIdx.x;
  const double conv = kH2kcal * 418.4 / kBohr2a;
  const size_t nfs = (size_t)nm * ns;
  const Fs3Rec &R = S.rec[sl];
  const double(*site)[kNs3][3] = S.site[sl];
  double vsite = 0.0;
  {
    const int item = tid >> 2, part = tid & 3;
    const bool act = item < 3 * kNs3;
    const int m = act ? item / kNs3 : 0, s = act ? item % kNs3 : 0, ps = sp(pidx(s));
    const double(*cv)[3] = R.cv;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    // the item's two pair families ("links"): family, whether this molecule is the second
    // of the family's pair (then the weight is G[partner][this] and the pair vector points
    // from the partner's site), the partner molecule; the virial counts each molecular
    // pair once (ij and ik from molecule i, jk from molecule j)
    const int fa = m == 2 ? 1 : 0, fb = m == 0 ? 1 : 2;
    const bool ta = m != 0, tb = m == 2;
    const int pa = m == 0 ? 1 : 0, pb = m == 2 ? 1 : 2;
    const double sga = ta ? -1.0 : 1.0, sgb = tb ? -1.0 : 1.0;
    const double wva = m == 0 ? 1.0 : 0.0, wvb = m != 2 ? 1.0 : 0.0;
    if (act) {
      const double x0 = site[m][s][0], x1 = site[m][s][1], x2 = site[m][s][2];
      const double *ga_row = &G[fa][0][0], *gb_row = &G[fb][0][0];
#pragma unroll 1
      for (int o = part; o < kNs3; o += 4) {
        const int po = sp(pidx(o));
        const double ga = ga_row[ta ? po * kRS + ps : ps * kRS + po];
        const double gb = gb_row[tb ? po * kRS + ps : ps * kRS + po];
        // (this - partner) site offsets, negated for a transposed link: exact
        const double a0 = cv[fa][0] + sga * (x0 - site[pa][o][0]);
        const double a1 = cv[fa][1] + sga * (x1 - site[pa][o][1]);
        const double a2 = cv[fa][2] + sga * (x2 - site[pa][o][2]);
        const double b0 = cv[fb][0] + sgb * (x0 - site[pb][o][0]);
        const double b1 = cv[fb][1] + sgb * (x1 - site[pb][o][1]);
        const double b2 = cv[fb][2] + sgb * (x2 - site[pb][o][2]);
        const double sa = sga * ga, sb = sgb * gb;
        fx -= sa * a0 + sb * b0;
        fy -= sa * a1 + sb * b1;
        fz -= sa * a2 + sb * b2;
        vsite += wva * ga * (a0 * a0 + a1 * a1 + a2 * a2) + wvb * gb * (b0 * b0 + b1 * b1 + b2 * b2);
      }
    }
#pragma unroll
    for (int off = 1; off < 4; off <<= 1) {
      fx += __shfl_xor_sync(0xffffffffu, fx, off);
      fy += __shfl_xor_sync(0xffffffffu, fy, off);
      fz += __shfl_xor_sync(0xffffffffu, fz, off);
    }
    if (act && part == 0) {
      const size_t o = (size_t)R.mol[m] * ns + s;
      atomicAdd(&f[o], fx * conv);
      atomicAdd(&f[nfs + o], fy * conv);
      atomicAdd(&f[2 * nfs + o], fz * conv);
    }
  }
  if (tid == kFs3Block - 1) {
    const double(*cv)[3] = R.cv;
    const double rij = R.rr[0], rik = R.rr[1], rjk = R.rr[2];
    const double iij = 1.0 / rij, iik = 1.0 / rik, ijk = 1.0 / rjk;
    const double ux = cv[0][0] * iij, uy = cv[0][1] * iij, uz = cv[0][2] * iij;
    const double wx = cv[1][0] * iik, wy = cv[1][1] * iik, wz = cv[1][2] * iik;
    const double sx = cv[2][0] * ijk, sy = cv[2][1] * ijk, sz = cv[2][2] * ijk;
    const int m0 = R.mol[0], m1 = R.mol[1], m2 = R.mol[2];
    atomicAdd(&fc3[m0], -comc * (ux + wx) * conv);
    atomicAdd(&fc3[nm + m0], -comc * (uy + wy) * conv);
    atomicAdd(&fc3[2 * nm + m0], -comc * (uz + wz) * conv);
    atomicAdd(&fc3[m1], -comc * (-ux + sx) * conv);
    atomicAdd(&fc3[nm + m1], -comc * (-uy + sy) * conv);
    atomicAdd(&fc3[2 * nm + m1], -comc * (-uz + sz) * conv);
    atomicAdd(&fc3[m2], -comc * (-wx - sx) * conv);
    atomicAdd(&fc3[nm + m2], -comc * (-wy - sy) * conv);
    atomicAdd(&fc3[2 * nm + m2], -comc * (-wz - sz) * conv);
    vsite += comc * (rij + rik + rjk);
  }
  return vsite;
}

// The gradient form holds one block per SM (its shared memory), so it may use more registers.
//
// Per sweep the block runs two barrier-separated phases: A, the pair phase of the sweep
// (threads < 289) -- on a triple's first sweep together with the site and COM forces of the
// block's previous triple (threads < 204 and the last thread) and the staging of its next
// triple (threads >= 289) -- and B, the three passes.  The force weights G alternate between
// two buffers by triple, and records and site offsets rotate through three staging slots, so
// that the previous triple's forces, this triple's tables and the next triple's staging
// never touch the same memory.
//
// The molecules may come in frames of frame_nm (the independent boxes of a batch, one list
// of triples): a frame's energy, virial and parameter-gradient sums go to scal + frame *
// scal_stride and gfs3 + frame * kFs3GradLen, flushed whenever a block's run of triples
// crosses into the next frame.  frame_nm = nm for a single box.
template <typename T, bool GRAD>
__global__ void __launch_bounds__(kFs3Block, GRAD ? 1 : CCP_FS3_MINBLOCKS)
    k_fs3(const Fs3Rec *__restrict__ recs, const int *__restrict__ icnt, int tri_cap,
          const double4 *__restrict__ s17, const double *__restrict__ coef,
          const double *__restrict__ bgr, int nm, int ns, double *f, double *fc3, double *scal,
          double *gfs3, int frame_nm, int scal_stride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Fs3Smem<T> &S = *reinterpret_cast<Fs3Smem<T> *>(smem_raw);
  Fs3Grad<T> *GS = GRAD ? reinterpret_cast<Fs3Grad<T> *>(smem_raw + fs3_grad_offset<T>()) : nullptr;
  const int tid = threadIdx.x;
  // each block takes a contiguous run of the triple list: the enumeration writes the triples
  // of one molecule pair (i, j) next to each other, so consecutive triples often share the
  // ij site-pair tables
  const int ntri = min(icnt[C_NTRI_FS3], tri_cap);
  const int chunk = (ntri + (int)gridDim.x - 1) / (int)gridDim.x;
  const int t_begin = (int)blockIdx.x * chunk, t_end = min(t_begin + chunk, ntri);
  if (t_begin >= t_end) return;  // no triple for this block
  if (GRAD) {
    for (int t = tid; t < 2 * kCoef; t += kFs3Block) (&GS->gc[0][0])[t] = 0.0;
    for (int t = tid; t < 2 * 3 * kPairs; t += kFs3Block) (&GS->gb[0][0][0])[t] = 0.0;
    for (int t = tid; t < 3 * kP * kRS; t += kFs3Block) (&GS->exd[0][0][0])[t] = 0.0;
  }
  for (int t = tid; t < 2 * kCoefT; t += kFs3Block) (&S.coef[0][0])[t] = 0.0;
  __syncthreads();
  for (int t = tid; t < 2 * kCoef / 2; t += kFs3Block) {
    const int v = t / (kCoef / 2), r = t % (kCoef / 2);
    const int tri = r / 4, j = r % 4;  // type triple ti*36 + tj*6 + tk, pair j of 4
    const int ti = tri / 36, tj = (tri / 6) % 6, tk = tri % 6;
    const double *src = coef + (size_t)v * kCoef + tri * 8 + 2 * j;
    double *dst = &S.coef[v][ti * kSi + tj * kSj + tk * kSk + 2 * j];
    dst[0] = src[0];
    dst[1] = src[1];
  }
  for (int t = tid; t < 2 * 3 * kPairs; t += kFs3Block) (&S.bgr[0][0][0])[t] = bgr[t];
  // padded dummy site: zero weight, unit distance (keeps e / d finite)
  for (int t = tid; t < 3 * kP; t += kFs3Block) {
    const int p = t / kP, q = t % kP;
    const double2 z = make_double2(0.0, 0.0), one = make_double2(GRAD ? 1.0 : 0.0, 0.0);
    S.uu[p][sp(1)][q] = z;
    S.uu[p][q][sp(1)] = z;
    S.dl[p][sp(1)][q] = one;
    S.dl[p][q][sp(1)] = one;
    if constexpr (sizeof(T) == 4) {
      S.uul.v[p][sp(1)][q] = make_float2(0.f, 0.f);
      S.uul.v[p][q][sp(1)] = make_float2(0.f, 0.f);
    }
  }
  fs3_stage(S, recs, s17, t_begin, 0);
  __syncthreads();
  CompSum e_tot, v_tot;  // this thread's energy and virial over the block's triples
  int have_i = -1, have_j = -1, have_v = -1;  // molecule pair and variant of the ij tables
  double comc_prev = 0.0;                     // COM-force weight of the previous triple
  int frame = S.rec[0].mol[0] / frame_nm;     // frame of the sums being accumulated
  // adds this block's sums of `frame` to its slots and clears them (every thread calls it;
  // the parameter-gradient table is complete: the last passes ended with a barrier, and the
  // next ones start after the next one)
  auto flush = [&]() {
    const double vt = warp_sum(v_tot.value()), et = warp_sum(e_tot.value());
    if ((tid & 31) == 0) {
      atomicAdd(&scal[(size_t)frame * scal_stride + S_FS3_VIR], vt);
      if (et != 0.0) atomicAdd(&scal[(size_t)frame * scal_stride + S_FS3_E], et);
    }
    v_tot = CompSum();
    e_tot = CompSum();
    if (GRAD) {
      double *gf = gfs3 + (size_t)frame * kFs3GradLen;
      for (int u = tid; u < 2 * kCoef; u += kFs3Block) {
        double &g = (&GS->gc[0][0])[u];
        if (g != 0.0) atomicAdd(&gf[u], g);
        g = 0.0;
      }
      for (int u = tid; u < 2 * 3 * kPairs; u += kFs3Block) {
        double &g = (&GS->gb[0][0][0])[u];
        if (g != 0.0) atomicAdd(&gf[2 * kCoef + u], g);
        g = 0.0;
      }
    }
  };
  for (int t = t_begin; t < t_end; t++) {
    const int k = t - t_begin, sl = k % 3, sl_prev = (k + 2) % 3, sl_next = (k + 1) % 3;
    const Fs3Rec &R = S.rec[sl];
    const double fdmp = R.fdmp, dfdmp = R.dfdmp;
    const int br = R.branch;
    const bool same_ij = R.mol[0] == have_i && R.mol[1] == have_j;
    have_i = R.mol[0];
    have_j = R.mol[1];
    // one sweep (SR or LR branch) or two (blend); of two, the one whose ij tables are already
    // in place goes first.  One call site keeps the kernel's instruction footprint small.
    const double smfun = R.smfun, smfun2 = 1.0 - smfun;
    const int nsweep = br == 2 ? 2 : 1;
    const bool lr_first = br == 2 && same_ij && have_v == 1;
    double Ssr = 0.0, Slr = 0.0;
#pragma unroll 1
    for (int w = 0; w < nsweep; w++) {
      const int v = br != 2 ? br : ((w == 0) == lr_first ? 1 : 0);
      const double ws = br != 2 ? fdmp : fdmp * (v == 0 ? smfun : smfun2);
      if (w == 0) {
        if (k > 0) v_tot.add(fs3_forces(S, sl_prev, S.G[(k - 1) & 1], comc_prev, nm, ns, f, fc3));
        if (R.mol[0] / frame_nm != frame) {  // the previous triple closed its frame's sums
          flush();
          frame = R.mol[0] / frame_nm;
        }
        if (t + 1 < t_end) fs3_stage(S, recs, s17, t + 1, sl_next);
      }
      fs3_pairs<T, GRAD>(S, GS, v, sl, w == 0 && same_ij && have_v == v);
      __syncthreads();
      const double Sv = fs3_passes<T, GRAD>(S, GS, v, ws, w == 0, S.G[k & 1]);
      if (v == 0)
        Ssr = Sv;
      else
        Slr = Sv;
      have_v = v;
    }
    if (br != 2) {
      const double Sv = br == 0 ? Ssr : Slr;
      if (tid == kFs3Block - 1) e_tot.add(fdmp * Sv);
      comc_prev = dfdmp * Sv;
    } else {
      const double cf = R.cf;
      if (tid == kFs3Block - 1) e_tot.add(fdmp * (smfun * Ssr + smfun2 * Slr));
      comc_prev = Ssr * (dfdmp * smfun + fdmp * cf) + Slr * (dfdmp * smfun2 - fdmp * cf);
    }
  }
  // the forces of the block's last triple (its G and slot are final after the last barrier)
  v_tot.add(fs3_forces(S, (t_end - 1 - t_begin) % 3, S.G[(t_end - 1 - t_begin) & 1], comc_prev,
                       nm, ns, f, fc3));
  if (GRAD) __syncthreads();  // every pass's atomics into the gradient table are done
  flush();
}

// Triples and blend-region triples of each frame (counts[2 f], counts[2 f + 1]).
__global__ void k_fs3_frame_counts(const Fs3Rec *__restrict__ recs, const int *__restrict__ icnt,
                                   int tri_cap, int frame_nm, int *counts) {
  const int ntri = min(icnt[C_NTRI_FS3], tri_cap);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntri; t += gridDim.x * blockDim.x) {
    const int fr = recs[t].mol[0] / frame_nm;
    atomicAdd(&counts[2 * fr], 1);
    if (recs[t].branch == 2) atomicAdd(&counts[2 * fr + 1], 1);
  }
}

}  // namespace

size_t fs3_record_bytes() { return sizeof(Fs3Rec); }

namespace {
// Persistent grid (one wave of resident blocks) when triples_per_block is 0; otherwise
// enough short blocks for the list's capacity, about triples_per_block triples each, so
// that blocks retire often and other streams' kernels can take their slots.
int fs3_grid(int resident, int tri_cap, int triples_per_block) {
  if (triples_per_block <= 0) return resident;
  const int g = (tri_cap + triples_per_block - 1) / triples_per_block;
  return g < 1 ? 1 : g;
}
}  // namespace

cudaError_t launch_fs3_enum(const double4 *comb, const int *nbr, const int *ncnt, int cap,
                            int nm, Fs3Params P, void *rec, int tri_cap, int *icnt,
                            cudaStream_t st) {
  const size_t smem = sizeof(int) * (size_t)((cap + 1) & ~1) + 3 * sizeof(double) * (size_t)cap;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_fs3_enum, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_fs3_enum<<<nm, 128, smem, st>>>(comb, nbr, ncnt, cap, nm, P, static_cast<Fs3Rec *>(rec),
                                    tri_cap, icnt);
  return cudaGetLastError();
}

namespace {
template <typename T, bool GRAD>
cudaError_t launch_fs3_t(const Fs3Rec *R, const int *icnt, int tri_cap, const double4 *s17,
                         const double *coef, const double *bgr, int nm, int ns, double *f,
                         double *fc3, double *scal, int nsm, int triples_per_block,
                         int blocks_per_sm, double *gfs3, int frame_nm, int scal_stride,
                         cudaStream_t st) {
  const size_t smem = GRAD ? fs3_grad_offset<T>() + sizeof(Fs3Grad<T>) : sizeof(Fs3Smem<T>);
  cudaError_t e = cudaFuncSetAttribute(k_fs3<T, GRAD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fs3<T, GRAD>, kFs3Block, smem);
  if (per_sm < 1) per_sm = 1;
  // the gradient form flushes per-block partial sums: a persistent grid keeps them few
  int grid = fs3_grid(nsm * per_sm, tri_cap, GRAD ? 0 : triples_per_block);
  // a cap makes the grid persistent on fewer slots, leaving the rest to concurrent kernels
  if (blocks_per_sm > 0 && blocks_per_sm < per_sm && grid > nsm * blocks_per_sm)
    grid = nsm * blocks_per_sm;
  k_fs3<T, GRAD><<<grid, kFs3Block, smem, st>>>(R, icnt, tri_cap, s17, coef, bgr, nm, ns, f, fc3,
                                                scal, gfs3, frame_nm, scal_stride);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_fs3_frame_counts(const void *rec, const int *icnt, int tri_cap, int frame_nm,
                                    int *counts, cudaStream_t st) {
  k_fs3_frame_counts<<<148 * 4, 256, 0, st>>>(static_cast<const Fs3Rec *>(rec), icnt, tri_cap,
                                              frame_nm, counts);
  return cudaGetLastError();
}

cudaError_t launch_fs3(int precision, const void *rec, const int *icnt, int tri_cap,
                       const double4 *s17, const double *coef, const double *bgr, int nm, int ns,
                       double *f, double *fc3, double *scal, int nsm, int triples_per_block,
                       int blocks_per_sm, double *gfs3, cudaStream_t st, int frame_nm,
                       int scal_stride) {
  const Fs3Rec *R = static_cast<const Fs3Rec *>(rec);
  if (frame_nm <= 0) frame_nm = nm;
  if (precision == 0) {
    if (gfs3)
      return launch_fs3_t<double, true>(R, icnt, tri_cap, s17, coef, bgr, nm, ns, f, fc3, scal,
                                        nsm, triples_per_block, blocks_per_sm, gfs3, frame_nm,
                                        scal_stride, st);
    return launch_fs3_t<double, false>(R, icnt, tri_cap, s17, coef, bgr, nm, ns, f, fc3, scal, nsm,
                                       triples_per_block, blocks_per_sm, nullptr, frame_nm,
                                       scal_stride, st);
  }
  if (gfs3)
    return launch_fs3_t<float, true>(R, icnt, tri_cap, s17, coef, bgr, nm, ns, f, fc3, scal, nsm,
                                     triples_per_block, blocks_per_sm, gfs3, frame_nm,
                                     scal_stride, st);
  return launch_fs3_t<float, false>(R, icnt, tri_cap, s17, coef, bgr, nm, ns, f, fc3, scal, nsm,
                                    triples_per_block, blocks_per_sm, nullptr, frame_nm,
                                    scal_stride, st);
}
