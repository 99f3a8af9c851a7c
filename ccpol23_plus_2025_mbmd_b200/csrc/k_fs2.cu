// k_fs2.cu -- FS2 nonadditive three-body kernel (sm_100a).
//
// FS2 (threebody_potential.f90:101-674): the exchange quadrupole of a pair (i, j),
// eta exp(-beta r) over the 3x3 O/H site pairs, interacting with the five 3-body charges of
// a spectator k, with long-range dampings of the two spectator distances.  The nine
// exchange terms of a pair do not depend on the spectator, so one warp per pair (i < j)
// computes them once; its lanes then test i's neighbours against both cut-offs, queue the
// spectators that pass, and evaluate them 32 at a time.
#include "ccp_device.cuh"

using namespace ccpd;

namespace {

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
__constant__ float kCharge3bf[5] = {0.258504607653328389f, 0.564050362569283648f,
                                    0.564050362569283648f, -0.693302666395947953f,
                                    -0.693302666395947953f};

// Mixed form: one spectator site ks of charge q seen from the pair, in FP32.  The FS2 terms
// are differences between the spectator's interaction with the pair's centres and with the
// exchange charges displaced by d = -+ g3 r_ij/|r_ij| (threebody_potential.f90:392-583), and
// formed literally they cancel to ~1e-3 of their parts.  Here every difference is formed from
// the displacement itself, with c the spectator site seen from a centre, e = c + d from the
// exchange charge, ic = 1/|c|, ie = 1/|e| and dl = |e|^2 - |c|^2 = d.(2c + d):
//   1/|c| - 1/|e| = dl ic^2 ie^2 / (ic + ie)                                (= D)
//   e/|e|^3 - c/|c|^3 = d ie^3 - D (ie^2 + ie ic + ic^2) c                  (= G)
// so the FP32 terms keep ~1e-7 relative accuracy.
struct Fs2Side {
  float D, ie3;   // 1/|c| - 1/|e| and 1/|e|^3
  float3 G, e;    // e/|e|^3 - c/|c|^3 and e
};
__device__ __forceinline__ Fs2Side fs2_side(float cx, float cy, float cz, float dx, float dy,
                                            float dz) {
  Fs2Side r;
  const float ex = cx + dx, ey = cy + dy, ez = cz + dz;
  const float ic = rsqrtf(cx * cx + cy * cy + cz * cz);
  const float ie = rsqrtf(ex * ex + ey * ey + ez * ez);
  const float dl = dx * (2.0f * cx + dx) + dy * (2.0f * cy + dy) + dz * (2.0f * cz + dz);
  const float ic2 = ic * ic, ie2 = ie * ie;
  r.D = dl * ic2 * ie2 / (ic + ie);
  r.ie3 = ie2 * ie;
  const float w = r.D * (ie2 + ie * ic + ic2);
  r.G = make_float3(dx * r.ie3 - w * cx, dy * r.ie3 - w * cy, dz * r.ie3 - w * cz);
  r.e = make_float3(ex, ey, ez);
  return r;
}

// 4 blocks (16 warps) per SM: 128 registers a thread, against 154 unbounded.  LOW: the mixed
// form, whose spectator terms run in FP32 (fs2_side) with per-spectator sums promoted into
// the FP64 accumulators; the pair's exchange sums, the cut-off tests and every accumulation
// across spectators stay FP64.
template <bool LOW>
__global__ void __launch_bounds__(128, 4)
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
  CompSum e_loc, v_loc;  // this lane's energy and virial over its spectators
  double A_loc = 0.0;
  double Ci[3] = {0, 0, 0}, Cj[3] = {0, 0, 0};
  int nspec = 0;
  // One spectator k that passed both cut-offs: its five 3-body charges against the pair's
  // exchange quadrupole.
  auto spectator = [&](int k) {
    const double4 ck = comb[k];
    const double xki = minimg(xsub(ck.x, ci.x), P.boxb);
    const double yki = minimg(xsub(ck.y, ci.y), P.boxb);
    const double zki = minimg(xsub(ck.z, ci.z), P.boxb);
    const double xkj = xadd(xki, xij), ykj = xadd(yki, yij), zkj = xadd(zki, zij);
    const double dki2 = norm2x(xki, yki, zki), dkj2 = norm2x(xkj, ykj, zkj);
    const double sdki = sqrt(dki2), sdkj = sqrt(dkj2);
    // flr = (1 / (1 + pom))^delta33, formed as exp(-delta33 log1p(pom))
    double pom = exp(P.alp3 * (sdki - P.r0dmp));
    const double pomki = 1.0 / (1.0 + pom);
    const double flrki = exp(-P.delta33 * log1p(pom));
    const double dflrki = -P.alp3 * P.delta33 * pom * pomki * flrki;
    const double dflrkiv = -P.alp3 * P.delta33 * pom * pomki * sdki;
    pom = exp(P.alp3 * (sdkj - P.r0dmp));
    const double pomkj = 1.0 / (1.0 + pom);
    const double flrkj = exp(-P.delta33 * log1p(pom));
    const double dflrkj = -P.alp3 * P.delta33 * pom * pomkj * flrkj;
    const double dflrkjv = -P.alp3 * P.delta33 * pom * pomkj * sdkj;
    const double fl = flrki * flrkj;
    const double cki = dflrki * flrkj / sdki, ckj = dflrkj * flrki / sdkj;
    nspec++;
    double ck_x = 0, ck_y = 0, ck_z = 0;  // COM force on k
    for (int ks = 0; ks < 5; ks++) {
      const double qks = kCharge3b[ks];
      const double4 sk = s17[(size_t)k * kNs3 + ks];
      const double dxkqi = xki + sk.x - g3 * xij * dij1i;
      const double dykqi = yki + sk.y - g3 * yij * dij1i;
      const double dzkqi = zki + sk.z - g3 * zij * dij1i;
      const double dkqi1i = rsqrt(dxkqi * dxkqi + dykqi * dykqi + dzkqi * dzkqi);
      const double dkqi3i = dkqi1i * dkqi1i * dkqi1i;
      const double dxkqj = xkj + sk.x + g3 * xij * dij1i;
      const double dykqj = ykj + sk.y + g3 * yij * dij1i;
      const double dzkqj = zkj + sk.z + g3 * zij * dij1i;
      const double dkqj1i = rsqrt(dxkqj * dxkqj + dykqj * dykqj + dzkqj * dzkqj);
      const double dkqj3i = dkqj1i * dkqj1i * dkqj1i;
      const double dxkci = xki + sk.x, dykci = yki + sk.y, dzkci = zki + sk.z;
      const double dkci1i = rsqrt(dxkci * dxkci + dykci * dykci + dzkci * dzkci);
      const double dkci3i = dkci1i * dkci1i * dkci1i;
      const double dxkcj = xkj + sk.x, dykcj = ykj + sk.y, dzkcj = zkj + sk.z;
      const double dkcj1i = rsqrt(dxkcj * dxkcj + dykcj * dykcj + dzkcj * dzkcj);
      const double dkcj3i = dkcj1i * dkcj1i * dkcj1i;
      const double term0 = dkci1i + dkcj1i - dkqi1i - dkqj1i;
      const double qE = qks * E;
      e_loc.add(qE * term0 * fl);
      const double termxy1 = (dxkqi * xij + dykqi * yij + dzkqi * zij) * g3 * dij1i * dkqi3i;
      const double termxy2 = (dxkqj * xij + dykqj * yij + dzkqj * zij) * g3 * dij1i * dkqj3i;
      v_loc.add((qks * Ev + (dflrkiv + dflrkjv) * qE) * term0 * fl + qE * (termxy1 - termxy2) * fl);
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
      const double tki = qE * term0 * cki;
      const double tkj = qE * term0 * ckj;
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
  };
  // The same spectator in FP32 (mixed form); identical terms, regrouped as in fs2_side.
  auto spectator32 = [&](int k) {
    const double4 ck = comb[k];
    const double xki = minimg(xsub(ck.x, ci.x), P.boxb);
    const double yki = minimg(xsub(ck.y, ci.y), P.boxb);
    const double zki = minimg(xsub(ck.z, ci.z), P.boxb);
    const float kix = (float)xki, kiy = (float)yki, kiz = (float)zki;
    const float kjx = (float)xadd(xki, xij), kjy = (float)xadd(yki, yij),
                kjz = (float)xadd(zki, zij);
    const float alp3 = (float)P.alp3, r0 = (float)P.r0dmp, d33 = (float)P.delta33;
    const float sdki = sqrtf(kix * kix + kiy * kiy + kiz * kiz);
    const float sdkj = sqrtf(kjx * kjx + kjy * kjy + kjz * kjz);
    float pom = expf(alp3 * (sdki - r0));
    const float pomki = 1.0f / (1.0f + pom);
    const float flrki = expf(-d33 * log1pf(pom));
    const float dflrki = -alp3 * d33 * pom * pomki * flrki;
    const float dflrkiv = -alp3 * d33 * pom * pomki * sdki;
    pom = expf(alp3 * (sdkj - r0));
    const float pomkj = 1.0f / (1.0f + pom);
    const float flrkj = expf(-d33 * log1pf(pom));
    const float dflrkj = -alp3 * d33 * pom * pomkj * flrkj;
    const float dflrkjv = -alp3 * d33 * pom * pomkj * sdkj;
    const float fl = flrki * flrkj;
    const float cki = dflrki * flrkj / sdki, ckj = dflrkj * flrki / sdkj;
    nspec++;
    const float rx = (float)xij, ry = (float)yij, rz = (float)zij;
    const float g = (float)g3, r1 = (float)dij1i, r3 = (float)dij3i;
    const float hx = g * rx * r1, hy = g * ry * r1, hz = g * rz * r1;  // g3 r_ij / |r_ij|
    const float Ef = (float)E, Evf = (float)Ev;
    float e_s = 0.f, v_s = 0.f, a_s = 0.f, ckx = 0.f, cky = 0.f, ckz = 0.f;
    float cix = 0.f, ciy = 0.f, ciz = 0.f, cjx = 0.f, cjy = 0.f, cjz = 0.f;
    for (int ks = 0; ks < 5; ks++) {
      const float qks = kCharge3bf[ks];
      const double4 sk = s17[(size_t)k * kNs3 + ks];
      const float skx = (float)sk.x, sky = (float)sk.y, skz = (float)sk.z;
      // from i's centre with the exchange charge at -g3 r^; from j's at +g3 r^
      const Fs2Side A = fs2_side(kix + skx, kiy + sky, kiz + skz, -hx, -hy, -hz);
      const Fs2Side B = fs2_side(kjx + skx, kjy + sky, kjz + skz, hx, hy, hz);
      const float term0 = A.D + B.D;
      const float qE = qks * Ef;
      e_s += qE * term0 * fl;
      const float dqi = rx * A.e.x + ry * A.e.y + rz * A.e.z;
      const float dqj = rx * B.e.x + ry * B.e.y + rz * B.e.z;
      const float h = dqi * A.ie3 - dqj * B.ie3;
      const float Hx = A.e.x * A.ie3 - B.e.x * B.ie3, Hy = A.e.y * A.ie3 - B.e.y * B.ie3,
                  Hz = A.e.z * A.ie3 - B.e.z * B.ie3;
      v_s += (qks * Evf + (dflrkiv + dflrkjv) * qE) * term0 * fl + qE * g * r1 * h * fl;
      a_s += qks * term0 * fl;
      // spectator site force
      const float fkx = qE * (A.G.x + B.G.x), fky = qE * (A.G.y + B.G.y),
                  fkz = qE * (A.G.z + B.G.z);
      const size_t so = (size_t)k * ns + ks;
      atomicAdd(&f[so], (double)(-fkx * fl) * conv);
      atomicAdd(&f[nfs + so], (double)(-fky * fl) * conv);
      atomicAdd(&f[2 * nfs + so], (double)(-fkz * fl) * conv);
      const float tki = qE * term0 * cki, tkj = qE * term0 * ckj;
      ckx += -tki * kix - tkj * kjx;
      cky += -tki * kiy - tkj * kjy;
      ckz += -tki * kiz - tkj * kjz;
      const float gh = g * r1, gh3 = g * r3 * h;
      const float fxi = qE * (-A.G.x - gh * Hx + gh3 * rx), fyi = qE * (-A.G.y - gh * Hy + gh3 * ry),
                  fzi = qE * (-A.G.z - gh * Hz + gh3 * rz);
      const float fxj = qE * (-B.G.x + gh * Hx - gh3 * rx), fyj = qE * (-B.G.y + gh * Hy - gh3 * ry),
                  fzj = qE * (-B.G.z + gh * Hz - gh3 * rz);
      cix += -fxi * fl + tki * kix;
      ciy += -fyi * fl + tki * kiy;
      ciz += -fzi * fl + tki * kiz;
      cjx += -fxj * fl + tkj * kjx;
      cjy += -fyj * fl + tkj * kjy;
      cjz += -fzj * fl + tkj * kjz;
    }
    e_loc.add((double)e_s);
    v_loc.add((double)v_s);
    A_loc += (double)a_s;
    Ci[0] += (double)cix;
    Ci[1] += (double)ciy;
    Ci[2] += (double)ciz;
    Cj[0] += (double)cjx;
    Cj[1] += (double)cjy;
    Cj[2] += (double)cjz;
    atomicAdd(&fc2[k], (double)ckx * conv);
    atomicAdd(&fc2[nm + k], (double)cky * conv);
    atomicAdd(&fc2[2 * nm + k], (double)ckz * conv);
  };
  // The spectators are i's neighbours k != j within the cut-off of both i and j; only a
  // fraction pass, so the warp first queues them (ballot + prefix into shared memory) and
  // evaluates them 32 at a time with every lane busy.
  __shared__ int kq_all[4][64];
  int *kq = kq_all[threadIdx.x >> 5];
  const unsigned below = (1u << lane) - 1u;
  int nq = 0, n0 = 0;
  const int cnt = ncnt[i];
  for (;;) {
    // fill the queue to 32 (or to the end of the list), then evaluate up to 32 spectators;
    // one call site keeps the kernel small
    while (nq < 32 && n0 < cnt) {
      const int n = n0 + lane;
      bool pass = false;
      int k = 0;
      if (n < cnt) {
        k = nbr[(size_t)i * cap + n];
        if (k != j) {
          const double4 ck = comb[k];
          const double xki = minimg(xsub(ck.x, ci.x), P.boxb);
          const double yki = minimg(xsub(ck.y, ci.y), P.boxb);
          const double zki = minimg(xsub(ck.z, ci.z), P.boxb);
          const double xkj = xadd(xki, xij), ykj = xadd(yki, yij), zkj = xadd(zki, zij);
          pass = norm2x(xki, yki, zki) < P.rc2 && norm2x(xkj, ykj, zkj) < P.rc2;
        }
      }
      const unsigned bal = __ballot_sync(0xffffffffu, pass);
      if (pass) kq[nq + __popc(bal & below)] = k;
      nq += __popc(bal);
      n0 += 32;
      __syncwarp();
    }
    if (nq == 0) break;
    if (lane < nq) {
      if constexpr (LOW)
        spectator32(kq[lane]);
      else
        spectator(kq[lane]);
    }
    __syncwarp();
    if (lane < nq - 32) kq[lane] = kq[32 + lane];
    nq = nq > 32 ? nq - 32 : 0;
    __syncwarp();
  }
  const double e_w = warp_sum(e_loc.value()), v_w = warp_sum(v_loc.value());
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
    atomicAdd(&scal[S_FS2_E], e_w);
    atomicAdd(&scal[S_FS2_VIR], v_w);
  }
  for (int o = 16; o > 0; o >>= 1) nspec += __shfl_xor_sync(0xffffffffu, nspec, o);
  if (lane == 0 && nspec) atomicAdd(ncomb, nspec);
}

}  // namespace

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
  // one warp per pair; the pair count is on the device, so launch for the capacity and
  // let surplus warps exit at once.
  const int warps = pair_cap;
  const int threads = 128;
  const int blocks = (warps * 32 + threads - 1) / threads;
  int *nc = const_cast<int *>(icnt) + C_NTRI_FS2;
  if (precision == 1)  // CCP_MIXED
    k_fs2<true><<<blocks, threads, 0, st>>>(pairs, icnt, pair_cap, comb, s17, nbr, ncnt, cap, P,
                                            nm, ns, f, fc2, scal, nc);
  else
    k_fs2<false><<<blocks, threads, 0, st>>>(pairs, icnt, pair_cap, comb, s17, nbr, ncnt, cap, P,
                                             nm, ns, f, fc2, scal, nc);
  return cudaGetLastError();
}
