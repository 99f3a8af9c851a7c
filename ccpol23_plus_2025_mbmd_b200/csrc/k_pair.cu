// k_pair.cu -- molecule-pair kernels of the hot path (sm_100a, FP64).
//
// One warp owns one molecule i and walks i's neighbour list; every quantity it produces
// belongs to i's own sites, so site forces and fields are written without atomics.  Each
// unordered pair is therefore visited from both sides; energies and virials are counted
// on the side with j > i only, which reproduces the reference's `do j = i+1, nm` sums.
// Only "active" sites enter (charged or polarisable): the reference loops over all 28x28
// site pairs, but every other pair multiplies by a zero charge and a zero dipole.
#include "ccp_device.cuh"

using namespace ccpd;

namespace {

__device__ __forceinline__ double4 ld4(const double4 *p) { return *p; }

// ------------------------------------------------------------------------ prep
__global__ void k_prep(const double *__restrict__ x, const double *__restrict__ y,
                       const double *__restrict__ z, const double *__restrict__ xs,
                       const double *__restrict__ ys, const double *__restrict__ zs, int nm,
                       int ld, SiteSets S, double4 *com, double4 *act, double4 *comb,
                       double4 *s17, int ns3, double *f, int nf, double *fc2, double *fc3,
                       double *scal, int *icnt) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int stride = gridDim.x * blockDim.x;
  // one thread per molecule, per (molecule, active site) and per (molecule, FS site): the
  // conversions to bohr are divisions, as the reference forms them
  bool bad = false;  // a coordinate that is not finite (NaN or infinite)
  for (int i = t; i < nm; i += stride) {
    bad |= !(isfinite(x[i]) && isfinite(y[i]) && isfinite(z[i]));
    com[i] = make_double4(x[i], y[i], z[i], 0.0);
    comb[i] = make_double4(x[i] / kBohr2a, y[i] / kBohr2a, z[i] / kBohr2a, 0.0);
    fc2[i] = fc2[nm + i] = fc2[2 * nm + i] = 0.0;
    fc3[i] = fc3[nm + i] = fc3[2 * nm + i] = 0.0;
  }
  for (int u = t; u < nm * S.na; u += stride) {
    const int i = u / S.na, a = u - i * S.na;
    const size_t o = (size_t)i * ld + S.asite[a];
    bad |= !(isfinite(xs[o]) && isfinite(ys[o]) && isfinite(zs[o]));
    act[u] = make_double4(xs[o], ys[o], zs[o], S.q[a]);
  }
  for (int u = t; u < nm * ns3; u += stride) {
    const int i = u / ns3, s = u - i * ns3;
    const size_t o = (size_t)i * ld + s;
    bad |= !(isfinite(xs[o]) && isfinite(ys[o]) && isfinite(zs[o]));
    s17[(size_t)i * kNs3 + s] = make_double4(xs[o] / kBohr2a, ys[o] / kBohr2a, zs[o] / kBohr2a, 0.0);
  }
  if (bad) atomicAdd(&icnt[C_NONFINITE], 1);
  for (int k = t; k < nf; k += stride) f[k] = 0.0;
  if (t < S_COUNT) scal[t] = 0.0;
  if (t < C_COUNT) icnt[t] = 0;
}

// ------------------------------------------------------------------- neighbours
// One block per molecule i: candidates j != i with the reference's minimum-image COM
// vector (computed exactly as the reference does) and |r|^2 < rlist2, written in
// increasing j.  The molecules come in frames of frame_nm (independent boxes of one batch;
// frame_nm = nm for a single box): the candidates of i are the molecules of its own frame.
__global__ void k_neighbors(const double4 *__restrict__ com, int nm, int frame_nm, double box,
                            double rlist2, int cap, int *nbr, double4 *nbrv, int *ncnt,
                            int *icnt) {
  __shared__ int warp_tot[32];
  __shared__ int base;
  const int i = blockIdx.x;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  const double4 ci = com[i];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int jb = (i / frame_nm) * frame_nm, je = min(jb + frame_nm, nm);
  for (int j0 = jb; j0 < je; j0 += blockDim.x) {
    int j = j0 + threadIdx.x;
    bool keep = false;
    double4 v;
    if (j < je && j != i) {
      double4 cj = com[j];
      double xcc = minimg(xsub(ci.x, cj.x), box);
      double ycc = minimg(xsub(ci.y, cj.y), box);
      double zcc = minimg(xsub(ci.z, cj.z), box);
      double r2 = norm2x(xcc, ycc, zcc);
      v = make_double4(xcc, ycc, zcc, r2);
      keep = r2 < rlist2;
    }
    unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) warp_tot[wid] = __popc(bal);
    __syncthreads();
    int off = base;
    for (int w = 0; w < wid; w++) off += warp_tot[w];
    int pos = off + __popc(bal & ((1u << lane) - 1u));
    if (keep) {
      if (pos < cap) {
        nbr[(size_t)i * cap + pos] = j;
        nbrv[(size_t)i * cap + pos] = v;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int w = 0; w < nw; w++) tot += warp_tot[w];
      base += tot;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    ncnt[i] = base < cap ? base : cap;
    if (base > cap) atomicMax(&icnt[C_OVERFLOW], base);
  }
}

// ------------------------------------------------------------ cell-list neighbours
// For boxes of at least five cells of side >= rlist/2 per axis: molecules are binned by their
// wrapped centre, and molecule i's candidates are the members of the 5 x 5 x 5 cells around
// its own (two cells of side >= rlist/2 on either side cover every centre within rlist under
// the minimum image, and five distinct cells per axis visit none twice).  Each candidate gets
// the same exact minimum-image test as in k_neighbors, and the kept ones are written in
// increasing j, so the list equals k_neighbors' entry for entry.
constexpr int kStencil = 125;

__device__ __forceinline__ int cell_axis(double x, double box, double side, int nc) {
  const double p = x - box * floor(x / box);
  int c = (int)(p / side);
  return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

__global__ void k_cell_assign(const double4 *__restrict__ com, int nm, double box, int nc,
                              int *cell_of, int *count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nm) return;
  const double side = box / nc;
  const double4 c = com[i];
  const int cell = (cell_axis(c.z, box, side, nc) * nc + cell_axis(c.y, box, side, nc)) * nc +
                   cell_axis(c.x, box, side, nc);
  cell_of[i] = cell;
  atomicAdd(&count[cell], 1);
}

// One block: exclusive scan of the cell counts into start[0..ncells] and cursor[0..ncells).
__global__ void __launch_bounds__(1024) k_cell_scan(int ncells, const int *__restrict__ count,
                                                    int *start, int *cursor) {
  __shared__ int part[1024];
  const int per = (ncells + 1023) / 1024;
  const int c0 = min(ncells, (int)threadIdx.x * per), c1 = min(ncells, c0 + per);
  int sum = 0;
  for (int c = c0; c < c1; c++) sum += count[c];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const int v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int o = part[threadIdx.x] - sum;
  for (int c = c0; c < c1; c++) {
    start[c] = o;
    cursor[c] = o;
    o += count[c];
  }
  if (threadIdx.x == 1023) start[ncells] = part[1023];
}

__global__ void k_cell_fill(int nm, const int *__restrict__ cell_of, int *cursor, int *members) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nm) members[atomicAdd(&cursor[cell_of[i]], 1)] = i;
}

// One block per molecule i; dynamic shared memory holds up to `cap` kept candidates.
__global__ void k_neighbors_cells(const double4 *__restrict__ com, int nm, double box,
                                  double rlist2, int cap, int nc, const int *__restrict__ cell_of,
                                  const int *__restrict__ start, const int *__restrict__ members,
                                  int *nbr, double4 *nbrv, int *ncnt, int *icnt) {
  extern __shared__ unsigned char smem_raw[];
  double4 *kv = reinterpret_cast<double4 *>(smem_raw);
  int *kj = reinterpret_cast<int *>(kv + cap);
  __shared__ int cs[kStencil], pre[kStencil + 1];
  __shared__ int nkept;
  const int i = blockIdx.x;
  const int t = threadIdx.x;
  const int c = cell_of[i];
  if (t < kStencil) {
    const int cx = c % nc, cy = (c / nc) % nc, cz = c / (nc * nc);
    const int dx = t % 5 - 2, dy = (t / 5) % 5 - 2, dz = t / 25 - 2;
    const int cell = (((cz + dz + nc) % nc) * nc + (cy + dy + nc) % nc) * nc + (cx + dx + nc) % nc;
    cs[t] = start[cell];
    pre[t + 1] = start[cell + 1] - start[cell];
  }
  if (t == 0) {
    nkept = 0;
    pre[0] = 0;
  }
  __syncthreads();
  if (t == 0)
    for (int k = 0; k < kStencil; k++) pre[k + 1] += pre[k];
  __syncthreads();
  const int total = pre[kStencil];
  const double4 ci = com[i];
  for (int e = t; e < total; e += blockDim.x) {
    int lo = 0, hi = kStencil;  // pre[lo] <= e < pre[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (pre[mid] <= e)
        lo = mid;
      else
        hi = mid;
    }
    const int j = members[cs[lo] + (e - pre[lo])];
    if (j == i) continue;
    const double4 cj = com[j];
    const double xcc = minimg(xsub(ci.x, cj.x), box);
    const double ycc = minimg(xsub(ci.y, cj.y), box);
    const double zcc = minimg(xsub(ci.z, cj.z), box);
    const double r2 = norm2x(xcc, ycc, zcc);
    if (!(r2 < rlist2)) continue;
    const int pos = atomicAdd(&nkept, 1);
    if (pos < cap) {
      kj[pos] = j;
      kv[pos] = make_double4(xcc, ycc, zcc, r2);
    }
  }
  __syncthreads();
  const int n = nkept, m = n < cap ? n : cap;
  // rank of each kept j among the kept (the j are distinct): increasing j
  for (int e = t; e < m; e += blockDim.x) {
    const int j = kj[e];
    int r = 0;
    for (int q = 0; q < m; q++) r += kj[q] < j;
    nbr[(size_t)i * cap + r] = j;
    nbrv[(size_t)i * cap + r] = kv[e];
  }
  if (t == 0) {
    ncnt[i] = m;
    if (n > cap) atomicMax(&icnt[C_OVERFLOW], n);
  }
}

// ------------------------------------------- Ewald real space + static field (real+TT)
// rspace_ewald (ewald.f90:177-405), rspace_efield_stat (nb_induction_model.f90:128-293),
// shortrange_efield_stat_damped (nb_induction_model.f90:5454-5629) and, with `with_self`,
// the intramolecular terms of ewald_self_correction (ewald.f90:101-147) and self_efield_stat
// (nb_induction_model.f90:977-1115).
//
// One block per molecule i, one warp per row: rows [0, nq) are i's charged sites (Ewald
// forces on them), rows [nq, nq + np) its polarisable sites (static field at them).  The 32
// lanes of a row stride over i's neighbours, so no warp mixes the two kinds of row, and the
// rows x 32 threads of every molecule keep enough warps resident to hide the latency of the
// erfc/exp chains.  The intramolecular pairs of a row go to its lanes (one partner each).
template <int R>
__global__ void __launch_bounds__(R * 32)
    k_pair_static(const double *__restrict__ x, const double *__restrict__ y,
                  const double *__restrict__ z, const double *__restrict__ xs,
                  const double *__restrict__ ys, const double *__restrict__ zs, int ld,
                  const double4 *__restrict__ act, const int *__restrict__ nbr,
                  const double4 *__restrict__ nbrv, const int *__restrict__ ncnt, int cap,
                  int nm, SiteSets S, EwaldParams P, double *f, double *e0r, double *e0s,
                  int with_self, double *fself, double *e0slf, double *scal) {
  __shared__ double red[R][4];
  const int i = blockIdx.x;
  const int row = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nq = S.nq, np = S.np, na = S.na, ns = S.ns;
  const bool qrow = row < nq, live = row < nq + np;
  const double alp = P.alpha;
  // row sums: a = force (charge row) or real-space field (polarisable row), b = short-range
  // field, s = intramolecular force or field
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, b0 = 0.0, b1 = 0.0, b2 = 0.0;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, e = 0.0, v = 0.0, sff = 0.0, svir = 0.0;
  if (live) {
    const int ai = qrow ? S.a_of_q[row] : S.a_of_p[row - nq];
    const double4 si = ld4(&act[(size_t)i * na + ai]);
    const int cnt = ncnt[i];
    for (int n = lane; n < cnt; n += 32) {
      const double4 c = ld4(&nbrv[(size_t)i * cap + n]);
      if (!(c.w < P.rcutsd)) continue;
      const int j = nbr[(size_t)i * cap + n];
      const bool half = j > i;
      for (int b = 0; b < nq; b++) {
        const double4 sj = ld4(&act[(size_t)j * na + S.a_of_q[b]]);
        if (qrow) {
          const double rx = (c.x + si.x) - sj.x;
          const double ry = (c.y + si.y) - sj.y;
          const double rz = (c.z + si.z) - sj.z;
          const double rssq = rx * rx + ry * ry + rz * rz;
          const double ri = rsqrt(rssq), drr = rssq * ri;
          const double ec = erfc(alp * drr);
          const double qq = kR4pie0 * si.w * sj.w;
          const double ad = alp * drr;
          const double fc = qq * (ec * ri + P.twosqpi * alp * exp(-(ad * ad)));
          const double cf = fc * (ri * ri);
          const double fx = rx * cf, fy = ry * cf, fz = rz * cf;
          a0 += fx;
          a1 += fy;
          a2 += fz;
          if (half) {
            e += qq * ec * ri;
            v -= rx * fx + ry * fy + rz * fz;
          }
        } else {
          const double qj = sj.w;
          const double dx = c.x + (si.x - sj.x);
          const double dy = c.y + (si.y - sj.y);
          const double dz = c.z + (si.z - sj.z);
          const double d2 = dx * dx + dy * dy + dz * dz;
          const double ri = rsqrt(d2), dist = d2 * ri;
          const double ad = alp * dist;
          const double expar2 = exp(-(ad * ad));
          const double d1i = erfc(alp * dist) * ri;
          const double d2i = ri * ri;
          const double d3i = d2i * (d1i + P.twosqpi * alp * expar2);
          a0 += qj * dx * d3i;
          a1 += qj * dy * d3i;
          a2 += qj * dz * d3i;
          if (P.damped) {
            const double r3 = ri * ri * ri;
            const double g = (tt<2>(P.delta2, dist) - 1.0) * qj * r3;
            b0 += g * dx;
            b1 += g * dy;
            b2 += g * dz;
          }
        }
      }
    }
    // intramolecular terms, as the reference forms them: (x + xs_a) - (x + xs_b), so that
    // coincident sites give exactly zero
    if (with_self) {
      const double xi = x[i], yi = y[i], zi = z[i];
      if (qrow) {
        const int b = lane;
        if (b < nq && b != row) {
          const int sa = S.qsite[row], sb = S.qsite[b];
          const double chg = S.q[S.a_of_q[row]] * S.q[S.a_of_q[b]];
          const size_t oa = (size_t)i * ld + sa, ob = (size_t)i * ld + sb;
          const double dx = (xi + xs[oa]) - (xi + xs[ob]);
          const double dy = (yi + ys[oa]) - (yi + ys[ob]);
          const double dz = (zi + zs[oa]) - (zi + zs[ob]);
          const double drr = sqrt(dx * dx + dy * dy + dz * dz);
          const double ef = erf(alp * drr);
          const double ad = alp * drr;
          const double fs = -kR4pie0 * chg *
                            (ef / (drr * drr * drr) - P.twosqpi * alp * exp(-(ad * ad)) / (drr * drr));
          s0 = dx * fs;
          s1 = dy * fs;
          s2 = dz * fs;
          if (row < b) {  // each unordered pair once, as the reference's a < b loop
            sff = ef * chg / drr;
            svir = -(dx * s0 + dy * s1 + dz * s2);
          }
        }
      } else if (lane < S.nself_q) {
        const int bq = S.self_q[lane];
        const int sp = S.psite[row - nq], sb = S.qsite[bq];
        const double qj = S.q[S.a_of_q[bq]];
        const size_t op = (size_t)i * ld + sp, ob = (size_t)i * ld + sb;
        const double dx = (xi + xs[op]) - (xi + xs[ob]);
        const double dy = (yi + ys[op]) - (yi + ys[ob]);
        const double dz = (zi + zs[op]) - (zi + zs[ob]);
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 != 0.0) {
          const double drr = sqrt(d2);
          const double d1i = 1.0 / drr, d2i = d1i * d1i, d3i = d2i * d1i;
          const double ad = alp * drr;
          const double g = erf(alp * drr) * d3i - P.twosqpi * alp * exp(-(ad * ad)) * d2i;
          s0 = -qj * dx * g;
          s1 = -qj * dy * g;
          s2 = -qj * dz * g;
        }
      }
    }
  }
  a0 = warp_sum(a0);
  a1 = warp_sum(a1);
  a2 = warp_sum(a2);
  b0 = warp_sum(b0);
  b1 = warp_sum(b1);
  b2 = warp_sum(b2);
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  e = warp_sum(e);
  v = warp_sum(v);
  sff = warp_sum(sff);
  svir = warp_sum(svir);
  if (lane == 0) {
    if (live) {
      const size_t nfs = (size_t)nm * ns;
      if (qrow) {
        const size_t o = (size_t)i * ns + S.qsite[row];
        f[o] += a0;
        f[nfs + o] += a1;
        f[2 * nfs + o] += a2;
        if (with_self) {
          fself[o] += s0;
          fself[nfs + o] += s1;
          fself[2 * nfs + o] += s2;
        }
      } else {
        const size_t o = ((size_t)i * np + (row - nq)) * 3;
        e0r[o] = a0;
        e0r[o + 1] = a1;
        e0r[o + 2] = a2;
        e0s[o] = b0;
        e0s[o + 1] = b1;
        e0s[o + 2] = b2;
        if (with_self) {
          e0slf[o] = s0;
          e0slf[o + 1] = s1;
          e0slf[o + 2] = s2;
        }
      }
    }
    red[row][0] = e;
    red[row][1] = v;
    red[row][2] = sff;
    red[row][3] = svir;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double te = 0.0, tv = 0.0, tf = 0.0, ts = 0.0;
    for (int r = 0; r < R; r++) {
      te += red[r][0];
      tv += red[r][1];
      tf += red[r][2];
      ts += red[r][3];
    }
    atomicAdd(&scal[S_RC_E], te);
    atomicAdd(&scal[S_RC_VIR], tv);
    if (with_self) {
      atomicAdd(&scal[S_SELF_SUMFF], tf);
      atomicAdd(&scal[S_SELF_VIR], ts);
    }
  }
}
// --------------------------------------------- intramolecular static terms (per molecule)
// ewald_self_correction intramolecular part (ewald.f90:101-147) and self_efield_stat
// (nb_induction_model.f90:977-1115).  Both use (x + xs_a) - (x + xs_b), as the reference
// does, so coincident sites give exactly zero and are skipped.
__global__ void k_self_static(const double *__restrict__ x, const double *__restrict__ y,
                              const double *__restrict__ z, const double *__restrict__ xs,
                              const double *__restrict__ ys, const double *__restrict__ zs,
                              int nm, int ld, SiteSets S, EwaldParams P, double *f,
                              double *e0slf, double *scal) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double sumff = 0.0, vir = 0.0;
  if (i < nm) {
    const double alp = P.alpha;
    const size_t nfs = (size_t)nm * S.ns;
    const double xi = x[i], yi = y[i], zi = z[i];
    for (int a = 0; a < S.nq; a++) {
      for (int b = a + 1; b < S.nq; b++) {
        const int sa = S.qsite[a], sb = S.qsite[b];
        const double chg = S.q[S.a_of_q[a]] * S.q[S.a_of_q[b]];
        const size_t oa = (size_t)i * ld + sa, ob = (size_t)i * ld + sb;
        const double dx = (xi + xs[oa]) - (xi + xs[ob]);
        const double dy = (yi + ys[oa]) - (yi + ys[ob]);
        const double dz = (zi + zs[oa]) - (zi + zs[ob]);
        const double drr = sqrt(dx * dx + dy * dy + dz * dz);
        const double ef = erf(alp * drr);
        sumff += ef * chg / drr;
        const double ad = alp * drr;
        const double fs = -kR4pie0 * chg *
                          (ef / (drr * drr * drr) - P.twosqpi * alp * exp(-(ad * ad)) / (drr * drr));
        const double fx = dx * fs, fy = dy * fs, fz = dz * fs;
        const size_t ca = (size_t)i * S.ns + sa, cb = (size_t)i * S.ns + sb;
        f[ca] += fx;
        f[nfs + ca] += fy;
        f[2 * nfs + ca] += fz;
        f[cb] -= fx;
        f[nfs + cb] -= fy;
        f[2 * nfs + cb] -= fz;
        vir -= dx * fx + dy * fy + dz * fz;
      }
    }
    for (int p = 0; p < S.np; p++) {
      const int sp = S.psite[p];
      double E[3] = {0.0, 0.0, 0.0};
      for (int u = 0; u < S.nself_q; u++) {
        const int b = S.self_q[u];
        const int sb = S.qsite[b];
        const double qj = S.q[S.a_of_q[b]];
        const size_t op = (size_t)i * ld + sp, ob = (size_t)i * ld + sb;
        const double dx = (xi + xs[op]) - (xi + xs[ob]);
        const double dy = (yi + ys[op]) - (yi + ys[ob]);
        const double dz = (zi + zs[op]) - (zi + zs[ob]);
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 == 0.0) continue;
        const double drr = sqrt(d2);
        const double d1i = 1.0 / drr, d2i = d1i * d1i, d3i = d2i * d1i;
        const double ad = alp * drr;
        const double g = erf(alp * drr) * d3i - P.twosqpi * alp * exp(-(ad * ad)) * d2i;
        E[0] -= qj * dx * g;
        E[1] -= qj * dy * g;
        E[2] -= qj * dz * g;
      }
      for (int k = 0; k < 3; k++) e0slf[((size_t)i * S.np + p) * 3 + k] = E[k];
    }
  }
  sumff = warp_sum(sumff);
  vir = warp_sum(vir);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&scal[S_SELF_SUMFF], sumff);
    atomicAdd(&scal[S_SELF_VIR], vir);
  }
}

// ------------------------------------------------------------ induction forces (real)
// real_forces (nb_induction_model.f90:3069-3631), shortrange_forces_damped (:5975-6557)
// and self_forces (:4841-5360).  Force on active site a of i from active site b of j:
//   F = q_a E_b(r_a) + (mu_a . grad) E_b(r_a),
// with the field/gradient of charge q_b and dipole mu_b in the reference's screened
// (erfc) and Tang-Toennies short-range forms, contracted as the reference contracts
// them.  The virial of a pair is -d . F, counted from the i < j side.
struct IndPair {
  double fx, fy, fz;
};

__device__ __forceinline__ void ind_pair(double dx, double dy, double dz, double qa,
                                         double max, double may, double maz, bool pa, double qb,
                                         double mbx, double mby, double mbz, bool pb,
                                         const EwaldParams &P, IndPair &out) {
  const double alp = P.alpha, alp3 = alp * alp * alp, alp5 = alp3 * alp * alp;
  const double d2 = dx * dx + dy * dy + dz * dz;
  const double d1i = rsqrt(d2), dist = d2 * d1i, d2i = d1i * d1i, d3i = d2i * d1i;
  const double d4i = d2i * d2i, d5i = d3i * d2i, d6i = d3i * d3i, d7i = d5i * d2i;
  const double ad = alp * dist;
  const double expar2 = exp(-(ad * ad));
  const double ec = erfc(alp * dist);
  const double ts = P.twosqpi;
  const double d3ii = ec * d3i + ts * alp * expar2 * d2i;
  const double d5ii = ec * d5i + ts * alp * expar2 * d4i + (2.0 / 3.0) * ts * alp3 * expar2 * d2i;
  const double d7ii = ec * d7i + ts * alp * expar2 * d6i + (2.0 / 3.0) * ts * alp3 * expar2 * d4i +
                      (4.0 / 15.0) * ts * alp5 * expar2 * d2i;
  const double doti = max * dx + may * dy + maz * dz;
  const double dotj = mbx * dx + mby * dy + mbz * dz;
  const double mm = max * mbx + may * mby + maz * mbz;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  // screened part: q_a E_mu_b + mu_a . grad (E_q_b + E_mu_b)
  if (pb && qa != 0.0) {
    const double s = 3.0 * d5ii * dotj;
    fx += qa * (s * dx - mbx * d3ii);
    fy += qa * (s * dy - mby * d3ii);
    fz += qa * (s * dz - mbz * d3ii);
  }
  if (pa) {
    // sum_x m_x G[x][y] = qb(-3 d5 doti d_y + m_y d3) - 15 d7 doti dotj d_y
    //                      + 3 d5 (m_y dotj + mm d_y + mb_y doti)
    const double c1 = -3.0 * qb * d5ii * doti - 15.0 * d7ii * doti * dotj + 3.0 * d5ii * mm;
    fx += c1 * dx + qb * max * d3ii + 3.0 * d5ii * (max * dotj + mbx * doti);
    fy += c1 * dy + qb * may * d3ii + 3.0 * d5ii * (may * dotj + mby * doti);
    fz += c1 * dz + qb * maz * d3ii + 3.0 * d5ii * (maz * dotj + mbz * doti);
  }
  if (P.damped) {
    const double f2 = tt<2>(P.delta2, dist), f3 = tt<3>(P.delta3, dist);
    const double df2 = dtt<2>(P.delta2, dist), df3 = dtt<3>(P.delta3, dist);
    if (pb && qa != 0.0) {
      const double s1 = (f2 - 1.0) * 3.0 * d5i * dotj - dotj * d3i * df2 * d1i;
      fx += qa * (s1 * dx - (f2 - 1.0) * mbx * d3i);
      fy += qa * (s1 * dy - (f2 - 1.0) * mby * d3i);
      fz += qa * (s1 * dz - (f2 - 1.0) * mbz * d3i);
    }
    if (pa) {
      // sum_c m_c g[x][c], g[x][c] = dE_c/dx of the short-range correction field
      const double c1 = (f2 - 1.0) * qb * (-3.0 * d5i * doti) + qb * doti * d3i * df2 * d1i +
                        (f3 - 1.0) * (-15.0 * dotj * d7i * doti + 3.0 * d5i * mm) +
                        (3.0 * doti * dotj * d5i - mm * d3i) * df3 * d1i;
      const double g2 = (f2 - 1.0) * qb * d3i;
      const double g3 = (f3 - 1.0) * 3.0 * d5i;
      fx += c1 * dx + g2 * max + g3 * (max * dotj + mbx * doti);
      fy += c1 * dy + g2 * may + g3 * (may * dotj + mby * doti);
      fz += c1 * dz + g2 * maz + g3 * (maz * dotj + mbz * doti);
    }
  }
  out.fx = fx;
  out.fy = fy;
  out.fz = fz;
}

// One block per molecule i, one warp per active site a of i (a row); the lanes of a row
// stride over i's neighbours and take one intramolecular partner each.
template <int R>
__global__ void __launch_bounds__(R * 32)
    k_pair_indforce(const double *__restrict__ x, const double *__restrict__ y,
                    const double *__restrict__ z, const double *__restrict__ xs,
                    const double *__restrict__ ys, const double *__restrict__ zs, int ld,
                    const double4 *__restrict__ act, const int *__restrict__ nbr,
                    const double4 *__restrict__ nbrv, const int *__restrict__ ncnt, int cap,
                    int nm, SiteSets S, EwaldParams P, const double *__restrict__ mu,
                    double *f, double *scal) {
  __shared__ double red[R];
  const int i = blockIdx.x;
  const int a = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int na = S.na, np = S.np;
  const bool live = a < na;
  double fx = 0.0, fy = 0.0, fz = 0.0, vir = 0.0;
  double qa = 0.0, max = 0.0, may = 0.0, maz = 0.0;
  if (live) {
    const double4 sa = ld4(&act[(size_t)i * na + a]);
    qa = sa.w;
    const int pai = S.p_of_a[a];
    const bool pa = pai >= 0;
    if (pa) {
      max = mu[((size_t)i * np + pai) * 3 + 0];
      may = mu[((size_t)i * np + pai) * 3 + 1];
      maz = mu[((size_t)i * np + pai) * 3 + 2];
    }
    const int cnt = ncnt[i];
    for (int n = lane; n < cnt; n += 32) {
      const double4 c = ld4(&nbrv[(size_t)i * cap + n]);
      if (!(c.w < P.rcutsd)) continue;
      const int j = nbr[(size_t)i * cap + n];
      const bool half = j > i;
      for (int b = 0; b < na; b++) {
        const int pbi = S.p_of_a[b];
        const bool pb = pbi >= 0;
        if (!pa && !(pb && qa != 0.0)) continue;
        const double4 sb = ld4(&act[(size_t)j * na + b]);
        double mbx = 0.0, mby = 0.0, mbz = 0.0;
        if (pb) {
          mbx = mu[((size_t)j * np + pbi) * 3 + 0];
          mby = mu[((size_t)j * np + pbi) * 3 + 1];
          mbz = mu[((size_t)j * np + pbi) * 3 + 2];
        }
        const double dx = c.x + (sa.x - sb.x);
        const double dy = c.y + (sa.y - sb.y);
        const double dz = c.z + (sa.z - sb.z);
        IndPair r;
        ind_pair(dx, dy, dz, qa, max, may, maz, pa, sb.w, mbx, mby, mbz, pb, P, r);
        fx += r.fx;
        fy += r.fy;
        fz += r.fz;
        if (half) vir -= dx * r.fx + dy * r.fy + dz * r.fz;
      }
    }
    // intramolecular (self_forces): lane w takes site a's side of the pair (a, w), with
    // d = (x + xs_a) - (x + xs_w); the pair's virial is counted once, on the a < w side
    const int w = lane;
    if (w < na && w != a) {
      const double alp = P.alpha, alp3 = alp * alp * alp, alp5 = alp3 * alp * alp;
      const double xi = x[i], yi = y[i], zi = z[i];
      const size_t oa = (size_t)i * ld + S.asite[a], ow = (size_t)i * ld + S.asite[w];
      const double ex = (xi + xs[oa]) - (xi + xs[ow]);
      const double ey = (yi + ys[oa]) - (yi + ys[ow]);
      const double ez = (zi + zs[oa]) - (zi + zs[ow]);
      const double d2 = ex * ex + ey * ey + ez * ez;
      if (d2 != 0.0) {
        const double drr = sqrt(d2);
        const double d1i = 1.0 / drr, d2i = d1i * d1i, d3i = d2i * d1i, d4i = d2i * d2i;
        const double d5i = d3i * d2i, d6i = d3i * d3i, d7i = d6i * d1i;
        const double ad = alp * drr;
        const double expar2 = exp(-(ad * ad));
        const double ef = erf(alp * drr);
        const double ts = P.twosqpi;
        // erf-screened kernels of the intramolecular correction (negated interactions)
        const double d3ii = ef * d3i - ts * alp * expar2 * d2i;
        const double d5ii = ef * d5i - ts * alp * expar2 * d4i - (2.0 / 3.0) * ts * alp3 * expar2 * d2i;
        const double d7ii = ef * d7i - ts * alp * expar2 * d6i - (2.0 / 3.0) * ts * alp3 * expar2 * d4i -
                            (4.0 / 15.0) * ts * alp5 * expar2 * d2i;
        const double4 sw = ld4(&act[(size_t)i * na + w]);
        const double qw = sw.w;
        const int pwi = S.p_of_a[w];
        double mwx = 0.0, mwy = 0.0, mwz = 0.0;
        if (pwi >= 0) {
          mwx = mu[((size_t)i * np + pwi) * 3 + 0];
          mwy = mu[((size_t)i * np + pwi) * 3 + 1];
          mwz = mu[((size_t)i * np + pwi) * 3 + 2];
        }
        const double doti = max * ex + may * ey + maz * ez;
        const double dotj = mwx * ex + mwy * ey + mwz * ez;
        const double mm = max * mwx + may * mwy + maz * mwz;
        // field E = -(3 d5 dotj e - mw d3); gradient = -(qw(...) + dipole part)
        const double s = 3.0 * d5ii * dotj;
        double gx = -qa * (s * ex - mwx * d3ii), gy = -qa * (s * ey - mwy * d3ii),
               gz = -qa * (s * ez - mwz * d3ii);
        const double c1 = -3.0 * qw * d5ii * doti - 15.0 * d7ii * doti * dotj + 3.0 * d5ii * mm;
        gx -= c1 * ex + qw * max * d3ii + 3.0 * d5ii * (max * dotj + mwx * doti);
        gy -= c1 * ey + qw * may * d3ii + 3.0 * d5ii * (may * dotj + mwy * doti);
        gz -= c1 * ez + qw * maz * d3ii + 3.0 * d5ii * (maz * dotj + mwz * doti);
        fx += gx;
        fy += gy;
        fz += gz;
        if (a < w) vir -= ex * gx + ey * gy + ez * gz;
      }
    }
  }
  fx = warp_sum(fx);
  fy = warp_sum(fy);
  fz = warp_sum(fz);
  vir = warp_sum(vir);
  if (lane == 0) {
    if (live) {
      // point self terms: field += selffac mu, gradient diagonal -= selffac q
      const double alp = P.alpha, alp3 = alp * alp * alp;
      const double selffac = 4.0 * alp3 / (3.0 * sqrt(kPi));
      const double px = qa * selffac * max - selffac * qa * max;
      const double py = qa * selffac * may - selffac * qa * may;
      const double pz = qa * selffac * maz - selffac * qa * maz;
      const size_t nfs = (size_t)nm * S.ns;
      const size_t o = (size_t)i * S.ns + S.asite[a];
      f[o] += kR4pie0 * (fx + px);
      f[nfs + o] += kR4pie0 * (fy + py);
      f[2 * nfs + o] += kR4pie0 * (fz + pz);
    }
    red[a] = vir;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int r = 0; r < R; r++) t += red[r];
    atomicAdd(&scal[S_IND_VIR_R], kR4pie0 * t);
  }
}

}  // namespace

// ------------------------------------------------------------------ launchers
namespace {
__global__ void k_add(int n, const double *__restrict__ a, double *b) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    b[t] += a[t];
}
}  // namespace

cudaError_t launch_add(int n, const double *a, double *b, cudaStream_t st) {
  int blocks = (n + 255) / 256;
  if (blocks > 4 * 148) blocks = 4 * 148;
  if (blocks < 1) blocks = 1;
  k_add<<<blocks, 256, 0, st>>>(n, a, b);
  return cudaGetLastError();
}

cudaError_t launch_prep(const double *x, const double *y, const double *z, const double *xs,
                        const double *ys, const double *zs, int nm, int ld, SiteSets S,
                        double4 *com, double4 *act, double4 *comb, double4 *s17, int ns3,
                        double *f, int nf, double *fc2, double *fc3, double *scal,
                        int *icnt, cudaStream_t st) {
  int threads = 256;
  int blocks = (nf + threads - 1) / threads;
  if (blocks < 1) blocks = 1;
  if (blocks > 4 * 148) blocks = 4 * 148;
  k_prep<<<blocks, threads, 0, st>>>(x, y, z, xs, ys, zs, nm, ld, S, com, act, comb, s17, ns3,
                                     f, nf, fc2, fc3, scal, icnt);
  return cudaGetLastError();
}

cudaError_t launch_neighbors(const double4 *com, int nm, double box, double rlist2, int cap,
                             int *nbr, double4 *nbrv, int *ncnt, int *icnt, cudaStream_t st,
                             int frame_nm) {
  k_neighbors<<<nm, 128, 0, st>>>(com, nm, frame_nm > 0 ? frame_nm : nm, box, rlist2, cap, nbr,
                                  nbrv, ncnt, icnt);
  return cudaGetLastError();
}

int cell_grid(double box, double rlist) {
  // five cells per axis are the minimum for distinct stencil cells, and at five the stencil
  // spans the whole box, so the cells pay from six on
  const int nc = (int)floor(2.0 * box / rlist);
  return nc >= 6 && nc <= kMaxCellsPerAxis ? nc : 0;
}

size_t cell_scratch_ints(int nc, int nm) {
  const size_t ncells = (size_t)nc * nc * nc;
  return 3 * ncells + 1 + 2 * (size_t)nm;
}

cudaError_t launch_neighbors_cells(const double4 *com, int nm, double box, double rlist2,
                                   int nc, int cap, int *scratch, int *nbr, double4 *nbrv,
                                   int *ncnt, int *icnt, cudaStream_t st) {
  const int ncells = nc * nc * nc;
  int *count = scratch, *cursor = count + ncells, *start = cursor + ncells;
  int *cell_of = start + ncells + 1, *members = cell_of + nm;
  cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int) * ncells, st);
  if (e != cudaSuccess) return e;
  const int nb = (nm + 255) / 256;
  k_cell_assign<<<nb, 256, 0, st>>>(com, nm, box, nc, cell_of, count);
  k_cell_scan<<<1, 1024, 0, st>>>(ncells, count, start, cursor);
  k_cell_fill<<<nb, 256, 0, st>>>(nm, cell_of, cursor, members);
  const size_t smem = (size_t)cap * (sizeof(double4) + sizeof(int));
  k_neighbors_cells<<<nm, 128, smem, st>>>(com, nm, box, rlist2, cap, nc, cell_of, start, members,
                                           nbr, nbrv, ncnt, icnt);
  return cudaGetLastError();
}

cudaError_t launch_pair_static(const double *x, const double *y, const double *z,
                               const double *xs, const double *ys, const double *zs, int ld,
                               const double4 *act, const int *nbr, const double4 *nbrv,
                               const int *ncnt, int cap, int nm, SiteSets S, EwaldParams P,
                               double *f, double *e0r, double *e0s, int with_self, double *fself,
                               double *e0slf, double *scal, cudaStream_t st) {
  if (nm < 1) return cudaSuccess;
  if (S.nq + S.np <= 8)
    k_pair_static<8><<<nm, 8 * 32, 0, st>>>(x, y, z, xs, ys, zs, ld, act, nbr, nbrv, ncnt, cap,
                                            nm, S, P, f, e0r, e0s, with_self, fself, e0slf, scal);
  else
    k_pair_static<kMaxQ + kMaxP><<<nm, (kMaxQ + kMaxP) * 32, 0, st>>>(
        x, y, z, xs, ys, zs, ld, act, nbr, nbrv, ncnt, cap, nm, S, P, f, e0r, e0s, with_self,
        fself, e0slf, scal);
  return cudaGetLastError();
}

cudaError_t launch_self_static(const double *x, const double *y, const double *z,
                               const double *xs, const double *ys, const double *zs, int nm,
                               int ld, SiteSets S, EwaldParams P, double *f, double *e0slf,
                               double *scal, cudaStream_t st) {
  const int threads = 128;
  k_self_static<<<(nm + threads - 1) / threads, threads, 0, st>>>(x, y, z, xs, ys, zs, nm, ld, S,
                                                                  P, f, e0slf, scal);
  return cudaGetLastError();
}

cudaError_t launch_pair_indforce(const double *x, const double *y, const double *z,
                                 const double *xs, const double *ys, const double *zs,
                                 int ld, const double4 *act, const int *nbr,
                                 const double4 *nbrv, const int *ncnt, int cap, int nm,
                                 SiteSets S, EwaldParams P, const double *mu, double *f,
                                 double *scal, cudaStream_t st) {
  if (nm < 1) return cudaSuccess;
  if (S.na <= 8)
    k_pair_indforce<8><<<nm, 8 * 32, 0, st>>>(x, y, z, xs, ys, zs, ld, act, nbr, nbrv, ncnt, cap,
                                              nm, S, P, mu, f, scal);
  else
    k_pair_indforce<kMaxA><<<nm, kMaxA * 32, 0, st>>>(x, y, z, xs, ys, zs, ld, act, nbr, nbrv,
                                                      ncnt, cap, nm, S, P, mu, f, scal);
  return cudaGetLastError();
}
