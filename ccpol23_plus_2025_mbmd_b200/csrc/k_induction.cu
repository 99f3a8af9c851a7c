// k_induction.cu -- the real-space part of the Jacobi induced-dipole iteration (sm_100a).
//
// The field of the induced dipoles at polarisable site p of molecule i is linear in the
// dipoles:  E_p = sum_j sum_q [ A (d . mu_q) d - B mu_q ],  d = r_p(i) - r_q(j), with
//   A = 3 d5ii + (tt3 - 1) 3 / r^5,  B = d3ii + (tt3 - 1) / r^3
// from the erfc-screened real-space term (rspace_efield_idm, nb_induction_model.f90:
// 1468-1517) plus the Tang-Toennies correction (shortrange_efield_idm_damped, :5716-5736),
// and, within the molecule, the erf-screened intramolecular term with the point self term
// (self_efield_idm, :2693-2783).  The geometry is fixed during the iteration, so the
// (d, A, B) of every site pair are computed once per evaluation, stored per polarisable site
// as T4/TB[i][p][n][q] (neighbour n of molecule i, its polarisable site q) so that the
// per-iteration product (k_iter.cu) reads them contiguously.
#include "ccp_device.cuh"

using namespace ccpd;

namespace {

__global__ void k_dip_tensor(const double *__restrict__ x, const double *__restrict__ y,
                             const double *__restrict__ z, const double *__restrict__ xs,
                             const double *__restrict__ ys, const double *__restrict__ zs, int ld,
                             const double4 *__restrict__ act, const int *__restrict__ nbr,
                             const double4 *__restrict__ nbrv, const int *__restrict__ ncnt,
                             int cap, int nm, SiteSets S, EwaldParams P, double4 *T4, double *TB,
                             double4 *S4, double *SB) {
  const int i = blockIdx.x;
  const int np = S.np, npp = np * np;
  const double alp = P.alpha, alp3 = alp * alp * alp;
  const int cnt = ncnt[i];
  for (int it = threadIdx.x; it < cnt * npp; it += blockDim.x) {
    const int n = it / npp, pq = it % npp, p = pq / np, q = pq % np;
    const size_t o = (((size_t)i * np + p) * cap + n) * np + q;
    const double4 c = nbrv[(size_t)i * cap + n];
    if (!(c.w < P.rcutsd)) {
      T4[o] = make_double4(0.0, 0.0, 0.0, 0.0);
      TB[o] = 0.0;
      continue;
    }
    const int j = nbr[(size_t)i * cap + n];
    const double4 sp = act[(size_t)i * S.na + S.a_of_p[p]];
    const double4 sq = act[(size_t)j * S.na + S.a_of_p[q]];
    const double dx = c.x + sp.x - sq.x, dy = c.y + sp.y - sq.y, dz = c.z + sp.z - sq.z;
    const double d2 = dx * dx + dy * dy + dz * dz;
    const double d1i = rsqrt(d2), drr = d2 * d1i, d2i = d1i * d1i, d3i = d2i * d1i;
    const double d5i = d3i * d2i;
    const double ad = alp * drr;
    const double expar2 = exp(-(ad * ad));
    const double ec = erfc(alp * drr);
    const double d3ii = ec * d3i + P.twosqpi * alp * expar2 * d2i;
    const double d5ii = ec * d5i + P.twosqpi * alp * expar2 * d2i * d2i +
                        (2.0 / 3.0) * P.twosqpi * alp3 * expar2 * d2i;
    double A = 3.0 * d5ii, B = d3ii;
    if (P.damped) {
      const double g = tt<3>(P.delta3, drr) - 1.0;
      A += g * 3.0 * d5i;
      B += g * d3i;
    }
    T4[o] = make_double4(dx, dy, dz, A);
    TB[o] = B;
  }
  // intramolecular: erf-screened pair terms (negated) and the point self term
  const double selffac = 4.0 * alp3 / (3.0 * sqrt(kPi));
  for (int pq = threadIdx.x; pq < npp; pq += blockDim.x) {
    const int p = pq / np, q = pq % np;
    const size_t o = (size_t)i * npp + pq;
    if (p == q) {
      S4[o] = make_double4(0.0, 0.0, 0.0, 0.0);
      SB[o] = -selffac;
      continue;
    }
    const size_t os = (size_t)i * ld + S.psite[p], ot = (size_t)i * ld + S.psite[q];
    const double xi = x[i], yi = y[i], zi = z[i];
    const double dx = (xi + xs[os]) - (xi + xs[ot]);
    const double dy = (yi + ys[os]) - (yi + ys[ot]);
    const double dz = (zi + zs[os]) - (zi + zs[ot]);
    const double drr = sqrt(dx * dx + dy * dy + dz * dz);
    const double d1i = 1.0 / drr, d2i = d1i * d1i, d3i = d2i * d1i, d5i = d3i * d2i;
    const double ad = alp * drr;
    const double expar2 = exp(-(ad * ad));
    const double ef = erf(alp * drr);
    const double d3ii = ef * d3i - P.twosqpi * alp * expar2 * d2i;
    const double d5ii = ef * d5i - P.twosqpi * alp * expar2 * d2i * d2i -
                        (2.0 / 3.0) * P.twosqpi * alp3 * expar2 * d2i;
    S4[o] = make_double4(dx, dy, dz, -3.0 * d5ii);
    SB[o] = -d3ii;
  }
}

// total static field E0 = r + k + self + short-range (nb_induction_model.f90:1320-1322)
__global__ void k_static_total(int n, const double *__restrict__ a, const double *__restrict__ b,
                               const double *__restrict__ c, const double *__restrict__ d,
                               double *out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = a[t] + b[t] + c[t] + d[t];
}

// Convergence test of the Jacobi loop (nb_induction_model.f90:1269-1372), run as the last
// node of the loop body: records the iteration count, the squared change and the energy of
// the iteration, clears the accumulators for the next one, and keeps the WHILE node going
// while change > thr and fewer than maxit iterations have run.
__global__ void k_dip_cond(cudaGraphConditionalHandle h, int use_graph, double *scal,
                           double *state, double thr, int maxit) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double ch = scal[S_IND_CHANGE], en = scal[S_IND_ENERGY];
  const int it = (int)state[0] + 1;
  state[0] = (double)it;
  state[1] = ch;
  state[2] = en;
  scal[S_IND_CHANGE] = 0.0;
  scal[S_IND_ENERGY] = 0.0;
  if (use_graph) cudaGraphSetConditional(h, (ch > thr && it < maxit) ? 1u : 0u);
}

}  // namespace

cudaError_t launch_dip_cond(cudaGraphConditionalHandle h, int use_graph, double *scal,
                            double *state, double thr, int maxit, cudaStream_t st) {
  k_dip_cond<<<1, 32, 0, st>>>(h, use_graph, scal, state, thr, maxit);
  return cudaGetLastError();
}

cudaError_t launch_dip_tensor(const double *x, const double *y, const double *z,
                              const double *xs, const double *ys, const double *zs, int ld,
                              const double4 *act, const int *nbr, const double4 *nbrv,
                              const int *ncnt, int cap, int nm, SiteSets S, EwaldParams P,
                              double4 *T4, double *TB, double4 *S4, double *SB,
                              cudaStream_t st) {
  k_dip_tensor<<<nm, 128, 0, st>>>(x, y, z, xs, ys, zs, ld, act, nbr, nbrv, ncnt, cap, nm, S, P, T4,
                                   TB, S4, SB);
  return cudaGetLastError();
}

cudaError_t launch_static_total(int n, const double *a, const double *b, const double *c,
                                const double *d, double *out, cudaStream_t st) {
  k_static_total<<<(n + 255) / 256, 256, 0, st>>>(n, a, b, c, d, out);
  return cudaGetLastError();
}
