// ccp_kspace_fixed.cu -- reciprocal-space Ewald sum (kspace_ewald, ewald.f90:754-1173) for
// callers that cannot let the library allocate device memory.
//
// Same kernels as the context form (k_kspace.cu, modes 0), but every temporary -- k-vector
// list, structure factors, per-site phase tables, packed positions, compact forces and the
// energy accumulators -- is carved out of one file-scope device array of fixed size
// (kFixedScratchBytes).  The entry point allocates no device or host memory on its success
// path and never synchronises: all work is enqueued on the caller's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "ccp_device.cuh"
#include "ccp_internal.h"

using namespace ccp;

namespace {

constexpr size_t kFixedScratchBytes = size_t(16) << 20;  // 16 MiB per device
constexpr int kMaxDevices = 64;

}  // namespace

// The scratch itself: one array per device that loads this library, kept until exit.  Host
// code must not pass its name to a kernel (that is a host-side stand-in); the device address
// comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_kspace_scratch[kFixedScratchBytes];

namespace {

std::mutex g_addr_mu;
unsigned char *g_addr[kMaxDevices] = {};

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

// Half-space k-vectors inside the sphere l^2+m^2+n^2 <= min(kmax)^2, in the reference's loop
// order (ewald.f90:936-1050): l ascending; for l = 0, m >= 0 and, for m = 0, n >= 1.
__host__ __device__ inline bool kvec_kept(int l, int m, int n, int klmsq) {
  if (l == 0 && (m < 0 || (m == 0 && n < 1))) return false;
  return l * l + m * m + n * n <= klmsq;
}

int count_kvecs(int lmax, int mmax, int nmax) {
  const int klm = std::min(lmax, std::min(mmax, nmax));
  int nk = 0;
  for (int l = 0; l <= lmax; l++)
    for (int m = -mmax; m <= mmax; m++)
      for (int n = -nmax; n <= nmax; n++) nk += kvec_kept(l, m, n, klm * klm);
  return nk;
}

// One block writes the ordered k-vector list: each thread takes a contiguous run of the
// lexicographic (l, m, n) candidates, and a block-wide exclusive scan of the kept counts
// gives each run its output offset.
__global__ void __launch_bounds__(1024)
    k_fixed_kvecs(int lmax, int mmax, int nmax, double alp, double box, KVec *kv) {
  __shared__ int scan[1024];
  const int M = 2 * mmax + 1, N = 2 * nmax + 1;
  const int total = (lmax + 1) * M * N;
  const int klm = min(lmax, min(mmax, nmax)), klmsq = klm * klm;
  const int per = (total + blockDim.x - 1) / blockDim.x;
  const int c0 = min(total, (int)threadIdx.x * per), c1 = min(total, c0 + per);
  int kept = 0;
  for (int c = c0; c < c1; c++) {
    const int l = c / (M * N), m = (c / N) % M - mmax, n = c % N - nmax;
    kept += kvec_kept(l, m, n, klmsq);
  }
  scan[threadIdx.x] = kept;
  __syncthreads();
  for (int off = 1; off < (int)blockDim.x; off <<= 1) {
    const int v = threadIdx.x >= (unsigned)off ? scan[threadIdx.x - off] : 0;
    __syncthreads();
    scan[threadIdx.x] += v;
    __syncthreads();
  }
  int o = scan[threadIdx.x] - kept;
  const double twopi = 2.0 * ccpd::kPi, volmi = box * box * box;
  for (int c = c0; c < c1; c++) {
    const int l = c / (M * N), m = (c / N) % M - mmax, n = c % N - nmax;
    if (!kvec_kept(l, m, n, klmsq)) continue;
    KVec k;
    k.rl = twopi * l / box;
    k.rm = twopi * m / box;
    k.rn = twopi * n / box;
    const double rksq = k.rl * k.rl + k.rm * k.rm + k.rn * k.rn;
    k.ak = twopi / volmi * exp(-0.25 * rksq / (alp * alp)) / rksq;
    k.l = l;
    k.m = m;
    k.n = n;
    k.pad = 0;
    kv[o++] = k;
  }
}

// Packs molecule centres and charged-site offsets, and clears the compact forces and the
// energy/virial accumulators (both are summed into with atomics).
__global__ void k_fixed_prep(const double *__restrict__ x, const double *__restrict__ y,
                             const double *__restrict__ z, const double *__restrict__ xs,
                             const double *__restrict__ ys, const double *__restrict__ zs, int nm,
                             int ld, SiteSets S, double4 *com, double4 *act, double *f,
                             double *scal) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = nm * S.nq;
  if (t < nm) com[t] = make_double4(x[t], y[t], z[t], 0.0);
  if (t < n) {
    const int i = t / S.nq, r = t % S.nq;
    const size_t o = (size_t)i * ld + S.qsite[r];
    act[t] = make_double4(xs[o], ys[o], zs[o], S.q[r]);
    f[t] = 0.0;
    f[(size_t)n + t] = 0.0;
    f[2 * (size_t)n + t] = 0.0;
  }
  if (t < S_COUNT) scal[t] = 0.0;
}

// Adds the compact charged-site forces into the caller's (molecule, ld) arrays and writes
// the energy (kcal/mol) and virial contribution with the reference's prefactors
// (ewald.f90:1151-1160).
__global__ void k_fixed_finish(const double *__restrict__ f, int nm, int ld, SiteSets S,
                               const double *__restrict__ scal, double *fxs, double *fys,
                               double *fzs, double *qkcpe, double *vir) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = nm * S.nq;
  if (t < n) {
    const int i = t / S.nq, r = t % S.nq;
    const size_t o = (size_t)i * ld + S.qsite[r];
    fxs[o] += f[t];
    fys[o] += f[(size_t)n + t];
    fzs[o] += f[2 * (size_t)n + t];
  }
  if (t == 0) {
    *qkcpe = 2.0 * ccpd::kR4pie0 * scal[S_KC_E] / 418.4;
    *vir += 2.0 * ccpd::kR4pie0 * scal[S_KC_VIR];
  }
}

int fail(int code, const std::string &msg) {
  set_error("ccp_kspace_ewald_fixed: " + msg);
  return code;
}

}  // namespace

extern "C" int ccp_kspace_ewald_fixed(const ccp_model *m, int nm, const double *x,
                                      const double *y, const double *z, const double *xs,
                                      const double *ys, const double *zs, int ld, int lmax,
                                      int mmax, int nmax, double alp, double box, double *qkcpe,
                                      double *fxs, double *fys, double *fzs, double *vir,
                                      void *stream) {
  if (!m || !x || !y || !z || !xs || !ys || !zs || !qkcpe || !fxs || !fys || !fzs || !vir)
    return fail(CCP_ERR_BAD_INPUT, "null argument");
  if (nm < 1 || ld < m->ns) return fail(CCP_ERR_BAD_INPUT, "need nm >= 1 and ld >= sites per molecule");
  if (lmax < 1 || mmax < 1 || nmax < 1) return fail(CCP_ERR_BAD_INPUT, "k-max must be >= 1");
  if (!(box > 0.0) || !(alp > 0.0)) return fail(CCP_ERR_BAD_INPUT, "box and alpha must be > 0");
  if (lmax > 64 || mmax > 64 || nmax > 64) return fail(CCP_ERR_CAPACITY, "k-max above 64");

  // charged sites only: the compact site set (active slot = charged slot)
  SiteSets S;
  std::memset(&S, 0, sizeof(S));
  for (int s = 0; s < m->ns; s++) {
    if (m->charge[s] == 0.0) continue;
    if (S.nq >= ccpd::kMaxQ) return fail(CCP_ERR_BAD_INPUT, "too many charged sites per molecule");
    S.qsite[S.nq] = s;
    S.a_of_q[S.nq] = S.nq;
    S.asite[S.nq] = S.nq;
    S.q[S.nq] = m->charge[s];
    S.p_of_a[S.nq] = -1;
    S.nq++;
  }
  S.na = S.nq;
  S.ns = S.nq;  // compact force layout: (molecule, charged slot)
  if (S.nq == 0) return fail(CCP_ERR_BAD_INPUT, "model has no charged sites");

  const int nk = count_kvecs(lmax, mmax, nmax);
  const int k1 = std::max(std::max(std::max(lmax, mmax), nmax) + 1, 2);
  const size_t nq = (size_t)nm * S.nq;
  const size_t b_kv = up256(sizeof(KVec) * (size_t)nk), b_sk = up256(sizeof(double) * 4 * (size_t)nk);
  const size_t b_com = up256(sizeof(double4) * (size_t)nm), b_act = up256(sizeof(double4) * nq);
  const size_t b_tab = up256(sizeof(double2) * 3 * (size_t)k1 * nq);
  const size_t b_f = up256(sizeof(double) * 3 * nq), b_scal = up256(sizeof(double) * S_COUNT);
  const size_t need = b_kv + b_sk + b_com + b_act + b_tab + b_f + b_scal;
  if (need > kFixedScratchBytes)
    return fail(CCP_ERR_CAPACITY, "needs " + std::to_string(need) + " bytes of scratch for " +
                                      std::to_string(nm) + " molecules and " + std::to_string(nk) +
                                      " k-vectors; the fixed scratch holds " +
                                      std::to_string(kFixedScratchBytes) + " bytes");

  // The launch checks below read the thread's last CUDA error.  An error that earlier work of
  // the caller left pending would be reported as this call's own, so such a call is refused
  // before anything is launched, and the pending error is left in place for its owner.
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return fail(CCP_ERR_CUDA, std::string("a CUDA error from earlier work is pending (nothing "
                                          "launched): ") + cudaGetErrorString(e));
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(CCP_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(CCP_ERR_BAD_INPUT, "device ordinal above 63");
  unsigned char *base;
  {
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (!g_addr[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_kspace_scratch);
      if (e != cudaSuccess)
        return fail(CCP_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_addr[dev] = static_cast<unsigned char *>(p);
    }
    base = g_addr[dev];
  }
  KVec *kv = reinterpret_cast<KVec *>(base);
  double *sk = reinterpret_cast<double *>(base + b_kv);
  double4 *com = reinterpret_cast<double4 *>(base + b_kv + b_sk);
  double4 *act = reinterpret_cast<double4 *>(base + b_kv + b_sk + b_com);
  double2 *tab = reinterpret_cast<double2 *>(base + b_kv + b_sk + b_com + b_act);
  double *f = reinterpret_cast<double *>(base + b_kv + b_sk + b_com + b_act + b_tab);
  double *scal = reinterpret_cast<double *>(base + b_kv + b_sk + b_com + b_act + b_tab + b_f);

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nthr = (int)std::max(nq, (size_t)S_COUNT);  // nq >= nm
  k_fixed_kvecs<<<1, 1024, 0, st>>>(lmax, mmax, nmax, alp, box, kv);
  k_fixed_prep<<<(nthr + 255) / 256, 256, 0, st>>>(x, y, z, xs, ys, zs, nm, ld, S, com, act, f,
                                                    scal);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(CCP_ERR_CUDA, cudaGetErrorString(e));
  if ((e = launch_ktab(com, act, nm, S, box, lmax, mmax, nmax, tab, st)) != cudaSuccess ||
      (e = launch_kspace_sums(0, kv, nk, tab, nm, S, lmax, mmax, nmax, nullptr, sk, st)) !=
          cudaSuccess ||
      (e = launch_kspace_energy(0, kv, nk, sk, alp, scal, st)) != cudaSuccess ||
      (e = launch_kspace_gather(0, kv, nk, tab, nm, S, lmax, mmax, nmax, nullptr, sk, nullptr, f,
                                st)) != cudaSuccess)
    return fail(CCP_ERR_CUDA, cudaGetErrorString(e));
  k_fixed_finish<<<(int)((nq + 255) / 256), 256, 0, st>>>(
      f, nm, ld, S, scal, fxs, fys, fzs, qkcpe, vir);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(CCP_ERR_CUDA, cudaGetErrorString(e));
  return CCP_OK;
}
