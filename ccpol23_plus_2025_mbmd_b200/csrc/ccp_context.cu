// ccp_context.cu -- device-resident state and the C-ABI entry points of the hot path.
//
// A context owns, on one GPU, the packed site arrays, neighbour/pair/triple lists,
// reciprocal-space tables, dipoles and force accumulators for boxes of nm molecules.
// The reference entry points (threebody_term, nb_induction, rspace_ewald, kspace_ewald,
// ewald_self_correction) map onto one evaluation with a subset of terms enabled.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ccp_device.cuh"
#include "ccp_internal.h"

using namespace ccp;

namespace {

enum TermMask : unsigned {
  T_SELF = 1u,
  T_RSPACE = 2u,
  T_KSPACE = 4u,
  T_INDUCTION = 8u,
  T_FS2 = 16u,
  T_FS3 = 32u,
  T_VDW = 64u,
};
static_assert(T_SELF == CCP_TERM_SELF && T_RSPACE == CCP_TERM_RSPACE && T_KSPACE == CCP_TERM_KSPACE &&
                  T_INDUCTION == CCP_TERM_INDUCTION && T_FS2 == CCP_TERM_FS2 && T_FS3 == CCP_TERM_FS3 &&
                  T_VDW == CCP_TERM_VDW,
              "term bits of the C ABI");

bool cuda_ok(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return false;
}

#define CK(call)                               \
  do {                                         \
    if (!cuda_ok((call), #call)) return CCP_ERR_CUDA; \
  } while (0)

template <typename T>
cudaError_t dalloc(T **p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  return cudaMalloc((void **)p, n * sizeof(T));
}

}  // namespace

struct ccp_context {
  int device = 0, precision = CCP_FP64, nm = 0, ns = 0, npol = 0, nsm = 148;
  size_t l2_bytes = size_t(126) << 20;  // the device's L2 size
  cudaStream_t own = nullptr, stream = nullptr;
  // model-derived constants
  SiteSets S{};
  double charge[kNsiteMax] = {0};
  double rcut = 0, rcutsd = 0, rcut3 = 0, rcutsd3 = 0, alpha3 = 0, delta33 = 0;
  bool s2 = false, s3 = false, induction = false, three_body = false, damped = false;
  bool have_fs3 = false;
  double alpha = 0;
  int kmax[3] = {0, 0, 0};
  int maxit = 500;
  int launches = 0;
  // inputs in the caller's layout (device copies)
  int ld_cap = 0;
  double *d_x = nullptr, *d_y = nullptr, *d_z = nullptr;
  double *d_xs = nullptr, *d_ys = nullptr, *d_zs = nullptr;
  // packed
  double4 *d_com = nullptr, *d_act = nullptr, *d_comb = nullptr, *d_s17 = nullptr;
  // accumulators
  // site forces f[3][nm*ns]; a second block of the same size takes the three-body forces
  // when those run concurrently on side streams (the Ewald/induction kernels add to f
  // without atomics), and is added to f after the join
  double *d_f = nullptr, *d_fc2 = nullptr, *d_fc3 = nullptr;
  double *d_scal = nullptr;
  int *d_icnt = nullptr;
  // induction
  double *d_mu = nullptr, *d_e0r = nullptr, *d_e0k = nullptr, *d_e0slf = nullptr, *d_e0s = nullptr;
  double *d_eir = nullptr, *d_eik = nullptr, *d_eislf = nullptr, *d_eis = nullptr;
  double *d_mu2 = nullptr, *d_e0tot = nullptr, *d_eim = nullptr;
  double *d_pcg = nullptr;  // PCG vectors u, w, s, p of the dipole solve (4 x npol x 3)
  double4 *d_T4 = nullptr, *d_S4 = nullptr;
  double *d_TB = nullptr, *d_SB = nullptr;
  // lists
  int cap = 0, tri_cap = 0, pair_cap = 0;
  int *d_nbr = nullptr, *d_ncnt = nullptr;
  int *d_cells = nullptr;  // cell-list scratch (launch_neighbors_cells)
  size_t cells_cap = 0;
  int opt_cells = 1;       // cell-list neighbour search where the box allows it
  bool cells_active = false;
  double4 *d_nbrv = nullptr;
  void *d_tri = nullptr;  // FS3 triple records
  int2 *d_pairs = nullptr;
  // reciprocal space
  KVec *d_kv = nullptr;
  KGather *d_kg = nullptr;
  int nk = 0, nk_cap = 0;
  // the rows of the k-vector list by decreasing length (KRow) and 2 pi n / L by n, for the
  // row form of the dipole step
  KRow *d_rows = nullptr;
  double *d_rn = nullptr;
  int nrow = 0, nrow_cap = 0, nrn_cap = 0, row_span = 0;
  double kv_box = -1, kv_alpha = -1;
  int kv_kmax[3] = {-1, -1, -1};
  double2 *d_tab = nullptr;
  size_t tab_cap = 0;
  double *d_sk = nullptr;
  double *d_skj = nullptr;  // the dipole loop's own S(k) buffers, so that the Ewald sums in
                            // d_sk can still be gathered while the loop runs
  // FS3 tables
  double *d_coef = nullptr, *d_bgr = nullptr;
  // rigid-molecule MD state (ccp_md_*), structure of arrays on the device
  double totm = 0, pmi[3] = {0, 0, 0};
  double *d_pcoord = nullptr;
  double *d_md_x = nullptr, *d_md_xs = nullptr, *d_md_v = nullptr, *d_md_q = nullptr,
         *d_md_j = nullptr, *d_md_red = nullptr, *h_md = nullptr;
  bool md_ready = false;
  double md_box = 0;
  double md_volm = 0;      // MD box volume (the barostat scales it, evolve.f90:7604-7606)
  int md_ens = 0;          // ensemble of ccp_md_run (CCP_MD_*)
  double md_temp0 = 0, md_taut = 0, md_pres0 = 0, md_taup = 0;  // pres0 in internal units
  double md_chit = 0, md_chip = 0, md_cint = 0;  // thermostat / barostat variables (REVCON)
  int md_eq_left = 0;      // MD steps still to be followed by the equilibration rescale
  double md_eq_temp = 0;   // its target temperature (K)
  ccp_energies md_e{};
  // ccpol23plus 2-body tables
  bool have_vdw = false;
  int vdw_nrows = 0, vdw_nv = 0;
  int *d_vdw_row = nullptr, *d_vdw_site = nullptr;
  double *d_vdw_qq = nullptr, *d_vdw_par = nullptr;
  // FS3 parameters of this context (host copies): class coefficients, the class of every
  // coefficient-table entry, site-pair (b, g, r0); and the parameter-gradient buffer
  std::vector<double> cs_sr, cs_lr, bgr_host;
  std::vector<int> class_of_type;
  int nclass = 0;
  double *d_gfs3 = nullptr;
  int opt_pgrad = 0;   // accumulate dE_FS3/d(parameters) in each evaluation
  bool pgrad_valid = false;
  int *d_types = nullptr;
  // host staging (pinned)
  double *h_scal = nullptr;
  int *h_icnt = nullptr;
  double *h_io = nullptr;
  size_t h_io_cap = 0;
  // pinned copies of the results of a host-buffer evaluation (site forces, FS2 and FS3 COM
  // forces, dipoles), queued before the evaluation's one synchronisation when dl_req is set
  double *h_out = nullptr;
  size_t h_out_cap = 0;
  bool dl_req = false;
  // constants for the Ewald self energy
  double sumq = 0, sumq2 = 0;
  // graph-resident Jacobi loop
  cudaStream_t cap_stream = nullptr;
  cudaGraph_t ind_graph = nullptr;
  cudaGraphExec_t ind_exec = nullptr;
  double *d_istate = nullptr;  // kIterStateLen slots (IterStateSlot)
  double *h_istate = nullptr;
  unsigned *d_ticket = nullptr;  // last-block ticket of the fused update kernel
  int ind_per_iter = 0;          // kernels per Jacobi iteration of the last solve
  std::vector<long long> ind_key;
  // phase factors of the polarisable sites for the dipole iteration (k_iter.cu), when they
  // fit kPhaseBudget: XY[site][l][m] then Z[site][n]
  double2 *d_P = nullptr;
  size_t P_cap = 0;
  bool use_P = false;
  // with the factor tables, the full phase matrix [site][k] of the polarisable sites when it
  // fits full_phase_budget (k_iter.cu, launch_phase_matrix)
  double2 *d_PM = nullptr;
  size_t PM_cap = 0;
  bool use_PM = false;
  int opt_pm = 1;  // the full phase matrix when it fits (1) or never (0)
  // without the full phase matrix, the row form of the dipole step (1) or the factor-table
  // kernels (0)
  int opt_rows = 1;
  bool use_rows = false;
  int opt_sum_sites = 32, opt_gather_sites = 4;  // block shapes of the dipole step (IterArgs)
  // options (ccp_context_set_option)
  int opt_graph = 1;  // Jacobi loop as a conditional graph (1) or driven from the host (0)
  int opt_phase = 1;  // phase-factor tables when they fit (1) or never (0)
  // dipole solver: Jacobi at the reference's criterion (0), PCG at the reference's criterion
  // (1), PCG at an RMS criterion of dip_tol_debye (2); PCG needs the phase tables and falls
  // back to Jacobi (at the reference's criterion) without them
  int opt_solver = 0;
  double dip_tol_debye = 1e-8;
  int opt_pdl = 1;  // the dipole-step kernels with programmatic dependent launch
  // mixed form: FS3's ik/jk gradient passes in FP32 (1) or FP64 (0, the default: in FP32 the
  // molecule forces of the 2048-water box are 1.45e-5 off, above the form's 1e-5 bar)
  int opt_fs3_low = 0;
  int opt_fs3_prio = 0;  // FS3's stream at the high priority of the Ewald/induction chain
  bool pcg_active = false;  // the solver of the last solve was PCG
  // phase timing (diagnostics)
  bool timing = false;
  cudaEvent_t ev[2 * CCP_NPHASE] = {};  // start/end of each phase, on the phase's stream
  unsigned phase_ran = 0;
  double phase_ms[CCP_NPHASE] = {0};
  // side streams of the three-body terms (forked from the main stream after the neighbour
  // list, joined before the scalars are read back)
  cudaStream_t s_fs3 = nullptr, s_fs2 = nullptr, s_main = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_j3 = nullptr, ev_j2 = nullptr, ev_jm = nullptr;
  // the reciprocal-space branch of the Ewald/induction chain (k tables, structure factors,
  // gathers) on its own high-priority stream beside the real-space kernels
  cudaStream_t s_kspace = nullptr;
  cudaEvent_t ev_k1 = nullptr, ev_k2 = nullptr, ev_lp = nullptr;
  int opt_overlap = 1;     // three-body terms concurrent with Ewald/induction
  int opt_fs3_tpb = 8;     // FS3 triples per block when concurrent (0 = persistent grid)
  int opt_fs3_bps = 0;     // when concurrent, at most this many FS3 blocks per SM (0 = no cap)
};

namespace {

void free_ctx(ccp_context *c) {
  cudaSetDevice(c->device);
  // d_y, d_z live in d_x's allocation and d_ys, d_zs in d_xs's
  void *dp[] = {c->d_x,   c->d_xs,  c->d_com,
                c->d_act, c->d_comb, c->d_s17,  c->d_f,     c->d_fc2,  c->d_fc3,   c->d_scal,
                c->d_icnt, c->d_mu, c->d_e0r,   c->d_e0k,   c->d_e0slf, c->d_e0s,  c->d_eir,
                c->d_eik, c->d_eislf, c->d_eis, c->d_nbr,   c->d_ncnt, c->d_nbrv,  c->d_tri,
                c->d_pairs, c->d_kv, c->d_kg, c->d_tab, c->d_sk, c->d_skj, c->d_coef, c->d_bgr,
                c->d_types,
                c->d_gfs3,  c->d_vdw_row, c->d_vdw_site, c->d_vdw_qq, c->d_vdw_par,
                c->d_pcoord, c->d_md_x, c->d_md_xs, c->d_md_v, c->d_md_q, c->d_md_j, c->d_md_red,
                c->d_mu2, c->d_e0tot, c->d_eim, c->d_T4, c->d_S4, c->d_TB, c->d_SB,
                c->d_pcg, c->d_cells};
  for (void *p : dp)
    if (p) cudaFree(p);
  if (c->h_scal) cudaFreeHost(c->h_scal);
  if (c->h_icnt) cudaFreeHost(c->h_icnt);
  if (c->h_io) cudaFreeHost(c->h_io);
  if (c->h_out) cudaFreeHost(c->h_out);
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->ind_exec) cudaGraphExecDestroy(c->ind_exec);
  if (c->ind_graph) cudaGraphDestroy(c->ind_graph);
  if (c->d_istate) cudaFree(c->d_istate);
  if (c->d_ticket) cudaFree(c->d_ticket);
  if (c->h_md) cudaFreeHost(c->h_md);
  if (c->d_P) cudaFree(c->d_P);
  if (c->d_PM) cudaFree(c->d_PM);
  if (c->d_rows) cudaFree(c->d_rows);
  if (c->d_rn) cudaFree(c->d_rn);
  if (c->h_istate) cudaFreeHost(c->h_istate);
  if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
  if (c->s_fs3) cudaStreamDestroy(c->s_fs3);
  if (c->s_fs2) cudaStreamDestroy(c->s_fs2);
  if (c->s_main) cudaStreamDestroy(c->s_main);
  if (c->s_kspace) cudaStreamDestroy(c->s_kspace);
  for (cudaEvent_t e : {c->ev_fork, c->ev_j3, c->ev_j2, c->ev_jm, c->ev_k1, c->ev_k2, c->ev_lp})
    if (e) cudaEventDestroy(e);
  if (c->own) cudaStreamDestroy(c->own);
}

int ensure_inputs(ccp_context *c, int ld) {
  if (ld <= c->ld_cap) return CCP_OK;
  // one allocation for the three site-offset arrays, so that an upload is one copy
  if (c->d_xs) cudaFree(c->d_xs);
  c->d_xs = c->d_ys = c->d_zs = nullptr;
  CK(dalloc(&c->d_xs, 3 * (size_t)c->nm * ld));
  c->d_ys = c->d_xs + (size_t)c->nm * ld;
  c->d_zs = c->d_ys + (size_t)c->nm * ld;
  c->ld_cap = ld;
  return CCP_OK;
}

int ensure_lists(ccp_context *c, int cap, int tri_cap, int pair_cap) {
  if (cap > c->cap) {
    if (c->d_nbr) cudaFree(c->d_nbr);
    if (c->d_nbrv) cudaFree(c->d_nbrv);
    if (c->d_T4) cudaFree(c->d_T4);
    if (c->d_TB) cudaFree(c->d_TB);
    CK(dalloc(&c->d_nbr, (size_t)c->nm * cap));
    CK(dalloc(&c->d_nbrv, (size_t)c->nm * cap));
    const size_t npp = (size_t)std::max(c->S.np, 1) * std::max(c->S.np, 1);
    CK(dalloc(&c->d_T4, (size_t)c->nm * cap * npp));
    CK(dalloc(&c->d_TB, (size_t)c->nm * cap * npp));
    c->cap = cap;
  }
  if (tri_cap > c->tri_cap) {
    if (c->d_tri) cudaFree(c->d_tri);
    CK(cudaMalloc(&c->d_tri, fs3_record_bytes() * (size_t)std::max(tri_cap, 1)));
    c->tri_cap = tri_cap;
  }
  if (pair_cap > c->pair_cap) {
    if (c->d_pairs) cudaFree(c->d_pairs);
    CK(dalloc(&c->d_pairs, (size_t)pair_cap));
    c->pair_cap = pair_cap;
  }
  return CCP_OK;
}

// Half-space k-vectors with the spherical cut-off, in the reference's loop order
// (ewald.f90:933-1082): ll = 0..lmax; mm from 0 (ll = 0) or -mmax; nn from 1 (first mm
// of ll = 0) or -nmax; keep ll^2 + mm^2 + nn^2 <= min(lmax,mmax,nmax)^2.
std::vector<KVec> build_kvecs(int lmax, int mmax, int nmax, double alp, double box) {
  std::vector<KVec> out;
  const double twopi = 2.0 * kPi;
  const int klm = std::min(lmax, std::min(mmax, nmax));
  const int klmsq = klm * klm;
  const double volmi = box * box * box;
  int mmin = 0, nmin = 1;
  for (int ll = 0; ll <= lmax; ll++) {
    const double rl = twopi * ll / box;
    if (ll > 0) mmin = -mmax;
    for (int mm = mmin; mm <= mmax; mm++) {
      const double rm = twopi * mm / box;
      for (int nn = nmin; nn <= nmax; nn++) {
        const double rn = twopi * nn / box;
        const int kk = ll * ll + mm * mm + nn * nn;
        if (kk <= klmsq) {
          const double rksq = rl * rl + rm * rm + rn * rn;
          KVec k;
          k.rl = rl;
          k.rm = rm;
          k.rn = rn;
          k.ak = twopi / volmi * std::exp(-0.25 * rksq / (alp * alp)) / rksq;
          k.l = ll;
          k.m = mm;
          k.n = nn;
          k.pad = 0;
          out.push_back(k);
        }
      }
      nmin = -nmax;
    }
  }
  return out;
}

// The rows of a k-vector list in the order build_kvecs makes it (n innermost): one per run
// of one (l, m), sorted by decreasing length (ties in list order), for the row form of the
// dipole step (k_iter.cu).
std::vector<KRow> build_krows(const std::vector<KVec> &kv, int mmax) {
  std::vector<KRow> rows;
  for (int k = 0; k < (int)kv.size(); k++) {
    const KVec &K = kv[k];
    if (k > 0 && K.l == kv[k - 1].l && K.m == kv[k - 1].m) {
      rows.back().len++;
      continue;
    }
    rows.push_back({K.rl, K.rm, k, 1, K.n, K.l * (2 * mmax + 1) + K.m + mmax});
  }
  std::stable_sort(rows.begin(), rows.end(),
                   [](const KRow &a, const KRow &b) { return a.len > b.len; });
  return rows;
}

int ensure_kspace(ccp_context *c, double box) {
  if (box == c->kv_box && c->alpha == c->kv_alpha && c->kmax[0] == c->kv_kmax[0] &&
      c->kmax[1] == c->kv_kmax[1] && c->kmax[2] == c->kv_kmax[2])
    return CCP_OK;
  std::vector<KVec> kv = build_kvecs(c->kmax[0], c->kmax[1], c->kmax[2], c->alpha, box);
  c->nk = (int)kv.size();
  if (c->nk > c->nk_cap) {
    if (c->d_kv) cudaFree(c->d_kv);
    if (c->d_kg) cudaFree(c->d_kg);
    if (c->d_sk) cudaFree(c->d_sk);
    if (c->d_skj) cudaFree(c->d_skj);
    CK(dalloc(&c->d_kv, (size_t)c->nk));
    CK(dalloc(&c->d_kg, (size_t)c->nk));
    CK(dalloc(&c->d_sk, (size_t)c->nk * 4));
    CK(dalloc(&c->d_skj, (size_t)c->nk * 4));
    c->nk_cap = c->nk;
  }
  if (c->nk) CK(cudaMemcpyAsync(c->d_kv, kv.data(), sizeof(KVec) * c->nk, cudaMemcpyHostToDevice, c->stream));
  std::vector<KGather> kg(c->nk);
  for (int k = 0; k < c->nk; k++) {
    const KVec &K = kv[k];
    kg[k] = {K.rl, K.rm, K.rn,
             ((K.l * (2 * c->kmax[1] + 1) + K.m + c->kmax[1]) << 8) | (K.n + c->kmax[2]), 0};
  }
  if (c->nk)
    CK(cudaMemcpyAsync(c->d_kg, kg.data(), sizeof(KGather) * c->nk, cudaMemcpyHostToDevice,
                       c->stream));
  {
    std::vector<KRow> rows = build_krows(kv, c->kmax[1]);
    c->nrow = (int)rows.size();
    c->row_span = 0;
    for (int t = 0; t < c->nrow; t += kRowTile) {
      int nb = rows[t].nlo, ne = nb + rows[t].len;
      for (int r = t + 1; r < std::min(c->nrow, t + kRowTile); r++) {
        nb = std::min(nb, rows[r].nlo);
        ne = std::max(ne, rows[r].nlo + rows[r].len);
      }
      c->row_span = std::max(c->row_span, ne - nb);
    }
    if (c->nrow > c->nrow_cap) {
      if (c->d_rows) cudaFree(c->d_rows);
      c->d_rows = nullptr;
      c->nrow_cap = 0;
      CK(dalloc(&c->d_rows, (size_t)c->nrow));
      c->nrow_cap = c->nrow;
    }
    const int nz = 2 * c->kmax[2] + 1;
    std::vector<double> rn(nz);
    for (int n = -c->kmax[2]; n <= c->kmax[2]; n++) rn[n + c->kmax[2]] = 2.0 * kPi * n / box;
    if (nz > c->nrn_cap) {
      if (c->d_rn) cudaFree(c->d_rn);
      c->d_rn = nullptr;
      c->nrn_cap = 0;
      CK(dalloc(&c->d_rn, (size_t)nz));
      c->nrn_cap = nz;
    }
    if (c->nrow)
      CK(cudaMemcpyAsync(c->d_rows, rows.data(), sizeof(KRow) * c->nrow, cudaMemcpyHostToDevice,
                         c->stream));
    CK(cudaMemcpyAsync(c->d_rn, rn.data(), sizeof(double) * nz, cudaMemcpyHostToDevice,
                       c->stream));
  }
  int k1 = std::max(c->kmax[0], std::max(c->kmax[1], c->kmax[2])) + 1;
  k1 = std::max(k1, 2);
  const size_t tab = (size_t)3 * k1 * c->nm * c->S.na;
  if (tab > c->tab_cap) {
    if (c->d_tab) cudaFree(c->d_tab);
    CK(dalloc(&c->d_tab, tab));
    c->tab_cap = tab;
  }
  c->kv_box = box;
  c->kv_alpha = c->alpha;
  for (int a = 0; a < 3; a++) c->kv_kmax[a] = c->kmax[a];
  return CCP_OK;
}

int ensure_host_io(ccp_context *c, size_t n) {
  if (n <= c->h_io_cap) return CCP_OK;
  if (c->h_io) cudaFreeHost(c->h_io);
  c->h_io = nullptr;
  CK(cudaMallocHost((void **)&c->h_io, n * sizeof(double)));
  c->h_io_cap = n;
  return CCP_OK;
}

struct EvalOut {
  double sumff = 0, self_vir = 0, rc_e = 0, rc_vir = 0, kc_e = 0, kc_vir = 0;
  double ind_e = 0, ind_vir = 0, fs2_e = 0, fs2_vir = 0, fs3_e = 0, fs3_vir = 0;
  double vdw_e = 0, vdw_vir = 0;
  int iters = 0, ntri = 0, nblend = 0, nfs2 = 0;
  bool converged = true;
};

// Largest phase-factor tables kept for the dipole iteration (nlm + nz complex numbers per
// polarisable site: 5 MB at 512 waters, 46 MB at 2048).
constexpr size_t kPhaseBudget = size_t(1) << 30;
// The full phase matrix (16 bytes per polarisable site and k-vector: 38 MB at 512 waters,
// 568 MB at 2048) pays only while it stays in L2, which it is read from twice per step: it
// is used when it fits in half of the L2.  Streamed from HBM (2048 waters) it made the dipole
// step slower than the factor tables and evicted the concurrent kernels' working sets.
size_t full_phase_budget(const ccp_context *c) { return c->l2_bytes / 2; }

constexpr double kIndThr = 1.0e-20;  // iteridm convergence threshold on sum |dmu|^2
constexpr double kDebyePerEA = 4.80320471;  // Debye per e*Angstrom (dipoles are in e*A)

// Whether the next solve is PCG, and its convergence threshold on sum |dmu|^2 (PCG: sum |u|^2
// at the iterate, the Jacobi update there).
bool pcg_solver(const ccp_context *c) { return c->opt_solver != 0 && c->use_P; }
double ind_threshold(const ccp_context *c) {
  if (!pcg_solver(c) || c->opt_solver == 1) return kIndThr;
  const double t = c->dip_tol_debye / kDebyePerEA;
  return (double)c->nm * c->S.np * t * t;
}

// Enqueues one Jacobi step: with the phase factors two kernels (k_iter.cu), otherwise T.mu,
// the tiled dipole structure factors and reciprocal field, the update and the convergence
// node.  `handle` is used only when use_graph is set.
IterArgs make_iter_args(ccp_context *c, cudaGraphConditionalHandle handle, int use_graph,
                        int par) {
  const SiteSets &S = c->S;
  IterArgs A{};
  A.nbr = c->d_nbr;
  A.ncnt = c->d_ncnt;
  A.cap = c->cap;
  A.nw = c->nm * S.np;
  A.np = S.np;
  A.T4 = c->d_T4;
  A.TB = c->d_TB;
  A.S4 = c->d_S4;
  A.SB = c->d_SB;
  A.mu = c->d_mu;
  A.eim = c->d_eim;
  A.e0 = c->d_e0tot;
  A.kv = c->d_kv;
  A.kg = c->d_kg;
  A.nk = c->nk;
  A.mmax = c->kmax[1];
  A.nmax = c->kmax[2];
  A.nlm = (c->kmax[0] + 1) * (2 * c->kmax[1] + 1);
  A.nz = 2 * c->kmax[2] + 1;
  A.XY = c->d_P;
  A.Z = c->d_P ? c->d_P + (size_t)A.nw * A.nlm : nullptr;
  A.PM = c->use_PM ? c->d_PM : nullptr;
  if (c->use_rows) {
    A.XY = nullptr;
    A.rows = c->d_rows;
    A.nrow = c->nrow;
    A.row_span = c->row_span;
    A.XYr = c->d_P;
    A.Z = c->d_P + (size_t)c->nrow * A.nw;
    A.ZT = A.Z + (size_t)A.nz * A.nw;
    A.rn = c->d_rn;
  }
  A.sk = c->d_skj;
  A.par = par;
  A.scal = c->d_scal;
  A.state = c->d_istate;
  A.ticket = c->d_ticket;
  A.thr = ind_threshold(c);
  A.pdl = c->opt_pdl;
  A.sum_sites = c->opt_sum_sites;
  A.gather_sites = c->opt_gather_sites;
  if (pcg_solver(c)) {
    const size_t np3 = (size_t)A.nw * 3;
    A.cu = c->d_pcg;
    A.cw = c->d_pcg + np3;
    A.cs = c->d_pcg + 2 * np3;
    A.cp = c->d_pcg + 3 * np3;
  }
  A.maxit = c->maxit;
  A.use_graph = use_graph;
  A.handle = handle;
  A.S = S;
  return A;
}

cudaError_t enqueue_dip_step(ccp_context *c, cudaStream_t st, cudaGraphConditionalHandle handle,
                             int use_graph, int par, int *nlaunch) {
  const SiteSets &S = c->S;
  if (c->use_P) {
    const IterArgs A = make_iter_args(c, handle, use_graph, par);
    *nlaunch = 2;
    cudaError_t e = launch_iter_a(A, st);
    return e == cudaSuccess ? launch_iter_b(A, st) : e;
  }
  *nlaunch = 5;
  cudaError_t e = launch_tmu(c->d_nbr, c->d_ncnt, c->cap, c->nm, S.np, c->d_T4, c->d_TB, c->d_S4,
                             c->d_SB, c->d_mu, c->d_eim, st);
  if (e == cudaSuccess)
    e = launch_kspace_sums(2, c->d_kv, c->nk, c->d_tab, c->nm, S, c->kmax[0], c->kmax[1],
                           c->kmax[2], c->d_mu, c->d_skj, st);
  if (e == cudaSuccess)
    e = launch_kspace_gather(2, c->d_kv, c->nk, c->d_tab, c->nm, S, c->kmax[0], c->kmax[1],
                             c->kmax[2], c->d_mu, c->d_skj, c->d_eik, nullptr, st);
  if (e == cudaSuccess)
    e = launch_dip_update(c->nm, S, c->d_e0tot, c->d_eim, c->d_eik, c->d_mu, c->d_mu, c->d_scal, st);
  if (e == cudaSuccess)
    e = launch_dip_cond(handle, use_graph, c->d_scal, c->d_istate, kIndThr, c->maxit, st);
  return e;
}

constexpr int kDipUnroll = 2;  // Jacobi steps per pass of the graph's WHILE body
static_assert(kDipUnroll % 2 == 0, "the steps of a pass alternate the S(k) buffer parity");

// Builds (once per set of buffers and sizes) the CUDA graph of the Jacobi iteration: a
// WHILE conditional node whose body is one or more Jacobi steps, each ending in the
// convergence test.
// The host launches it once per evaluation and never synchronises inside the loop.
int ensure_ind_graph(ccp_context *c) {
  std::vector<long long> key = {
      (long long)c->d_nbr, (long long)c->d_ncnt, (long long)c->d_T4,  (long long)c->d_TB,
      (long long)c->d_S4,  (long long)c->d_SB,   (long long)c->d_mu,  (long long)c->d_eim,
      (long long)c->d_kv,  (long long)c->d_tab,  (long long)c->d_skj, (long long)c->d_eik,
      (long long)c->d_kg,
      (long long)c->d_e0tot, (long long)c->d_scal, (long long)c->d_istate, (long long)c->d_P,
      (long long)c->use_P, (long long)c->d_PM, (long long)c->use_PM, c->cap, c->nm, c->nk, c->kmax[0], c->kmax[1], c->kmax[2], c->maxit,
      (long long)pcg_solver(c), (long long)c->opt_solver, (long long)c->d_pcg,
      (long long)c->opt_pdl, c->opt_sum_sites, c->opt_gather_sites, (long long)c->use_rows,
      (long long)c->d_rows, c->nrow, c->row_span, (long long)c->d_rn};
  double thr = ind_threshold(c);
  long long thr_bits;
  std::memcpy(&thr_bits, &thr, sizeof thr_bits);
  key.push_back(thr_bits);
  if (c->ind_exec && key == c->ind_key) return CCP_OK;
  if (c->ind_exec) cudaGraphExecDestroy(c->ind_exec);
  if (c->ind_graph) cudaGraphDestroy(c->ind_graph);
  c->ind_exec = nullptr;
  c->ind_graph = nullptr;
  CK(cudaGraphCreate(&c->ind_graph, 0));
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, c->ind_graph, 1, cudaGraphCondAssignDefault));
  cudaStream_t cs = c->cap_stream;
  // the first Jacobi step (from mu = 0) is one kernel node ahead of the WHILE node, whose
  // condition it sets
  CK(cudaStreamBeginCaptureToGraph(cs, c->ind_graph, nullptr, nullptr, 0,
                                   cudaStreamCaptureModeRelaxed));
  const IterArgs A0 = make_iter_args(c, h, 1, 0);
  const cudaError_t ef = A0.cu ? launch_pcg_first(A0, cs) : launch_dip_first(A0, cs);
  cudaGraph_t captured_first = nullptr;
  const cudaError_t ef2 = cudaStreamEndCapture(cs, &captured_first);
  if (!cuda_ok(ef, "capture of the first dipole step")) return CCP_ERR_CUDA;
  CK(ef2);
  cudaGraphNode_t first = nullptr;
  size_t nfirst = 1;
  CK(cudaGraphGetNodes(c->ind_graph, &first, &nfirst));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, c->ind_graph, &first, 1, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  CK(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  int nl = 0;
  // with the phase tables the body holds kDipUnroll Jacobi steps: a step's update kernel
  // returns at once when an earlier step of the same pass has finished the solve, so the
  // count of steps taken is unchanged while the per-pass cost of the WHILE node is shared
  const int unroll = c->use_P ? kDipUnroll : 1;
  cudaError_t e = cudaSuccess;
  for (int u = 0; u < unroll && e == cudaSuccess; u++) e = enqueue_dip_step(c, cs, h, 1, u & 1, &nl);
  cudaGraph_t captured = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(cs, &captured);
  if (!cuda_ok(e, "capture of the dipole loop")) return CCP_ERR_CUDA;
  CK(e2);
  CK(cudaGraphInstantiate(&c->ind_exec, c->ind_graph, 0));
  c->ind_key = key;
  return CCP_OK;
}

// The whole Jacobi solve from mu = 0.  The state {iterations, change, energy} is copied to
// h_istate; in the graph form the copy completes at the evaluation's final synchronisation.
int run_dipole_loop(ccp_context *c, cudaStream_t st) {
  // the first step writes every dipole, so d_mu needs no clearing
  const bool pcg = pcg_solver(c);
  c->pcg_active = pcg;
  if (pcg && !c->d_pcg) CK(dalloc(&c->d_pcg, 4 * (size_t)c->nm * c->S.np * 3));
  const double thr = ind_threshold(c);
  CK(cudaMemsetAsync(c->d_istate, 0, kIterStateLen * sizeof(double), st));
  CK(cudaMemsetAsync(c->d_scal + S_IND_CHANGE, 0, 2 * sizeof(double), st));
  CK(cudaMemsetAsync(c->d_ticket, 0, sizeof(unsigned), st));
  if (c->use_P) CK(cudaMemsetAsync(c->d_skj, 0, sizeof(double) * 4 * (size_t)c->nk, st));
  int per = 0;
  if (c->opt_graph) {
    int r = ensure_ind_graph(c);
    if (r) return r;
    CK(cudaGraphLaunch(c->ind_exec, st));
    CK(cudaMemcpyAsync(c->h_istate, c->d_istate, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    per = c->use_P ? 2 : 5;
  } else {
    const IterArgs A0 = make_iter_args(c, 0, 0, 0);
    if (!cuda_ok(pcg ? launch_pcg_first(A0, st) : launch_dip_first(A0, st), "first dipole step"))
      return CCP_ERR_CUDA;
    for (int step = 0;; step++) {
      // the PCG start takes no step, so its first step always runs
      if (!pcg || step > 0) {
        CK(cudaMemcpyAsync(c->h_istate, c->d_istate, 3 * sizeof(double), cudaMemcpyDeviceToHost,
                           st));
        CK(cudaStreamSynchronize(st));
        const int it = (int)c->h_istate[0];
        if (!(c->h_istate[1] > thr && it < c->maxit)) break;
      }
      if (!cuda_ok(enqueue_dip_step(c, st, 0, 0, step & 1, &per), "dipole step"))
        return CCP_ERR_CUDA;
    }
    if (!per) per = c->use_P ? 2 : 5;
  }
  c->ind_per_iter = per;
  return CCP_OK;
}

// Allocates the phase-factor tables when the dipole iteration can use them.
int ensure_phase_matrix(ccp_context *c) {
  const size_t nw = (size_t)c->nm * c->S.np, nz = 2 * (size_t)c->kmax[2] + 1;
  // XY[site][l][m] and Z[site][n], or in the row form XYr[row][site], Z and ZT[n][site]
  const size_t n = nw * std::max((size_t)(c->kmax[0] + 1) * (2 * c->kmax[1] + 1) + nz,
                                 (size_t)c->nrow + 2 * nz);
  // the gather records pack the phase-table row of n in 8 bits
  c->use_P = c->opt_phase && c->nk > 0 && n * sizeof(double2) <= kPhaseBudget &&
             2 * c->kmax[2] + 1 <= 255;
  const size_t npm = (size_t)c->nm * c->S.np * (size_t)c->nk;
  c->use_PM = c->use_P && c->opt_pm && npm * sizeof(double2) <= full_phase_budget(c);
  c->use_rows = c->use_P && !c->use_PM && c->opt_rows &&
                iter_rows_fit(c->opt_sum_sites, 2 * c->kmax[2] + 1, c->row_span);
  if (c->use_P && n > c->P_cap) {
    if (c->d_P) cudaFree(c->d_P);
    c->d_P = nullptr;
    c->P_cap = 0;
    CK(dalloc(&c->d_P, n));
    c->P_cap = n;
  }
  if (c->use_PM && npm > c->PM_cap) {
    if (c->d_PM) cudaFree(c->d_PM);
    c->d_PM = nullptr;
    c->PM_cap = 0;
    CK(dalloc(&c->d_PM, npm));
    c->PM_cap = npm;
  }
  return CCP_OK;
}

#define LK(call)                                        \
  do {                                                  \
    c->launches++;                                      \
    if (!cuda_ok((call), #call)) return CCP_ERR_CUDA;   \
  } while (0)

// FS3's cut-off, damping and switch constants (threebody_potential.f90:860-904, 1418-1423) in
// bohr for a box of `box` Angstrom.
Fs3Params fs3_params(const ccp_context *c, double box) {
  Fs3Params F3;
  F3.boxb = box / kBohr2a;
  F3.rc2 = std::pow(6.3, 2.0) * std::pow(kBohr2a, -2.0);
  F3.alp3 = c->alpha3 * kBohr2a;
  F3.r0dmp = 6.20446 / kBohr2a;
  F3.delta33 = c->delta33;
  F3.rmin = 4.5 / kBohr2a;
  F3.rmax = 5.5 / kBohr2a;
  return F3;
}

// Runs the enabled terms on inputs already in the context's device buffers
// (x, y, z at px.., sites at pxs.. with leading dimension ld).
int evaluate_impl(ccp_context *c, const double *px, const double *py, const double *pz,
             const double *pxs, const double *pys, const double *pzs, int ld, double box,
             unsigned mask, EvalOut &o) {
  cudaStream_t st = c->stream;
  const int nm = c->nm, ns = c->ns;
  const SiteSets &S = c->S;
  if ((mask & (T_FS2 | T_FS3)) && !c->three_body) mask &= ~(T_FS2 | T_FS3);
  if ((mask & T_FS2) && !c->s2) mask &= ~T_FS2;
  if ((mask & T_VDW) && !c->have_vdw) mask &= ~T_VDW;
  if ((mask & T_FS3) && (!c->s3 || !c->have_fs3)) mask &= ~T_FS3;
  if ((mask & T_FS3) && ns < kNs3) {
    set_error("FS3 needs 17 sites per molecule");
    return CCP_ERR_BAD_INPUT;
  }
  if ((mask & T_FS2) && ns < 5) {
    set_error("FS2 needs 5 sites per molecule");
    return CCP_ERR_BAD_INPUT;
  }
  EwaldParams P;
  P.alpha = c->alpha;
  P.rcutsd = c->rcutsd;
  P.box = box;
  P.twosqpi = 2.0 / std::sqrt(kPi);
  P.delta2 = 1.65 / kBohr2a;
  P.delta3 = 1.55 / kBohr2a;
  P.damped = c->damped ? 1 : 0;
  const double boxb = box / kBohr2a;
  const Fs3Params F3 = fs3_params(c, box);
  Fs2Params F2;
  F2.boxb = boxb;
  F2.rc2 = c->rcutsd3 * std::pow(kBohr2a, -2.0);
  F2.alp3 = c->alpha3 * kBohr2a;
  F2.r0dmp = 7.40446 / kBohr2a;
  F2.delta33 = c->delta33;
  if (mask & T_KSPACE || mask & T_INDUCTION) {
    int r = ensure_kspace(c, box);
    if (r) return r;
  }
  if (mask & T_INDUCTION) {
    int r = ensure_phase_matrix(c);
    if (r) return r;
  }
  // neighbour-list radius covering every consumer (each re-tests with its exact cut-off)
  double rl = c->rcut;
  if (mask & T_FS3) rl = std::max(rl, 6.3);
  if (mask & T_FS2) rl = std::max(rl, c->rcut3);
  rl += 0.05;

  // phase k runs between ev[2k] and ev[2k+1], recorded on the stream it runs on
  auto pbeg = [&](int k, cudaStream_t s) {
    if (c->timing) {
      cudaEventRecord(c->ev[2 * k], s);
      c->phase_ran |= 1u << k;
    }
  };
  auto pend = [&](int k, cudaStream_t s) {
    if (c->timing) cudaEventRecord(c->ev[2 * k + 1], s);
  };
  const bool side = c->opt_overlap && (mask & (T_FS2 | T_FS3 | T_VDW));
  // Ewald + induction run on a high-priority internal stream, the three-body terms on
  // low-priority ones, so that freed SM slots go to the latency-bound induction chain first
  cudaStream_t s3 = side ? c->s_fs3 : st, s2 = side ? c->s_fs2 : st, sm = side ? c->s_main : st;
  for (int attempt = 0; attempt < 3; attempt++) {
    c->launches = 0;
    c->phase_ran = 0;
    pbeg(0, st);
    LK(launch_prep(px, py, pz, pxs, pys, pzs, nm, ld, S, c->d_com, c->d_act, c->d_comb, c->d_s17,
                   std::min(ns, kNs3), c->d_f, 6 * nm * ns, c->d_fc2, c->d_fc3, c->d_scal,
                   c->d_icnt, st));
    const bool need_nbr = mask & (T_RSPACE | T_INDUCTION | T_FS2 | T_FS3 | T_VDW);
    if (need_nbr) {
      // the cell-list search when the box holds 5+ cells of side >= rl/2 per axis and its
      // kept candidates fit a block's shared memory; the all-pairs scan otherwise (same lists)
      const int nc = c->opt_cells && (size_t)c->cap * (sizeof(double4) + sizeof(int)) <= 48 * 1024
                         ? cell_grid(box, rl)
                         : 0;
      c->cells_active = nc > 0;
      if (nc) {
        const size_t need = cell_scratch_ints(nc, nm);
        if (need > c->cells_cap) {
          if (c->d_cells) cudaFree(c->d_cells);
          c->d_cells = nullptr;
          c->cells_cap = 0;
          CK(dalloc(&c->d_cells, need));
          c->cells_cap = need;
        }
        c->launches += 3;  // four kernels; LK counts one
        LK(launch_neighbors_cells(c->d_com, nm, box, rl * rl, nc, c->cap, c->d_cells, c->d_nbr,
                                  c->d_nbrv, c->d_ncnt, c->d_icnt, st));
      } else {
        LK(launch_neighbors(c->d_com, nm, box, rl * rl, c->cap, c->d_nbr, c->d_nbrv, c->d_ncnt,
                            c->d_icnt, st));
      }
    }
    pend(0, st);
    // with the terms overlapping, the reciprocal-space branch runs on its own stream; its
    // forces go to the three-body block f3, which receives atomic additions only, while the
    // real-space kernels add to d_f without atomics
    const bool kfork = side && (mask & (T_KSPACE | T_INDUCTION));
    cudaStream_t sk = kfork ? c->s_kspace : sm;
    if (side) {
      CK(cudaEventRecord(c->ev_fork, st));
      CK(cudaStreamWaitEvent(s3, c->ev_fork, 0));
      CK(cudaStreamWaitEvent(s2, c->ev_fork, 0));
      CK(cudaStreamWaitEvent(sm, c->ev_fork, 0));
      if (kfork) CK(cudaStreamWaitEvent(sk, c->ev_fork, 0));
    }
    // three-body terms first, so that on side streams they start at once
    double *f3 = side ? c->d_f + (size_t)3 * nm * ns : c->d_f;
    double *gfs3 = nullptr;
    if ((mask & T_FS3) && c->opt_pgrad) {
      gfs3 = c->d_gfs3;
      CK(cudaMemsetAsync(gfs3, 0, sizeof(double) * kFs3GradLen, s3));
    }
    if (mask & T_FS3) {
      pbeg(7, s3);
      LK(launch_fs3_enum(c->d_comb, c->d_nbr, c->d_ncnt, c->cap, nm, F3, c->d_tri, c->tri_cap,
                         c->d_icnt, s3));
      pend(7, s3);
      pbeg(8, s3);
      const int fs3_prec = c->precision == CCP_MIXED && c->opt_fs3_low ? CCP_MIXED : CCP_FP64;
      LK(launch_fs3(fs3_prec, c->d_tri, c->d_icnt, c->tri_cap, c->d_s17, c->d_coef, c->d_bgr,
                    nm, ns, f3, c->d_fc3, c->d_scal, c->nsm, side ? c->opt_fs3_tpb : 0,
                    side ? c->opt_fs3_bps : 0, gfs3,
                    s3));
      pend(8, s3);
    }
    if (mask & T_FS2) {
      pbeg(6, s2);
      LK(launch_fs2_enum(c->d_comb, c->d_nbr, c->d_ncnt, c->cap, nm, F2, c->d_pairs, c->pair_cap,
                         c->d_icnt, s2));
      LK(launch_fs2(c->precision, c->d_pairs, c->d_icnt, c->pair_cap, c->d_comb, c->d_s17, c->d_nbr,
                    c->d_ncnt, c->cap, F2, nm, ns, f3, c->d_fc2, c->d_scal, s2));
      pend(6, s2);
    }
    if (mask & T_VDW) {
      pbeg(9, s2);
      LK(launch_vdw(pxs, pys, pzs, ld, c->d_nbr, c->d_nbrv, c->d_ncnt, c->cap, nm, ns,
                    c->rcutsd, c->d_vdw_row, c->d_vdw_qq, c->d_vdw_par, c->vdw_nrows,
                    c->d_vdw_site, c->vdw_nv, f3, c->d_scal, s2));
      pend(9, s2);
    }
    pbeg(1, sm);
    if (mask & (T_RSPACE | T_INDUCTION)) {
      // one kernel gives the real-space Ewald forces, the static field and (for the self
      // term or the induction) the intramolecular terms; an output that the mask does not
      // ask for goes to the scratch field buffer
      const bool with_self = mask & (T_SELF | T_INDUCTION);
      LK(launch_pair_static(px, py, pz, pxs, pys, pzs, ld, c->d_act, c->d_nbr, c->d_nbrv,
                            c->d_ncnt, c->cap, nm, S, P, (mask & T_RSPACE) ? c->d_f : c->d_eir,
                            c->d_e0r, c->d_e0s, with_self ? 1 : 0,
                            (mask & T_SELF) ? c->d_f : c->d_eir, c->d_e0slf, c->d_scal, sm));
    } else if (mask & T_SELF) {
      LK(launch_self_static(px, py, pz, pxs, pys, pzs, nm, ld, S, P, c->d_f, c->d_e0slf,
                            c->d_scal, sm));
    }
    pend(1, sm);
    double *fk = kfork ? f3 : c->d_f;
    pbeg(2, sk);
    if (mask & (T_KSPACE | T_INDUCTION))
      LK(launch_ktab(c->d_com, c->d_act, nm, S, box, c->kmax[0], c->kmax[1], c->kmax[2], c->d_tab,
                     sk));
    if (mask & T_KSPACE)
      LK(launch_kspace_sums(0, c->d_kv, c->nk, c->d_tab, nm, S, c->kmax[0], c->kmax[1], c->kmax[2],
                            c->d_mu, c->d_sk, sk));
    // the Ewald energy and forces from those sums: here when the chain is serial, or after
    // the dipole loop's inputs on the reciprocal branch's stream, beside the loop (which uses
    // its own S(k) buffers)
    const bool ewald_late = kfork && (mask & T_INDUCTION);
    if ((mask & T_KSPACE) && !ewald_late) {
      LK(launch_kspace_energy(0, c->d_kv, c->nk, c->d_sk, c->alpha, c->d_scal, sk));
      LK(launch_kspace_gather(0, c->d_kv, c->nk, c->d_tab, nm, S, c->kmax[0], c->kmax[1],
                              c->kmax[2], c->d_mu, c->d_sk, nullptr, fk, sk));
    }
    pend(2, sk);
    if (mask & T_INDUCTION) {
      pbeg(3, sm);
      // the static field's structure factors (charges, mode 1) are the Ewald sums' (mode 0):
      // when those ran, d_sk still holds them
      if (!(mask & T_KSPACE))
        LK(launch_kspace_sums(1, c->d_kv, c->nk, c->d_tab, nm, S, c->kmax[0], c->kmax[1],
                              c->kmax[2], c->d_mu, c->d_sk, sk));
      LK(launch_kspace_gather(1, c->d_kv, c->nk, c->d_tab, nm, S, c->kmax[0], c->kmax[1],
                              c->kmax[2], c->d_mu, c->d_sk, c->d_e0k, fk, sk));
      if (c->use_rows) {
        const size_t nw = (size_t)nm * S.np, nz = 2 * c->kmax[2] + 1;
        double2 *XYr = c->d_P, *Z = XYr + (size_t)c->nrow * nw, *ZT = Z + nz * nw;
        LK(launch_phase_rows(c->d_tab, nm, S, c->kmax[0], c->kmax[1], c->kmax[2], c->d_rows,
                             c->nrow, XYr, Z, ZT, sk));
      } else if (c->use_P) {
        const int nlm = (c->kmax[0] + 1) * (2 * c->kmax[1] + 1), nz = 2 * c->kmax[2] + 1;
        double2 *XY = c->d_P, *Z = c->d_P + (size_t)nm * S.np * nlm;
        LK(launch_phase_factors(c->d_tab, nm, S, c->kmax[0], c->kmax[1], c->kmax[2], XY, Z, sk));
        if (c->use_PM)
          LK(launch_phase_matrix(c->d_kg, c->nk, nm * S.np, nlm, nz, XY, Z, c->d_PM, sk));
      }
      if (kfork) CK(cudaEventRecord(c->ev_k1, sk));
      if ((mask & T_KSPACE) && ewald_late) {
        LK(launch_kspace_energy(0, c->d_kv, c->nk, c->d_sk, c->alpha, c->d_scal, sk));
        LK(launch_kspace_gather(0, c->d_kv, c->nk, c->d_tab, nm, S, c->kmax[0], c->kmax[1],
                                c->kmax[2], c->d_mu, c->d_sk, nullptr, fk, sk));
      }
      if (!c->damped) CK(cudaMemsetAsync(c->d_e0s, 0, sizeof(double) * nm * S.np * 3, sm));
      LK(launch_dip_tensor(px, py, pz, pxs, pys, pzs, ld, c->d_act, c->d_nbr, c->d_nbrv, c->d_ncnt,
                           c->cap, nm, S, P, c->d_T4, c->d_TB, c->d_S4, c->d_SB, sm));
      if (kfork) CK(cudaStreamWaitEvent(sm, c->ev_k1, 0));
      LK(launch_static_total(nm * S.np * 3, c->d_e0r, c->d_e0k, c->d_e0slf, c->d_e0s, c->d_e0tot,
                             sm));
      pend(3, sm);
      pbeg(4, sm);
      {
        int r = run_dipole_loop(c, sm);
        if (r) return r;
      }
      pend(4, sm);
      pbeg(5, sm);
      if (kfork) {
        CK(cudaEventRecord(c->ev_lp, sm));
        CK(cudaStreamWaitEvent(sk, c->ev_lp, 0));
      }
      LK(launch_pair_indforce(px, py, pz, pxs, pys, pzs, ld, c->d_act, c->d_nbr, c->d_nbrv,
                              c->d_ncnt, c->cap, nm, S, P, c->d_mu, c->d_f, c->d_scal, sm));
      LK(launch_kspace_sums(3, c->d_kv, c->nk, c->d_tab, nm, S, c->kmax[0], c->kmax[1], c->kmax[2],
                            c->d_mu, c->d_sk, sk));
      LK(launch_kspace_energy(3, c->d_kv, c->nk, c->d_sk, c->alpha, c->d_scal, sk));
      LK(launch_kspace_gather(3, c->d_kv, c->nk, c->d_tab, nm, S, c->kmax[0], c->kmax[1],
                              c->kmax[2], c->d_mu, c->d_sk, nullptr, fk, sk));
      if (kfork) {
        CK(cudaEventRecord(c->ev_k2, sk));
        CK(cudaStreamWaitEvent(sm, c->ev_k2, 0));
      }
      pend(5, sm);
    } else if (kfork) {
      CK(cudaEventRecord(c->ev_k2, sk));
      CK(cudaStreamWaitEvent(sm, c->ev_k2, 0));
    }
    if (side) {
      CK(cudaEventRecord(c->ev_j3, s3));
      CK(cudaEventRecord(c->ev_j2, s2));
      CK(cudaEventRecord(c->ev_jm, sm));
      CK(cudaStreamWaitEvent(st, c->ev_j3, 0));
      CK(cudaStreamWaitEvent(st, c->ev_j2, 0));
      CK(cudaStreamWaitEvent(st, c->ev_jm, 0));
      LK(launch_add(3 * nm * ns, f3, c->d_f, st));
    }
    if (c->dl_req) {
      const size_t n = (size_t)nm * c->ns, np3 = (size_t)nm * c->S.np * 3;
      double *h = c->h_out;
      CK(cudaMemcpyAsync(h, c->d_f, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(h + 3 * n, c->d_fc2, 3 * nm * sizeof(double), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(h + 3 * n + 3 * nm, c->d_fc3, 3 * nm * sizeof(double),
                         cudaMemcpyDeviceToHost, st));
      if (np3)
        CK(cudaMemcpyAsync(h + 3 * n + 6 * nm, c->d_mu, np3 * sizeof(double),
                           cudaMemcpyDeviceToHost, st));
    }
    CK(cudaMemcpyAsync(c->h_scal, c->d_scal, sizeof(double) * S_COUNT, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(c->h_icnt, c->d_icnt, sizeof(int) * C_ALLOC, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const int *ic = c->h_icnt;
    if (ic[C_NONFINITE] > 0) {
      CK(cudaMemset(c->d_icnt + C_NONFINITE, 0, sizeof(int)));
      set_error("non-finite coordinates (NaN or infinite) in the positions or site offsets");
      return CCP_ERR_BAD_INPUT;
    }
    bool grow = false;
    int ncap = c->cap, ntcap = c->tri_cap, npcap = c->pair_cap;
    if (ic[C_OVERFLOW] > 0) {
      ncap = std::min(nm, ic[C_OVERFLOW] + 32);
      grow = true;
    }
    if (ic[C_NTRI_FS3] > c->tri_cap) {
      ntcap = ic[C_NTRI_FS3] + ic[C_NTRI_FS3] / 4 + 64;
      grow = true;
    }
    if (ic[C_NPAIR_FS2] > c->pair_cap) {
      npcap = ic[C_NPAIR_FS2] + ic[C_NPAIR_FS2] / 4 + 64;
      grow = true;
    }
    if (grow) {
      int r = ensure_lists(c, ncap, ntcap, npcap);
      if (r) return r;
      continue;
    }
    c->pgrad_valid = gfs3 != nullptr;
    if (mask & T_INDUCTION) {
      o.iters = (int)c->h_istate[0];
      o.ind_e = c->h_istate[2];
      // the Jacobi first step is one kernel; the PCG start takes no step
      c->launches += 1 + c->ind_per_iter * (c->pcg_active ? o.iters : o.iters - 1);
      o.converged = o.iters < c->maxit;
      if (!o.converged) {
        set_error("No convergence in the induced-dipole iteration (maxit reached)");
        return CCP_ERR_NOT_CONVERGED;
      }
    }
    if (c->timing)
      for (int k = 0; k < CCP_NPHASE; k++) {
        float ms = 0.f;
        if (c->phase_ran & (1u << k)) cudaEventElapsedTime(&ms, c->ev[2 * k], c->ev[2 * k + 1]);
        c->phase_ms[k] = ms;
      }
    const double *h = c->h_scal;
    o.sumff = h[S_SELF_SUMFF];
    o.self_vir = h[S_SELF_VIR];
    o.rc_e = h[S_RC_E];
    o.rc_vir = h[S_RC_VIR];
    o.kc_e = h[S_KC_E];
    o.kc_vir = h[S_KC_VIR];
    o.ind_vir = h[S_IND_VIR_R] + 2.0 * kR4pie0 * h[S_IND_VIR_K];
    o.fs2_e = h[S_FS2_E];
    o.fs2_vir = h[S_FS2_VIR];
    o.fs3_e = h[S_FS3_E];
    o.fs3_vir = h[S_FS3_VIR];
    o.vdw_e = h[S_VDW_E];
    o.vdw_vir = h[S_VDW_VIR];
    o.ntri = ic[C_NTRI_FS3];
    o.nblend = ic[C_NBLEND_FS3];
    o.nfs2 = ic[C_NTRI_FS2];
    return CCP_OK;
  }
  set_error("internal list capacity kept overflowing");
  return CCP_ERR_CAPACITY;
}

int evaluate(ccp_context *c, const double *px, const double *py, const double *pz,
             const double *pxs, const double *pys, const double *pzs, int ld, double box,
             unsigned mask, EvalOut &o) {
  const int r = evaluate_impl(c, px, py, pz, pxs, pys, pzs, ld, box, mask, o);
  if (r) {  // no side-stream work of a failed evaluation may outlive it
    cudaStreamSynchronize(c->s_fs3);
    cudaStreamSynchronize(c->s_fs2);
    cudaStreamSynchronize(c->s_main);
    cudaStreamSynchronize(c->s_kspace);
  }
  return r;
}

int check_args(ccp_context *c, const void *const *ptrs, int n, int ld) {
  if (!c) {
    set_error("null context");
    return CCP_ERR_BAD_INPUT;
  }
  for (int k = 0; k < n; k++)
    if (!ptrs[k]) {
      set_error("null array argument");
      return CCP_ERR_BAD_INPUT;
    }
  if (ld < c->ns) {
    set_error("leading dimension ld is smaller than the number of sites");
    return CCP_ERR_BAD_INPUT;
  }
  return CCP_OK;
}

// Upload the caller's host arrays (through pinned staging) into the context buffers.
int upload(ccp_context *c, const double *x, const double *y, const double *z, const double *xs,
           const double *ys, const double *zs, int ld) {
  int r = ensure_inputs(c, ld);
  if (r) return r;
  const size_t nm = c->nm, ns = (size_t)nm * ld;
  r = ensure_host_io(c, 3 * nm + 3 * ns);
  if (r) return r;
  double *h = c->h_io;
  std::memcpy(h, x, nm * sizeof(double));
  std::memcpy(h + nm, y, nm * sizeof(double));
  std::memcpy(h + 2 * nm, z, nm * sizeof(double));
  std::memcpy(h + 3 * nm, xs, ns * sizeof(double));
  std::memcpy(h + 3 * nm + ns, ys, ns * sizeof(double));
  std::memcpy(h + 3 * nm + 2 * ns, zs, ns * sizeof(double));
  cudaStream_t st = c->stream;
  // d_x, d_y, d_z and d_xs, d_ys, d_zs are two contiguous blocks
  CK(cudaMemcpyAsync(c->d_x, h, 3 * nm * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(c->d_xs, h + 3 * nm, 3 * ns * sizeof(double), cudaMemcpyHostToDevice, st));
  return CCP_OK;
}

// Pinned result buffer of ccp_hot_path: site forces, FS2 and FS3 COM forces and dipoles.
int ensure_host_out(ccp_context *c) {
  const size_t n = 3 * (size_t)c->nm * c->ns + 6 * (size_t)c->nm + (size_t)c->nm * c->S.np * 3;
  if (n <= c->h_out_cap) return CCP_OK;
  if (c->h_out) cudaFreeHost(c->h_out);
  c->h_out = nullptr;
  CK(cudaMallocHost((void **)&c->h_out, n * sizeof(double)));
  c->h_out_cap = n;
  return CCP_OK;
}

// Unpack the results that evaluate() copied into h_out into the caller's arrays: site forces
// added into the ld layout, COM forces copied, dipoles written at the polarisable sites.
void unpack_host_out(const ccp_context *c, int ld, double *fxs, double *fys, double *fzs,
                     double *fxfs2, double *fyfs2, double *fzfs2, double *fxfs3, double *fyfs3,
                     double *fzfs3, double *mx, double *my, double *mz) {
  const size_t nm = c->nm, n = nm * c->ns;
  const double *h = c->h_out;
  double *f[3] = {fxs, fys, fzs};
  for (int a = 0; a < 3; a++) {
    if (!f[a]) continue;
    const double *src = h + a * n;
    for (size_t i = 0; i < nm; i++)
      for (int s = 0; s < c->ns; s++) f[a][i * ld + s] += src[i * c->ns + s];
  }
  double *com[6] = {fxfs2, fyfs2, fzfs2, fxfs3, fyfs3, fzfs3};
  for (int a = 0; a < 6; a++)
    if (com[a]) std::memcpy(com[a], h + 3 * n + a * nm, nm * sizeof(double));
  double *m[3] = {mx, my, mz};
  const double *mu = h + 3 * n + 6 * nm;
  for (int a = 0; a < 3; a++) {
    if (!m[a]) continue;
    for (size_t i = 0; i < nm; i++) {
      for (int s = 0; s < c->ns; s++) m[a][i * ld + s] = 0.0;
      for (int p = 0; p < c->S.np; p++)
        m[a][i * ld + c->S.psite[p]] = mu[(i * c->S.np + p) * 3 + a];
    }
  }
}

// Download the compact site forces and add them into the caller's (ld-layout) arrays.
int download_forces(ccp_context *c, int ld, double *fxs, double *fys, double *fzs) {
  if (!fxs && !fys && !fzs) return CCP_OK;
  const size_t n = (size_t)c->nm * c->ns;
  int r = ensure_host_io(c, 3 * n);
  if (r) return r;
  CK(cudaMemcpyAsync(c->h_io, c->d_f, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double *out[3] = {fxs, fys, fzs};
  for (int a = 0; a < 3; a++) {
    if (!out[a]) continue;
    const double *src = c->h_io + a * n;
    for (int i = 0; i < c->nm; i++)
      for (int s = 0; s < c->ns; s++) out[a][(size_t)i * ld + s] += src[(size_t)i * c->ns + s];
  }
  return CCP_OK;
}

int download_com(ccp_context *c, const double *d, double *fx, double *fy, double *fz) {
  if (!fx && !fy && !fz) return CCP_OK;
  const size_t nm = c->nm;
  int r = ensure_host_io(c, 3 * nm);
  if (r) return r;
  CK(cudaMemcpyAsync(c->h_io, d, 3 * nm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (fx) std::memcpy(fx, c->h_io, nm * sizeof(double));
  if (fy) std::memcpy(fy, c->h_io + nm, nm * sizeof(double));
  if (fz) std::memcpy(fz, c->h_io + 2 * nm, nm * sizeof(double));
  return CCP_OK;
}

int download_dipoles(ccp_context *c, int ld, double *mx, double *my, double *mz) {
  if (!mx && !my && !mz) return CCP_OK;
  const size_t n = (size_t)c->nm * c->S.np * 3;
  int r = ensure_host_io(c, n);
  if (r) return r;
  CK(cudaMemcpyAsync(c->h_io, c->d_mu, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double *out[3] = {mx, my, mz};
  for (int a = 0; a < 3; a++) {
    if (!out[a]) continue;
    for (int i = 0; i < c->nm; i++) {
      for (int s = 0; s < c->ns; s++) out[a][(size_t)i * ld + s] = 0.0;
      for (int p = 0; p < c->S.np; p++)
        out[a][(size_t)i * ld + c->S.psite[p]] = c->h_io[((size_t)i * c->S.np + p) * 3 + a];
    }
  }
  return CCP_OK;
}

double self_point_energy(const ccp_context *c, double alp, double box) {
  // ewald.f90:79-88: -pi (sum q / alpha)^2 / (2 V) - alpha sum q^2 / sqrt(pi)
  const double t = c->sumq / alp;
  double e = -kPi * (t * t) / (2.0 * box * box * box);
  e = e - alp * c->sumq2 / std::sqrt(kPi);
  return e;
}

void fill_energies(ccp_context *c, const EvalOut &o, double box, ccp_energies *e) {
  e->scpe = kR4pie0 * (self_point_energy(c, c->alpha, box) - o.sumff) / 418.4;
  e->rcpe = o.rc_e / 418.4;
  e->kcpe = 2.0 * kR4pie0 * o.kc_e / 418.4;
  e->indpe = kR4pie0 * o.ind_e / 418.4;
  e->fs2pe = o.fs2_e * kH2kcal;
  e->fs3pe = o.fs3_e * kH2kcal;
  e->vdwpe = o.vdw_e / 418.4;
  e->vir = o.self_vir + o.rc_vir + 2.0 * kR4pie0 * o.kc_vir + o.ind_vir +
           o.fs2_vir * kH2kcal * 418.4 + o.fs3_vir * kH2kcal * 418.4 + o.vdw_vir;
  e->ind_iters = o.iters;
  e->n_fs3_triples = o.ntri;
  e->n_fs3_blend = o.nblend;
  e->n_fs2_triples = o.nfs2;
}

unsigned allowed_mask(const ccp_context *c);

unsigned hot_mask(const ccp_context *c) {
  unsigned m = T_SELF | T_RSPACE | T_KSPACE;
  if (c->induction) m |= T_INDUCTION;
  if (c->three_body) m |= T_FS2 | T_FS3;
  return m;
}

// Every term this context can evaluate: the hot path plus the 2-body term when the model is
// ccpol23plus.
unsigned allowed_mask(const ccp_context *c) {
  return hot_mask(c) | (c->have_vdw ? unsigned(T_VDW) : 0u);
}

__global__ void k_scatter_out(const double *__restrict__ f, int nm, int ns, int ld, double *fx,
                              double *fy, double *fz) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = nm * ns;
  if (t >= n) return;
  const int i = t / ns, s = t % ns;
  const size_t o = (size_t)i * ld + s;
  if (fx) fx[o] += f[t];
  if (fy) fy[o] += f[(size_t)n + t];
  if (fz) fz[o] += f[2 * (size_t)n + t];
}

__global__ void k_scatter_dip(const double *__restrict__ mu, int nm, int ns, int np, int p0,
                              int ld, double *mx, double *my, double *mz) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nm * ns) return;
  const int i = t / ns, s = t % ns;
  const int p = s - p0;
  const size_t o = (size_t)i * ld + s;
  double v[3] = {0, 0, 0};
  if (p >= 0 && p < np)
    for (int a = 0; a < 3; a++) v[a] = mu[((size_t)i * np + p) * 3 + a];
  if (mx) mx[o] = v[0];
  if (my) my[o] = v[1];
  if (mz) mz[o] = v[2];
}

}  // namespace

extern "C" {

int ccp_context_create(const ccp_model *m, int nm, double box0, int device, int precision,
                       ccp_context **out) {
  if (!m || !out || nm < 1 || !(box0 > 0.0) || (precision != CCP_FP64 && precision != CCP_MIXED)) {
    set_error("ccp_context_create: bad argument (null model or output, nm < 1, box0 <= 0 or an "
              "unknown precision)");
    return CCP_ERR_BAD_INPUT;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("no CUDA device");
    return CCP_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) {
    set_error("device ordinal out of range");
    return CCP_ERR_BAD_INPUT;
  }
  auto *c = new ccp_context();
  c->device = device;
  c->precision = precision;
  // the mixed form solves for the dipoles by PCG to 1e-8 D RMS, the FP64 form by the
  // reference's Jacobi iteration and criterion
  c->opt_solver = precision == CCP_MIXED ? 2 : 0;
  c->nm = nm;
  c->ns = m->ns;
  c->npol = m->npol;
  if (!cuda_ok(cudaSetDevice(device), "cudaSetDevice")) {
    delete c;
    return CCP_ERR_CUDA;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) {
    c->nsm = prop.multiProcessorCount;
    if (prop.l2CacheSize > 0) c->l2_bytes = (size_t)prop.l2CacheSize;
  }
  // site sets from the model's charges and polarisabilities
  SiteSets &S = c->S;
  std::memset(&S, 0, sizeof(S));
  S.ns = m->ns;
  const int p0 = m->ns - m->npol;
  for (int s = 0; s < m->ns; s++) c->charge[s] = m->charge[s];
  for (int s = 0; s < m->ns; s++) {
    const bool q = m->charge[s] != 0.0;
    const bool pol = s >= p0;
    if (!q && !pol) continue;
    if (S.na >= ccpd::kMaxA || (q && S.nq >= ccpd::kMaxQ) || (pol && S.np >= ccpd::kMaxP)) {
      set_error("too many charged/polarisable sites per molecule");
      delete c;
      return CCP_ERR_BAD_INPUT;
    }
    const int a = S.na++;
    S.asite[a] = s;
    S.q[a] = m->charge[s];
    S.p_of_a[a] = -1;
    if (q) {
      S.qsite[S.nq] = s;
      S.a_of_q[S.nq] = a;
      if (s < p0) S.self_q[S.nself_q++] = S.nq;
      S.nq++;
    }
    if (pol) {
      S.psite[S.np] = s;
      S.a_of_p[S.np] = a;
      S.apol[S.np] = m->polarizability[s] * std::pow(kBohr2a, 3.0);
      S.p_of_a[a] = S.np;
      S.np++;
    }
  }
  c->sumq = 0;
  c->sumq2 = 0;
  for (int i = 0; i < nm; i++)
    for (int s = 0; s < m->ns; s++) {
      c->sumq = c->sumq + m->charge[s];
      c->sumq2 = c->sumq2 + m->charge[s] * m->charge[s];
    }
  c->rcut = m->rcut;
  c->rcutsd = m->rcut * m->rcut;
  c->rcut3 = m->rcut3;
  c->rcutsd3 = m->rcut3 * m->rcut3;
  c->alpha3 = m->alpha3;
  c->delta33 = m->delta33;
  c->s2 = m->s2_term;
  c->s3 = m->s3_term;
  c->three_body = m->nonadditive_3b;
  c->induction = m->induction && m->ind_model == "point_dipole";
  c->damped = m->induction_type == "damped";
  c->have_fs3 = m->have_fs3;
  ccp_ewald_setup(kEwp, m->rcut, box0, &c->alpha, &c->kmax[0], &c->kmax[1], &c->kmax[2]);

  auto fail = [&](const char *what) {
    set_error(std::string("ccp_context_create: ") + what + ": " + cudaGetErrorString(cudaGetLastError()));
    free_ctx(c);
    delete c;
    return CCP_ERR_CUDA;
  };
  if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) return fail("stream");
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  if (cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->s_fs3, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->s_fs2, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->s_main, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->s_kspace, cudaStreamNonBlocking, prio_hi) != cudaSuccess)
    return fail("stream");
  if (cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_j3, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_j2, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_jm, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_k1, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_k2, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_lp, cudaEventDisableTiming) != cudaSuccess)
    return fail("event");
  c->stream = c->own;
  if (cudaMalloc(&c->d_istate, kIterStateLen * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->d_ticket, sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(c->d_ticket, 0, sizeof(unsigned)) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_istate, 3 * sizeof(double)) != cudaSuccess)
    return fail("loop state");
  const size_t n = nm, nsi = (size_t)nm * m->ns, np3 = (size_t)nm * std::max(S.np, 1) * 3;
  bool ok = dalloc(&c->d_x, 3 * n) == cudaSuccess && dalloc(&c->d_com, n) == cudaSuccess &&
            dalloc(&c->d_comb, n) == cudaSuccess &&
            dalloc(&c->d_act, n * std::max(S.na, 1)) == cudaSuccess &&
            dalloc(&c->d_s17, n * kNs3) == cudaSuccess && dalloc(&c->d_f, 6 * nsi) == cudaSuccess &&
            dalloc(&c->d_fc2, 3 * n) == cudaSuccess && dalloc(&c->d_fc3, 3 * n) == cudaSuccess &&
            dalloc(&c->d_scal, (size_t)S_COUNT) == cudaSuccess &&
            dalloc(&c->d_icnt, (size_t)C_ALLOC) == cudaSuccess &&
            dalloc(&c->d_mu, np3) == cudaSuccess && dalloc(&c->d_e0r, np3) == cudaSuccess &&
            dalloc(&c->d_e0k, np3) == cudaSuccess && dalloc(&c->d_e0slf, np3) == cudaSuccess &&
            dalloc(&c->d_e0s, np3) == cudaSuccess && dalloc(&c->d_eir, std::max(np3, 3 * nsi)) == cudaSuccess &&
            dalloc(&c->d_eik, np3) == cudaSuccess && dalloc(&c->d_eislf, np3) == cudaSuccess &&
            dalloc(&c->d_eis, np3) == cudaSuccess && dalloc(&c->d_ncnt, n) == cudaSuccess &&
            dalloc(&c->d_mu2, np3) == cudaSuccess && dalloc(&c->d_e0tot, np3) == cudaSuccess &&
            dalloc(&c->d_eim, np3) == cudaSuccess &&
            dalloc(&c->d_S4, n * std::max(S.np, 1) * std::max(S.np, 1)) == cudaSuccess &&
            dalloc(&c->d_SB, n * std::max(S.np, 1) * std::max(S.np, 1)) == cudaSuccess;
  if (!ok) return fail("device allocation");
  c->d_y = c->d_x + n;  // x, y, z share one allocation, so that an upload is one copy
  c->d_z = c->d_y + n;
  if (cudaMemset(c->d_e0s, 0, np3 * sizeof(double)) != cudaSuccess) return fail("memset");
  if (cudaMemset(c->d_mu, 0, np3 * sizeof(double)) != cudaSuccess) return fail("memset");
  if (cudaMemset(c->d_icnt, 0, C_ALLOC * sizeof(int)) != cudaSuccess) return fail("memset");
  if (cudaMallocHost((void **)&c->h_scal, sizeof(double) * S_COUNT) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_icnt, sizeof(int) * C_ALLOC) != cudaSuccess)
    return fail("pinned allocation");
  if (ensure_inputs(c, m->ns) != CCP_OK) return fail("inputs");
  const int cap0 = std::min(nm - 1, 192);
  if (ensure_lists(c, std::max(cap0, 1), 96 * nm, 48 * nm) != CCP_OK) return fail("lists");
  c->totm = m->totm;
  for (int a = 0; a < 3; a++) c->pmi[a] = m->pmi[a];
  if (dalloc(&c->d_pcoord, m->pcoord.size()) != cudaSuccess ||
      cudaMemcpy(c->d_pcoord, m->pcoord.data(), m->pcoord.size() * sizeof(double),
                 cudaMemcpyHostToDevice) != cudaSuccess)
    return fail("principal-frame sites");
  if (m->pot_name == "ccpol23plus" && !m->vdw.empty()) {
    // parameter row of every site pair (name match in either order, first row wins, as the
    // reference's row loop), charge products, and the sites that have any row
    const int ns = m->ns;
    std::vector<int> row(ns * ns, -1), vs;
    std::vector<double> qq(ns * ns), par;
    for (int a = 0; a < ns; a++)
      for (int b = 0; b < ns; b++) {
        qq[a * ns + b] = m->charge[a] * m->charge[b];
        for (size_t k = 0; k < m->vdw.size(); k++) {
          const auto &r = m->vdw[k];
          if ((m->names[a] == r.a && m->names[b] == r.b) || (m->names[b] == r.a && m->names[a] == r.b)) {
            row[a * ns + b] = (int)k;
            break;
          }
        }
      }
    for (int a = 0; a < ns; a++) {
      bool any = false;
      for (int b = 0; b < ns; b++) any = any || row[a * ns + b] >= 0;
      if (any) vs.push_back(a);
    }
    // initialization.f90:612-628: c0..c3, c6, c8, c10 to internal energy units
    for (const auto &r : m->vdw) {
      const double *p = r.p;
      const double v[kVdwPar] = {p[0], p[1] * 418.4, p[2] * 418.4, p[3] * 418.4, p[4] * 418.4,
                                 p[5] * 418.4, p[6] * 418.4, p[7] * 418.4, p[8], p[9], p[10], p[11]};
      par.insert(par.end(), v, v + kVdwPar);
    }
    if ((int)m->vdw.size() > kVdwMaxRows || vs.size() > 32 || vs.empty()) {
      set_error("ccp_context_create: ccpol23plus needs at most 64 parameter rows and 32 sites with rows");
      free_ctx(c);
      delete c;
      return CCP_ERR_BAD_INPUT;
    }
    c->vdw_nrows = (int)m->vdw.size();
    c->vdw_nv = (int)vs.size();
    if (dalloc(&c->d_vdw_row, row.size()) != cudaSuccess || dalloc(&c->d_vdw_site, vs.size()) != cudaSuccess ||
        dalloc(&c->d_vdw_qq, qq.size()) != cudaSuccess || dalloc(&c->d_vdw_par, par.size()) != cudaSuccess)
      return fail("2-body tables");
    if (cudaMemcpy(c->d_vdw_row, row.data(), row.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->d_vdw_site, vs.data(), vs.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->d_vdw_qq, qq.data(), qq.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->d_vdw_par, par.data(), par.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail("2-body upload");
    c->have_vdw = true;
  }
  if (m->have_fs3) {
    std::vector<double> coef(2 * m->coef_sr.size());
    std::copy(m->coef_sr.begin(), m->coef_sr.end(), coef.begin());
    std::copy(m->coef_lr.begin(), m->coef_lr.end(), coef.begin() + m->coef_sr.size());
    c->cs_sr = m->sr.cs;
    c->cs_lr = m->lr.cs;
    c->class_of_type = m->class_of_type;
    c->nclass = m->nclass;
    std::vector<double> bgr(2 * 3 * 289);
    for (int q = 0; q < 289; q++) {
      bgr[0 * 289 + q] = m->sr.b[q];
      bgr[1 * 289 + q] = m->sr.g[q];
      bgr[2 * 289 + q] = m->sr.r0[q];
      bgr[3 * 289 + q] = m->lr.b[q];
      bgr[4 * 289 + q] = m->lr.g[q];
      bgr[5 * 289 + q] = m->lr.r0[q];
    }
    c->bgr_host = bgr;
    if (dalloc(&c->d_coef, coef.size()) != cudaSuccess || dalloc(&c->d_bgr, bgr.size()) != cudaSuccess ||
        dalloc(&c->d_gfs3, (size_t)kFs3GradLen) != cudaSuccess ||
        dalloc(&c->d_types, (size_t)kNs3) != cudaSuccess)
      return fail("FS3 tables");
    if (cudaMemcpy(c->d_coef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->d_bgr, bgr.data(), bgr.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->d_types, m->fs3_type, kNs3 * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail("FS3 upload");
  }
  *out = c;
  return CCP_OK;
}

int ccp_context_destroy(ccp_context *ctx) {
  if (!ctx) return CCP_ERR_BAD_INPUT;
  free_ctx(ctx);
  delete ctx;
  return CCP_OK;
}

int ccp_context_set_ewald(ccp_context *ctx, double alpha, int k1, int k2, int k3) {
  if (!ctx || !(alpha > 0.0) || k1 < 1 || k2 < 1 || k3 < 1) {
    set_error("ccp_context_set_ewald: bad argument");
    return CCP_ERR_BAD_INPUT;
  }
  ctx->alpha = alpha;
  ctx->kmax[0] = k1;
  ctx->kmax[1] = k2;
  ctx->kmax[2] = k3;
  return CCP_OK;
}

int ccp_context_set_maxit(ccp_context *ctx, int maxit) {
  if (!ctx || maxit < 1) {
    set_error("ccp_context_set_maxit: bad argument");
    return CCP_ERR_BAD_INPUT;
  }
  ctx->maxit = maxit;
  return CCP_OK;
}

int ccp_context_set_stream(ccp_context *ctx, void *stream) {
  if (!ctx) return CCP_ERR_BAD_INPUT;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own;
  return CCP_OK;
}

int ccp_context_set_timing(ccp_context *ctx, int on) {
  if (!ctx) return CCP_ERR_BAD_INPUT;
  CK(cudaSetDevice(ctx->device));
  if (on && !ctx->ev[0])
    for (auto &e : ctx->ev) CK(cudaEventCreate(&e));
  ctx->timing = on != 0;
  return CCP_OK;
}

int ccp_context_set_option(ccp_context *ctx, const char *name, int value) {
  if (!ctx || !name) return CCP_ERR_BAD_INPUT;
  const std::string n(name);
  if (n == "graph_loop") {
    ctx->opt_graph = value != 0;
  } else if (n == "phase_matrix") {
    ctx->opt_phase = value != 0;
  } else if (n == "phase_matrix_full") {
    ctx->opt_pm = value != 0;
  } else if (n == "dipole_row_form") {
    ctx->opt_rows = value != 0;
  } else if (n == "dipole_sum_sites") {
    if (value < 1 || value > 128) {
      set_error("ccp_context_set_option: dipole_sum_sites must be 1..128");
      return CCP_ERR_BAD_INPUT;
    }
    ctx->opt_sum_sites = value;
  } else if (n == "dipole_gather_sites") {
    if (value != 2 && value != 3 && value != 4 && value != 6 && value != 8) {
      set_error("ccp_context_set_option: dipole_gather_sites must be 2, 3, 4, 6 or 8");
      return CCP_ERR_BAD_INPUT;
    }
    ctx->opt_gather_sites = value;
  } else if (n == "cell_list") {
    ctx->opt_cells = value != 0;
  } else if (n == "pdl") {
    ctx->opt_pdl = value != 0;
  } else if (n == "fs3_fp32_passes") {
    ctx->opt_fs3_low = value != 0;
  } else if (n == "fs3_high_priority") {
    // FS3's side stream at the chain's high priority (1) or the low one (0)
    if ((value != 0) != (ctx->opt_fs3_prio != 0)) {
      CK(cudaSetDevice(ctx->device));
      CK(cudaStreamSynchronize(ctx->s_fs3));
      int prio_lo = 0, prio_hi = 0;
      cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
      cudaStream_t s = nullptr;
      CK(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, value ? prio_hi : prio_lo));
      cudaStreamDestroy(ctx->s_fs3);
      ctx->s_fs3 = s;
      ctx->opt_fs3_prio = value != 0;
    }
  } else if (n == "dipole_solver") {
    if (value < 0 || value > 2) {
      set_error("ccp_context_set_option: dipole_solver must be 0 (Jacobi), 1 (PCG, the "
                "reference's criterion) or 2 (PCG, 1e-8 D RMS)");
      return CCP_ERR_BAD_INPUT;
    }
    ctx->opt_solver = value;
  } else if (n == "overlap") {
    ctx->opt_overlap = value != 0;
  } else if (n == "fs3_param_grad") {
    ctx->opt_pgrad = value != 0;
  } else if (n == "fs3_triples_per_block") {
    if (value < 0 || value > 4096) {
      set_error("ccp_context_set_option: fs3_triples_per_block must be 0..4096");
      return CCP_ERR_BAD_INPUT;
    }
    ctx->opt_fs3_tpb = value;
  } else if (n == "fs3_blocks_per_sm") {
    if (value < 0 || value > 32) {
      set_error("ccp_context_set_option: fs3_blocks_per_sm must be 0..32");
      return CCP_ERR_BAD_INPUT;
    }
    ctx->opt_fs3_bps = value;
  } else {
    set_error("ccp_context_set_option: unknown option " + n);
    return CCP_ERR_BAD_INPUT;
  }
  return CCP_OK;
}

int ccp_context_get_option(const ccp_context *ctx, const char *name, int *value) {
  if (!ctx || !name || !value) return CCP_ERR_BAD_INPUT;
  const std::string n(name);
  if (n == "graph_loop") {
    *value = ctx->opt_graph;
  } else if (n == "phase_matrix") {
    *value = ctx->opt_phase;
  } else if (n == "phase_matrix_active") {
    *value = ctx->use_P ? 1 : 0;
  } else if (n == "phase_matrix_full") {
    *value = ctx->opt_pm;
  } else if (n == "dipole_sum_sites") {
    *value = ctx->opt_sum_sites;
  } else if (n == "dipole_gather_sites") {
    *value = ctx->opt_gather_sites;
  } else if (n == "phase_matrix_full_active") {
    *value = ctx->use_PM ? 1 : 0;
  } else if (n == "dipole_row_form") {
    *value = ctx->opt_rows;
  } else if (n == "dipole_row_form_active") {
    *value = ctx->use_rows ? 1 : 0;
  } else if (n == "dipole_solver") {
    *value = ctx->opt_solver;
  } else if (n == "cell_list") {
    *value = ctx->opt_cells;
  } else if (n == "fs3_available") {
    *value = ctx->three_body && ctx->s3 && ctx->have_fs3 && ctx->ns >= kNs3 ? 1 : 0;
  } else if (n == "pdl") {
    *value = ctx->opt_pdl;
  } else if (n == "fs3_fp32_passes") {
    *value = ctx->opt_fs3_low;
  } else if (n == "fs3_high_priority") {
    *value = ctx->opt_fs3_prio;
  } else if (n == "cell_list_active") {
    *value = ctx->cells_active ? 1 : 0;
  } else if (n == "dipole_solver_pcg_active") {
    *value = ctx->pcg_active ? 1 : 0;
  } else if (n == "overlap") {
    *value = ctx->opt_overlap;
  } else if (n == "fs3_param_grad") {
    *value = ctx->opt_pgrad;
  } else if (n == "fs3_triples_per_block") {
    *value = ctx->opt_fs3_tpb;
  } else if (n == "fs3_blocks_per_sm") {
    *value = ctx->opt_fs3_bps;
  } else {
    set_error("ccp_context_get_option: unknown option " + n);
    return CCP_ERR_BAD_INPUT;
  }
  return CCP_OK;
}

int ccp_context_phase_ms(const ccp_context *ctx, double *ms, int n) {
  if (!ctx || !ms || n < 1 || n > CCP_NPHASE) return CCP_ERR_BAD_INPUT;
  for (int k = 0; k < n; k++) ms[k] = ctx->phase_ms[k];
  return CCP_OK;
}

int ccp_context_last_launches(const ccp_context *ctx, int *launches) {
  if (!ctx || !launches) return CCP_ERR_BAD_INPUT;
  *launches = ctx->launches;
  return CCP_OK;
}

int ccp_ewald_self_correction(ccp_context *ctx, double alp, double box, const double *x,
                              const double *y, const double *z, const double *xs,
                              const double *ys, const double *zs, int ld, double *qscpe,
                              double *fxs, double *fys, double *fzs, double *vir) {
  const void *p[] = {x, y, z, xs, ys, zs, qscpe, fxs, fys, fzs, vir};
  int r = check_args(ctx, p, 11, ld);
  if (r) return r;
  CK(cudaSetDevice(ctx->device));
  const double keep = ctx->alpha;
  ctx->alpha = alp;
  r = upload(ctx, x, y, z, xs, ys, zs, ld);
  EvalOut o;
  if (!r) r = evaluate(ctx, ctx->d_x, ctx->d_y, ctx->d_z, ctx->d_xs, ctx->d_ys, ctx->d_zs, ld, box, T_SELF, o);
  if (!r) r = download_forces(ctx, ld, fxs, fys, fzs);
  if (!r) {
    *qscpe = kR4pie0 * (self_point_energy(ctx, alp, box) - o.sumff) / 418.4;
    *vir += o.self_vir;
  }
  ctx->alpha = keep;
  return r;
}

int ccp_rspace_ewald(ccp_context *ctx, const double *x, const double *y, const double *z,
                     const double *xs, const double *ys, const double *zs, int ld, double box,
                     double alp, double *qrcpe, double *fxs, double *fys, double *fzs,
                     double *vir) {
  const void *p[] = {x, y, z, xs, ys, zs, qrcpe, fxs, fys, fzs, vir};
  int r = check_args(ctx, p, 11, ld);
  if (r) return r;
  CK(cudaSetDevice(ctx->device));
  const double keep = ctx->alpha;
  ctx->alpha = alp;
  r = upload(ctx, x, y, z, xs, ys, zs, ld);
  EvalOut o;
  if (!r) r = evaluate(ctx, ctx->d_x, ctx->d_y, ctx->d_z, ctx->d_xs, ctx->d_ys, ctx->d_zs, ld, box, T_RSPACE, o);
  if (!r) r = download_forces(ctx, ld, fxs, fys, fzs);
  if (!r) {
    *qrcpe = o.rc_e / 418.4;
    *vir += o.rc_vir;
  }
  ctx->alpha = keep;
  return r;
}

int ccp_ccpol23plus(ccp_context *ctx, const double *x, const double *y, const double *z,
                    const double *xs, const double *ys, const double *zs, int ld, double box,
                    double *qvdwe, double *fxs, double *fys, double *fzs, double *vir) {
  const void *p[] = {x, y, z, xs, ys, zs, qvdwe, fxs, fys, fzs, vir};
  int r = check_args(ctx, p, 11, ld);
  if (r) return r;
  if (!ctx->have_vdw) {
    set_error("ccp_ccpol23plus: the model's potential is not ccpol23plus");
    return CCP_ERR_BAD_INPUT;
  }
  CK(cudaSetDevice(ctx->device));
  r = upload(ctx, x, y, z, xs, ys, zs, ld);
  EvalOut o;
  if (!r) r = evaluate(ctx, ctx->d_x, ctx->d_y, ctx->d_z, ctx->d_xs, ctx->d_ys, ctx->d_zs, ld, box, T_VDW, o);
  if (r) return r;
  // vdw_ccpol23plus.f90:212-221: the site forces and the virial start from zero
  for (int i = 0; i < ctx->nm; i++)
    for (int s = 0; s < ctx->ns; s++) {
      fxs[(size_t)i * ld + s] = 0.0;
      fys[(size_t)i * ld + s] = 0.0;
      fzs[(size_t)i * ld + s] = 0.0;
    }
  r = download_forces(ctx, ld, fxs, fys, fzs);
  if (!r) {
    *qvdwe = o.vdw_e / 418.4;
    *vir = o.vdw_vir;
  }
  return r;
}

int ccp_kspace_ewald(ccp_context *ctx, const double *x, const double *y, const double *z,
                     const double *xs, const double *ys, const double *zs, int ld, int lmax,
                     int mmax, int nmax, double alp, double box, double *qkcpe, double *fxs,
                     double *fys, double *fzs, double *vir) {
  const void *p[] = {x, y, z, xs, ys, zs, qkcpe, fxs, fys, fzs, vir};
  int r = check_args(ctx, p, 11, ld);
  if (r) return r;
  if (lmax < 1 || mmax < 1 || nmax < 1) {
    set_error("kspace_ewald: k-max must be >= 1");
    return CCP_ERR_BAD_INPUT;
  }
  CK(cudaSetDevice(ctx->device));
  const double keep = ctx->alpha;
  int kk[3] = {ctx->kmax[0], ctx->kmax[1], ctx->kmax[2]};
  ctx->alpha = alp;
  ctx->kmax[0] = lmax;
  ctx->kmax[1] = mmax;
  ctx->kmax[2] = nmax;
  r = upload(ctx, x, y, z, xs, ys, zs, ld);
  EvalOut o;
  if (!r) r = evaluate(ctx, ctx->d_x, ctx->d_y, ctx->d_z, ctx->d_xs, ctx->d_ys, ctx->d_zs, ld, box, T_KSPACE, o);
  if (!r) r = download_forces(ctx, ld, fxs, fys, fzs);
  if (!r) {
    *qkcpe = 2.0 * kR4pie0 * o.kc_e / 418.4;
    *vir += 2.0 * kR4pie0 * o.kc_vir;
  }
  ctx->alpha = keep;
  for (int a = 0; a < 3; a++) ctx->kmax[a] = kk[a];
  return r;
}

int ccp_nb_induction(ccp_context *ctx, const double *x, const double *y, const double *z,
                     const double *xs, const double *ys, const double *zs, int ld, double box,
                     double *qindpe, double *idmx, double *idmy, double *idmz, double *fxs,
                     double *fys, double *fzs, double *vir, int *iters) {
  const void *p[] = {x, y, z, xs, ys, zs, qindpe, idmx, idmy, idmz, fxs, fys, fzs, vir};
  int r = check_args(ctx, p, 14, ld);
  if (r) return r;
  CK(cudaSetDevice(ctx->device));
  r = upload(ctx, x, y, z, xs, ys, zs, ld);
  EvalOut o;
  if (!r) r = evaluate(ctx, ctx->d_x, ctx->d_y, ctx->d_z, ctx->d_xs, ctx->d_ys, ctx->d_zs, ld, box, T_INDUCTION, o);
  if (iters) *iters = o.iters;
  if (r) return r;
  r = download_forces(ctx, ld, fxs, fys, fzs);
  if (!r) r = download_dipoles(ctx, ld, idmx, idmy, idmz);
  if (!r) {
    *qindpe = kR4pie0 * o.ind_e / 418.4;
    *vir += o.ind_vir;
  }
  return r;
}

int ccp_threebody_term(ccp_context *ctx, const double *x, const double *y, const double *z,
                       const double *xs, const double *ys, const double *zs, int ld,
                       double box, double *qfs2, double *qfs3, double *fxs, double *fys,
                       double *fzs, double *fxfs2, double *fyfs2, double *fzfs2,
                       double *fxfs3, double *fyfs3, double *fzfs3, double *vir) {
  const void *p[] = {x, y, z, xs, ys, zs, qfs2, qfs3, fxs, fys, fzs, vir};
  int r = check_args(ctx, p, 12, ld);
  if (r) return r;
  CK(cudaSetDevice(ctx->device));
  r = upload(ctx, x, y, z, xs, ys, zs, ld);
  EvalOut o;
  if (!r) r = evaluate(ctx, ctx->d_x, ctx->d_y, ctx->d_z, ctx->d_xs, ctx->d_ys, ctx->d_zs, ld, box, T_FS2 | T_FS3, o);
  if (r) return r;
  r = download_forces(ctx, ld, fxs, fys, fzs);
  if (!r && ctx->three_body && ctx->s2) r = download_com(ctx, ctx->d_fc2, fxfs2, fyfs2, fzfs2);
  if (!r && ctx->three_body && ctx->s3) r = download_com(ctx, ctx->d_fc3, fxfs3, fyfs3, fzfs3);
  if (!r) {
    if (ctx->three_body && ctx->s2) *qfs2 = o.fs2_e * kH2kcal;
    if (ctx->three_body && ctx->s3) *qfs3 = o.fs3_e * kH2kcal;
    *vir += (o.fs2_vir + o.fs3_vir) * kH2kcal * 418.4;
  }
  return r;
}

int ccp_hot_path(ccp_context *ctx, const double *x, const double *y, const double *z,
                 const double *xs, const double *ys, const double *zs, int ld, double box,
                 ccp_energies *e, double *fxs, double *fys, double *fzs, double *fxfs2,
                 double *fyfs2, double *fzfs2, double *fxfs3, double *fyfs3, double *fzfs3,
                 double *idmx, double *idmy, double *idmz) {
  const void *p[] = {x, y, z, xs, ys, zs, e};
  int r = check_args(ctx, p, 7, ld);
  if (r) return r;
  CK(cudaSetDevice(ctx->device));
  r = upload(ctx, x, y, z, xs, ys, zs, ld);
  if (!r) r = ensure_host_out(ctx);
  EvalOut o;
  // the results' copies are queued before the evaluation's one synchronisation
  ctx->dl_req = true;
  if (!r) r = evaluate(ctx, ctx->d_x, ctx->d_y, ctx->d_z, ctx->d_xs, ctx->d_ys, ctx->d_zs, ld, box, hot_mask(ctx), o);
  ctx->dl_req = false;
  if (r) return r;
  fill_energies(ctx, o, box, e);
  unpack_host_out(ctx, ld, fxs, fys, fzs, fxfs2, fyfs2, fzfs2, fxfs3, fyfs3, fzfs3, idmx, idmy,
                  idmz);
  return CCP_OK;
}

int ccp_terms_device(ccp_context *ctx, unsigned terms, const double *x, const double *y,
                     const double *z, const double *xs, const double *ys, const double *zs,
                     int ld, double box, ccp_energies *e, double *fxs, double *fys, double *fzs, double *fxfs2,
                        double *fyfs2, double *fzfs2, double *fxfs3, double *fyfs3,
                        double *fzfs3, double *idmx, double *idmy, double *idmz) {
  const void *p[] = {x, y, z, xs, ys, zs, e};
  int r = check_args(ctx, p, 7, ld);
  if (r) return r;
  CK(cudaSetDevice(ctx->device));
  if (terms & ~unsigned(CCP_TERM_ALL)) {
    set_error("ccp_terms_device: unknown term bits");
    return CCP_ERR_BAD_INPUT;
  }
  const unsigned mask = terms & allowed_mask(ctx);
  EvalOut o;
  r = evaluate(ctx, x, y, z, xs, ys, zs, ld, box, mask, o);
  if (r) return r;
  fill_energies(ctx, o, box, e);
  if (!(mask & T_SELF)) e->scpe = 0.0;  // the point self energy is part of that term
  cudaStream_t st = ctx->stream;
  const int n = ctx->nm * ctx->ns;
  if (fxs || fys || fzs) {
    k_scatter_out<<<(n + 255) / 256, 256, 0, st>>>(ctx->d_f, ctx->nm, ctx->ns, ld, fxs, fys, fzs);
    ctx->launches++;
    CK(cudaGetLastError());
  }
  const size_t nb = (size_t)ctx->nm * sizeof(double);
  double *c2[3] = {fxfs2, fyfs2, fzfs2}, *c3[3] = {fxfs3, fyfs3, fzfs3};
  for (int a = 0; a < 3; a++) {
    if (c2[a]) CK(cudaMemcpyAsync(c2[a], ctx->d_fc2 + (size_t)a * ctx->nm, nb, cudaMemcpyDeviceToDevice, st));
    if (c3[a]) CK(cudaMemcpyAsync(c3[a], ctx->d_fc3 + (size_t)a * ctx->nm, nb, cudaMemcpyDeviceToDevice, st));
  }
  if (idmx || idmy || idmz) {
    k_scatter_dip<<<(n + 255) / 256, 256, 0, st>>>(ctx->d_mu, ctx->nm, ctx->ns, ctx->S.np,
                                                   ctx->ns - ctx->npol, ld, idmx, idmy, idmz);
    ctx->launches++;
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(st));
  return CCP_OK;
}

int ccp_hot_path_device(ccp_context *ctx, const double *x, const double *y, const double *z,
                        const double *xs, const double *ys, const double *zs, int ld, double box,
                        ccp_energies *e, double *fxs, double *fys, double *fzs, double *fxfs2,
                        double *fyfs2, double *fzfs2, double *fxfs3, double *fyfs3,
                        double *fzfs3, double *idmx, double *idmy, double *idmz) {
  return ccp_terms_device(ctx, CCP_TERM_HOT, x, y, z, xs, ys, zs, ld, box, e, fxs, fys, fzs, fxfs2,
                          fyfs2, fzfs2, fxfs3, fyfs3, fzfs3, idmx, idmy, idmz);
}

int ccp_context_get_fs3_params(const ccp_context *ctx, double *cs_sr, double *cs_lr, int ncoef,
                               double *bgr_sr, double *bgr_lr) {
  if (!ctx) return CCP_ERR_BAD_INPUT;
  if (!ctx->have_fs3 || ncoef != ctx->nclass) {
    set_error("FS3 parameters: the model has no FS3 tables or ncoef differs from its " +
              std::to_string(ctx->nclass) + " coefficients");
    return CCP_ERR_BAD_INPUT;
  }
  for (int k = 0; k < ncoef; k++) {
    if (cs_sr) cs_sr[k] = ctx->cs_sr[k];
    if (cs_lr) cs_lr[k] = ctx->cs_lr[k];
  }
  for (int k = 0; k < 3 * 289; k++) {
    if (bgr_sr) bgr_sr[k] = ctx->bgr_host[k];
    if (bgr_lr) bgr_lr[k] = ctx->bgr_host[3 * 289 + k];
  }
  return CCP_OK;
}

int ccp_context_set_fs3_params(ccp_context *ctx, const double *cs_sr, const double *cs_lr,
                               int ncoef, const double *bgr_sr, const double *bgr_lr) {
  if (!ctx || !cs_sr || !cs_lr || !bgr_sr || !bgr_lr) return CCP_ERR_BAD_INPUT;
  if (!ctx->have_fs3 || ncoef != ctx->nclass) {
    set_error("FS3 parameters: the model has no FS3 tables or ncoef differs from its " +
              std::to_string(ctx->nclass) + " coefficients");
    return CCP_ERR_BAD_INPUT;
  }
  CK(cudaSetDevice(ctx->device));
  for (int k = 0; k < ncoef; k++) {
    ctx->cs_sr[k] = cs_sr[k];
    ctx->cs_lr[k] = cs_lr[k];
  }
  for (int k = 0; k < 3 * 289; k++) {
    ctx->bgr_host[k] = bgr_sr[k];
    ctx->bgr_host[3 * 289 + k] = bgr_lr[k];
  }
  const size_t nt = ctx->class_of_type.size();
  std::vector<double> coef(2 * nt);
  for (size_t t = 0; t < nt; t++) {
    coef[t] = ctx->cs_sr[ctx->class_of_type[t]];
    coef[nt + t] = ctx->cs_lr[ctx->class_of_type[t]];
  }
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(ctx->d_coef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->d_bgr, ctx->bgr_host.data(), ctx->bgr_host.size() * sizeof(double),
                     cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  ctx->pgrad_valid = false;
  return CCP_OK;
}

int ccp_context_fs3_param_grad(ccp_context *ctx, double *dcs_sr, double *dcs_lr, int ncoef,
                               double *dbgr_sr, double *dbgr_lr) {
  if (!ctx) return CCP_ERR_BAD_INPUT;
  if (!ctx->have_fs3 || ncoef != ctx->nclass) {
    set_error("FS3 parameter gradient: the model has no FS3 tables or ncoef differs from its " +
              std::to_string(ctx->nclass) + " coefficients");
    return CCP_ERR_BAD_INPUT;
  }
  if (!ctx->pgrad_valid) {
    set_error("FS3 parameter gradient: set the fs3_param_grad option and evaluate FS3 first");
    return CCP_ERR_BAD_INPUT;
  }
  CK(cudaSetDevice(ctx->device));
  std::vector<double> g(kFs3GradLen);
  CK(cudaMemcpyAsync(g.data(), ctx->d_gfs3, sizeof(double) * kFs3GradLen, cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const size_t nt = ctx->class_of_type.size();
  std::vector<double> gs(ncoef, 0.0), gl(ncoef, 0.0);
  for (size_t t = 0; t < nt; t++) {
    gs[ctx->class_of_type[t]] += g[t];
    gl[ctx->class_of_type[t]] += g[nt + t];
  }
  for (int k = 0; k < ncoef; k++) {
    if (dcs_sr) dcs_sr[k] = gs[k] * kH2kcal;
    if (dcs_lr) dcs_lr[k] = gl[k] * kH2kcal;
  }
  const double *gb = g.data() + 2 * nt;
  for (int k = 0; k < 3 * 289; k++) {
    if (dbgr_sr) dbgr_sr[k] = gb[k] * kH2kcal;
    if (dbgr_lr) dbgr_lr[k] = gb[3 * 289 + k] * kH2kcal;
  }
  return CCP_OK;
}

// ------------------------------------------------------------- NVE molecular dynamics
namespace {
constexpr double kBoltz = 8.31451115e-1;  // (10 J/mol)/K
constexpr double kPrsunt = 0.163882576;   // internal pressure unit to katm

int md_alloc(ccp_context *c) {
  if (c->d_md_x) return CCP_OK;
  const size_t nm = c->nm;
  CK(dalloc(&c->d_md_x, 3 * nm));
  CK(dalloc(&c->d_md_xs, 3 * nm * (size_t)c->ns));
  CK(dalloc(&c->d_md_v, 3 * nm));
  CK(dalloc(&c->d_md_q, 4 * nm));
  CK(dalloc(&c->d_md_j, 3 * nm));
  CK(dalloc(&c->d_md_red, (size_t)9));
  // 13 doubles per molecule for the state, and at least 32 for the per-step scalar slots
  CK(cudaMallocHost((void **)&c->h_md, sizeof(double) * std::max<size_t>(13 * nm, 40)));
  return CCP_OK;
}

// sites from the quaternions, then every term (the 2-body one too when the model has it)
int md_forces(ccp_context *c, EvalOut &o) {
  const size_t nm = c->nm, nsi = nm * c->ns;
  double *x = c->d_md_x, *xs = c->d_md_xs;
  CK(launch_md_sites(c->nm, c->ns, c->d_md_q, c->d_pcoord, xs, xs + nsi, xs + 2 * nsi,
                     c->stream));
  c->launches = 0;
  int r = evaluate(c, x, x + nm, x + 2 * nm, xs, xs + nsi, xs + 2 * nsi, c->ns, c->md_box,
                   allowed_mask(c), o);
  if (r) return r;
  fill_energies(c, o, c->md_box, &c->md_e);
  return CCP_OK;
}
}  // namespace

int ccp_md_set_state(ccp_context *ctx, double box, const double *x, const double *y,
                     const double *z, const double *v, const double *q, const double *j) {
  if (!ctx || !x || !y || !z || !v || !q || !j || !(box > 0.0)) return CCP_ERR_BAD_INPUT;
  CK(cudaSetDevice(ctx->device));
  int r = md_alloc(ctx);
  if (r) return r;
  const size_t nm = ctx->nm;
  double *h = ctx->h_md;
  for (size_t i = 0; i < nm; i++) {
    h[i] = x[i];
    h[nm + i] = y[i];
    h[2 * nm + i] = z[i];
    for (int a = 0; a < 3; a++) h[(3 + a) * nm + i] = v[3 * i + a];
    for (int a = 0; a < 4; a++) h[(6 + a) * nm + i] = q[4 * i + a];
    for (int a = 0; a < 3; a++) h[(10 + a) * nm + i] = j[3 * i + a];
  }
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(ctx->d_md_x, h, 3 * nm * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->d_md_v, h + 3 * nm, 3 * nm * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->d_md_q, h + 6 * nm, 4 * nm * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->d_md_j, h + 10 * nm, 3 * nm * sizeof(double), cudaMemcpyHostToDevice, st));
  ctx->md_box = box;
  ctx->md_volm = pow(box, 3.0);
  EvalOut o;
  r = md_forces(ctx, o);
  ctx->md_ready = r == CCP_OK;
  return r;
}

int ccp_md_get_state(ccp_context *ctx, double *x, double *y, double *z, double *v, double *q,
                     double *j) {
  if (!ctx || !ctx->md_ready) {
    set_error("ccp_md_get_state: no MD state (call ccp_md_set_state first)");
    return CCP_ERR_BAD_INPUT;
  }
  CK(cudaSetDevice(ctx->device));
  const size_t nm = ctx->nm;
  double *h = ctx->h_md;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(h, ctx->d_md_x, 3 * nm * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(h + 3 * nm, ctx->d_md_v, 3 * nm * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(h + 6 * nm, ctx->d_md_q, 4 * nm * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(h + 10 * nm, ctx->d_md_j, 3 * nm * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (size_t i = 0; i < nm; i++) {
    if (x) x[i] = h[i];
    if (y) y[i] = h[nm + i];
    if (z) z[i] = h[2 * nm + i];
    for (int a = 0; a < 3; a++)
      if (v) v[3 * i + a] = h[(3 + a) * nm + i];
    for (int a = 0; a < 4; a++)
      if (q) q[4 * i + a] = h[(6 + a) * nm + i];
    for (int a = 0; a < 3; a++)
      if (j) j[3 * i + a] = h[(10 + a) * nm + i];
  }
  return CCP_OK;
}

int ccp_md_get_dipoles(ccp_context *ctx, int ld, double *idmx, double *idmy, double *idmz) {
  if (!ctx || !ctx->md_ready || ld < ctx->ns) {
    set_error("ccp_md_get_dipoles: no MD state or ld below the sites per molecule");
    return CCP_ERR_BAD_INPUT;
  }
  CK(cudaSetDevice(ctx->device));
  return download_dipoles(ctx, ld, idmx, idmy, idmz);
}

}  // extern "C"

namespace {
constexpr double kBetta = 0.007372;  // Berendsen barostat compressibility (evolve.f90:7514)

// md.f90:169-176 and evolve.f90:1020-1052 (initialization.f90:76-89, 386-399 for the initial
// state): energies of the last evaluation, the given kinetic energies (internal units), the
// temperature, virial (vir + the sum f . xs in h_md[2]) and pressure over md_volm.
// `e` and `red` (the step's reductions, red[2] = sum f . xs) default to the context's last.
void md_fill_stats(const ccp_context *ctx, double tke, double rke, ccp_md_stats &S,
                   const ccp_energies *ep = nullptr, const double *red = nullptr) {
  const ccp_energies &e = ep ? *ep : ctx->md_e;
  const double qvir = e.vir + (red ? red : ctx->h_md)[2];
  S.vdwpe = e.vdwpe;
  S.cpe = e.scpe + e.rcpe + e.kcpe;
  S.indpe = e.indpe;
  S.pe3b = e.fs2pe + e.fs3pe;
  S.pe = S.vdwpe + S.cpe + S.indpe + S.pe3b;
  S.tke = tke / 418.4;
  S.rke = rke / 418.4;
  S.te = S.tke + S.rke + S.pe;
  S.sys_temp = 2.0 * (tke + rke) / (3.0 * kBoltz * (2.0 * ctx->nm - 1.0));
  S.vir = qvir / 418.4;
  S.pres = kPrsunt * (2.0 * tke - qvir) / (3.0 * ctx->md_volm);
  S.ind_iters = e.ind_iters;
  S.box = ctx->md_box;
  S.volm = ctx->md_volm;
  S.chit = ctx->md_chit;
  S.chip = ctx->md_chip;
  // nvt_hov_3's conserved part of the thermostat (evolve.f90:3797): 0.5 qmass chit^2 + ceng cint
  const double sigma0 = (6.0 * ctx->nm - 3.0) * kBoltz * ctx->md_temp0 / 2.0;
  S.consv = ctx->md_ens == CCP_MD_NVT_H
                ? 0.5 * (2.0 * sigma0 * ctx->md_taut * ctx->md_taut) * ctx->md_chit * ctx->md_chit +
                      2.0 * sigma0 * ctx->md_cint
                : 0.0;
}

void md_fill_stats(const ccp_context *ctx, ccp_md_stats &S) {
  md_fill_stats(ctx, 0.5 * ctx->totm * ctx->h_md[0], 0.5 * ctx->h_md[1], S);
}

// npt_b_1 before the step (evolve.f90:7568-7607): the pressure of the current state sets
// the Berendsen barostat chip; volume times chip, box times chip^(1/3), k-max for the new
// box (ewald_setup).  Returns the centres' scale chip^(1/3) in *scale.
int md_barostat(ccp_context *ctx, double dt, double *scale) {
  const size_t nm = ctx->nm, nsi = nm * ctx->ns;
  double *xs = ctx->d_md_xs;
  cudaStream_t st = ctx->stream;
  CK(launch_md_sums(ctx->nm, ctx->ns, ctx->d_f, ctx->d_fc2, ctx->d_fc3, xs, xs + nsi,
                    xs + 2 * nsi, ctx->d_md_v, ctx->d_md_j, ctx->d_md_x, ctx->pmi,
                    ctx->d_md_red, st));
  CK(cudaMemcpyAsync(ctx->h_md, ctx->d_md_red, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const double tke0 = 0.5 * ctx->totm * ctx->h_md[0];
  const double qpres = (2.0 * tke0 - (ctx->md_e.vir + ctx->h_md[2])) / (3.0 * ctx->md_volm);
  const double chip = 1.0 + kBetta * dt * (qpres - ctx->md_pres0) / ctx->md_taup;
  ctx->md_chip = chip;
  *scale = pow(chip, 1.0 / 3.0);
  ctx->md_volm = ctx->md_volm * chip;
  ctx->md_box = *scale * ctx->md_box;
  double a;
  int k1, k2, k3;
  const int r = ccp_ewald_setup(kEwp, ctx->rcut, ctx->md_box, &a, &k1, &k2, &k3);
  if (r) return r;
  ctx->kmax[0] = k1;
  ctx->kmax[1] = k2;
  ctx->kmax[2] = k3;
  return CCP_OK;
}

// Nose-Hoover thermostat and barostat variables of nvt_hov_3 / npt_hov_2 (evolve.f90:
// 3391-3398, 5642-5650; sigma_Text utility.f90:240-255): masses and the thermostat's energy.
struct NhConsts {
  double qmass, ceng, pmass, fmtk;  // fmtk: npt_mtk's 3/(dof - dofr) (evolve.f90:8510), else 0
};
NhConsts nh_consts(const ccp_context *ctx, int kind) {
  const double dof = 6.0 * ctx->nm - 3.0, dofr = 3.0 * ctx->nm;
  const double sigma0 = dof * kBoltz * ctx->md_temp0 / 2.0;
  NhConsts c{2.0 * sigma0 * ctx->md_taut * ctx->md_taut, 2.0 * sigma0, 0.0, 0.0};
  if (kind == CCP_MD_NPT_MTK) c.fmtk = 3.0 / (dof - dofr);
  if (kind == CCP_MD_NPT_H || kind == CCP_MD_NPT_MTK) {
    const double tmpt = (2.0 * sigma0) / (kBoltz * dof);
    c.ceng = 2.0 * sigma0 + kBoltz * tmpt;
    c.pmass = ((dof - dofr) + 3.0) * kBoltz * tmpt * ctx->md_taup * ctx->md_taup;
  }
  return c;
}

// The kinetic energies and velocity scale factors a thermostat / barostat sequence acts on:
// the scalings are products, applied to the device state once the sequence is done.
struct NhState {
  double tke, rke, fv, fj;
};

// nptqscl_t_dl4 (evolve.f90:8305-8369) with time step ttt
void nh_thermo(ccp_context *ctx, const NhConsts &c, double ttt, NhState &s) {
  const double h = 0.5 * ttt, q = 0.25 * ttt, f1 = c.pmass * pow(ctx->md_chip, 2.0);
  double chit = ctx->md_chit, cint = ctx->md_cint;
  cint = cint + q * chit;
  chit = chit + h * (2.0 * (s.tke + s.rke) + f1 - c.ceng) / c.qmass;
  cint = cint + h * chit;
  const double sc = exp(-ttt * chit);
  s.fv *= sc;
  s.fj *= sc;
  s.tke = s.tke * pow(sc, 2.0);
  s.rke = s.rke * pow(sc, 2.0);
  chit = chit + h * (2.0 * (s.tke + s.rke) + f1 - c.ceng) / c.qmass;
  cint = cint + q * chit;
  ctx->md_chit = chit;
  ctx->md_cint = cint;
}

// nptqscl_p_dl4 (evolve.f90:8435-8495), or nptqscl_p_dl4_mtk (:8497-8558) when c.fmtk is
// set, with time step ttt, box boxi and virial qvir
void nh_baro(ccp_context *ctx, const NhConsts &c, double ttt, double boxi, double qvir,
             NhState &s) {
  const double h = 0.5 * ttt, q = 0.25 * ttt, vi = pow(boxi, 3.0), chit = ctx->md_chit;
  double chip = ctx->md_chip;
  chip = chip * exp(-q * chit);
  chip = chip + h * ((2.0 * (1.0 + c.fmtk) * s.tke - qvir) - 3.0 * ctx->md_pres0 * vi) / c.pmass;
  chip = chip * exp(-q * chit);
  const double sc = exp(-ttt * (1.0 + c.fmtk) * chip);
  s.fv *= sc;
  s.tke = s.tke * pow(sc, 2.0);
  chip = chip * exp(-q * chit);
  chip = chip + h * ((2.0 * (1.0 + c.fmtk) * s.tke - qvir) - 3.0 * ctx->md_pres0 * vi) / c.pmass;
  chip = chip * exp(-q * chit);
  ctx->md_chip = chip;
}

// npt_hov_2's thermostat / barostat / thermostat sequence (evolve.f90:5661-5665, 6061-6065)
void nh_sequence(ccp_context *ctx, const NhConsts &c, double dt, double boxi, double qvir,
                 NhState &s) {
  nh_thermo(ctx, c, 0.25 * dt, s);
  nh_baro(ctx, c, 0.5 * dt, boxi, qvir, s);
  nh_thermo(ctx, c, 0.25 * dt, s);
}

// nsteps steps of the ensemble `kind` (CCP_MD_*): nve_1 (evolve.f90:621-1061), nvt_b
// (:1063-1644) or npt_b_1 (:7485-8104).  They share the kicks, drift and nosquish rotation
// (stage 1 and 2 kernels); nvt_b does not wrap the centres, npt_b_1 wraps them after its
// thermostat into the new box.
int md_steps(ccp_context *ctx, int kind, int nsteps, double dt, ccp_md_stats *stats) {
  CK(cudaSetDevice(ctx->device));
  const size_t nm = ctx->nm, nsi = nm * ctx->ns;
  const int ns = ctx->ns;
  double *x = ctx->d_md_x, *xs = ctx->d_md_xs, *v = ctx->d_md_v, *q = ctx->d_md_q,
         *jv = ctx->d_md_j;
  cudaStream_t st = ctx->stream;
  const double zero[3] = {0.0, 0.0, 0.0};
  const double dof_sys = 3.0 * kBoltz * (2.0 * ctx->nm - 1.0);
  // NVE steps without an equilibration rescale take no host decision from their kinetic
  // energies: a step's reductions are copied without a synchronisation, and its statistics
  // are filled after the next step's evaluation, whose own synchronisation covers the copy
  int pend = -1;
  ccp_energies pend_e{};
  const double *pend_red = nullptr;
  for (int k = 0; k < nsteps; k++) {
    double scale = 1.0;
    if (kind == CCP_MD_NPT_B) {
      const int r = md_barostat(ctx, dt, &scale);
      if (r) return r;
    }
    const double *centre = nullptr;
    double cen[3] = {0.0, 0.0, 0.0}, boxi = 0.0, volmi = 0.0;
    NhConsts nhc{0.0, 0.0, 0.0};
    const bool nh_baro = kind == CCP_MD_NPT_H || kind == CCP_MD_NPT_MTK;
    if (nh_baro) {
      // npt_hov_2 / npt_mtk before the step (evolve.f90:5661-5712): thermostat / barostat / thermostat
      // on the current state, new volume exp(3 dt chip) V, centres scaled by exp(dt chip)
      // about the system's centre (the mean of the centres: the site offsets of a molecule
      // sum to zero about it) in the drift
      nhc = nh_consts(ctx, kind);
      CK(launch_md_sums(ctx->nm, ns, ctx->d_f, ctx->d_fc2, ctx->d_fc3, xs, xs + nsi, xs + 2 * nsi,
                        v, jv, x, ctx->pmi, ctx->d_md_red, st));
      CK(cudaMemcpyAsync(ctx->h_md, ctx->d_md_red, 9 * sizeof(double), cudaMemcpyDeviceToHost,
                         st));
      CK(cudaStreamSynchronize(st));
      const double *h0 = ctx->h_md;
      NhState ns0{0.5 * ctx->totm * h0[0], 0.5 * h0[1], 1.0, 1.0};
      nh_sequence(ctx, nhc, dt, ctx->md_box, ctx->md_e.vir + h0[2], ns0);
      for (int a = 0; a < 3; a++) cen[a] = h0[6 + a] / (double)nm;
      CK(launch_md_scale(ctx->nm, v, zero, ns0.fv, jv, ns0.fj, st));
      volmi = pow(ctx->md_box, 3.0) * exp(3.0 * dt * ctx->md_chip);
      boxi = pow(volmi, 1.0 / 3.0);
      scale = exp(dt * ctx->md_chip);
      if (kind == CCP_MD_NPT_H) centre = cen;  // npt_mtk scales about the origin
    }
    // first half kick, drift and rotation with the previous evaluation's forces
    CK(launch_md_stage1(ctx->nm, ns, ctx->d_f, ctx->d_fc2, ctx->d_fc3, xs, xs + nsi, xs + 2 * nsi,
                        x, x + nm, x + 2 * nm, v, q, jv, ctx->pmi, ctx->totm, dt, scale, centre,
                        st));
    EvalOut o;
    int r = md_forces(ctx, o);
    if (r) {
      ctx->md_ready = false;
      return r;
    }
    CK(launch_md_stage2(ctx->nm, ns, ctx->d_f, ctx->d_fc2, ctx->d_fc3, xs, xs + nsi, xs + 2 * nsi,
                        x, x + nm, x + 2 * nm, v, q, jv, ctx->pmi, ctx->totm, dt, ctx->md_box,
                        (kind == CCP_MD_NVE || kind == CCP_MD_NVT_H) ? 1 : 0, ctx->d_md_red, st));
    if (pend >= 0) {  // the previous step's copy completed in this step's evaluation
      if (stats) {
        const double *r0 = pend_red;
        md_fill_stats(ctx, 0.5 * ctx->totm * r0[0], 0.5 * r0[1], stats[pend], &pend_e, r0);
      }
      pend = -1;
    }
    if (kind == CCP_MD_NVE && ctx->md_eq_left == 0) {
      double *slot = ctx->h_md + 16 + 8 * (k & 1);  // h_md holds >= 40 doubles
      CK(cudaMemcpyAsync(slot, ctx->d_md_red, 6 * sizeof(double), cudaMemcpyDeviceToHost, st));
      pend = k;
      pend_e = ctx->md_e;
      pend_red = slot;
      continue;
    }
    CK(cudaMemcpyAsync(ctx->h_md, ctx->d_md_red, 6 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const double *h = ctx->h_md;
    double tke = 0.5 * ctx->totm * h[0];
    const double rke = 0.5 * h[1];
    if (kind == CCP_MD_NVE) {
      if (stats) md_fill_stats(ctx, tke, rke, stats[k]);
      if (ctx->md_eq_left > 0) {
        // md.f90:187-193: after the step, velocities and angular momenta to temp0
        // (equilibrationGRU, utility.f90:353-368; trans_temp / rot_temp :196-227)
        const double ttemp = 2.0 * tke / ((3.0 * nm - 3.0) * kBoltz);
        const double rtemp = 2.0 * rke / ((3.0 * nm) * kBoltz);
        CK(launch_md_scale(ctx->nm, v, zero, sqrt(ctx->md_eq_temp / ttemp), jv,
                           sqrt(ctx->md_eq_temp / rtemp), st));
        ctx->md_eq_left--;
      }
      continue;
    }
    if (nh_baro) {
      // npt_hov_2 / npt_mtk after the step (evolve.f90:6061-6103): the sequence again with the new box
      // and virial, then the new box, COM-velocity removal and the wrap into the new box
      NhState ns1{tke, rke, 1.0, 1.0};
      nh_sequence(ctx, nhc, dt, boxi, ctx->md_e.vir + h[2], ns1);
      ctx->md_box = boxi;
      ctx->md_volm = volmi;
      double a_;
      int k1, k2, k3;
      r = ccp_ewald_setup(kEwp, ctx->rcut, ctx->md_box, &a_, &k1, &k2, &k3);
      if (r) return r;
      ctx->kmax[0] = k1;
      ctx->kmax[1] = k2;
      ctx->kmax[2] = k3;
      double c[3], c2 = 0.0, cs = 0.0;
      for (int a = 0; a < 3; a++) {
        c[a] = h[3 + a] / (double)nm;
        c2 += c[a] * c[a];
        cs += c[a] * h[3 + a];
      }
      const double tk = ns1.fv * ns1.fv * 0.5 * ctx->totm * (h[0] - 2.0 * cs + (double)nm * c2);
      CK(launch_md_scale(ctx->nm, v, c, ns1.fv, jv, ns1.fj, st));
      CK(launch_md_wrap(ctx->nm, x, x + nm, x + 2 * nm, ctx->md_box, st));
      if (stats) {
        md_fill_stats(ctx, tk, ns1.rke, stats[k]);
        stats[k].consv = 0.5 * nhc.qmass * pow(ctx->md_chit, 2.0) +
                         0.5 * nhc.pmass * pow(ctx->md_chip, 2.0) + nhc.ceng * ctx->md_cint +
                         ctx->md_pres0 * volmi;
      }
      continue;
    }
    if (kind == CCP_MD_NVT_H) {
      // nvt_hov_3 (evolve.f90:3590-3600): the Nose-Hoover thermostat of nptqscl_t_dl4
      // (:8305-8369) with its time step dt/4, pmass = chip = 0
      const double sigma0 = (6.0 * nm - 3.0) * kBoltz * ctx->md_temp0 / 2.0;
      const double qmass = 2.0 * sigma0 * ctx->md_taut * ctx->md_taut, ceng = 2.0 * sigma0;
      const double tq = 0.25 * dt, hq = 0.5 * tq, qq = 0.25 * tq;
      double chit = ctx->md_chit, cint = ctx->md_cint;
      cint = cint + qq * chit;
      chit = chit + hq * (2.0 * (tke + rke) - ceng) / qmass;
      cint = cint + hq * chit;
      const double sc = exp(-tq * chit);
      CK(launch_md_scale(ctx->nm, v, zero, sc, jv, sc, st));
      const double tk2 = tke * pow(sc, 2.0), rk2 = rke * pow(sc, 2.0);
      chit = chit + hq * (2.0 * (tk2 + rk2) - ceng) / qmass;
      cint = cint + qq * chit;
      ctx->md_chit = chit;
      ctx->md_cint = cint;
      if (stats) md_fill_stats(ctx, tk2, rk2, stats[k]);
      continue;
    }
    double c[3] = {0.0, 0.0, 0.0};
    if (kind == CCP_MD_NPT_B) {
      // utility.f90:293-351: the system's COM velocity (every molecule of mass totm), removed
      // before the thermostat; sum (v - c)^2 = sum v^2 - 2 c . sum v + nm c^2
      double c2 = 0.0, cs = 0.0;
      for (int a = 0; a < 3; a++) {
        c[a] = h[3 + a] / (double)nm;
        c2 += c[a] * c[a];
        cs += c[a] * h[3 + a];
      }
      tke = 0.5 * ctx->totm * (h[0] - 2.0 * cs + (double)nm * c2);
    }
    // evolve.f90:1598-1606 / 8047-8055: Berendsen thermostat on the system temperature
    const double tsys = 2.0 * (tke + rke) / dof_sys;
    const double chit = sqrt(1.0 + dt / ctx->md_taut * (ctx->md_temp0 / tsys - 1.0));
    ctx->md_chit = chit;
    CK(launch_md_scale(ctx->nm, v, c, chit, jv, chit, st));
    if (kind == CCP_MD_NPT_B) CK(launch_md_wrap(ctx->nm, x, x + nm, x + 2 * nm, ctx->md_box, st));
    if (stats) md_fill_stats(ctx, chit * chit * tke, chit * chit * rke, stats[k]);
  }
  if (pend >= 0) {
    CK(cudaStreamSynchronize(st));
    if (stats)
      md_fill_stats(ctx, 0.5 * ctx->totm * pend_red[0], 0.5 * pend_red[1], stats[pend], &pend_e,
                    pend_red);
  }
  return CCP_OK;
}
}  // namespace

extern "C" {

int ccp_md_nve(ccp_context *ctx, int nsteps, double dt, ccp_md_stats *stats) {
  if (!ctx || nsteps < 0 || !(dt > 0.0)) return CCP_ERR_BAD_INPUT;
  if (!ctx->md_ready) {
    set_error("ccp_md_nve: no MD state (call ccp_md_set_state first)");
    return CCP_ERR_BAD_INPUT;
  }
  return md_steps(ctx, CCP_MD_NVE, nsteps, dt, stats);
}

int ccp_md_set_ensemble(ccp_context *ctx, int ensemble, double temp0, double taut,
                        double pres0_katm, double taup) {
  if (!ctx || ensemble < CCP_MD_NVE || ensemble > CCP_MD_NPT_MTK ||
      (ensemble != CCP_MD_NVE && !(temp0 > 0.0 && taut > 0.0)) ||
      (ensemble >= CCP_MD_NPT_B && ensemble != CCP_MD_NVT_H && !(taup > 0.0))) {
    set_error("ccp_md_set_ensemble: unknown ensemble or non-positive temp0 / taut / taup");
    return CCP_ERR_BAD_INPUT;
  }
  ctx->md_ens = ensemble;
  ctx->md_temp0 = temp0;
  ctx->md_taut = taut;
  ctx->md_pres0 = pres0_katm / kPrsunt;  // initialization.f90:160
  ctx->md_taup = taup;
  return CCP_OK;
}

int ccp_md_set_thermostat(ccp_context *ctx, double chit, double chip) {
  if (!ctx) return CCP_ERR_BAD_INPUT;
  ctx->md_chit = chit;
  ctx->md_chip = chip;
  ctx->md_cint = 0.0;  // initialization.f90:172
  return CCP_OK;
}

int ccp_md_run(ccp_context *ctx, int nsteps, double dt, ccp_md_stats *stats) {
  if (!ctx || nsteps < 0 || !(dt > 0.0)) return CCP_ERR_BAD_INPUT;
  if (!ctx->md_ready) {
    set_error("ccp_md_run: no MD state (call ccp_md_set_state first)");
    return CCP_ERR_BAD_INPUT;
  }
  return md_steps(ctx, ctx->md_ens, nsteps, dt, stats);
}

int ccp_md_set_equilibration(ccp_context *ctx, double temp0, int nsteps) {
  if (!ctx || nsteps < 0 || (nsteps > 0 && !(temp0 > 0.0))) {
    set_error("ccp_md_set_equilibration: need temp0 > 0 and nsteps >= 0");
    return CCP_ERR_BAD_INPUT;
  }
  ctx->md_eq_temp = temp0;
  ctx->md_eq_left = nsteps;
  return CCP_OK;
}

int ccp_md_get_stats(ccp_context *ctx, ccp_md_stats *stats) {
  if (!ctx || !stats) return CCP_ERR_BAD_INPUT;
  if (!ctx->md_ready) {
    set_error("ccp_md_get_stats: no MD state (call ccp_md_set_state first)");
    return CCP_ERR_BAD_INPUT;
  }
  CK(cudaSetDevice(ctx->device));
  const size_t nm = ctx->nm, nsi = nm * ctx->ns;
  cudaStream_t st = ctx->stream;
  const double *xs = ctx->d_md_xs;
  CK(launch_md_sums(ctx->nm, ctx->ns, ctx->d_f, ctx->d_fc2, ctx->d_fc3, xs, xs + nsi, xs + 2 * nsi,
                    ctx->d_md_v, ctx->d_md_j, ctx->d_md_x, ctx->pmi, ctx->d_md_red, st));
  CK(cudaMemcpyAsync(ctx->h_md, ctx->d_md_red, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  md_fill_stats(ctx, *stats);
  return CCP_OK;
}

}  // extern "C"

// ------------------------------------------------------------ batches: fused FS3
namespace {

// Packs the centres (Angstrom and bohr) and FS3 site offsets (bohr) of every molecule of a
// batch, frames one after another as the caller's arrays hold them, with the same
// conversions as k_prep; clears the force, counter and energy buffers.
__global__ void k_batch_fs3_prep(const double *__restrict__ x, const double *__restrict__ y,
                                 const double *__restrict__ z, const double *__restrict__ xs,
                                 const double *__restrict__ ys, const double *__restrict__ zs,
                                 int nt, int ld, int ns, double4 *com, double4 *comb, double4 *s17,
                                 double *f, double *fc3, int *icnt, double *scal, int nscal,
                                 int *counts, int ncounts) {
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int i = t0; i < nt; i += stride) {
    com[i] = make_double4(x[i], y[i], z[i], 0.0);
    comb[i] = make_double4(x[i] / kBohr2a, y[i] / kBohr2a, z[i] / kBohr2a, 0.0);
    fc3[i] = fc3[nt + i] = fc3[2 * nt + i] = 0.0;
  }
  for (int u = t0; u < nt * kNs3; u += stride) {
    const int i = u / kNs3, s = u - i * kNs3;
    const size_t o = (size_t)i * ld + s;
    s17[u] = make_double4(xs[o] / kBohr2a, ys[o] / kBohr2a, zs[o] / kBohr2a, 0.0);
  }
  for (size_t u = t0; u < 3 * (size_t)nt * ns; u += stride) f[u] = 0.0;
  for (int u = t0; u < nscal; u += stride) scal[u] = 0.0;
  for (int u = t0; u < ncounts; u += stride) counts[u] = 0;
  if (t0 < C_COUNT) icnt[t0] = 0;
}

int batch_fs3_alloc(ccp_context *c, BatchFs3 &B, int nframes, int cap, int tri_cap) {
  const int nt = nframes * c->nm;
  if (B.device == c->device && nt <= B.nm_total && nframes <= B.nframes && cap <= B.cap &&
      tri_cap <= B.tri_cap)
    return CCP_OK;
  const int nt_a = std::max(nt, B.nm_total), nf_a = std::max(nframes, B.nframes);
  const int cap_a = std::max(cap, B.cap), tri_a = std::max(tri_cap, B.tri_cap);
  void *stream = B.stream;
  B.stream = nullptr;
  batch_fs3_free(B);
  B.stream = stream;
  B.device = c->device;
  B.nm_total = nt_a;
  B.nframes = nf_a;
  B.cap = cap_a;
  B.tri_cap = tri_a;
  const size_t n = nt_a, ns = c->ns;
  double4 *com, *comb, *s17, *nbrv;
  CK(dalloc(&com, n));
  B.com = com;
  CK(dalloc(&comb, n));
  B.comb = comb;
  CK(dalloc(&s17, n * kNs3));
  B.s17 = s17;
  CK(dalloc(&nbrv, n * cap_a));
  B.nbrv = nbrv;
  CK(dalloc(&B.nbr, n * cap_a));
  CK(dalloc(&B.ncnt, n));
  CK(dalloc(&B.icnt, (size_t)C_COUNT));
  CK(dalloc(&B.counts, 2 * (size_t)nf_a));
  CK(cudaMalloc(&B.tri, fs3_record_bytes() * (size_t)tri_a));
  CK(dalloc(&B.f, 3 * n * ns));
  CK(dalloc(&B.fc3, 3 * n));
  CK(dalloc(&B.scal, (size_t)nf_a * S_COUNT));
  CK(dalloc(&B.gfs3, (size_t)nf_a * kFs3GradLen));
  CK(cudaMallocHost((void **)&B.h_icnt, sizeof(int) * C_COUNT));
  CK(cudaMallocHost((void **)&B.h_counts, sizeof(int) * 2 * nf_a));
  CK(cudaMallocHost((void **)&B.h_scal, sizeof(double) * ((size_t)nf_a * S_COUNT +
                                                          (size_t)nf_a * kFs3GradLen)));
  return CCP_OK;
}

}  // namespace

namespace ccp {

void batch_fs3_free(BatchFs3 &B) {
  if (B.device >= 0) cudaSetDevice(B.device);
  void *dp[] = {B.com, B.comb, B.s17, B.nbrv, B.nbr, B.ncnt, B.icnt, B.counts, B.tri,
                B.f, B.fc3, B.scal, B.gfs3};
  for (void *p : dp)
    if (p) cudaFree(p);
  if (B.h_icnt) cudaFreeHost(B.h_icnt);
  if (B.h_counts) cudaFreeHost(B.h_counts);
  if (B.h_scal) cudaFreeHost(B.h_scal);
  if (B.stream) cudaStreamDestroy(static_cast<cudaStream_t>(B.stream));
  B = BatchFs3();
}

// Enqueues the FS3 term of `nframes` frames of c->nm molecules (the caller's frame-strided
// device arrays, one box length for all) as one neighbour search, one triple enumeration and
// one FS3 launch on the batch's own stream.  The list capacities are checked once (one
// synchronisation after the enumeration) and grown if a frame needed more.  `grad`: also
// the per-frame FS3 parameter gradients.  batch_fs3_finish completes the call.
int batch_fs3_launch(ccp_context *c, BatchFs3 &B, int nframes, double box, const double *x,
                     const double *y, const double *z, const double *xs, const double *ys,
                     const double *zs, int ld, bool grad) {
  CK(cudaSetDevice(c->device));
  if (!c->three_body || !c->s3 || !c->have_fs3 || c->ns < kNs3) {
    set_error("fused FS3: the model has no FS3 term");
    return CCP_ERR_BAD_INPUT;
  }
  if (!B.stream) {
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    cudaStream_t st;
    CK(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio_lo));
    B.stream = st;
  }
  cudaStream_t st = static_cast<cudaStream_t>(B.stream);
  const int nm = c->nm, nt = nframes * nm;
  int cap = std::max(B.cap, std::max(1, std::min(nm - 1, c->cap)));
  int tri_cap = std::max(B.tri_cap, c->tri_cap * nframes);
  const double rl = 6.3 + 0.05;  // FS3's cut-off and the list margin of an evaluation
  const Fs3Params F3 = fs3_params(c, box);
  for (int attempt = 0;; attempt++) {
    int r = batch_fs3_alloc(c, B, nframes, cap, tri_cap);
    if (r) return r;
    cap = B.cap;
    tri_cap = B.tri_cap;
    k_batch_fs3_prep<<<148 * 4, 256, 0, st>>>(
        x, y, z, xs, ys, zs, nt, ld, c->ns, static_cast<double4 *>(B.com),
        static_cast<double4 *>(B.comb), static_cast<double4 *>(B.s17), B.f, B.fc3, B.icnt,
        B.scal, nframes * S_COUNT, B.counts, 2 * nframes);
    CK(cudaGetLastError());
    if (grad) CK(cudaMemsetAsync(B.gfs3, 0, sizeof(double) * nframes * kFs3GradLen, st));
    CK(launch_neighbors(static_cast<double4 *>(B.com), nt, box, rl * rl, cap, B.nbr,
                        static_cast<double4 *>(B.nbrv), B.ncnt, B.icnt, st, nm));
    CK(launch_fs3_enum(static_cast<double4 *>(B.comb), B.nbr, B.ncnt, cap, nt, F3, B.tri, tri_cap,
                       B.icnt, st));
    CK(cudaMemcpyAsync(B.h_icnt, B.icnt, sizeof(int) * C_COUNT, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const int *ic = B.h_icnt;
    bool grow = false;
    if (ic[C_OVERFLOW] > 0) {
      cap = std::min(nm, ic[C_OVERFLOW] + 32);
      grow = true;
    }
    if (ic[C_NTRI_FS3] > tri_cap) {
      tri_cap = ic[C_NTRI_FS3] + ic[C_NTRI_FS3] / 4 + 64;
      grow = true;
    }
    if (!grow) break;
    if (attempt == 2) {
      set_error("fused FS3: the lists overflowed after growing");
      return CCP_ERR_CAPACITY;
    }
  }
  const int prec = c->precision == CCP_MIXED && c->opt_fs3_low ? CCP_MIXED : CCP_FP64;
  CK(launch_fs3(prec, B.tri, B.icnt, tri_cap, static_cast<double4 *>(B.s17), c->d_coef, c->d_bgr,
                nt, c->ns, B.f, B.fc3, B.scal, c->nsm, c->opt_fs3_tpb, 0, grad ? B.gfs3 : nullptr,
                st, nm, S_COUNT));
  CK(launch_fs3_frame_counts(B.tri, B.icnt, tri_cap, nm, B.counts, st));
  return CCP_OK;
}

// Completes batch_fs3_launch: adds the FS3 site forces into the caller's (frame-strided)
// fxs.., writes the FS3 COM forces, adds each frame's FS3 energy, virial and triple counts
// to e[f] and, with pgrad, writes each frame's parameter gradient (layout of
// ccp_batch_terms_device).
int batch_fs3_finish(ccp_context *c, BatchFs3 &B, int nframes, int ld, ccp_energies *e,
                     double *fxs, double *fys, double *fzs, double *fxfs3, double *fyfs3,
                     double *fzfs3, double *pgrad, int pgrad_len) {
  CK(cudaSetDevice(c->device));
  cudaStream_t st = static_cast<cudaStream_t>(B.stream);
  const int nt = nframes * c->nm;
  if (fxs || fys || fzs) {
    k_scatter_out<<<(nt * c->ns + 255) / 256, 256, 0, st>>>(B.f, nt, c->ns, ld, fxs, fys, fzs);
    CK(cudaGetLastError());
  }
  double *c3[3] = {fxfs3, fyfs3, fzfs3};
  for (int a = 0; a < 3; a++)
    if (c3[a])
      CK(cudaMemcpyAsync(c3[a], B.fc3 + (size_t)a * nt, sizeof(double) * nt,
                         cudaMemcpyDeviceToDevice, st));
  double *hs = B.h_scal, *hg = B.h_scal + (size_t)nframes * S_COUNT;
  CK(cudaMemcpyAsync(hs, B.scal, sizeof(double) * nframes * S_COUNT, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(B.h_counts, B.counts, sizeof(int) * 2 * nframes, cudaMemcpyDeviceToHost, st));
  if (pgrad)
    CK(cudaMemcpyAsync(hg, B.gfs3, sizeof(double) * nframes * kFs3GradLen,
                       cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const size_t ntype = c->class_of_type.size();
  const int ncoef = c->nclass;
  for (int f = 0; f < nframes; f++) {
    const double *sc = hs + (size_t)f * S_COUNT;
    e[f].fs3pe = sc[S_FS3_E] * kH2kcal;
    e[f].vir += sc[S_FS3_VIR] * kH2kcal * 418.4;
    e[f].n_fs3_triples = B.h_counts[2 * f];
    e[f].n_fs3_blend = B.h_counts[2 * f + 1];
    if (!pgrad) continue;
    // fold the coefficient-table entries onto the classes (ccp_context_fs3_param_grad)
    const double *g = hg + (size_t)f * kFs3GradLen;
    double *out = pgrad + (size_t)f * pgrad_len;
    for (int k = 0; k < 2 * ncoef; k++) out[k] = 0.0;
    for (size_t t = 0; t < ntype; t++) {
      out[c->class_of_type[t]] += g[t];
      out[ncoef + c->class_of_type[t]] += g[ntype + t];
    }
    for (int k = 0; k < 2 * ncoef; k++) out[k] *= kH2kcal;
    for (int k = 0; k < 2 * 3 * 289; k++) out[2 * ncoef + k] = g[2 * ntype + k] * kH2kcal;
  }
  return CCP_OK;
}

}  // namespace ccp
