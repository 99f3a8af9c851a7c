// ccp_internal.h -- host-side model description shared by the C++ loader and the CUDA
// context.  Not part of the public ABI (include/ccpol23_b200.h is).
#pragma once

#include <string>
#include <vector>

#include "../../include/ccpol23_b200.h"

namespace ccp {

constexpr int kNsiteMax = 50;   // common_arrays.f90:22 (nsite)
constexpr int kNs3 = 17;        // FS3 sites per molecule (threebody_potential.f90:736)
constexpr int kNtype = 6;       // FS3 site types (threebody_potential.f90:2076)
constexpr int kMaxCharged = 8;  // compile-time caps of the compact site lists
constexpr int kMaxPolar = 4;
constexpr int kMaxActive = 12;

// Physical constants of the reference (common_arrays.f90:28-36, 189-190).
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kR4pie0 = 138935.4835;
constexpr double kBohr2a = 0.529177249;
constexpr double kH2kcal = 627.510;
constexpr double kEwp = 1.0e-6;

void set_error(const std::string &msg);

// Device state of a batch's fused FS3 evaluation: the molecules of all frames packed one
// frame after another, one neighbour search, one triple list and one FS3 launch for the
// whole batch (ccp_context.cu: batch_fs3_*; used by ccp_batch.cpp).
struct BatchFs3 {
  int nm_total = 0, nframes = 0, cap = 0, tri_cap = 0;
  void *com = nullptr, *comb = nullptr, *s17 = nullptr, *nbrv = nullptr;  // double4 arrays
  int *nbr = nullptr, *ncnt = nullptr, *icnt = nullptr, *counts = nullptr;
  void *tri = nullptr;
  double *f = nullptr, *fc3 = nullptr, *scal = nullptr, *gfs3 = nullptr;
  int *h_icnt = nullptr, *h_counts = nullptr;
  double *h_scal = nullptr;
  void *stream = nullptr;  // cudaStream_t
  int device = -1;
};
void batch_fs3_free(BatchFs3 &B);
int batch_fs3_launch(ccp_context *c, BatchFs3 &B, int nframes, double box, const double *x,
                     const double *y, const double *z, const double *xs, const double *ys,
                     const double *zs, int ld, bool grad);
int batch_fs3_finish(ccp_context *c, BatchFs3 &B, int nframes, int ld, ccp_energies *e,
                     double *fxs, double *fys, double *fzs, double *fxfs3, double *fyfs3,
                     double *fzfs3, double *pgrad, int pgrad_len);

struct Fs3Table {
  double b[289], g[289], r0[289];  // [is*17 + js]
  std::vector<double> cs;          // linear coefficients in file order
};

}  // namespace ccp

struct ccp_model {
  // CONTROL (initialization.f90:463-489)
  std::string pot_name, ensemble, initial_config, ind_model, induction_type, method;
  double taut = 0, taup = 0, temp0 = 0, pres0 = 0, dt = 0, rcut = 0, rcut3 = 0, alpha3 = 0;
  double r0_tilda = 0, delta33 = 0, hsize = 0;
  int nsteps = 0, nequil = 0, hist_freq = 0;
  bool rand_vcom = false, rand_quat = false, induction = false, nonadditive_3b = false;
  bool s3_term = false, s2_term = false, restart = false, check_forces = false;
  // FIELD (initialization.f90:491-636)
  std::string system_name;
  int nm = 0, ns = 0, npol = 0;
  std::vector<std::string> names;
  std::vector<double> coords, mass, charge, polarizability;  // coords: ns*3
  struct VdwRow {
    std::string a, b;
    double p[14];
  };
  std::vector<VdwRow> vdw;
  // FS3 tables: SR from data3b_full, LR from data3b_full_LR_4p5
  bool have_fs3 = false;
  ccp::Fs3Table sr, lr;
  // derived
  double totm = 0;
  std::vector<double> pcoord;  // ns*3, principal-axis frame
  double pmi[3] = {0, 0, 0};
  std::vector<int> ind_lin;    // 17^3*8, 1-based coefficient index
  int nclass = 0;
  int fs3_type[ccp::kNs3];     // 0-based type of each FS3 site
  // coefficient by type: [ti*36 + tj*6 + tk][ip*4 + jp*2 + kp] for SR and LR
  std::vector<double> coef_sr, coef_lr;
  std::vector<int> class_of_type;  // same layout: 0-based coefficient (class) index
};
