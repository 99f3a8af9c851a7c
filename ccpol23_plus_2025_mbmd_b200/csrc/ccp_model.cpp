// ccp_model.cpp -- parameter loading and host-side set-up for the CCpol23+(2025) hot path.
//
// Reads the reference's own input files and derives what its start-up code derives:
//   CONTROL                     initialization.f90:463-489 (control_parameters)
//   FIELD, data3b_full(_LR_4p5)  initialization.f90:491-720 (molecule)
//   COM shift + principal axes   initialization.f90:728-845, Jacobi: utility.f90:458-596
//   site placement               molecular_sites.f90:14-111
//   Ewald alpha / k-max          ewald.f90:17-43
//   FS3 coefficient index        threebody_potential.f90:909-946, 2064-2131
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "ccp_internal.h"

namespace ccp {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }

namespace {

std::vector<std::string> split(const std::string &s) {
  std::vector<std::string> out;
  std::string cur;
  for (char c : s) {
    if (c == ' ' || c == '\t' || c == ',' || c == '\r' || c == '\n') {
      if (!cur.empty()) out.push_back(cur), cur.clear();
    } else {
      cur.push_back(c);
    }
  }
  if (!cur.empty()) out.push_back(cur);
  return out;
}

bool read_lines(const std::string &path, std::vector<std::string> &lines) {
  std::ifstream f(path);
  if (!f) return false;
  std::string ln;
  while (std::getline(f, ln)) lines.push_back(ln);
  return true;
}

// Fortran list-directed logical: T/.TRUE./t...
bool flog(const std::string &t) {
  size_t i = 0;
  while (i < t.size() && t[i] == '.') i++;
  return i < t.size() && (t[i] == 'T' || t[i] == 't');
}

// Fortran reads "3.7E-002" and "1.0D0"; map D exponents to E for strtod.
double fnum(std::string t) {
  for (char &c : t)
    if (c == 'D' || c == 'd') c = 'E';
  return std::strtod(t.c_str(), nullptr);
}

struct Tok {
  std::vector<std::vector<std::string>> rows;
  bool need(size_t r, size_t n) const { return r < rows.size() && rows[r].size() >= n; }
};

bool parse_control(const std::string &path, ccp_model &m) {
  std::vector<std::string> lines;
  if (!read_lines(path, lines)) return false;
  Tok t;
  for (auto &l : lines) t.rows.push_back(split(l));
  const size_t need[17] = {1, 3, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 4, 3, 4, 1, 2};
  for (size_t r = 0; r < 17; r++)
    if (!t.need(r, need[r])) {
      set_error("CONTROL: record " + std::to_string(r + 1) + " is short");
      return false;
    }
  auto &R = t.rows;
  m.pot_name = R[0][0];
  m.ensemble = R[1][0];
  m.taut = fnum(R[1][1]);
  m.taup = fnum(R[1][2]);
  m.initial_config = R[2][0];
  m.temp0 = fnum(R[3][0]);
  m.pres0 = fnum(R[4][0]);
  m.nsteps = (int)fnum(R[5][0]);
  m.dt = fnum(R[6][0]);
  m.nequil = (int)fnum(R[7][0]);
  m.rcut = fnum(R[8][0]);
  m.hist_freq = (int)fnum(R[9][0]);
  m.rand_vcom = flog(R[10][0]);
  m.rand_quat = flog(R[11][0]);
  m.induction = flog(R[12][0]);
  m.ind_model = R[12][1];
  m.induction_type = R[12][2];
  m.method = R[12][3];
  m.nonadditive_3b = flog(R[13][0]);
  m.s3_term = flog(R[13][1]);
  m.s2_term = flog(R[13][2]);
  m.rcut3 = fnum(R[14][0]);
  m.alpha3 = fnum(R[14][1]);
  m.r0_tilda = fnum(R[14][2]);
  m.delta33 = fnum(R[14][3]);
  m.restart = flog(R[15][0]);
  m.check_forces = flog(R[16][0]);
  m.hsize = fnum(R[16][1]);
  return true;
}

bool parse_field(const std::string &path, ccp_model &m) {
  std::vector<std::string> lines;
  if (!read_lines(path, lines)) return false;
  std::vector<std::vector<std::string>> R;
  for (auto &l : lines) R.push_back(split(l));
  auto bad = [&](const char *what) {
    set_error(std::string("FIELD: ") + what);
    return false;
  };
  if (R.size() < 5 || R[0].empty() || R[1].empty() || R[2].empty() || R[3].empty())
    return bad("header is short");
  m.system_name = R[0][0];
  m.nm = (int)fnum(R[1][0]);
  m.ns = (int)fnum(R[2][0]);
  m.npol = (int)fnum(R[3][0]);
  if (m.ns < 1 || m.ns > kNsiteMax || m.npol < 0 || m.npol > m.ns) return bad("bad ns/npol");
  if (R.size() < (size_t)(5 + m.ns + 3)) return bad("site table is short");
  for (int s = 0; s < m.ns; s++) {
    auto &r = R[5 + s];
    if (r.size() < 7) return bad("site row is short");
    m.names.push_back(r[0]);
    for (int a = 0; a < 3; a++) m.coords.push_back(fnum(r[1 + a]));
    m.mass.push_back(fnum(r[4]));
    m.charge.push_back(fnum(r[5]));
    m.polarizability.push_back(fnum(r[6]));
  }
  size_t row = 5 + m.ns + 1;
  int npi = (int)fnum(R[row][0]);
  row += 2;
  for (int k = 0; k < npi && row + k < R.size(); k++) {
    auto &r = R[row + k];
    if (r.size() < 16) break;  // other potentials have other row shapes; not needed here
    ccp_model::VdwRow v;
    v.a = r[0];
    v.b = r[1];
    for (int q = 0; q < 14; q++) v.p[q] = fnum(r[2 + q]);
    m.vdw.push_back(v);
  }
  return true;
}

bool parse_fs3(const std::string &path, Fs3Table &T) {
  std::vector<std::string> lines;
  if (!read_lines(path, lines)) return false;
  if (lines.size() < 1 + 289 + 2) {
    set_error(path + ": too short");
    return false;
  }
  for (int n = 0; n < 289; n++) {
    auto r = split(lines[1 + n]);
    if (r.size() < 3) {
      set_error(path + ": short table row");
      return false;
    }
    T.b[n] = fnum(r[0]);
    T.g[n] = fnum(r[1]);
    T.r0[n] = fnum(r[2]);
  }
  int nlin = (int)fnum(split(lines[1 + 289 + 1]).at(0));
  if (nlin < 1 || nlin > 5000 || lines.size() < (size_t)(1 + 289 + 2 + nlin)) {
    set_error(path + ": bad number of linear parameters");
    return false;
  }
  T.cs.assign(nlin, 0.0);
  for (int n = 0; n < nlin; n++) {
    auto r = split(lines[1 + 289 + 2 + n]);
    if (r.size() < 2) {
      set_error(path + ": short coefficient row");
      return false;
    }
    T.cs[n] = fnum(r[1]);  // the reference fills cs3(is3) by row, ignoring the index column
  }
  return true;
}

// DL_POLY cyclic Jacobi diagonalisation of a symmetric matrix using its lower triangle
// (published algorithm; utility.f90:458-596 uses the same one).  a is row-major n x n.
void jacobi(double *a, double *v, int n) {
  const double rho = 1.0e-16;
  double tes = 0.0, scl = 0.0;
  auto A = [&](int i, int j) -> double & { return a[i * n + j]; };
  auto V = [&](int i, int j) -> double & { return v[i * n + j]; };
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) V(i, j) = (i == j) ? 1.0 : 0.0;
  for (int i = 0; i < n; i++)
    if (std::fabs(A(i, i)) > scl) scl = std::fabs(A(i, i));
  for (int i = 0; i < n; i++)
    for (int j = 0; j <= i; j++) A(i, j) = A(i, j) / scl;
  for (int i = 1; i < n; i++)
    for (int j = 0; j < i; j++) tes = tes + 2.0 * A(i, j) * A(i, j);
  tes = std::sqrt(tes);
  while (tes > rho) {
    tes = tes / (double)n;
    if (tes < rho) tes = rho;
    bool again = true;
    while (again) {
      again = false;
      for (int i = 1; i < n; i++)
        for (int j = 0; j < i; j++) {
          if (!(std::fabs(A(i, j)) >= tes)) continue;
          again = true;
          double v1 = A(j, j), v2 = A(i, j), v3 = A(i, i);
          double u = 0.5 * (v1 - v3), omg;
          if (std::fabs(u) < rho) {
            omg = -1.0;
          } else {
            omg = -v2 / std::sqrt(v2 * v2 + u * u);
            if (u < 0.0) omg = -omg;
          }
          double s = omg / std::sqrt(2.0 * (1.0 + std::sqrt(1.0 - omg * omg)));
          double c = std::sqrt(1.0 - s * s);
          for (int k = 0; k < n; k++) {
            double tem;
            if (k >= i) {
              tem = A(k, j) * c - A(k, i) * s;
              A(k, i) = A(k, j) * s + A(k, i) * c;
              A(k, j) = tem;
            } else if (k < j) {
              tem = A(j, k) * c - A(i, k) * s;
              A(i, k) = A(j, k) * s + A(i, k) * c;
              A(j, k) = tem;
            } else {
              tem = A(k, j) * c - A(i, k) * s;
              A(i, k) = A(k, j) * s + A(i, k) * c;
              A(k, j) = tem;
            }
            tem = V(k, j) * c - V(k, i) * s;
            V(k, i) = V(k, j) * s + V(k, i) * c;
            V(k, j) = tem;
          }
          A(j, j) = v1 * c * c + v3 * s * s - 2.0 * v2 * s * c;
          A(i, i) = v1 * s * s + v3 * c * c + 2.0 * v2 * s * c;
          A(i, j) = (v1 - v3) * s * c + v2 * (c * c - s * s);
        }
    }
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j <= i; j++) A(i, j) = scl * A(i, j);
}

bool principal_frame(ccp_model &m) {
  const int ns = m.ns;
  double totm = 0.0;
  for (int s = 0; s < ns; s++)
    if (m.mass[s] != 0.0) totm = totm + m.mass[s];
  if (!(totm > 0.0)) {
    set_error("FIELD: molecule has no mass");
    return false;
  }
  std::vector<double> c = m.coords;
  double r[3] = {0, 0, 0};
  for (int s = 0; s < ns; s++)
    for (int a = 0; a < 3; a++) r[a] = r[a] + m.mass[s] * c[s * 3 + a] / totm;
  for (int s = 0; s < ns; s++)
    for (int a = 0; a < 3; a++) c[s * 3 + a] = c[s * 3 + a] - r[a];
  double rmi[9] = {0}, rot[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int s = 0; s < ns; s++) {
        rmi[i * 3 + j] = rmi[i * 3 + j] - m.mass[s] * c[s * 3 + i] * c[s * 3 + j];
        if (i == j) {
          double x = c[s * 3], y = c[s * 3 + 1], z = c[s * 3 + 2];
          rmi[i * 3 + j] = rmi[i * 3 + j] + m.mass[s] * (x * x + y * y + z * z);
        }
      }
  jacobi(rmi, rot, 3);
  // initialization.f90:801-812: symmetrise and reject a degenerate tensor
  rmi[1] = rmi[3];
  rmi[2] = rmi[6];
  rmi[5] = rmi[7];
  double size = std::sqrt(rmi[0] * rmi[0] + rmi[4] * rmi[4] + rmi[8] * rmi[8]) / 3.0;
  if (rmi[0] / size < 1.0e-8 || rmi[4] / size < 1.0e-8 || rmi[8] / size < 1.0e-8) {
    set_error("FIELD: molecule off-diagonal inertia error");
    return false;
  }
  m.pmi[0] = rmi[0];
  m.pmi[1] = rmi[4];
  m.pmi[2] = rmi[8];
  m.totm = totm;
  m.pcoord.assign(ns * 3, 0.0);
  for (int s = 0; s < ns; s++) {
    double rx = c[s * 3], ry = c[s * 3 + 1], rz = c[s * 3 + 2];
    for (int a = 0; a < 3; a++)
      m.pcoord[s * 3 + a] = rx * rot[0 * 3 + a] + ry * rot[1 * 3 + a] + rz * rot[2 * 3 + a];
  }
  return true;
}

// FS3 symmetric coefficient index.  Site types come in consecutive blocks; a class is a
// multiset of three (type, power) pairs, numbered in the order the reference's sweep
// over (iat, jat, kat, ip, jp, kp) first meets it, and every site triple of those types
// and every one of the six permutations gets the same number.
const int kFs3Type1[kNs3] = {1, 2, 2, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 6, 6, 6, 6};

inline int tpos(int kp, int jp, int ip, int k, int j, int i) {  // 1-based sites
  return kp + 2 * jp + 4 * ip + 8 * (k - 1) + 136 * (j - 1) + 2312 * (i - 1);
}

void block_of(int site, int &first, int &last) {
  int t = kFs3Type1[site - 1];
  first = last = 0;
  for (int s = 1; s <= kNs3; s++)
    if (kFs3Type1[s - 1] == t) {
      if (!first) first = s;
      last = s;
    }
}

int build_index(std::vector<int> &ind) {
  ind.assign(kNs3 * kNs3 * kNs3 * 8, 0);
  int count = 0;
  for (int ia = 1; ia <= kNs3; ia++)
    for (int ja = 1; ja <= kNs3; ja++)
      for (int ka = 1; ka <= kNs3; ka++)
        for (int ip = 0; ip < 2; ip++)
          for (int jp = 0; jp < 2; jp++)
            for (int kp = 0; kp < 2; kp++) {
              if (ind[tpos(kp, jp, ip, ka, ja, ia)] != 0) continue;
              ++count;
              int i0, i1, j0, j1, k0, k1;
              block_of(ia, i0, i1);
              block_of(ja, j0, j1);
              block_of(ka, k0, k1);
              for (int ii = i0; ii <= i1; ii++)
                for (int jj = j0; jj <= j1; jj++)
                  for (int kk = k0; kk <= k1; kk++) {
                    ind[tpos(kp, jp, ip, kk, jj, ii)] = count;  // (i,j,k)
                    ind[tpos(jp, kp, ip, jj, kk, ii)] = count;  // (i,k,j)
                    ind[tpos(ip, kp, jp, ii, kk, jj)] = count;  // (j,k,i)
                    ind[tpos(kp, ip, jp, kk, ii, jj)] = count;  // (j,i,k)
                    ind[tpos(ip, jp, kp, ii, jj, kk)] = count;  // (k,j,i)
                    ind[tpos(jp, ip, kp, jj, ii, kk)] = count;  // (k,i,j)
                  }
            }
  return count;
}

// Collapse the per-site-triple index to a per-type-triple coefficient table and check
// that the index really depends on types only (it does by construction).
bool type_coefficients(ccp_model &m) {
  for (int s = 0; s < kNs3; s++) m.fs3_type[s] = kFs3Type1[s] - 1;
  const int nt = kNtype;
  m.coef_sr.assign(nt * nt * nt * 8, 0.0);
  m.coef_lr.assign(nt * nt * nt * 8, 0.0);
  m.class_of_type.assign(nt * nt * nt * 8, -1);
  std::vector<int> seen(nt * nt * nt * 8, 0);
  for (int is = 0; is < kNs3; is++)
    for (int js = 0; js < kNs3; js++)
      for (int ks = 0; ks < kNs3; ks++)
        for (int p = 0; p < 8; p++) {
          int ip = p >> 2, jp = (p >> 1) & 1, kp = p & 1;
          int idx = m.ind_lin[tpos(kp, jp, ip, ks + 1, js + 1, is + 1)];
          if (idx < 1 || idx > (int)m.sr.cs.size() || idx > (int)m.lr.cs.size()) {
            set_error("FS3 coefficient index outside the parameter files");
            return false;
          }
          int t = ((m.fs3_type[is] * nt + m.fs3_type[js]) * nt + m.fs3_type[ks]) * 8 + p;
          if (seen[t] && seen[t] != idx) {
            set_error("FS3 index is not a function of site types");
            return false;
          }
          seen[t] = idx;
          m.class_of_type[t] = idx - 1;
          m.coef_sr[t] = m.sr.cs[idx - 1];
          m.coef_lr[t] = m.lr.cs[idx - 1];
        }
  return true;
}

}  // namespace
}  // namespace ccp

using namespace ccp;

extern "C" {

const char *ccp_last_error(void) { return g_err.c_str(); }

int ccp_model_load(const char *dir, ccp_model **out) {
  if (!dir || !out) {
    set_error("ccp_model_load: null argument");
    return CCP_ERR_BAD_INPUT;
  }
  *out = nullptr;
  auto *m = new ccp_model();
  std::string d(dir);
  if (!d.empty() && d.back() != '/') d += '/';
  if (!parse_control(d + "CONTROL", *m)) {
    if (g_err.empty() || g_err.rfind("CONTROL", 0) != 0) set_error("cannot read " + d + "CONTROL");
    delete m;
    return CCP_ERR_IO;
  }
  set_error("");
  if (!parse_field(d + "FIELD", *m)) {
    if (g_err.empty()) set_error("cannot read " + d + "FIELD");
    delete m;
    return g_err.rfind("FIELD:", 0) == 0 ? CCP_ERR_BAD_INPUT : CCP_ERR_IO;
  }
  // The reference opens the FS3 files whenever the 3-body term is on; they are required
  // here only when FS3 itself is on, so an FS2-only parameter set needs no FS3 tables.
  if (m->nonadditive_3b && m->s3_term) {
    if (!parse_fs3(d + "data3b_full", m->sr) || !parse_fs3(d + "data3b_full_LR_4p5", m->lr)) {
      if (g_err.empty()) set_error("cannot read the FS3 parameter files in " + d);
      delete m;
      return CCP_ERR_IO;
    }
    m->have_fs3 = true;
  }
  if (!principal_frame(*m)) {
    delete m;
    return CCP_ERR_BAD_INPUT;
  }
  m->nclass = build_index(m->ind_lin);
  if (m->have_fs3 && !type_coefficients(*m)) {
    delete m;
    return CCP_ERR_BAD_INPUT;
  }
  set_error("");
  *out = m;
  return CCP_OK;
}

void ccp_model_free(ccp_model *m) { delete m; }

int ccp_model_get_int(const ccp_model *m, const char *name, int *value) {
  if (!m || !name || !value) return CCP_ERR_BAD_INPUT;
  std::string n(name);
  if (n == "nm") *value = m->nm;
  else if (n == "ns") *value = m->ns;
  else if (n == "npol") *value = m->npol;
  else if (n == "nsteps") *value = m->nsteps;
  else if (n == "nequil") *value = m->nequil;
  else if (n == "hist_freq") *value = m->hist_freq;
  else if (n == "S2_term") *value = m->s2_term;
  else if (n == "S3_term") *value = m->s3_term;
  else if (n == "nonadditive_3B") *value = m->nonadditive_3b;
  else if (n == "induction") *value = m->induction;
  else if (n == "damped") *value = (m->induction_type == "damped");
  else if (n == "restart") *value = m->restart;
  else if (n == "nclass") *value = m->nclass;
  else if (n == "nlin") *value = (int)m->sr.cs.size();
  else if (n == "have_fs3") *value = m->have_fs3;
  else if (n == "ensemble_nve") *value = m->ensemble == "nve";
  else if (n == "ensemble_kind")  // CCP_MD_* of the ensembles the device integrator runs, else -1
    *value = m->ensemble == "nve" ? CCP_MD_NVE
                                  : (m->ensemble == "nvt_b" ? CCP_MD_NVT_B
                                                            : (m->ensemble == "npt_b" ? CCP_MD_NPT_B
                                                               : (m->ensemble == "nvt_h" ? CCP_MD_NVT_H
                                                                  : (m->ensemble == "npt_h" ? CCP_MD_NPT_H
                                                                     : (m->ensemble == "npt_mtk" ? CCP_MD_NPT_MTK : -1)))));
  else {
    set_error("unknown int parameter " + n);
    return CCP_ERR_BAD_INPUT;
  }
  return CCP_OK;
}

int ccp_model_get_double(const ccp_model *m, const char *name, double *value) {
  if (!m || !name || !value) return CCP_ERR_BAD_INPUT;
  std::string n(name);
  if (n == "rcut") *value = m->rcut;
  else if (n == "rcut3") *value = m->rcut3;
  else if (n == "alpha3") *value = m->alpha3;
  else if (n == "delta33") *value = m->delta33;
  else if (n == "r0_tilda") *value = m->r0_tilda;
  else if (n == "dt") *value = m->dt;
  else if (n == "temp0") *value = m->temp0;
  else if (n == "pres0") *value = m->pres0;
  else if (n == "taut") *value = m->taut;
  else if (n == "taup") *value = m->taup;
  else if (n == "hsize") *value = m->hsize;
  else if (n == "totm") *value = m->totm;
  else {
    set_error("unknown double parameter " + n);
    return CCP_ERR_BAD_INPUT;
  }
  return CCP_OK;
}

int ccp_model_set_int(ccp_model *m, const char *name, int value) {
  if (!m || !name) return CCP_ERR_BAD_INPUT;
  std::string n(name);
  if (n == "nm") m->nm = value;
  else if (n == "S2_term") m->s2_term = value != 0;
  else if (n == "S3_term") m->s3_term = value != 0;
  else if (n == "nonadditive_3B") m->nonadditive_3b = value != 0;
  else if (n == "induction") m->induction = value != 0;
  else if (n == "damped") m->induction_type = value ? "damped" : "undamped";
  else {
    set_error("unknown or read-only int parameter " + n);
    return CCP_ERR_BAD_INPUT;
  }
  return CCP_OK;
}

int ccp_model_set_double(ccp_model *m, const char *name, double value) {
  if (!m || !name) return CCP_ERR_BAD_INPUT;
  std::string n(name);
  if (n == "rcut") m->rcut = value;
  else if (n == "rcut3") m->rcut3 = value;
  else if (n == "alpha3") m->alpha3 = value;
  else if (n == "delta33") m->delta33 = value;
  else {
    set_error("unknown or read-only double parameter " + n);
    return CCP_ERR_BAD_INPUT;
  }
  return CCP_OK;
}

int ccp_model_get_array(const ccp_model *m, const char *name, double *out, int n) {
  if (!m || !name || !out) return CCP_ERR_BAD_INPUT;
  std::string k(name);
  const std::vector<double> *src = nullptr;
  std::vector<double> tmp;
  if (k == "charge") src = &m->charge;
  else if (k == "polarizability") src = &m->polarizability;
  else if (k == "mass") src = &m->mass;
  else if (k == "pcoord") src = &m->pcoord;
  else if (k == "coords") src = &m->coords;
  else if (k == "pmi") {
    tmp.assign(m->pmi, m->pmi + 3);
    src = &tmp;
  } else if (k == "coef_sr") src = &m->coef_sr;
  else if (k == "coef_lr") src = &m->coef_lr;
  else if (k == "ind_lin") {
    tmp.assign(m->ind_lin.begin(), m->ind_lin.end());
    src = &tmp;
  } else {
    set_error("unknown array " + k);
    return CCP_ERR_BAD_INPUT;
  }
  if ((int)src->size() != n) {
    set_error("array " + k + " has " + std::to_string(src->size()) + " values");
    return CCP_ERR_BAD_INPUT;
  }
  std::memcpy(out, src->data(), sizeof(double) * n);
  return CCP_OK;
}

int ccp_sites(const ccp_model *m, int nm, const double *q, int ld, double *xs, double *ys,
              double *zs) {
  if (!m || !q || !xs || !ys || !zs || nm < 0 || ld < m->ns) {
    set_error("ccp_sites: bad argument");
    return CCP_ERR_BAD_INPUT;
  }
  for (int j = 0; j < nm; j++) {
    const double q0 = q[j * 4], q1 = q[j * 4 + 1], q2 = q[j * 4 + 2], q3 = q[j * 4 + 3];
    // quat_to_rot (molecular_sites.f90:93-111)
    const double r[9] = {q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3, 2.0 * (q1 * q2 - q0 * q3),
                         2.0 * (q1 * q3 + q0 * q2),           2.0 * (q1 * q2 + q0 * q3),
                         q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3, 2.0 * (q2 * q3 - q0 * q1),
                         2.0 * (q1 * q3 - q0 * q2),           2.0 * (q2 * q3 + q0 * q1),
                         q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3};
    for (int s = 0; s < m->ns; s++) {
      const double a = m->pcoord[s * 3], b = m->pcoord[s * 3 + 1], c = m->pcoord[s * 3 + 2];
      xs[(size_t)j * ld + s] = a * r[0] + b * r[1] + c * r[2];
      ys[(size_t)j * ld + s] = a * r[3] + b * r[4] + c * r[5];
      zs[(size_t)j * ld + s] = a * r[6] + b * r[7] + c * r[8];
    }
  }
  return CCP_OK;
}

int ccp_ewald_setup(double ewps, double rcut, double box, double *alp, int *k1, int *k2,
                    int *k3) {
  if (!alp || !k1 || !k2 || !k3 || !(rcut > 0.0) || !(box > 0.0)) {
    set_error("ccp_ewald_setup: bad argument");
    return CCP_ERR_BAD_INPUT;
  }
  double eprec = std::fmin(std::fabs(ewps), 0.5);
  double tol = std::sqrt(std::fabs(std::log(eprec * rcut)));
  double a = std::sqrt(std::fabs(std::log(eprec * rcut * tol))) / rcut;
  double t2 = 2.0 * tol * a;
  double tol1 = std::sqrt(-std::log(eprec * rcut * (t2 * t2)));
  int k = (int)std::round(0.25 + 1.0 * box * a * tol1 / kPi);
  *alp = a;
  *k1 = *k2 = *k3 = k;
  return CCP_OK;
}

}  // extern "C"
