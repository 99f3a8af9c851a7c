// k_md.cu -- the rigid-molecule NVE integrator of the reference (nve_1 with the nosquish
// rotation, evolve.f90:621-1061 and 8107-8203) on the device, FP64.
//
// State (structure of arrays): COM x, y, z; COM velocity v[3][nm]; unit quaternion
// q[4][nm]; principal-frame angular momentum j[3][nm].  A step is
//   stage 1 (one thread per molecule): force and torque from the previous evaluation's
//     site forces, quaternion momenta from j, half kick, COM drift, nosquish rotation,
//     j from the new momenta;
//   sites: site offsets R(q) pcoord (molecular_sites.f90:14-47);
//   the force evaluation (every term);
//   stage 2: force and torque again, half kick, j, periodic wrap of the COM, and the
//     kinetic-energy and molecular-virial sums.
#include "ccp_device.cuh"

using namespace ccpd;

namespace {

struct Rot {
  double r[9];  // row-major rott(1..9) of quat_to_rot (molecular_sites.f90:95-111)
};

__device__ __forceinline__ Rot quat_rot(double q0, double q1, double q2, double q3) {
  Rot R;
  R.r[0] = q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3;
  R.r[1] = 2.0 * (q1 * q2 - q0 * q3);
  R.r[2] = 2.0 * (q1 * q3 + q0 * q2);
  R.r[3] = 2.0 * (q1 * q2 + q0 * q3);
  R.r[4] = q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3;
  R.r[5] = 2.0 * (q2 * q3 - q0 * q1);
  R.r[6] = 2.0 * (q1 * q3 - q0 * q2);
  R.r[7] = 2.0 * (q2 * q3 + q0 * q1);
  R.r[8] = q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3;
  return R;
}

// Force and torque of molecule i (evolve.f90:664-704); lvir = sum_s f_s . s.
__device__ __forceinline__ void force_torque(int i, int nm, int ns, const double *__restrict__ f,
                                             const double *__restrict__ fc2,
                                             const double *__restrict__ fc3,
                                             const double *__restrict__ xs,
                                             const double *__restrict__ ys,
                                             const double *__restrict__ zs, double F[3],
                                             double T[3], double &lvir) {
  const size_t nfs = (size_t)nm * ns;
  F[0] = F[1] = F[2] = T[0] = T[1] = T[2] = 0.0;
  lvir = 0.0;
  for (int s = 0; s < ns; s++) {
    const size_t o = (size_t)i * ns + s;
    const double fx = f[o], fy = f[nfs + o], fz = f[2 * nfs + o];
    const double sx = xs[o], sy = ys[o], sz = zs[o];
    F[0] += fx;
    F[1] += fy;
    F[2] += fz;
    T[0] += sy * fz - sz * fy;
    T[1] += sz * fx - sx * fz;
    T[2] += sx * fy - sy * fx;
    lvir += fx * sx + fy * sy + fz * sz;
  }
  F[0] += fc2[i] + fc3[i];
  F[1] += fc2[nm + i] + fc3[nm + i];
  F[2] += fc2[2 * nm + i] + fc3[2 * nm + i];
}

// Quaternion torque and quaternion momenta from j (evolve.f90:712-741), then the half kick.
__device__ __forceinline__ void half_kick_p(const double q[4], const double T[3],
                                            const double J[3], double dt, double p[4]) {
  const Rot R = quat_rot(q[0], q[1], q[2], q[3]);
  const double tqx = T[0] * R.r[0] + T[1] * R.r[3] + T[2] * R.r[6];
  const double tqy = T[0] * R.r[1] + T[1] * R.r[4] + T[2] * R.r[7];
  const double tqz = T[0] * R.r[2] + T[1] * R.r[5] + T[2] * R.r[8];
  const double qt[4] = {2.0 * (-q[1] * tqx - q[2] * tqy - q[3] * tqz),
                        2.0 * (q[0] * tqx - q[3] * tqy + q[2] * tqz),
                        2.0 * (q[3] * tqx + q[0] * tqy - q[1] * tqz),
                        2.0 * (-q[2] * tqx + q[1] * tqy + q[0] * tqz)};
  const double ox = J[0], oy = J[1], oz = J[2];
  p[0] = 2.0 * (-q[1] * ox - q[2] * oy - q[3] * oz);
  p[1] = 2.0 * (q[0] * ox - q[3] * oy + q[2] * oz);
  p[2] = 2.0 * (q[3] * ox + q[0] * oy - q[1] * oz);
  p[3] = 2.0 * (-q[2] * ox + q[1] * oy + q[0] * oz);
  for (int k = 0; k < 4; k++) p[k] = p[k] + qt[k] * 0.5 * dt;
}

__device__ __forceinline__ void momenta_to_j(const double q[4], const double p[4], double J[3]) {
  J[0] = 0.5 * (-q[1] * p[0] + q[0] * p[1] + q[3] * p[2] - q[2] * p[3]);
  J[1] = 0.5 * (-q[2] * p[0] - q[3] * p[1] + q[0] * p[2] + q[1] * p[3]);
  J[2] = 0.5 * (-q[3] * p[0] + q[2] * p[1] - q[1] * p[2] + q[0] * p[3]);
}

// One rotation of the nosquish splitting about a principal axis: q and p rotate in the two
// planes (a, b) and (c, d) of their components by the angle zeta.
__device__ __forceinline__ void rot_pair(double zeta, double *q, double *p, int a, int b, int c,
                                         int d, double sa, double sc) {
  double sn, cs;
  sincos(zeta, &sn, &cs);
  const double qa = q[a], qb = q[b], qc = q[c], qd = q[d];
  const double pa = p[a], pb = p[b], pc = p[c], pd = p[d];
  q[a] = cs * qa - sn * qb;
  q[b] = cs * qb + sa * sn * qa;
  q[c] = cs * qc + sc * sn * qd;
  q[d] = cs * qd - sc * sn * qc;
  p[a] = cs * pa - sn * pb;
  p[b] = cs * pb + sa * sn * pa;
  p[c] = cs * pc + sc * sn * pd;
  p[d] = cs * pd - sc * sn * pc;
}

// nosquish (evolve.f90:8107-8203): mrot = 10 sub-steps of z/2, y/2, x, y/2, z/2.
__device__ void nosquish(double tstep, double q[4], double p[4], const double pmi[3]) {
  const double trstep = tstep / 10.0;
  for (int m = 0; m < 10; m++) {
    // z: (0,3) with q0' = c q0 - s q3, q3' = c q3 + s q0; (1,2): q1' = c q1 + s q2, q2' = c q2 - s q1
    double zeta = 0.125 / pmi[2] * trstep * (-p[0] * q[3] + p[1] * q[2] - p[2] * q[1] + p[3] * q[0]);
    rot_pair(zeta, q, p, 0, 3, 1, 2, 1.0, 1.0);
    // y: (0,2) q0' = c q0 - s q2, q2' = c q2 + s q0; (1,3) q1' = c q1 - s q3, q3' = c q3 + s q1
    zeta = 0.125 / pmi[1] * trstep * (-p[0] * q[2] - p[1] * q[3] + p[2] * q[0] + p[3] * q[1]);
    rot_pair(zeta, q, p, 0, 2, 1, 3, 1.0, -1.0);
    // x: (0,1) q0' = c q0 - s q1, q1' = c q1 + s q0; (2,3) q2' = c q2 + s q3, q3' = c q3 - s q2
    zeta = 0.25 / pmi[0] * trstep * (-p[0] * q[1] + p[1] * q[0] + p[2] * q[3] - p[3] * q[2]);
    rot_pair(zeta, q, p, 0, 1, 2, 3, 1.0, 1.0);
    zeta = 0.125 / pmi[1] * trstep * (-p[0] * q[2] - p[1] * q[3] + p[2] * q[0] + p[3] * q[1]);
    rot_pair(zeta, q, p, 0, 2, 1, 3, 1.0, -1.0);
    zeta = 0.125 / pmi[2] * trstep * (-p[0] * q[3] + p[1] * q[2] - p[2] * q[1] + p[3] * q[0]);
    rot_pair(zeta, q, p, 0, 3, 1, 2, 1.0, 1.0);
  }
}

__global__ void k_md_stage1(int nm, int ns, const double *__restrict__ f,
                            const double *__restrict__ fc2, const double *__restrict__ fc3,
                            const double *__restrict__ xs, const double *__restrict__ ys,
                            const double *__restrict__ zs, double *x, double *y, double *z,
                            double *v, double *qv, double *jv, double pmi0, double pmi1,
                            double pmi2, double totm, double dt, double scale, double cx,
                            double cy, double cz, int centred) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nm) return;
  double F[3], T[3], lvir;
  force_torque(i, nm, ns, f, fc2, fc3, xs, ys, zs, F, T, lvir);
  double q[4] = {qv[i], qv[nm + i], qv[2 * nm + i], qv[3 * nm + i]};
  const double J[3] = {jv[i], jv[nm + i], jv[2 * nm + i]};
  double p[4];
  half_kick_p(q, T, J, dt, p);
  double vx = v[i] + 0.5 * F[0] * dt / totm;
  double vy = v[nm + i] + 0.5 * F[1] * dt / totm;
  double vz = v[2 * nm + i] + 0.5 * F[2] * dt / totm;
  v[i] = vx;
  v[nm + i] = vy;
  v[2 * nm + i] = vz;
  if (centred) {  // npt_hov_2 (evolve.f90:5708-5712): scaled about the system's centre
    x[i] = scale * (x[i] - cx) + dt * vx + cx;
    y[i] = scale * (y[i] - cy) + dt * vy + cy;
    z[i] = scale * (z[i] - cz) + dt * vz + cz;
  } else if (scale == 1.0) {
    x[i] = x[i] + dt * vx;
    y[i] = y[i] + dt * vy;
    z[i] = z[i] + dt * vz;
  } else {  // npt_b_1 (evolve.f90:7612-7616): the barostat scales the centres in the drift
    x[i] = scale * x[i] + dt * vx;
    y[i] = scale * y[i] + dt * vy;
    z[i] = scale * z[i] + dt * vz;
  }
  const double pmi[3] = {pmi0, pmi1, pmi2};
  nosquish(dt, q, p, pmi);
  double Jn[3];
  momenta_to_j(q, p, Jn);
  for (int k = 0; k < 4; k++) qv[k * nm + i] = q[k];
  for (int k = 0; k < 3; k++) jv[k * nm + i] = Jn[k];
}

// site offsets of every molecule from its quaternion (transform, iway = 1)
__global__ void k_md_sites(int nm, int ns, const double *__restrict__ qv,
                           const double *__restrict__ pcoord, double *xs, double *ys, double *zs) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nm * ns) return;
  const int i = t / ns, s = t - i * ns;
  const Rot R = quat_rot(qv[i], qv[nm + i], qv[2 * nm + i], qv[3 * nm + i]);
  const double r1 = pcoord[3 * s], r2 = pcoord[3 * s + 1], r3 = pcoord[3 * s + 2];
  xs[t] = r1 * R.r[0] + r2 * R.r[1] + r3 * R.r[2];
  ys[t] = r1 * R.r[3] + r2 * R.r[4] + r3 * R.r[5];
  zs[t] = r1 * R.r[6] + r2 * R.r[7] + r3 * R.r[8];
}

// stage 2; red[0] += sum v^2, red[1] += sum j^2/pmi, red[2] += sum f.s
__global__ void k_md_stage2(int nm, int ns, const double *__restrict__ f,
                            const double *__restrict__ fc2, const double *__restrict__ fc3,
                            const double *__restrict__ xs, const double *__restrict__ ys,
                            const double *__restrict__ zs, double *x, double *y, double *z,
                            double *v, const double *__restrict__ qv, double *jv, double pmi0,
                            double pmi1, double pmi2, double totm, double dt, double box,
                            int wrap, double *red) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v2 = 0.0, j2 = 0.0, lv = 0.0, sv[3] = {0.0, 0.0, 0.0};
  if (i < nm) {
    double F[3], T[3], lvir;
    force_torque(i, nm, ns, f, fc2, fc3, xs, ys, zs, F, T, lvir);
    const double q[4] = {qv[i], qv[nm + i], qv[2 * nm + i], qv[3 * nm + i]};
    const double J[3] = {jv[i], jv[nm + i], jv[2 * nm + i]};
    double p[4];
    half_kick_p(q, T, J, dt, p);
    const double vx = v[i] + 0.5 * F[0] * dt / totm;
    const double vy = v[nm + i] + 0.5 * F[1] * dt / totm;
    const double vz = v[2 * nm + i] + 0.5 * F[2] * dt / totm;
    v[i] = vx;
    v[nm + i] = vy;
    v[2 * nm + i] = vz;
    double Jn[3];
    momenta_to_j(q, p, Jn);
    for (int k = 0; k < 3; k++) jv[k * nm + i] = Jn[k];
    if (wrap) {  // evolve.f90:1009-1015: periodic wrap of the centres of mass
      x[i] = minimg(x[i], box);
      y[i] = minimg(y[i], box);
      z[i] = minimg(z[i], box);
    }
    v2 = vx * vx + vy * vy + vz * vz;
    sv[0] = vx;
    sv[1] = vy;
    sv[2] = vz;
    j2 = Jn[0] * Jn[0] / pmi0 + Jn[1] * Jn[1] / pmi1 + Jn[2] * Jn[2] / pmi2;
    lv = lvir;
  }
  v2 = warp_sum(v2);
  j2 = warp_sum(j2);
  lv = warp_sum(lv);
  for (int k = 0; k < 3; k++) sv[k] = warp_sum(sv[k]);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&red[0], v2);
    atomicAdd(&red[1], j2);
    atomicAdd(&red[2], lv);
    for (int k = 0; k < 3; k++) atomicAdd(&red[3 + k], sv[k]);
  }
}

// Periodic wrap of the centres into the box (npt_b_1 does it after its thermostat,
// evolve.f90:8094-8098).
__global__ void k_md_wrap(int nm, double *x, double *y, double *z, double box) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += gridDim.x * blockDim.x) {
    x[i] = minimg(x[i], box);
    y[i] = minimg(y[i], box);
    z[i] = minimg(z[i], box);
  }
}

// Kinetic sums and the COM virial of the current state without moving it (the statistics
// of initialization.f90:76-89, 386-399): v^2, J^2 / I and sum f . xs.
__global__ void k_md_sums(int nm, int ns, const double *__restrict__ f,
                          const double *__restrict__ fc2, const double *__restrict__ fc3,
                          const double *__restrict__ xs, const double *__restrict__ ys,
                          const double *__restrict__ zs, const double *__restrict__ v,
                          const double *__restrict__ jv, const double *__restrict__ x,
                          double pmi0, double pmi1, double pmi2, double *red) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v2 = 0.0, j2 = 0.0, lv = 0.0, sv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (i < nm) {
    double F[3], T[3], lvir;
    force_torque(i, nm, ns, f, fc2, fc3, xs, ys, zs, F, T, lvir);
    const double vx = v[i], vy = v[nm + i], vz = v[2 * nm + i];
    const double J0 = jv[i], J1 = jv[nm + i], J2 = jv[2 * nm + i];
    v2 = vx * vx + vy * vy + vz * vz;
    j2 = J0 * J0 / pmi0 + J1 * J1 / pmi1 + J2 * J2 / pmi2;
    lv = lvir;
    sv[0] = vx;
    sv[1] = vy;
    sv[2] = vz;
    sv[3] = x[i];
    sv[4] = x[nm + i];
    sv[5] = x[2 * nm + i];
  }
  v2 = warp_sum(v2);
  j2 = warp_sum(j2);
  lv = warp_sum(lv);
  for (int k = 0; k < 6; k++) sv[k] = warp_sum(sv[k]);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&red[0], v2);
    atomicAdd(&red[1], j2);
    atomicAdd(&red[2], lv);
    for (int k = 0; k < 6; k++) atomicAdd(&red[3 + k], sv[k]);
  }
}

// Velocity rescaling (rescale_velocities, utility.f90:257-275, and the Berendsen thermostat
// of nvt_b / npt_b_1): COM velocities v = fv (v - c), angular momenta by fj; c is the
// system's COM velocity that npt_b_1 removes first (evolve.f90:8029-8055), else 0.
__global__ void k_md_scale(int nm, double *v, double cx, double cy, double cz, double fv,
                           double *jv, double fj) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * nm; t += gridDim.x * blockDim.x) {
    const double c = t < nm ? cx : (t < 2 * nm ? cy : cz);
    v[t] = fv * (v[t] - c);
    jv[t] *= fj;
  }
}

}  // namespace

cudaError_t launch_md_sums(int nm, int ns, const double *f, const double *fc2, const double *fc3,
                           const double *xs, const double *ys, const double *zs, const double *v,
                           const double *j, const double *x, const double pmi[3], double *red,
                           cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(red, 0, 9 * sizeof(double), st);
  if (e != cudaSuccess) return e;
  k_md_sums<<<(nm + 127) / 128, 128, 0, st>>>(nm, ns, f, fc2, fc3, xs, ys, zs, v, j, x, pmi[0],
                                              pmi[1], pmi[2], red);
  return cudaGetLastError();
}

cudaError_t launch_md_scale(int nm, double *v, const double c[3], double fv, double *j, double fj,
                            cudaStream_t st) {
  const int n = 3 * nm;
  k_md_scale<<<(n + 255) / 256, 256, 0, st>>>(nm, v, c[0], c[1], c[2], fv, j, fj);
  return cudaGetLastError();
}

cudaError_t launch_md_wrap(int nm, double *x, double *y, double *z, double box, cudaStream_t st) {
  k_md_wrap<<<(nm + 255) / 256, 256, 0, st>>>(nm, x, y, z, box);
  return cudaGetLastError();
}

cudaError_t launch_md_stage1(int nm, int ns, const double *f, const double *fc2,
                             const double *fc3, const double *xs, const double *ys,
                             const double *zs, double *x, double *y, double *z, double *v,
                             double *q, double *j, const double pmi[3], double totm, double dt,
                             double scale, const double centre[3], cudaStream_t st) {
  k_md_stage1<<<(nm + 127) / 128, 128, 0, st>>>(nm, ns, f, fc2, fc3, xs, ys, zs, x, y, z, v, q, j,
                                                pmi[0], pmi[1], pmi[2], totm, dt, scale,
      centre ? centre[0] : 0.0, centre ? centre[1] : 0.0, centre ? centre[2] : 0.0, centre ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_md_sites(int nm, int ns, const double *q, const double *pcoord, double *xs,
                            double *ys, double *zs, cudaStream_t st) {
  const int n = nm * ns;
  k_md_sites<<<(n + 255) / 256, 256, 0, st>>>(nm, ns, q, pcoord, xs, ys, zs);
  return cudaGetLastError();
}

cudaError_t launch_md_stage2(int nm, int ns, const double *f, const double *fc2,
                             const double *fc3, const double *xs, const double *ys,
                             const double *zs, double *x, double *y, double *z, double *v,
                             const double *q, double *j, const double pmi[3], double totm,
                             double dt, double box, int wrap, double *red, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(red, 0, 6 * sizeof(double), st);
  if (e != cudaSuccess) return e;
  k_md_stage2<<<(nm + 127) / 128, 128, 0, st>>>(nm, ns, f, fc2, fc3, xs, ys, zs, x, y, z, v, q, j,
                                                pmi[0], pmi[1], pmi[2], totm, dt, box, wrap, red);
  return cudaGetLastError();
}
