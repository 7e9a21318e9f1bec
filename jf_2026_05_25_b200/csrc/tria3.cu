// tria3.cu -- CTRIA3 element stiffness (FP64) on the device.
//
// Default SOL101 CTRIA3 of FEMKernels.jl:9375-9809
// (stiffness_tria3_matrices_generic): constant-strain membrane, constant-
// curvature bending, MITC3 transverse shear on the recovered tying rigidity
// with the residual bending flexibility of the directional-pairing law and
// its guard (:9281-9313), lumped K6ROT drilling; element frame
// helpers.jl:1487-1490, local coordinates about the centroid and the
// congruence Ke = T' Ke_loc T of assembly.jl:5395-5503.  Isotropic PSHELL
// sections without MID4 coupling, offsets or SNORM.
//
// Two phases per CTA of T3_THREADS threads and T3_ELEMS elements: one thread
// per element reduces its geometry and section to a compact record in shared
// memory (membrane and bending operands, the 3 x 9 shear tying rows, the 3 x 3
// tying rigidity, the drilling weight and the three nodal frame rotations);
// then all threads write the T3_ELEMS x 324 global entries, consecutive
// threads on consecutive addresses, each entry contracted from the record.
#include "jfg_internal.h"

namespace jfg {
namespace {

constexpr int T3_THREADS = 128;
constexpr int T3_ELEMS = 32;
// record: A, bv[3], cv[3], Dm[9], Db[9], D3[27] (3 x 9 col-major), W[9],
// alpha, T[27] (per node 3 x 3, row k col i = (Rel node_R)[k][i])
constexpr int R_A = 0, R_BV = 1, R_CV = 4, R_DM = 7, R_DB = 16, R_D3 = 25, R_W = 52, R_AL = 61, R_T = 62;
constexpr int T3_REC = 89;

__device__ inline void t3_record_error(DevError* err, int32_t code, int64_t idx) {
  if (atomicCAS(&err->code, 0, code) == 0) err->index = idx;
}

// inverse of a 3 x 3 (col-major) by Gauss-Jordan elimination with partial
// pivoting (the flexibilities inverted here are ill-conditioned on slivers;
// elimination keeps the backward error at the level of one rounding);
// false if singular
__device__ inline bool inv3(const double* A, double* X) {
  double M[9];
  for (int q = 0; q < 9; ++q) { M[q] = A[q]; X[q] = (q % 4 == 0) ? 1.0 : 0.0; }
  for (int k = 0; k < 3; ++k) {
    int p = k;
    double best = fabs(M[k + 3 * k]);
    for (int i = k + 1; i < 3; ++i)
      if (fabs(M[i + 3 * k]) > best) { best = fabs(M[i + 3 * k]); p = i; }
    if (best == 0.0 || !isfinite(best)) return false;
    if (p != k)
      for (int j = 0; j < 3; ++j) {
        double t = M[k + 3 * j]; M[k + 3 * j] = M[p + 3 * j]; M[p + 3 * j] = t;
        t = X[k + 3 * j]; X[k + 3 * j] = X[p + 3 * j]; X[p + 3 * j] = t;
      }
    const double piv = M[k + 3 * k];
    for (int j = 0; j < 3; ++j) { M[k + 3 * j] /= piv; X[k + 3 * j] /= piv; }
    for (int i = 0; i < 3; ++i) {
      if (i == k) continue;
      const double f = M[i + 3 * k];
      if (f == 0.0) continue;
      for (int j = 0; j < 3; ++j) {
        M[i + 3 * j] -= f * M[k + 3 * j];
        X[i + 3 * j] -= f * X[k + 3 * j];
      }
    }
  }
  return true;
}

// FEMKernels.jl:9281-9313: bounds on the two residual bending channels in
// orthogonal work coordinates; false when the normal flexibility is not
// positive (the reference raises an error there)
__device__ inline bool t3_guard(double* Zb, double La, double Lb, double c, double s, double Dn) {
  const double scale = 6 * (La / Lb) * s * Dn;
  if (!(scale > 0.0 && Zb[8] > 0.0)) return true;
  const double z13 = Zb[6], z23 = Zb[7], z33 = Zb[8];
  const double h11 = scale * (Zb[0] - z13 * z13 / z33) / (La * La);
  const double h22 = scale * (Zb[4] - z23 * z23 / z33) / (Lb * Lb);
  const double h12 = scale * (Zb[3] - z13 * z23 / z33) / (La * Lb);
  const double p11 = h11, p12 = (h12 - c * h11) / s, p22 = (h22 - 2 * c * h12 + c * c * h11) / (s * s);
  if (!(isfinite(p22) && p22 > 0.0)) return false;
  const double a = fmax(p11, 1.0 / 10000);
  const double q = fmax(p22, a / 10000);
  const double lim = sqrt((85.0 / 100) * a * q);
  const double b = fmin(fmax(p12, -lim), lim);
  if (a == p11 && b == p12 && q == p22) return true;
  const double n11 = a, n12 = c * a + s * b, n22 = c * c * a + 2 * c * s * b + s * s * q;
  Zb[0] += (n11 - h11) * La * La / scale;
  Zb[3] += (n12 - h12) * La * Lb / scale;
  Zb[1] = Zb[3];
  Zb[4] += (n22 - h22) * Lb * Lb / scale;
  return true;
}

// Fills the compact record of one element; returns an error code or 0.
__device__ int t3_prepare(const double* __restrict__ xyz, const double* __restrict__ nodeR,
                          const int32_t* __restrict__ nd, const double* __restrict__ sect, double* rec) {
  double p[3][3];
  for (int k = 0; k < 3; ++k)
    for (int a = 0; a < 3; ++a) p[k][a] = xyz[3 * (int64_t)nd[k] + a];
  double v1[3], e13[3], v2[3], v3[3];
  for (int a = 0; a < 3; ++a) { v1[a] = p[1][a] - p[0][a]; e13[a] = p[2][a] - p[0][a]; }
  const double l1 = sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
  for (int a = 0; a < 3; ++a) v1[a] /= l1;
  v3[0] = v1[1] * e13[2] - v1[2] * e13[1];
  v3[1] = v1[2] * e13[0] - v1[0] * e13[2];
  v3[2] = v1[0] * e13[1] - v1[1] * e13[0];
  const double l3 = sqrt(v3[0] * v3[0] + v3[1] * v3[1] + v3[2] * v3[2]);
  for (int a = 0; a < 3; ++a) v3[a] /= l3;
  v2[0] = v3[1] * v1[2] - v3[2] * v1[1];
  v2[1] = v3[2] * v1[0] - v3[0] * v1[2];
  v2[2] = v3[0] * v1[1] - v3[1] * v1[0];
  double x[3], y[3];
  {
    double c[3];
    for (int a = 0; a < 3; ++a) c[a] = (p[0][a] + p[1][a] + p[2][a]) / 3.0;
    for (int k = 0; k < 3; ++k) {
      const double d0 = p[k][0] - c[0], d1 = p[k][1] - c[1], d2 = p[k][2] - c[2];
      x[k] = d0 * v1[0] + d1 * v1[1] + d2 * v1[2];
      y[k] = d0 * v2[0] + d1 * v2[1] + d2 * v2[2];
    }
  }
  // nodal congruence blocks T_k = Rel node_R_k
  for (int k = 0; k < 3; ++k) {
    const double* R = nodeR + 9 * (int64_t)nd[k];
    for (int r = 0; r < 3; ++r)
      for (int i = 0; i < 3; ++i) {
        const double* Rel = r == 0 ? v1 : (r == 1 ? v2 : v3);
        rec[R_T + 9 * k + 3 * r + i] = Rel[0] * R[3 * i] + Rel[1] * R[3 * i + 1] + Rel[2] * R[3 * i + 2];
      }
  }
  for (int q = 0; q < 9; ++q) { rec[R_DM + q] = sect[q]; rec[R_DB + q] = sect[9 + q]; }
  const double* Db = sect + 9;
  const double* Ds = sect + 18;
  const double A2 = x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]);
  const double A = 0.5 * fabs(A2);
  rec[R_A] = A;
  if (!(A >= 1e-12)) {   // degenerate: the reference returns a zero matrix
    rec[R_A] = 0.0;
    rec[R_AL] = 0.0;
    for (int q = 0; q < 6; ++q) rec[R_BV + q] = 0.0;
    for (int q = 0; q < 27; ++q) rec[R_D3 + q] = 0.0;
    for (int q = 0; q < 9; ++q) rec[R_W + q] = 0.0;
    return 0;
  }
  rec[R_BV + 0] = (y[1] - y[2]) / (2 * A);
  rec[R_BV + 1] = (y[2] - y[0]) / (2 * A);
  rec[R_BV + 2] = (y[0] - y[1]) / (2 * A);
  rec[R_CV + 0] = (x[2] - x[1]) / (2 * A);
  rec[R_CV + 1] = (x[0] - x[2]) / (2 * A);
  rec[R_CV + 2] = (x[1] - x[0]) / (2 * A);
  // MITC3 tying rows grA = g_r(1/2, 0), gsB = g_s(0, 1/2) and the linear mode
  // c = (g_r(C) - grA) - (g_s(C) - gsB); J = [x2-x1 y2-y1; x3-x1 y3-y1]
  const double J11 = x[1] - x[0], J12 = y[1] - y[0], J21 = x[2] - x[0], J22 = y[2] - y[0];
  for (int i = 0; i < 3; ++i) {
    const double NA = i == 0 ? 0.5 : (i == 1 ? 0.5 : 0.0);   // N at (1/2, 0)
    const double NB = i == 0 ? 0.5 : (i == 2 ? 0.5 : 0.0);   // N at (0, 1/2)
    const double NC = i == 0 ? 0.0 : 0.5;                    // N at (1/2, 1/2)
    const double dwdr = i == 0 ? -1.0 : (i == 1 ? 1.0 : 0.0);
    const double dwds = i == 0 ? -1.0 : (i == 2 ? 1.0 : 0.0);
    // columns w, rx, ry of node i
    const double grA[3] = {dwdr, -NA * J12, NA * J11};
    const double gsB[3] = {dwds, -NB * J22, NB * J21};
    const double grC[3] = {dwdr, -NC * J12, NC * J11};
    const double gsC[3] = {dwds, -NC * J22, NC * J21};
    for (int d = 0; d < 3; ++d) {
      const int col = 3 * i + d;
      rec[R_D3 + 3 * col + 0] = grA[d];
      rec[R_D3 + 3 * col + 1] = gsB[d];
      rec[R_D3 + 3 * col + 2] = (grC[d] - grA[d]) - (gsC[d] - gsB[d]);
    }
  }
  // tying rigidity W in the metric G = J^-T Ds J^-1
  const double detJ = J11 * J22 - J12 * J21;
  const double i11 = J22 / detJ, i12 = -J12 / detJ, i21 = -J21 / detJ, i22 = J11 / detJ;   // Jinv
  const double t11 = Ds[0] * i11 + Ds[2] * i21, t12 = Ds[0] * i12 + Ds[2] * i22;
  const double t21 = Ds[1] * i11 + Ds[3] * i21, t22 = Ds[1] * i12 + Ds[3] * i22;
  const double G11 = i11 * t11 + i21 * t21, G12 = i11 * t12 + i21 * t22, G22 = i12 * t12 + i22 * t22;
  const double La = hypot(J11, J12), Lb = hypot(J21, J22), Lc = hypot(x[2] - x[1], y[2] - y[1]);
  const double Pp = La + Lb + Lc;
  const double cth = fmin(fmax((J11 * J21 + J12 * J22) / fmax(La * Lb, 1e-30), -1.0), 1.0);
  const double sth = sqrt(fmax(1.0 - cth * cth, 0.0));
  const double uu = 3 * La / Pp, vv = 3 * Lb / Pp;
  double W[9];
  W[0] = G11 * A;
  W[3] = W[1] = G12 * A;
  W[4] = G22 * A;
  W[6] = W[2] = (A / 3) * (uu * G11 - vv * G12);
  W[7] = W[5] = (A / 3) * (uu * G12 - vv * G22);
  W[8] = uu * uu * G11 * (A / 6) - 2 * uu * vv * G12 * (A * (2 - cth) / 18) + vv * vv * G22 * (A / 6);
  const double Dbend = fabs(Db[0]);
  if (sth > 1e-9 && Dbend > 1e-30 && La > 1e-30 && Lb > 1e-30) {
    const double D22e = fabs(Db[4]);
    const bool dir = D22e > 1e-30;
    const double s6 = 1.0 / 6;
    const double rho = La / Lb, R2 = rho + 1 / rho - 2, T2 = rho - 1 / rho;
    const double omc2 = (1 - cth) * (1 - cth);
    double c11, c22, c12, Gd, Dn12;
    if (dir) {
      const double fr = (omc2 - (rho - cth)) / (6 * sth) + R2 * (1 + cth * cth) / (12 * sth) + T2 * sth / 12;
      const double fri = (omc2 - (1 / rho - cth)) / (6 * sth) + R2 * (1 + cth * cth) / (12 * sth) - T2 * sth / 12;
      const double w12 = (1 / rho - cth) / (6 * sth), w13 = (rho - cth) / (6 * sth), w23 = cth / (6 * sth);
      const double o12 = (R2 * cth - omc2 - T2 * cth) / (12 * sth);
      const double o13 = (R2 * cth - omc2 + T2 * cth) / (12 * sth);
      const double o23 = (1 + cth * cth) / (12 * sth);
      // directional stiffness w' Db w along the normal of each edge
      auto ddir = [&](double vx, double vy) {
        const double n = hypot(vx, vy);
        if (n < 1e-30) return Dbend;
        const double nx = -vy / n, ny = vx / n;
        const double w[3] = {nx * nx, ny * ny, 2 * nx * ny};
        double d = 0;
        for (int ii = 0; ii < 3; ++ii)
          for (int jj = 0; jj < 3; ++jj) d += w[ii] * Db[ii + 3 * jj] * w[jj];
        return fabs(d) > 1e-30 ? d : Dbend;
      };
      Dn12 = ddir(J11, J12);
      const double Dn13 = ddir(J21, J22);
      const double Dn23 = ddir(x[2] - x[1], y[2] - y[1]);
      Gd = sqrt(Dbend * D22e);
      c11 = s6 / Gd + fr / Dn12 + w13 / Dn13 + w23 / Dn23;
      c22 = s6 / Gd + w12 / Dn12 + fri / Dn13 + w23 / Dn23;
      c12 = -s6 / Gd + o12 / Dn12 + o13 / Dn13 + o23 / Dn23;
    } else {
      const double Rr = (La - Lb) * (La - Lb) / (La * Lb), Tt = (La * La - Lb * Lb) / (La * Lb);
      const double sum_d = 2 * ((1 - cth + cth * cth) / (6 * sth) + s6) + Rr * (1 + cth * cth) / (6 * sth);
      const double dif_d = Tt * sth / 6;
      c11 = ((sum_d + dif_d) / 2) / Dbend;
      c22 = ((sum_d - dif_d) / 2) / Dbend;
      c12 = ((-1 + 4 * cth - cth * cth) / (12 * sth) - s6 + Rr * cth / (6 * sth)) / Dbend;
      Gd = Dbend;
      Dn12 = Dbend;
    }
    const double S1 = La, S2 = Lb, S3 = Pp;
    double Zb[9];
    Zb[0] = c11 * S1 * S1;
    Zb[3] = Zb[1] = c12 * S1 * S2;
    Zb[4] = c22 * S2 * S2;
    Zb[6] = Zb[2] = -s6 / Gd * S1 * S3;
    Zb[7] = Zb[5] = s6 / Gd * S2 * S3;
    Zb[8] = s6 / Gd * S3 * S3;
    if (!t3_guard(Zb, La, Lb, cth, sth, Dn12)) return EE_T3_FLEX;
    double Wi[9], Zt[9];
    if (!inv3(W, Wi)) return EE_T3_FLEX;
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) Zt[i + 3 * j] = 0.5 * ((Wi[i + 3 * j] + Zb[i + 3 * j]) + (Wi[j + 3 * i] + Zb[j + 3 * i]));
    if (!inv3(Zt, W)) return EE_T3_FLEX;
  }
  for (int q = 0; q < 9; ++q) rec[R_W + q] = W[q];
  rec[R_AL] = (sect[24] * 1e-6) * sect[8] * (2 * A);
  return 0;
}

// local stiffness entry (r, c) of the record (DOFs u v w rx ry rz per node)
__device__ inline double t3_kloc(const double* rec, int r, int c) {
  const int a = r / 6, p = r - 6 * a, b = c / 6, q = c - 6 * b;
  const double A = rec[R_A];
  const double bva = rec[R_BV + a], cva = rec[R_CV + a], bvb = rec[R_BV + b], cvb = rec[R_CV + b];
  double v = 0.0;
  if (p < 2 && q < 2) {   // membrane: Bm columns (bv, 0, cv) for u and (0, cv, bv) for v
    const double xr[3] = {p == 0 ? bva : 0.0, p == 0 ? 0.0 : cva, p == 0 ? cva : bva};
    const double xc[3] = {q == 0 ? bvb : 0.0, q == 0 ? 0.0 : cvb, q == 0 ? cvb : bvb};
    const double* Dm = rec + R_DM;
    double s = 0.0;
    for (int l = 0; l < 3; ++l) s += (xr[0] * Dm[3 * l] + xr[1] * Dm[3 * l + 1] + xr[2] * Dm[3 * l + 2]) * xc[l];
    v += A * s;
  }
  if (p >= 2 && p <= 4 && q >= 2 && q <= 4) {
    // bending: Bb columns 0 for w, (0, -cv, -bv) for rx, (bv, 0, cv) for ry
    if (p > 2 && q > 2) {
      const double xr[3] = {p == 4 ? bva : 0.0, p == 3 ? -cva : 0.0, p == 3 ? -bva : cva};
      const double xc[3] = {q == 4 ? bvb : 0.0, q == 3 ? -cvb : 0.0, q == 3 ? -bvb : cvb};
      const double* Db = rec + R_DB;
      double s = 0.0;
      for (int l = 0; l < 3; ++l) s += (xr[0] * Db[3 * l] + xr[1] * Db[3 * l + 1] + xr[2] * Db[3 * l + 2]) * xc[l];
      v += A * s;
    }
    // MITC3 shear: D3[:, i]' W D3[:, j]
    const double* di = rec + R_D3 + 3 * (3 * a + p - 2);
    const double* dj = rec + R_D3 + 3 * (3 * b + q - 2);
    const double* W = rec + R_W;
    double s = 0.0;
    for (int l = 0; l < 3; ++l) s += (di[0] * W[3 * l] + di[1] * W[3 * l + 1] + di[2] * W[3 * l + 2]) * dj[l];
    v += s;
  }
  // lumped drilling: sum over nodes i of alpha (g + e_i)(g + e_i)', g the
  // membrane rotation row (cv/2 on u, -bv/2 on v), e_i the rz of node i
  const double gr = p == 0 ? 0.5 * cva : (p == 1 ? -0.5 * bva : 0.0);
  const double gc = q == 0 ? 0.5 * cvb : (q == 1 ? -0.5 * bvb : 0.0);
  const double er = p == 5 ? 1.0 : 0.0, ec = q == 5 ? 1.0 : 0.0;
  const double drill = 3.0 * gr * gc + gr * ec + er * gc + ((p == 5 && q == 5 && a == b) ? 1.0 : 0.0);
  v += rec[R_AL] * drill;
  return v;
}

__global__ void __launch_bounds__(T3_THREADS)
k_t3(int64_t n, const int32_t* __restrict__ nodes, const double* __restrict__ sect, const double* __restrict__ xyz,
     const double* __restrict__ nodeR, double* __restrict__ ev, DevError* err) {
  __shared__ double recs[T3_ELEMS][T3_REC];
  const int64_t e0 = (int64_t)blockIdx.x * T3_ELEMS;
  const int64_t left = n - e0;
  const int ne = left < T3_ELEMS ? (int)left : T3_ELEMS;
  if (threadIdx.x < ne) {
    const int64_t e = e0 + threadIdx.x;
    const int code = t3_prepare(xyz, nodeR, nodes + 3 * e, sect + JFG_Q4_SECT_STRIDE * e, recs[threadIdx.x]);
    if (code) t3_record_error(err, code, e);
  }
  __syncthreads();
  for (int ent = threadIdx.x; ent < ne * 324; ent += T3_THREADS) {
    const int le = ent / 324, k = ent - 324 * le;
    const int rr = k % 18, cc = k / 18;
    const double* rec = recs[le];
    const int I = rr / 3, i = rr - 3 * I, J = cc / 3, j = cc - 3 * J;
    const double* Ta = rec + R_T + 9 * (I / 2);
    const double* Tb = rec + R_T + 9 * (J / 2);
    double v = 0.0;
    for (int kk = 0; kk < 3; ++kk) {
      double row = 0.0;
      for (int ll = 0; ll < 3; ++ll) row += t3_kloc(rec, 3 * I + kk, 3 * J + ll) * Tb[3 * ll + j];
      v += Ta[3 * kk + i] * row;
    }
    ev[(e0 + le) * 324 + k] = v;
  }
}

}  // namespace

jfg_status launch_t3(const jfg_model* m, cudaStream_t st, double* ev, DevError* err) {
  if (m->n_t3 <= 0) return JFG_OK;
  const int64_t blocks = (m->n_t3 + T3_ELEMS - 1) / T3_ELEMS;
  k_t3<<<(unsigned)blocks, T3_THREADS, 0, st>>>(m->n_t3, m->d_t3n, m->d_t3s, m->d_xyz, m->d_R, ev, err);
  count_launch();
  JFG_CUDA(cudaGetLastError());
  return JFG_OK;
}

}  // namespace jfg
