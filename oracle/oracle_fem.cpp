// oracle_fem.cpp -- CPU FP64 restatement of OpenJFEM's SOL101 element and
// assembly path.  TEST INFRASTRUCTURE ONLY: this file is the checker that the
// CUDA library is compared against (tests/, the smoke check and the CPU
// baseline leg of bench.py).  Nothing in the product links or calls it.
//
// Each function cites the reference file:line whose behaviour it restates.
// All matrices are column-major (Julia layout): A[r + nrow*c].
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <vector>
#include <numeric>

namespace {

inline double& at(double* A, int n, int r, int c) { return A[r + n * c]; }
inline double at(const double* A, int n, int r, int c) { return A[r + n * c]; }

// C(m x n) += alpha * A(k x m)^T * B(k x n)  (FEMKernels.jl:649 ts_mul_At_add!)
void mul_At_add(double* C, int m, int n, const double* A, int k, const double* B,
                double alpha) {
  for (int j = 0; j < n; ++j)
    for (int l = 0; l < k; ++l) {
      double v = alpha * B[l + k * j];
      for (int i = 0; i < m; ++i) C[i + m * j] += A[l + k * i] * v;
    }
}
// C(m x n) = A(m x k) * B(k x n)  (FEMKernels.jl:663 ts_mul!)
void mul(double* C, int m, int n, const double* A, int k, const double* B) {
  for (int i = 0; i < m * n; ++i) C[i] = 0.0;
  for (int j = 0; j < n; ++j)
    for (int l = 0; l < k; ++l) {
      double v = B[l + k * j];
      for (int i = 0; i < m; ++i) C[i + m * j] += A[i + m * l] * v;
    }
}

// Small dense inverse by Gauss-Jordan with partial pivoting.  Returns false if
// singular.  (Julia's inv(SMatrix) / LU replicas; 1e-12 parity needs only the
// mathematically same inverse, not identical rounding.)
bool inv_small(const double* A, int n, double* Ainv) {
  std::vector<double> M(A, A + n * n);
  for (int i = 0; i < n * n; ++i) Ainv[i] = 0.0;
  for (int i = 0; i < n; ++i) Ainv[i + n * i] = 1.0;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = std::fabs(M[k + n * k]);
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(M[i + n * k]) > best) { best = std::fabs(M[i + n * k]); p = i; }
    if (best == 0.0 || !std::isfinite(best)) return false;
    if (p != k)
      for (int j = 0; j < n; ++j) {
        std::swap(M[k + n * j], M[p + n * j]);
        std::swap(Ainv[k + n * j], Ainv[p + n * j]);
      }
    double piv = M[k + n * k];
    for (int j = 0; j < n; ++j) { M[k + n * j] /= piv; Ainv[k + n * j] /= piv; }
    for (int i = 0; i < n; ++i) {
      if (i == k) continue;
      double f = M[i + n * k];
      if (f == 0.0) continue;
      for (int j = 0; j < n; ++j) {
        M[i + n * j] -= f * M[k + n * j];
        Ainv[i + n * j] -= f * Ainv[k + n * j];
      }
    }
  }
  return true;
}

// FEMKernels.jl:762 shape_derivs_quad
inline void shape_derivs_quad(double xi, double eta, double dNr[4], double dNs[4]) {
  dNr[0] = -0.25 * (1 - eta); dNr[1] = 0.25 * (1 - eta);
  dNr[2] = 0.25 * (1 + eta);  dNr[3] = -0.25 * (1 + eta);
  dNs[0] = -0.25 * (1 - xi);  dNs[1] = -0.25 * (1 + xi);
  dNs[2] = 0.25 * (1 + xi);   dNs[3] = 0.25 * (1 - xi);
}
inline void shape_vals_quad(double xi, double eta, double N[4]) {
  N[0] = 0.25 * (1 - xi) * (1 - eta); N[1] = 0.25 * (1 + xi) * (1 - eta);
  N[2] = 0.25 * (1 + xi) * (1 + eta); N[3] = 0.25 * (1 - xi) * (1 + eta);
}
inline void jac_quad(const double* lc /*4x2 col-major*/, const double dNr[4],
                     const double dNs[4], double& J11, double& J12, double& J21,
                     double& J22) {
  J11 = J12 = J21 = J22 = 0.0;
  for (int k = 0; k < 4; ++k) {
    J11 += dNr[k] * lc[k]; J12 += dNr[k] * lc[k + 4];
    J21 += dNs[k] * lc[k]; J22 += dNs[k] * lc[k + 4];
  }
}
// FEMKernels.jl:2867 _quad4_jacobian_measure
inline bool jac_ok(double detj, double j11, double j12, double j21, double j22) {
  double scale = std::fabs(j11 * j22) + std::fabs(j12 * j21);
  return std::isfinite(detj) && std::isfinite(scale) &&
         std::fabs(detj) > 64.0 * 2.220446049250313e-16 * scale;
}

// MacNeal shear block on the default path: full edge MITC rows (D_edge) and
// the natural residual-flexibility law.
//   rows:          FEMKernels.jl:4599-4783 (shear_mitc, row_full, pt_row = 1)
//   flexibility:   FEMKernels.jl:4223-4339 quad4_natural_shear_flexibility!
//   K_plate:       FEMKernels.jl:6187-6200, added at plate dofs :6278-6285
int macneal_shear(const double* lc, const double* Cb, const double* Cs, double h,
                  double* Ke, double* KP_out = nullptr) {
  double csmax = 0;
  for (int i = 0; i < 4; ++i) csmax = std::max(csmax, std::fabs(Cs[i]));
  if (h < 1e-30 || csmax < 1e-30) return 0;
  const double pt = 1.0 / std::sqrt(3.0);
  // sample (xi, eta, comp) at Gauss offsets and their edge (row) points
  const double sxi[4] = {0.0, 0.0, -pt, pt}, seta[4] = {-pt, pt, 0.0, 0.0};
  const int comp[4] = {1, 1, 2, 2};
  double Ce[4][12];
  double Je[4][4];
  for (int sp = 0; sp < 4; ++sp) {
    double xr = sxi[sp] == 0.0 ? 0.0 : std::copysign(1.0, sxi[sp]);
    double er = seta[sp] == 0.0 ? 0.0 : std::copysign(1.0, seta[sp]);
    double dNr[4], dNs[4], N[4];
    shape_derivs_quad(xr, er, dNr, dNs);
    shape_vals_quad(xr, er, N);
    double J11, J12, J21, J22;
    jac_quad(lc, dNr, dNs, J11, J12, J21, J22);
    Je[sp][0] = J11; Je[sp][1] = J12; Je[sp][2] = J21; Je[sp][3] = J22;
    double tx = comp[sp] == 1 ? J11 : J21;
    double ty = comp[sp] == 1 ? J12 : J22;
    for (int k = 0; k < 4; ++k) {
      Ce[sp][3 * k + 0] = comp[sp] == 1 ? dNr[k] : dNs[k];
      Ce[sp][3 * k + 1] = -N[k] * ty;
      Ce[sp][3 * k + 2] = N[k] * tx;
    }
  }
  double D[4 * 12];  // 4 x 12 column-major
  for (int sp = 0; sp < 4; ++sp) {
    double J11 = Je[sp][0], J12 = Je[sp][1], J21 = Je[sp][2], J22 = Je[sp][3];
    double det = J11 * J22 - J12 * J21;
    double adet = std::fabs(det) < 1e-14 ? (det < 0 ? -1e-14 : 1e-14) : det;
    double i11 = J22 / adet, i12 = -J12 / adet, i21 = -J21 / adet, i22 = J11 / adet;
    double xi = sxi[sp], eta = seta[sp];
    double w1 = 0.5 * (1.0 - eta / pt), w2 = 0.5 * (1.0 + eta / pt);
    double w3 = 0.5 * (1.0 - xi / pt), w4 = 0.5 * (1.0 + xi / pt);
    for (int j = 0; j < 12; ++j) {
      double gxi = w1 * Ce[0][j] + w2 * Ce[1][j];
      double geta = w3 * Ce[2][j] + w4 * Ce[3][j];
      D[sp + 4 * j] = sp < 2 ? (i11 * gxi + i12 * geta) : (i21 * gxi + i22 * geta);
    }
  }
  // natural residual flexibility
  double tr[16] = {0};  // transport 4x4 col-major
  const double rn[4] = {-1, 1, 1, -1}, sn[4] = {-1, -1, 1, 1};
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 4; ++k) {
      int b = 3 * k;
      tr[i + 4 * 0] += D[i + 4 * (b + 2)];
      tr[i + 4 * 1] += sn[k] * D[i + 4 * (b + 2)];
      tr[i + 4 * 2] -= D[i + 4 * (b + 1)];
      tr[i + 4 * 3] -= rn[k] * D[i + 4 * (b + 1)];
    }
  const double* x = lc; const double* y = lc + 4;
  double ax = 0.25 * (-x[0] + x[1] + x[2] - x[3]), ay = 0.25 * (-y[0] + y[1] + y[2] - y[3]);
  double bx = 0.25 * (-x[0] - x[1] + x[2] + x[3]), by = 0.25 * (-y[0] - y[1] + y[2] + y[3]);
  double cx = 0.25 * (x[0] - x[1] + x[2] - x[3]), cy = 0.25 * (y[0] - y[1] + y[2] - y[3]);
  double det0 = ax * by - ay * bx;
  double det_scale = std::max(std::hypot(ax, ay) * std::hypot(bx, by), 2.220446049250313e-16);
  if (!(std::fabs(det0) > 64 * 2.220446049250313e-16 * det_scale)) return 2;
  double area = 4.0 * std::fabs(det0);
  double dx2 = (2 * ax) * (2 * ax), dy2 = (2 * by) * (2 * by);
  double fxx = std::fabs(2 * ax) > 1e-30 ? (cx / (2 * ax)) * (cx / (2 * ax)) : 0.0;
  double fyy = std::fabs(2 * by) > 1e-30 ? (cy / (2 * by)) * (cy / (2 * by)) : 0.0;
  if (fxx + fyy > 1e-24 && ((Cb[0] == 0.0) != (Cb[4] == 0.0))) return 3;
  double dxr = Cb[0], dyr = Cb[4];
  double ux = dx2 / (12 * area * std::max(std::fabs(dxr), 1e-30));
  double uy = dy2 / (12 * area * std::max(std::fabs(dyr), 1e-30));
  double zb[4] = {ux, 3 * dy2 / (dy2 + 39 * dx2) * ux, uy, 3 * dx2 / (dx2 + 39 * dy2) * uy};
  double Z[16] = {0};
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i)
      for (int k = 0; k < 4; ++k) Z[i + 4 * j] += tr[i + 4 * k] * zb[k] * tr[j + 4 * k];
  // Zs = tr * inv(H) * tr'
  const double gp = pt;
  auto jac = [&](double r, double s) {
    return std::fabs((ax + cx * s) * (by + cy * r) - (ay + cy * s) * (bx + cx * r));
  };
  double va = std::sqrt(2 * jac(0.0, -gp)), vb = std::sqrt(2 * jac(0.0, gp));
  double vc = std::sqrt(2 * jac(-gp, 0.0)), vd = std::sqrt(2 * jac(gp, 0.0));
  double pxa[4] = {va, -gp * va, 0, 0}, pxb[4] = {vb, gp * vb, 0, 0};
  double pyc[4] = {0, 0, vc, -gp * vc}, pyd[4] = {0, 0, vd, gp * vd};
  double H[16];
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i)
      H[i + 4 * j] = Cs[0] * (pxa[i] * pxa[j] + pxb[i] * pxb[j]) +
                     Cs[3] * (pyc[i] * pyc[j] + pyd[i] * pyd[j]) +
                     Cs[2] * (pxa[i] + pxb[i]) * (pyc[j] + pyd[j]) / 2 +
                     Cs[1] * (pyc[i] + pyd[i]) * (pxa[j] + pxb[j]) / 2;
  double Hi[16];
  if (!inv_small(H, 4, Hi)) return 4;
  double t4[16], Zs[16];
  mul(t4, 4, 4, tr, 4, Hi);
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += t4[i + 4 * k] * tr[j + 4 * k];
      Zs[i + 4 * j] = s;
    }
  for (int i = 0; i < 16; ++i) Z[i] += Zs[i];
  double Zi[16];
  if (!inv_small(Z, 4, Zi)) return 5;
  double sol[4 * 12];
  mul(sol, 4, 12, Zi, 4, D);
  double KP[144] = {0};
  mul_At_add(KP, 12, 12, D, 4, sol, 1.0);
  if (KP_out) std::memcpy(KP_out, KP, sizeof KP);
  const int pd[12] = {2, 3, 4, 8, 9, 10, 14, 15, 16, 20, 21, 22};
  for (int j = 0; j < 12; ++j)
    for (int i = 0; i < 12; ++i)
      Ke[pd[i] + 24 * pd[j]] += 0.5 * (KP[i + 12 * j] + KP[j + 12 * i]);
  return 0;
}

// CQUAD4 element frame (shell_element_frame_quad4, diagonal mode) and the
// local in-plane coordinates of the corners about their centroid, as the
// stiffness and the stress recovery both take them
// (stress_recovery.jl:774-781, assembly.jl:5858-5870).  xyz: 4 x 3, node
// major.  zmax / xmax: largest out-of-plane offset and in-plane coordinate.
void q4_frame(const double* xyz, double v1[3], double v2[3], double v3[3], double lc[8],
              double& zmax, double& xmax) {
  double p[4][3];
  for (int k = 0; k < 4; ++k)
    for (int a = 0; a < 3; ++a) p[k][a] = xyz[3 * k + a];
  auto sub = [](const double* a, const double* b, double* o) {
    o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2];
  };
  auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  auto cross = [](const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1]; o[1] = a[2] * b[0] - a[0] * b[2]; o[2] = a[0] * b[1] - a[1] * b[0];
  };
  auto nrm = [&](double* a) {
    double l = std::sqrt(dot(a, a));
    a[0] /= l; a[1] /= l; a[2] /= l;
  };
  double gxi[3], geta[3];
  for (int a = 0; a < 3; ++a) {
    gxi[a] = 0.25 * (-p[0][a] + p[1][a] + p[2][a] - p[3][a]);
    geta[a] = 0.25 * (-p[0][a] - p[1][a] + p[2][a] + p[3][a]);
  }
  cross(gxi, geta, v3);
  double d13[3], d24[3];
  sub(p[2], p[0], d13); sub(p[3], p[1], d24);
  if (dot(v3, v3) <= 1e-24) cross(d13, d24, v3);
  nrm(v3);
  double d13n[3] = {d13[0], d13[1], d13[2]}, d24n[3] = {d24[0], d24[1], d24[2]};
  nrm(d13n); nrm(d24n);
  double xr[3];
  for (int a = 0; a < 3; ++a) xr[a] = d13n[a] - d24n[a];
  if (dot(xr, xr) < 1e-20)
    for (int a = 0; a < 3; ++a) xr[a] = d13n[a] + d24n[a];
  double xp[3];
  double dv = dot(xr, v3);
  for (int a = 0; a < 3; ++a) xp[a] = xr[a] - dv * v3[a];
  if (dot(xp, xp) <= 1e-24) {
    double ge = dot(geta, v3);
    for (int a = 0; a < 3; ++a) xp[a] = geta[a] - ge * v3[a];
    if (dot(xp, xp) <= 1e-24) {
      double e12[3];
      sub(p[1], p[0], e12);
      double de = dot(e12, v3);
      for (int a = 0; a < 3; ++a) xp[a] = e12[a] - de * v3[a];
    }
  }
  for (int a = 0; a < 3; ++a) v1[a] = xp[a];
  nrm(v1);
  cross(v3, v1, v2);
  double c[3];
  for (int a = 0; a < 3; ++a) c[a] = (p[0][a] + p[1][a] + p[2][a] + p[3][a]) / 4.0;
  zmax = 0;
  xmax = 0;
  for (int k = 0; k < 4; ++k) {
    double d[3];
    sub(p[k], c, d);
    lc[k] = dot(d, v1);
    lc[k + 4] = dot(d, v2);
    zmax = std::max(zmax, std::fabs(dot(d, v3)));
    xmax = std::max(xmax, std::fabs(lc[k]));
  }
}

// Principal values of a 2-D symmetric tensor (xx, yy, xy) without
// cancellation (_recovery_principal_2d, stress_recovery.jl:17-34).
void principal_2d(double xx, double yy, double xy, double& major, double& minor) {
  if (xy == 0.0) {
    major = std::max(xx, yy);
    minor = std::min(xx, yy);
    return;
  }
  double scale = std::max(std::max(std::fabs(xx), std::fabs(yy)), std::fabs(xy));
  double a = xx / scale, b = yy / scale, c = xy / scale;
  double mean = (a + b) / 2, radius = std::hypot((a - b) / 2, c);
  double large = (mean + std::copysign(radius, mean)) * scale;
  if (!std::isfinite(large)) {
    major = (mean + radius) * scale;
    minor = (mean - radius) * scale;
    return;
  }
  double hi = std::fabs(xx) >= std::fabs(yy) ? xx : yy, lo = std::fabs(xx) >= std::fabs(yy) ? yy : xx;
  double small = (hi / large) * lo - (xy / large) * xy;
  major = std::max(large, small);
  minor = std::min(large, small);
}

}  // namespace

extern "C" {

// 24x24 local CQUAD4 stiffness on the default SOL101 path for a flat element
// (FEMKernels.jl:2874-4166 _stiffness_quad4_core! with kernel_mode="macneal",
// kernel_planar=true, membrane_incomp=true, bending_incomp=true,
// section_kinematic enrichment, lumped reference drilling, flat => warp map
// skipped).  lc: 4x2 local coordinates (col-major).  Returns 0 or an error code.
int or_q4_local(const double* lc, const double* Cm, const double* Cb,
                const double* Cs, double h, double k6rot, double drill_scale,
                double* Ke) {
  std::memset(Ke, 0, sizeof(double) * 576);
  double K_ab[96] = {0}, K_bb[16] = {0}, K_abb[96] = {0}, K_bbb[16] = {0};
  double K_abs[96] = {0}, K_bbs[16] = {0};
  const double dNr_c[4] = {-0.25, 0.25, 0.25, -0.25};
  const double dNs_c[4] = {-0.25, -0.25, 0.25, 0.25};
  double J11c, J12c, J21c, J22c;
  jac_quad(lc, dNr_c, dNs_c, J11c, J12c, J21c, J22c);
  double detJc = J11c * J22c - J12c * J21c;
  double abs_detJc = std::fabs(detJc);
  double idc = 1.0 / detJc;
  double iJ11c = J22c * idc, iJ12c = -J12c * idc, iJ21c = -J21c * idc, iJ22c = J11c * idc;
  double cmmax = 0;
  for (int i = 0; i < 9; ++i) cmmax = std::max(cmmax, std::fabs(Cm[i]));
  const double* shape = cmmax > 0 ? Cm : Cb;   // FEMKernels.jl:3555
  const double pt = 1.0 / std::sqrt(3.0);
  const double gr[4] = {-pt, pt, pt, -pt}, gs[4] = {-pt, -pt, pt, pt};
  for (int g = 0; g < 4; ++g) {
    double r = gr[g], s = gs[g];
    double dNr[4], dNs[4];
    shape_derivs_quad(r, s, dNr, dNs);
    double J11, J12, J21, J22;
    jac_quad(lc, dNr, dNs, J11, J12, J21, J22);
    double detJ = J11 * J22 - J12 * J21;
    if (!jac_ok(detJ, J11, J12, J21, J22)) return 1;
    double w = std::fabs(detJ);
    double id = 1.0 / detJ;
    double iJ11 = J22 * id, iJ12 = -J12 * id, iJ21 = -J21 * id, iJ22 = J11 * id;
    double Bm[72] = {0}, Bb[72] = {0};
    for (int k = 0; k < 4; ++k) {
      double dx = iJ11 * dNr[k] + iJ12 * dNs[k];
      double dy = iJ21 * dNr[k] + iJ22 * dNs[k];
      int c = 6 * k;
      Bm[0 + 3 * (c + 0)] = dx; Bm[1 + 3 * (c + 1)] = dy;
      Bm[2 + 3 * (c + 0)] = dy; Bm[2 + 3 * (c + 1)] = dx;
      Bb[0 + 3 * (c + 4)] = dx; Bb[1 + 3 * (c + 3)] = -dy;
      Bb[2 + 3 * (c + 4)] = dy; Bb[2 + 3 * (c + 3)] = -dx;
    }
    // membrane incompatible modes, patch-consistent Jacobian (FEMKernels.jl:1847-1895)
    double ratio = (iJ11 * iJ22 - iJ12 * iJ21) / (iJ11c * iJ22c - iJ12c * iJ21c);
    double m11 = ratio * iJ11c, m12 = ratio * iJ12c, m21 = ratio * iJ21c, m22 = ratio * iJ22c;
    double Bi[12] = {0};
    double p1x = m11 * (-2 * r), p1y = m21 * (-2 * r), p2x = m12 * (-2 * s), p2y = m22 * (-2 * s);
    Bi[0 + 3 * 0] = p1x; Bi[2 + 3 * 0] = p1y; Bi[1 + 3 * 1] = p1y; Bi[2 + 3 * 1] = p1x;
    Bi[0 + 3 * 2] = p2x; Bi[2 + 3 * 2] = p2y; Bi[1 + 3 * 3] = p2y; Bi[2 + 3 * 3] = p2x;
    // bending incompatible modes, qm6 Jacobian (FEMKernels.jl:3474-3488)
    double gq = detJc / detJ;
    double b1x = (iJ11c * (-2 * r)) * gq, b1y = (iJ21c * (-2 * r)) * gq;
    double b2x = (iJ12c * (-2 * s)) * gq, b2y = (iJ22c * (-2 * s)) * gq;
    double Bib[12] = {0};
    Bib[1 + 3 * 0] = -b1y; Bib[1 + 3 * 1] = -b2y;
    Bib[0 + 3 * 2] = b1x;  Bib[0 + 3 * 3] = b2x;
    Bib[2 + 3 * 0] = -b1x; Bib[2 + 3 * 1] = -b2x;
    Bib[2 + 3 * 2] = b1y;  Bib[2 + 3 * 3] = b2y;
    double t324[72], t34[12];
    mul(t324, 3, 24, Cm, 3, Bm);  mul_At_add(Ke, 24, 24, Bm, 3, t324, w);
    mul(t324, 3, 24, Cb, 3, Bb);  mul_At_add(Ke, 24, 24, Bb, 3, t324, w);
    mul(t34, 3, 4, Cm, 3, Bi);
    mul_At_add(K_ab, 24, 4, Bm, 3, t34, w);
    mul_At_add(K_bb, 4, 4, Bi, 3, t34, w);
    mul(t34, 3, 4, shape, 3, Bib);
    mul_At_add(K_abs, 24, 4, Bb, 3, t34, w);
    mul_At_add(K_bbs, 4, 4, Bib, 3, t34, w);
    mul(t34, 3, 4, Cb, 3, Bib);
    mul_At_add(K_abb, 24, 4, Bb, 3, t34, w);
    mul_At_add(K_bbb, 4, 4, Bib, 3, t34, w);
  }
  int st = macneal_shear(lc, Cb, Cs, h, Ke);
  if (st) return 10 + st;
  // lumped reference drilling (FEMKernels.jl:3749-3818)
  double A_drill = 4.0 * abs_detJc;
  double alphaL = drill_scale * (k6rot * 1e-6) * Cm[8] * A_drill;
  if (alphaL != 0.0) {
    const double cr[4] = {-1, 1, 1, -1}, cs[4] = {-1, -1, 1, 1};
    for (int i = 0; i < 4; ++i) {
      double dNr[4], dNs[4];
      shape_derivs_quad(cr[i], cs[i], dNr, dNs);
      double J11, J12, J21, J22;
      jac_quad(lc, dNr, dNs, J11, J12, J21, J22);
      double detJ = J11 * J22 - J12 * J21;
      if (!jac_ok(detJ, J11, J12, J21, J22)) return 1;
      double id = 1.0 / detJ;
      double iJ11 = J22 * id, iJ12 = -J12 * id, iJ21 = -J21 * id, iJ22 = J11 * id;
      double Bd[24] = {0};
      for (int k = 0; k < 4; ++k) {
        double dx = iJ11 * dNr[k] + iJ12 * dNs[k];
        double dy = iJ21 * dNr[k] + iJ22 * dNs[k];
        Bd[6 * k + 0] = 0.5 * dy; Bd[6 * k + 1] = -0.5 * dx;
      }
      Bd[6 * i + 5] = 1.0;
      double wc = std::fabs(detJ) / std::max(abs_detJc, 1e-30);
      mul_At_add(Ke, 24, 24, Bd, 1, Bd, alphaL * wc);
    }
  }
  // section-kinematic enrichment (FEMKernels.jl:1989-2024)
  double Pm[96] = {0}, Pb[96] = {0};  // 4 x 24
  double mx = 0;
  for (int i = 0; i < 16; ++i) mx = std::max(mx, std::fabs(K_bb[i]));
  if (mx > 0) {
    double C[16];
    if (!inv_small(K_bb, 4, C)) return 20;
    for (int j = 0; j < 24; ++j)
      for (int i = 0; i < 4; ++i)
        for (int k = 0; k < 4; ++k) Pm[i + 4 * j] -= C[i + 4 * k] * K_ab[j + 24 * k];
  }
  mx = 0;
  for (int i = 0; i < 16; ++i) mx = std::max(mx, std::fabs(K_bbs[i]));
  if (mx > 0) {
    double C[16];
    if (!inv_small(K_bbs, 4, C)) return 21;
    for (int j = 0; j < 24; ++j)
      for (int i = 0; i < 4; ++i)
        for (int k = 0; k < 4; ++k) Pb[i + 4 * j] -= C[i + 4 * k] * K_abs[j + 24 * k];
  }
  for (int j = 0; j < 24; ++j)
    for (int i = 0; i < 24; ++i) {
      double v = 0;
      for (int k = 0; k < 4; ++k) {
        v += K_ab[i + 24 * k] * Pm[k + 4 * j] + Pm[k + 4 * i] * K_ab[j + 24 * k] +
             K_abb[i + 24 * k] * Pb[k + 4 * j] + Pb[k + 4 * i] * K_abb[j + 24 * k];
        for (int l = 0; l < 4; ++l)
          v += Pm[k + 4 * i] * K_bb[k + 4 * l] * Pm[l + 4 * j] +
               Pb[k + 4 * i] * K_bbb[k + 4 * l] * Pb[l + 4 * j];
      }
      Ke[i + 24 * j] += v;
    }
  return 0;
}

// Element frame + local coordinates + PSHELL material-axis rotation + the
// 24x24 transform to node DOF frames and the positional emit.
//   frame:    helpers.jl:1422-1481 shell_element_frame_quad4 (mode :diag)
//   lc:       assembly.jl:3672-3677
//   beta:     assembly.jl:4392-4420 (PSHELL, macneal) with helpers.jl:1749
//   rotation: assembly.jl:2440 _rotate_constitutive_3x3!
//   emit:     assembly.jl:359-440 _quad4_transform_emit!
// xyz: 4 nodes x 3 (row per node, i.e. xyz[3*k + a]); nodeR: 4 x 9 col-major
// 3x3 blocks; sect: JFG_Q4_SECT_STRIDE record.  Ke_global: 24x24 col-major.
int or_q4_element(const double* xyz, const double* nodeR, const double* sect,
                  double* Ke_global) {
  double p[4][3];
  for (int k = 0; k < 4; ++k)
    for (int a = 0; a < 3; ++a) p[k][a] = xyz[3 * k + a];
  auto sub = [](const double* a, const double* b, double* o) {
    o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2];
  };
  auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  double v1[3], v2[3], v3[3], lc[8], zmax, xmax;
  q4_frame(xyz, v1, v2, v3, lc, zmax, xmax);
  // Only flat elements: the finite-warp multiplier is then skipped by the
  // reference itself (FEMKernels.jl:1100-1102).
  if (!(zmax <= 1e-12 * std::max(xmax, 1e-30))) return 100;
  if (sect[25] != 0.0) return 101;
  double Cm[9], Cb[9], Cs[4];
  std::memcpy(Cm, sect, sizeof Cm);
  std::memcpy(Cb, sect + 9, sizeof Cb);
  std::memcpy(Cs, sect + 18, sizeof Cs);
  double h = sect[22], k6rot = sect[24];
  // PSHELL material frame angle (projected edge G1-G2 measured from v1)
  double e12[3];
  sub(p[1], p[0], e12);
  double de = dot(e12, v3);
  double e12p[3] = {e12[0] - de * v3[0], e12[1] - de * v3[1], e12[2] - de * v3[2]};
  double l2 = dot(e12p, e12p);
  double beta = 0.0;
  if (l2 > 1e-24) {
    double lx = std::sqrt(l2);
    double xm[3] = {e12p[0] / lx, e12p[1] / lx, e12p[2] / lx};
    beta = std::atan2(dot(xm, v2), dot(xm, v1));
  }
  if (std::fabs(beta) > 1e-10) {
    double cb = std::cos(beta), sb = std::sin(beta);
    double c2 = cb * cb, s2 = sb * sb, cs = cb * sb;
    double T[9] = {c2, s2, -2 * cs, s2, c2, 2 * cs, cs, -cs, c2 - s2};  // col-major T
    for (double* C : {Cm, Cb}) {
      double t[9], o[9];
      mul(t, 3, 3, C, 3, T);
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
          double s = 0;
          for (int k = 0; k < 3; ++k) s += T[k + 3 * i] * t[k + 3 * j];
          o[i + 3 * j] = s;
        }
      std::memcpy(C, o, sizeof o);
    }
    double a11 = Cs[0], a12 = Cs[2], a22 = Cs[3];
    Cs[0] = cb * cb * a11 - 2 * cb * sb * a12 + sb * sb * a22;
    Cs[2] = cb * sb * a11 + (cb * cb - sb * sb) * a12 - cb * sb * a22;
    Cs[1] = Cs[2];
    Cs[3] = sb * sb * a11 + 2 * cb * sb * a12 + cb * cb * a22;
  }
  double Ke[576];
  int st = or_q4_local(lc, Cm, Cb, Cs, h, k6rot, 1.0, Ke);
  if (st) return st;
  // T = blockdiag(Rel * node_R) for translations and rotations of each node
  double T[576] = {0};
  const double Rel[3][3] = {{v1[0], v1[1], v1[2]}, {v2[0], v2[1], v2[2]}, {v3[0], v3[1], v3[2]}};
  for (int k = 0; k < 4; ++k) {
    const double* R = nodeR + 9 * k;
    for (int rr = 0; rr < 3; ++rr)
      for (int cc = 0; cc < 3; ++cc) {
        double v = Rel[rr][0] * R[0 + 3 * cc] + Rel[rr][1] * R[1 + 3 * cc] + Rel[rr][2] * R[2 + 3 * cc];
        T[(6 * k + rr) + 24 * (6 * k + cc)] = v;
        T[(6 * k + 3 + rr) + 24 * (6 * k + 3 + cc)] = v;
      }
  }
  double tmp[576] = {0};
  for (int jj = 0; jj < 24; ++jj)
    for (int ll = 0; ll < 24; ++ll) {
      double v = T[ll + 24 * jj];
      if (v != 0.0)
        for (int ii = 0; ii < 24; ++ii) tmp[ii + 24 * jj] += Ke[ii + 24 * ll] * v;
    }
  std::memset(Ke_global, 0, sizeof(double) * 576);
  for (int jj = 0; jj < 24; ++jj)
    for (int ll = 0; ll < 24; ++ll) {
      double v = tmp[ll + 24 * jj];
      if (v != 0.0)
        for (int ii = 0; ii < 24; ++ii) Ke_global[ii + 24 * jj] += T[ll + 24 * ii] * v;
    }
  return 0;
}

// CQUAD4 stress recovery on the default isotropic PSHELL path
// (recover_shell_stresses!, stress_recovery.jl:505-1237, n == 4: no offset,
// no SNORM, no thermal load, flat so the warp map is the identity).
//   element displacements: (Rel * node_R) u per node            (:774-781)
//   centre fields: stress_strain_quad4's default branch, FEMKernels.jl:6794-6978
//     (Wilson membrane modes condensed with Cm = h D, patch-consistent
//     Jacobian :1847-1895; area-weighted Gauss-point means of eps and kappa)
//   Q: the area-mean MacNeal shear resultant, FEMKernels.jl:6623-6646, which
//     replaces the centre shear when _pshell_macneal_mean_shear_data applies
//     (stress_recovery.jl:248-292, :917-927)
//   fibres -T/2, +T/2; strains: membrane (tag 0) and -kappa (tag -1)
//     (stress_recovery.jl:1118-1123, :1239-1255)
// xyz: 4 x 3 node major; nodeR: 4 x 9; E, nu: MAT1 of MID1; h = T; br =
// BEND_RATIO; sect: the element's 26-double section record (its Cs gives the
// shear law); u: the 24 node-frame displacements.  out (31 doubles):
//   0-7   fx fy fxy mx my mxy qx qy
//   8-13  fibre z1: sx sy txy von_mises major minor;  14-19  fibre z2
//   20-24 membrane strain ex ey gxy major minor;  25-29 -kappa, same layout
//   30    major principal stress at z1 (compute_principal_2d, FEMKernels.jl:6509)
int or_q4_stress(const double* xyz, const double* nodeR, double E, double nu, double h, double br,
                 const double* sect, const double* u, double* out) {
  double v1[3], v2[3], v3[3], lc[8], zmax, xmax;
  q4_frame(xyz, v1, v2, v3, lc, zmax, xmax);
  if (!(zmax <= 1e-12 * std::max(xmax, 1e-30))) return 100;
  const double Rel[3][3] = {{v1[0], v1[1], v1[2]}, {v2[0], v2[1], v2[2]}, {v3[0], v3[1], v3[2]}};
  double ue[24];
  for (int k = 0; k < 4; ++k) {
    const double* R = nodeR + 9 * k;
    double Tn[3][3];
    for (int rr = 0; rr < 3; ++rr)
      for (int cc = 0; cc < 3; ++cc)
        Tn[rr][cc] = Rel[rr][0] * R[0 + 3 * cc] + Rel[rr][1] * R[1 + 3 * cc] + Rel[rr][2] * R[2 + 3 * cc];
    for (int rr = 0; rr < 3; ++rr) {
      double a = 0, b = 0;
      for (int cc = 0; cc < 3; ++cc) {
        a += Tn[rr][cc] * u[6 * k + cc];
        b += Tn[rr][cc] * u[6 * k + 3 + cc];
      }
      ue[6 * k + rr] = a;
      ue[6 * k + 3 + rr] = b;
    }
  }
  const double cmem = E / (1 - nu * nu);
  const double D[9] = {cmem, cmem * nu, 0, cmem * nu, cmem, 0, 0, 0, cmem * (1 - nu) / 2};  // col-major
  double Cm[9];
  for (int i = 0; i < 9; ++i) Cm[i] = D[i] * h;
  const double dNr_c[4] = {-0.25, 0.25, 0.25, -0.25};
  const double dNs_c[4] = {-0.25, -0.25, 0.25, 0.25};
  double J11c, J12c, J21c, J22c;
  jac_quad(lc, dNr_c, dNs_c, J11c, J12c, J21c, J22c);
  double detJc = J11c * J22c - J12c * J21c;
  double idc = 1.0 / detJc;
  double iJ11c = J22c * idc, iJ12c = -J12c * idc, iJ21c = -J21c * idc, iJ22c = J11c * idc;
  const double pt = 1.0 / std::sqrt(3.0);
  const double gr[4] = {-pt, pt, pt, -pt}, gs[4] = {-pt, -pt, pt, pt};
  double Bm[4][72], Bb[4][72], Bi[4][12], wgt[4];
  double K_ab[96] = {0}, K_bb[16] = {0};
  for (int g = 0; g < 4; ++g) {
    double r = gr[g], s = gs[g];
    double dNr[4], dNs[4];
    shape_derivs_quad(r, s, dNr, dNs);
    double J11, J12, J21, J22;
    jac_quad(lc, dNr, dNs, J11, J12, J21, J22);
    double detJ = J11 * J22 - J12 * J21;
    if (!jac_ok(detJ, J11, J12, J21, J22)) return 1;
    wgt[g] = std::fabs(detJ);
    double id = 1.0 / detJ;
    double iJ11 = J22 * id, iJ12 = -J12 * id, iJ21 = -J21 * id, iJ22 = J11 * id;
    std::memset(Bm[g], 0, sizeof Bm[g]);
    std::memset(Bb[g], 0, sizeof Bb[g]);
    for (int k = 0; k < 4; ++k) {
      double dx = iJ11 * dNr[k] + iJ12 * dNs[k];
      double dy = iJ21 * dNr[k] + iJ22 * dNs[k];
      int c = 6 * k;
      Bm[g][0 + 3 * (c + 0)] = dx; Bm[g][1 + 3 * (c + 1)] = dy;
      Bm[g][2 + 3 * (c + 0)] = dy; Bm[g][2 + 3 * (c + 1)] = dx;
      Bb[g][0 + 3 * (c + 4)] = dx; Bb[g][1 + 3 * (c + 3)] = -dy;
      Bb[g][2 + 3 * (c + 4)] = dy; Bb[g][2 + 3 * (c + 3)] = -dx;
    }
    double ratio = (iJ11 * iJ22 - iJ12 * iJ21) / (iJ11c * iJ22c - iJ12c * iJ21c);
    double m11 = ratio * iJ11c, m12 = ratio * iJ12c, m21 = ratio * iJ21c, m22 = ratio * iJ22c;
    double p1x = m11 * (-2 * r), p1y = m21 * (-2 * r), p2x = m12 * (-2 * s), p2y = m22 * (-2 * s);
    std::memset(Bi[g], 0, sizeof Bi[g]);
    Bi[g][0 + 3 * 0] = p1x; Bi[g][2 + 3 * 0] = p1y; Bi[g][1 + 3 * 1] = p1y; Bi[g][2 + 3 * 1] = p1x;
    Bi[g][0 + 3 * 2] = p2x; Bi[g][2 + 3 * 2] = p2y; Bi[g][1 + 3 * 3] = p2y; Bi[g][2 + 3 * 3] = p2x;
    double t34[12];
    mul(t34, 3, 4, Cm, 3, Bi[g]);
    mul_At_add(K_ab, 24, 4, Bm[g], 3, t34, wgt[g]);
    mul_At_add(K_bb, 4, 4, Bi[g], 3, t34, wgt[g]);
  }
  // alpha = -(K_bb \ (K_ab' u))
  double rhs[4];
  for (int j = 0; j < 4; ++j) {
    double acc = 0;
    for (int i = 0; i < 24; ++i) acc += K_ab[i + 24 * j] * ue[i];
    rhs[j] = acc;
  }
  double Kbi[16];
  if (!inv_small(K_bb, 4, Kbi)) return 2;
  double alpha[4];
  for (int i = 0; i < 4; ++i) {
    double acc = 0;
    for (int j = 0; j < 4; ++j) acc += Kbi[i + 4 * j] * rhs[j];
    alpha[i] = -acc;
  }
  double eps[3] = {0, 0, 0}, kap[3] = {0, 0, 0}, area = 0;
  for (int g = 0; g < 4; ++g) {
    for (int a = 0; a < 3; ++a) {
      double e = 0, k = 0;
      for (int i = 0; i < 24; ++i) {
        e += Bm[g][a + 3 * i] * ue[i];
        k += Bb[g][a + 3 * i] * ue[i];
      }
      for (int j = 0; j < 4; ++j) e += Bi[g][a + 3 * j] * alpha[j];
      eps[a] += e * wgt[g];
      kap[a] += k * wgt[g];
    }
    area += wgt[g];
  }
  for (int a = 0; a < 3; ++a) { eps[a] /= area; kap[a] /= area; }
  double N[3], M[3];
  for (int a = 0; a < 3; ++a) {
    double n = 0, m = 0;
    for (int b = 0; b < 3; ++b) { n += Cm[a + 3 * b] * eps[b]; m += D[a + 3 * b] * kap[b]; }
    N[a] = n;
    M[a] = -br * m * (h * h * h / 12.0);
  }
  // area-mean MacNeal shear resultant from the plate operator K_plate
  double q[2] = {0, 0};
  if (br > 1e-12) {
    double Cb[9];
    for (int i = 0; i < 9; ++i) Cb[i] = br * (h * h * h) / 12 * D[i];
    double Kscratch[576] = {0}, KP[144] = {0};
    int st = macneal_shear(lc, Cb, sect + 18, h, Kscratch, KP);
    if (st) return 10 + st;
    double qx = 0, qy = 0;
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j)
        for (int c = 0; c < 3; ++c) {
          qx += KP[(3 * i + 2) + 12 * (3 * j + c)] * ue[6 * j + c + 2];
          qy -= KP[(3 * i + 1) + 12 * (3 * j + c)] * ue[6 * j + c + 2];
        }
    double a4 = 4 * std::fabs(detJc);
    q[0] = qx / a4;
    q[1] = qy / a4;
  }
  double ez1[3], ez2[3], sz1[3], sz2[3];
  for (int a = 0; a < 3; ++a) {
    ez1[a] = eps[a] + (-h / 2.0) * kap[a];
    ez2[a] = eps[a] + (h / 2.0) * kap[a];
  }
  for (int a = 0; a < 3; ++a) {
    double x = 0, y = 0;
    for (int b = 0; b < 3; ++b) { x += D[a + 3 * b] * ez1[b]; y += D[a + 3 * b] * ez2[b]; }
    sz1[a] = x;
    sz2[a] = y;
  }
  for (int a = 0; a < 3; ++a) { out[a] = N[a]; out[3 + a] = M[a]; }
  out[6] = q[0];
  out[7] = q[1];
  auto stress_row = [&](const double* sg, double* o) {
    o[0] = sg[0]; o[1] = sg[1]; o[2] = sg[2];
    o[3] = std::sqrt(sg[0] * sg[0] - sg[0] * sg[1] + sg[1] * sg[1] + 3 * sg[2] * sg[2]);
    principal_2d(sg[0], sg[1], sg[2], o[4], o[5]);
  };
  stress_row(sz1, out + 8);
  stress_row(sz2, out + 14);
  double em[3], kn[3];
  for (int a = 0; a < 3; ++a) {
    em[a] = (ez1[a] + ez2[a]) / 2.0;
    kn[a] = (ez1[a] - ez2[a]) / h;
  }
  auto strain_row = [&](const double* e, double* o) {
    o[0] = e[0]; o[1] = e[1]; o[2] = e[2];
    principal_2d(e[0], e[1], e[2] / 2, o[3], o[4]);
  };
  strain_row(em, out + 20);
  strain_row(kn, out + 25);
  double savg = (sz1[0] + sz1[1]) / 2.0;
  out[30] = savg + std::sqrt(((sz1[0] - sz1[1]) / 2.0) * ((sz1[0] - sz1[1]) / 2.0) + sz1[2] * sz1[2]);
  return 0;
}

// ---------------------------------------------------------------------------
// CQUAD8 (src/quad8_shell.jl:24-204, shape_quad8 FEMKernels.jl:11583-11600)
static void shape_quad8(double r, double s, double N[8], double dr[8], double ds[8]) {
  const double rc[4] = {-1, 1, 1, -1}, sc[4] = {-1, -1, 1, 1};
  for (int k = 0; k < 4; ++k) {
    double a = 1 + rc[k] * r, b = 1 + sc[k] * s, c = rc[k] * r + sc[k] * s - 1;
    N[k] = 0.25 * a * b * c;
    dr[k] = 0.25 * rc[k] * b * (c + a);
    ds[k] = 0.25 * sc[k] * a * (c + b);
  }
  N[4] = 0.5 * (1 - r * r) * (1 - s); dr[4] = -r * (1 - s);     ds[4] = -0.5 * (1 - r * r);
  N[5] = 0.5 * (1 + r) * (1 - s * s); dr[5] = 0.5 * (1 - s * s); ds[5] = -s * (1 + r);
  N[6] = 0.5 * (1 - r * r) * (1 + s); dr[6] = -r * (1 + s);     ds[6] = 0.5 * (1 - r * r);
  N[7] = 0.5 * (1 - r) * (1 - s * s); dr[7] = -0.5 * (1 - s * s); ds[7] = -s * (1 - r);
}
static void q8_point(const double* xy /*8x2 col-major*/, double r, double s, double N[8],
                     double dx[8], double dy[8], double& detJ, double jj[4]) {
  double dr[8], ds[8];
  shape_quad8(r, s, N, dr, ds);
  double j11 = 0, j12 = 0, j21 = 0, j22 = 0;
  for (int k = 0; k < 8; ++k) {
    j11 += dr[k] * xy[k]; j12 += dr[k] * xy[k + 8];
    j21 += ds[k] * xy[k]; j22 += ds[k] * xy[k + 8];
  }
  detJ = j11 * j22 - j12 * j21;
  for (int k = 0; k < 8; ++k) {
    dx[k] = (j22 * dr[k] - j12 * ds[k]) / detJ;
    dy[k] = (-j21 * dr[k] + j11 * ds[k]) / detJ;
  }
  jj[0] = j11; jj[1] = j12; jj[2] = j21; jj[3] = j22;
}
static double norm3(const double* a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

// quad8_shell.jl:34-46
int or_q8_parallelogram(const double* xyz /*8 rows x 3*/) {
  auto P = [&](int k, int a) { return xyz[3 * k + a]; };
  double d21[3], d41[3];
  for (int a = 0; a < 3; ++a) { d21[a] = P(1, a) - P(0, a); d41[a] = P(3, a) - P(0, a); }
  double scale = std::max(norm3(d21), norm3(d41));
  if (!(scale > 0)) return 0;
  double lim = 1e-6 * scale;
  double t[3];
  for (int a = 0; a < 3; ++a) t[a] = P(0, a) + P(2, a) - P(1, a) - P(3, a);
  if (norm3(t) > lim) return 0;
  const int mab[4][3] = {{4, 0, 1}, {5, 1, 2}, {6, 2, 3}, {7, 3, 0}};
  for (auto& m : mab) {
    for (int a = 0; a < 3; ++a) t[a] = P(m[0], a) - (P(m[1], a) + P(m[2], a)) / 2;
    if (norm3(t) > lim) return 0;
  }
  double n[3] = {d21[1] * d41[2] - d21[2] * d41[1], d21[2] * d41[0] - d21[0] * d41[2],
                 d21[0] * d41[1] - d21[1] * d41[0]};
  return norm3(n) > 1e-12 * scale * scale ? 1 : 0;
}

// quad8_shell.jl:96-204 stiffness_quad8_shell, then T'KT with node_R
// (assembly.jl:5893-5915).  sect: JFG_Q8_SECT_STRIDE record.
int or_q8_element(const double* xyz, const double* nodeR, const double* sect,
                  double* Ke_global) {
  if (!or_q8_parallelogram(xyz)) return 100;
  auto P = [&](int k, int a) { return xyz[3 * k + a]; };
  double gxi[3], geta[3], ez[3], a[3], b[3], ex[3], ey[3], cen[3];
  for (int q = 0; q < 3; ++q) {
    gxi[q] = (P(1, q) + P(2, q) - P(0, q) - P(3, q)) / 4;
    geta[q] = (P(2, q) + P(3, q) - P(0, q) - P(1, q)) / 4;
    cen[q] = (P(0, q) + P(1, q) + P(2, q) + P(3, q)) / 4;
  }
  ez[0] = gxi[1] * geta[2] - gxi[2] * geta[1];
  ez[1] = gxi[2] * geta[0] - gxi[0] * geta[2];
  ez[2] = gxi[0] * geta[1] - gxi[1] * geta[0];
  double l = norm3(ez);
  for (int q = 0; q < 3; ++q) ez[q] /= l;
  double lg = norm3(gxi), le = norm3(geta);
  for (int q = 0; q < 3; ++q) a[q] = gxi[q] / lg + geta[q] / le;
  l = norm3(a);
  for (int q = 0; q < 3; ++q) a[q] /= l;
  b[0] = ez[1] * a[2] - ez[2] * a[1];
  b[1] = ez[2] * a[0] - ez[0] * a[2];
  b[2] = ez[0] * a[1] - ez[1] * a[0];
  for (int q = 0; q < 3; ++q) { ex[q] = (a[q] - b[q]) / std::sqrt(2.0); ey[q] = (a[q] + b[q]) / std::sqrt(2.0); }
  double R[9] = {ex[0], ex[1], ex[2], ey[0], ey[1], ey[2], ez[0], ez[1], ez[2]};  // columns
  double xy[16];
  for (int k = 0; k < 8; ++k) {
    double d[3] = {P(k, 0) - cen[0], P(k, 1) - cen[1], P(k, 2) - cen[2]};
    xy[k] = d[0] * ex[0] + d[1] * ex[1] + d[2] * ex[2];
    xy[k + 8] = d[0] * ey[0] + d[1] * ey[1] + d[2] * ey[2];
  }
  std::vector<double> Kl(48 * 48, 0.0);
  const double g2p[2] = {-1 / std::sqrt(3.0), 1 / std::sqrt(3.0)}, g2w[2] = {1.0, 1.0};
  const double g3p[3] = {-std::sqrt(0.6), 0.0, std::sqrt(0.6)}, g3w[3] = {5.0 / 9, 8.0 / 9, 5.0 / 9};
  bool hasA = sect[20] != 0.0, hasD = sect[21] != 0.0;
  const double* A = sect;
  const double* Dm = sect + 9;
  double shear = sect[18], dref = sect[19];
  double N[8], dx[8], dy[8], detJ, jj[4];
  if (hasA) {
    for (double r : g2p)
      for (double s : g2p) {
        q8_point(xy, r, s, N, dx, dy, detJ, jj);
        std::vector<double> B(3 * 48, 0.0), t(3 * 48);
        for (int k = 0; k < 8; ++k) {
          int c = 6 * k;
          B[0 + 3 * (c + 0)] = dx[k]; B[1 + 3 * (c + 1)] = dy[k];
          B[2 + 3 * (c + 0)] = dy[k]; B[2 + 3 * (c + 1)] = dx[k];
        }
        mul(t.data(), 3, 48, A, 3, B.data());
        mul_At_add(Kl.data(), 48, 48, B.data(), 3, t.data(), detJ);
      }
    for (int row = 1; row <= 2; ++row) {
      double modulus = row == 1 ? A[0] : A[4];
      for (int pass = 0; pass < 2; ++pass) {
        const double *pr, *wr, *ps, *ws;
        int npr, nps;
        double sign = pass == 0 ? 1.0 : -1.0;
        if (row == 1) {
          pr = g2p; wr = g2w; npr = 2;
          if (pass == 0) { ps = g3p; ws = g3w; nps = 3; } else { ps = g2p; ws = g2w; nps = 2; }
        } else {
          if (pass == 0) { pr = g3p; wr = g3w; npr = 3; } else { pr = g2p; wr = g2w; npr = 2; }
          ps = g2p; ws = g2w; nps = 2;
        }
        for (int i = 0; i < npr; ++i)
          for (int j = 0; j < nps; ++j) {
            q8_point(xy, pr[i], ps[j], N, dx, dy, detJ, jj);
            double bv[48] = {0};
            for (int k = 0; k < 8; ++k) bv[6 * k + row - 1] = row == 1 ? dx[k] : dy[k];
            double f = 0.25 * sign * wr[i] * ws[j] * detJ * modulus;
            for (int q = 0; q < 48; ++q)
              for (int p = 0; p < 48; ++p) Kl[p + 48 * q] += f * (bv[p] * bv[q]);
          }
      }
    }
  }
  if (hasD) {
    double Dx[9] = {Dm[0], Dm[3], 0.0, Dm[3], Dm[4], 0.0, 0.0, 0.0, 4 * Dm[8]};
    // NOTE: Dx = [D11 D12 0; D12 D22 0; 0 0 4 D33] (quad8_shell.jl:139), column-major
    Dx[1] = Dm[3]; Dx[3] = Dm[3];
    auto curv = [&](double* B) {
      for (int i = 0; i < 3 * 48; ++i) B[i] = 0.0;
      for (int k = 0; k < 8; ++k) {
        int c = 6 * k;
        B[0 + 3 * (c + 4)] = dx[k]; B[1 + 3 * (c + 3)] = -dy[k];
        B[2 + 3 * (c + 4)] = dy[k]; B[2 + 3 * (c + 3)] = -dx[k];
      }
    };
    std::vector<double> B(3 * 48), t(3 * 48);
    for (double r : g2p)
      for (double s : g2p) {
        q8_point(xy, r, s, N, dx, dy, detJ, jj);
        curv(B.data());
        mul(t.data(), 3, 48, Dm, 3, B.data());
        std::vector<double> K1(48 * 48, 0.0), K2(48 * 48, 0.0);
        mul_At_add(K1.data(), 48, 48, B.data(), 3, t.data(), 1.0);
        mul(t.data(), 3, 48, Dx, 3, B.data());
        mul_At_add(K2.data(), 48, 48, B.data(), 3, t.data(), 1.0);
        for (int i = 0; i < 48 * 48; ++i) Kl[i] += detJ * K1[i] - (2 * detJ) * K2[i];
      }
    for (int pass = 0; pass < 2; ++pass) {
      const double* pr = pass == 0 ? g2p : g3p;
      const double* wr = pass == 0 ? g2w : g3w;
      const double* ps = pass == 0 ? g3p : g2p;
      const double* ws = pass == 0 ? g3w : g2w;
      int npr = pass == 0 ? 2 : 3, nps = pass == 0 ? 3 : 2;
      for (int i = 0; i < npr; ++i)
        for (int j = 0; j < nps; ++j) {
          q8_point(xy, pr[i], ps[j], N, dx, dy, detJ, jj);
          curv(B.data());
          mul(t.data(), 3, 48, Dx, 3, B.data());
          mul_At_add(Kl.data(), 48, 48, B.data(), 3, t.data(), wr[i] * ws[j] * detJ);
        }
    }
    if (!(dref > 0)) return 101;
    std::vector<double> Bs(8 * 48, 0.0);
    double detJ0 = 0, jac[4] = {0, 0, 0, 0};
    int sample = 0;
    for (double r : g2p)
      for (double s : g2p) {
        q8_point(xy, r, s, N, dx, dy, detJ, jj);
        detJ0 = detJ;
        for (int q = 0; q < 4; ++q) jac[q] = jj[q];
        for (int k = 0; k < 8; ++k) {
          int c = 6 * k;
          Bs[(2 * sample) + 8 * (c + 2)] = dx[k];
          Bs[(2 * sample) + 8 * (c + 4)] = N[k];
          Bs[(2 * sample + 1) + 8 * (c + 2)] = dy[k];
          Bs[(2 * sample + 1) + 8 * (c + 3)] = -N[k];
        }
        ++sample;
      }
    double rx = detJ0 / (jac[0] * jac[0]), ry = detJ0 / (jac[3] * jac[3]);
    const double pat[4][4] = {{1, 1, 1, 1}, {-1, -1, 1, 1}, {-1, 1, -1, 1}, {1, -1, -1, 1}};
    double sx[4] = {12 * rx + 1200 * ry, 9.6 * rx, 12 * rx + 400 * ry, 12 * rx + 120 * ry};
    double sy[4] = {12 * ry + 1200 * rx, 12 * ry + 400 * rx, 9.6 * ry, 12 * ry + 120 * rx};
    double F[64] = {0};
    double base = std::isfinite(shear) ? 1 / (shear * detJ0) : 0.0;
    for (int q = 0; q < 8; ++q) F[q + 8 * q] = base;
    for (int comp = 1; comp <= 2; ++comp)
      for (int k = 0; k < 4; ++k) {
        double stiff = comp == 1 ? sx[k] : sy[k];
        double f = 1 / (stiff * dref) / 4;
        for (int aa = 0; aa < 4; ++aa)
          for (int cc = 0; cc < 4; ++cc)
            F[(2 * aa + comp - 1) + 8 * (2 * cc + comp - 1)] += f * pat[k][aa] * pat[k][cc];
      }
    double Fi[64];
    if (!inv_small(F, 8, Fi)) return 102;
    std::vector<double> X(8 * 48);
    mul(X.data(), 8, 48, Fi, 8, Bs.data());
    mul_At_add(Kl.data(), 48, 48, Bs.data(), 8, X.data(), 1.0);
  }
  // local = R' * frame for both blocks; K = T' Kl T; (K + K')/2
  std::vector<double> T(48 * 48, 0.0), t1(48 * 48), K(48 * 48);
  for (int k = 0; k < 8; ++k)
    for (int blk = 0; blk < 2; ++blk) {
      int c = 6 * k + 3 * blk;
      for (int aa = 0; aa < 3; ++aa)
        for (int bb = 0; bb < 3; ++bb) T[(c + aa) + 48 * (c + bb)] = R[bb + 3 * aa];
    }
  mul(t1.data(), 48, 48, Kl.data(), 48, T.data());
  for (int j = 0; j < 48; ++j)
    for (int i = 0; i < 48; ++i) {
      double s = 0;
      for (int k = 0; k < 48; ++k) s += T[k + 48 * i] * t1[k + 48 * j];
      K[i + 48 * j] = s;
    }
  std::vector<double> Ks(48 * 48);
  for (int j = 0; j < 48; ++j)
    for (int i = 0; i < 48; ++i) Ks[i + 48 * j] = (K[i + 48 * j] + K[j + 48 * i]) / 2;
  // node_R congruence (assembly.jl:5899-5911)
  std::vector<double> Tn(48 * 48, 0.0);
  for (int k = 0; k < 8; ++k) {
    const double* Rn = nodeR + 9 * k;
    for (int blk = 0; blk < 2; ++blk) {
      int r0 = 6 * k + 3 * blk;
      for (int aa = 0; aa < 3; ++aa)
        for (int bb = 0; bb < 3; ++bb) Tn[(r0 + aa) + 48 * (r0 + bb)] = Rn[aa + 3 * bb];
    }
  }
  mul(t1.data(), 48, 48, Ks.data(), 48, Tn.data());
  for (int j = 0; j < 48; ++j)
    for (int i = 0; i < 48; ++i) {
      double s = 0;
      for (int k = 0; k < 48; ++k) s += Tn[k + 48 * i] * t1[k + 48 * j];
      Ke_global[i + 48 * j] = s;
    }
  return 0;
}

// ---------------------------------------------------------------------------
// CTETRA10 (src/tetra10.jl:6-79; iso_3d_constitutive FEMKernels.jl:12056-12069)
// xyz: 10 rows x 3.  Ke: 30x30 col-major, transformed by node_R (assembly.jl:5858-5870).
int or_t10_element(const double* xyz, const double* nodeR, double E, double nu,
                   double* Ke_global) {
  if (!(std::isfinite(E) && E > 0 && std::isfinite(nu) && nu > -1 && nu < 0.5)) return 2;
  double c = E / ((1.0 + nu) * (1.0 - 2.0 * nu)), d = 1.0 - nu, s = (1.0 - 2.0 * nu) / 2.0;
  double D[36] = {0};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) D[i + 6 * j] = (i == j) ? c * d : c * nu;
  for (int i = 3; i < 6; ++i) D[i + 6 * i] = c * s;
  const double A = (5.0 + 3.0 * std::sqrt(5.0)) / 20.0, Bq = (5.0 - std::sqrt(5.0)) / 20.0;
  const double pts[4][3] = {{Bq, Bq, Bq}, {A, Bq, Bq}, {Bq, A, Bq}, {Bq, Bq, A}};
  const int edges[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
  const double dL[3][4] = {{-1, 1, 0, 0}, {-1, 0, 1, 0}, {-1, 0, 0, 1}};
  double K[900] = {0};
  for (auto& q : pts) {
    double L[4] = {1.0 - q[0] - q[1] - q[2], q[0], q[1], q[2]};
    double dN[3][10];
    for (int i = 0; i < 4; ++i)
      for (int k = 0; k < 3; ++k) dN[k][i] = (4.0 * L[i] - 1.0) * dL[k][i];
    for (int e = 0; e < 6; ++e) {
      int i = edges[e][0], j = edges[e][1];
      for (int k = 0; k < 3; ++k) dN[k][e + 4] = 4.0 * (L[j] * dL[k][i] + L[i] * dL[k][j]);
    }
    double J[9];  // J[a][b] = sum_k dN[a][k] X[k][b], col-major J[a + 3b]
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double sm = 0;
        for (int k = 0; k < 10; ++k) sm += dN[a][k] * xyz[3 * k + b];
        J[a + 3 * b] = sm;
      }
    double det = J[0] * (J[4] * J[8] - J[7] * J[5]) - J[3] * (J[1] * J[8] - J[7] * J[2]) +
                 J[6] * (J[1] * J[5] - J[4] * J[2]);
    if (!(std::isfinite(det) && det > 0.0)) return 1;
    double Ji[9];
    if (!inv_small(J, 3, Ji)) return 1;
    double g[3][10];
    for (int a = 0; a < 3; ++a)
      for (int k = 0; k < 10; ++k) g[a][k] = Ji[a] * dN[0][k] + Ji[a + 3] * dN[1][k] + Ji[a + 6] * dN[2][k];
    double B[6 * 30] = {0};
    for (int i = 0; i < 10; ++i) {
      int cc = 3 * i;
      double gx = g[0][i], gy = g[1][i], gz = g[2][i];
      B[0 + 6 * (cc + 0)] = gx; B[1 + 6 * (cc + 1)] = gy; B[2 + 6 * (cc + 2)] = gz;
      B[3 + 6 * (cc + 0)] = gy; B[3 + 6 * (cc + 1)] = gx;
      B[4 + 6 * (cc + 1)] = gz; B[4 + 6 * (cc + 2)] = gy;
      B[5 + 6 * (cc + 0)] = gz; B[5 + 6 * (cc + 2)] = gx;
    }
    double t[6 * 30];
    mul(t, 6, 30, D, 6, B);
    mul_At_add(K, 30, 30, B, 6, t, det / 24.0);
  }
  // Matrix(Symmetric(K)): upper triangle mirrored
  for (int j = 0; j < 30; ++j)
    for (int i = j + 1; i < 30; ++i) K[i + 30 * j] = K[j + 30 * i];
  double T[900] = {0};
  for (int k = 0; k < 10; ++k)
    for (int aa = 0; aa < 3; ++aa)
      for (int bb = 0; bb < 3; ++bb) T[(3 * k + aa) + 30 * (3 * k + bb)] = nodeR[9 * k + aa + 3 * bb];
  double t1[900];
  mul(t1, 30, 30, K, 30, T);
  for (int j = 0; j < 30; ++j)
    for (int i = 0; i < 30; ++i) {
      double sm = 0;
      for (int k = 0; k < 30; ++k) sm += T[k + 30 * i] * t1[k + 30 * j];
      Ke_global[i + 30 * j] = sm;
    }
  return 0;
}

// ---------------------------------------------------------------------------
// CTRIA3 (FEMKernels.jl:9375-9809 stiffness_tria3_matrices_generic on the
// default SOL101 settings: plate kernel "mitc3", the recovered tying rigidity
// (JFEM_TRIA3_MITC3_SHEAR_REF), the residual bending flexibility with
// directional pairing (JFEM_TRIA3_MITC3_ZB, JFEM_TRIA3_ZB_DIRECTIONAL), the
// lumped drilling penalty (JFEM_TRIA3_DRILL_LUMPED), no Bmb coupling, no
// residual-bending shear relaxation (JFEM_TRIA3_RBF_C = 0)).

// FEMKernels.jl:9281-9313 tria3_guard_bending_flexibility!: Zb 3x3 col-major,
// modified in place; returns 1 when a bound changed it, 0 when not, -1 when
// the residual normal flexibility is not positive (the reference throws).
int or_tria3_guard(double* Zb, double La, double Lb, double c, double s, double Dnormal) {
  const double scale = 6 * (La / Lb) * s * Dnormal;
  if (!(scale > 0.0 && Zb[8] > 0.0)) return 0;
  const double z11 = Zb[0], z12 = Zb[3], z13 = Zb[6], z22 = Zb[4], z23 = Zb[7], z33 = Zb[8];
  const double h11 = scale * (z11 - z13 * z13 / z33) / (La * La);
  const double h22 = scale * (z22 - z23 * z23 / z33) / (Lb * Lb);
  const double h12 = scale * (z12 - z13 * z23 / z33) / (La * Lb);
  const double p11 = h11, p12 = (h12 - c * h11) / s, p22 = (h22 - 2 * c * h12 + c * c * h11) / (s * s);
  if (!(std::isfinite(p22) && p22 > 0.0)) return -1;
  const double a = std::max(p11, 1.0 / 10000);
  const double q = std::max(p22, a / 10000);
  const double limit = std::sqrt((85.0 / 100) * a * q);
  const double b = std::min(std::max(p12, -limit), limit);
  if (a == p11 && b == p12 && q == p22) return 0;
  const double n11 = a, n12 = c * a + s * b, n22 = c * c * a + 2 * c * s * b + s * s * q;
  Zb[0] += (n11 - h11) * La * La / scale;
  Zb[3] += (n12 - h12) * La * Lb / scale;
  Zb[1] = Zb[3];
  Zb[4] += (n22 - h22) * Lb * Lb / scale;
  return 1;
}

// 18x18 local CTRIA3 stiffness (col-major), DOFs (u v w rx ry rz) per node.
// coords: 3x2 local coordinates (col-major); Dm, Db: 3x3; Ds: 2x2.  Returns 0,
// or 111 when the residual flexibility guard fails (the reference throws).
int or_tria3_local(const double* coords, const double* Dm, const double* Db, const double* Ds,
                   double k6rot, double* Ke) {
  std::memset(Ke, 0, sizeof(double) * 324);
  const double x[3] = {coords[0], coords[1], coords[2]}, y[3] = {coords[3], coords[4], coords[5]};
  const double A2 = x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]);
  const double A = 0.5 * std::fabs(A2);
  if (A < 1e-12) return 0;   // :9380
  // membrane CST (:9389-9396)
  const double bv[3] = {(y[1] - y[2]) / (2 * A), (y[2] - y[0]) / (2 * A), (y[0] - y[1]) / (2 * A)};
  const double cv[3] = {(x[2] - x[1]) / (2 * A), (x[0] - x[2]) / (2 * A), (x[1] - x[0]) / (2 * A)};
  double Bm[18] = {0};   // 3 x 6
  for (int i = 0; i < 3; ++i) {
    at(Bm, 3, 0, 2 * i) = bv[i];
    at(Bm, 3, 1, 2 * i + 1) = cv[i];
    at(Bm, 3, 2, 2 * i) = cv[i];
    at(Bm, 3, 2, 2 * i + 1) = bv[i];
  }
  double DB[18], Kmem[36] = {0};
  mul(DB, 3, 6, Dm, 3, Bm);
  mul_At_add(Kmem, 6, 6, Bm, 3, DB, A);
  const int m_idx[6] = {0, 1, 6, 7, 12, 13};
  for (int j = 0; j < 6; ++j)
    for (int i = 0; i < 6; ++i) at(Ke, 18, m_idx[i], m_idx[j]) = at(Kmem, 6, i, j);
  // constant-curvature bending (:9399-9408)
  double Bb[27] = {0};   // 3 x 9
  for (int i = 0; i < 3; ++i) {
    const int crx = 3 * i + 1, cry = 3 * i + 2;
    at(Bb, 3, 0, cry) = bv[i];
    at(Bb, 3, 1, crx) = -cv[i];
    at(Bb, 3, 2, crx) = -bv[i];
    at(Bb, 3, 2, cry) = cv[i];
  }
  double DBb[27], Kb[81] = {0};
  mul(DBb, 3, 9, Db, 3, Bb);
  mul_At_add(Kb, 9, 9, Bb, 3, DBb, A);
  // MITC3 covariant shear rows (:9482-9502)
  const double x1 = x[0], y1 = y[0], x2 = x[1], y2 = y[1], x3 = x[2], y3 = y[2];
  const double J[4] = {x2 - x1, x3 - x1, y2 - y1, y3 - y1};   // [x2-x1 y2-y1; x3-x1 y3-y1] col-major
  double Ji[4];
  inv_small(J, 2, Ji);
  auto gcov = [&](double r, double s_, double* Br, double* Bs) {
    const double N[3] = {1 - r - s_, r, s_};
    const double dwdr[3] = {-1, 1, 0}, dwds[3] = {-1, 0, 1};
    for (int i = 0; i < 3; ++i) {
      const int cw = 3 * i, crx = 3 * i + 1, cry = 3 * i + 2;
      Br[cw] = dwdr[i]; Bs[cw] = dwds[i];
      Br[cry] = N[i] * at(J, 2, 0, 0); Bs[cry] = N[i] * at(J, 2, 1, 0);
      Br[crx] = -N[i] * at(J, 2, 0, 1); Bs[crx] = -N[i] * at(J, 2, 1, 1);
    }
  };
  double grA[9], gsA[9], grB[9], gsB[9], grC[9], gsC[9], cvec[9];
  gcov(0.5, 0.0, grA, gsA);
  gcov(0.0, 0.5, grB, gsB);
  gcov(0.5, 0.5, grC, gsC);
  for (int k = 0; k < 9; ++k) cvec[k] = (grC[k] - grA[k]) - (gsC[k] - gsB[k]);
  // tying rigidity (:9507-9557)
  const double La = std::hypot(x2 - x1, y2 - y1), Lb = std::hypot(x3 - x1, y3 - y1);
  const double Lc = std::hypot(x3 - x2, y3 - y2), Pper = La + Lb + Lc;
  const double cth = std::min(std::max(((x2 - x1) * (x3 - x1) + (y2 - y1) * (y3 - y1)) / std::max(La * Lb, 1e-30), -1.0), 1.0);
  const double sth = std::sqrt(std::max(1.0 - cth * cth, 0.0));
  double t2[4], G[4];
  mul(t2, 2, 2, Ds, 2, Ji);   // Ds * Jinv
  for (int j = 0; j < 2; ++j)
    for (int i = 0; i < 2; ++i) at(G, 2, i, j) = at(Ji, 2, 0, i) * at(t2, 2, 0, j) + at(Ji, 2, 1, i) * at(t2, 2, 1, j);
  const double uu = 3 * La / Pper, vv = 3 * Lb / Pper;
  double W[9];
  W[0] = at(G, 2, 0, 0) * A;
  W[3] = at(G, 2, 0, 1) * A; W[1] = W[3];
  W[4] = at(G, 2, 1, 1) * A;
  W[6] = (A / 3) * (uu * at(G, 2, 0, 0) - vv * at(G, 2, 0, 1)); W[2] = W[6];
  W[7] = (A / 3) * (uu * at(G, 2, 0, 1) - vv * at(G, 2, 1, 1)); W[5] = W[7];
  W[8] = uu * uu * at(G, 2, 0, 0) * (A / 6) - 2 * uu * vv * at(G, 2, 0, 1) * (A * (2 - cth) / 18) +
         vv * vv * at(G, 2, 1, 1) * (A / 6);
  // residual bending flexibility with directional pairing (:9581-9756)
  const double Dbend = std::fabs(Db[0]);
  if (sth > 1e-9 && Dbend > 1e-30 && La > 1e-30 && Lb > 1e-30) {
    const double Rr = (La - Lb) * (La - Lb) / (La * Lb);
    const double Tt = (La * La - Lb * Lb) / (La * Lb);
    const double sum_d = 2 * ((1 - cth + cth * cth) / (6 * sth) + 1.0 / 6) + Rr * (1 + cth * cth) / (6 * sth);
    const double dif_d = Tt * sth / 6;
    const double a11 = (sum_d + dif_d) / 2, a22 = (sum_d - dif_d) / 2;
    const double a12 = (-1 + 4 * cth - cth * cth) / (12 * sth) - 1.0 / 6 + Rr * cth / (6 * sth);
    const double S1 = La, S2 = Lb, S3 = Pper, s6 = 1.0 / 6;
    const double D11e = Dbend, D22e = std::fabs(Db[4]);
    const bool dir_pair = D11e > 1e-30 && D22e > 1e-30;
    const double rho = La / Lb, Rr2 = rho + 1 / rho - 2, Tt2 = rho - 1 / rho;
    const double fr = ((1 - cth) * (1 - cth) - (rho - cth)) / (6 * sth) + Rr2 * (1 + cth * cth) / (12 * sth) + Tt2 * sth / 12;
    const double fri = ((1 - cth) * (1 - cth) - (1 / rho - cth)) / (6 * sth) + Rr2 * (1 + cth * cth) / (12 * sth) - Tt2 * sth / 12;
    const double w12 = (1 / rho - cth) / (6 * sth), w13 = (rho - cth) / (6 * sth), w23 = cth / (6 * sth);
    const double o12 = (Rr2 * cth - (1 - cth) * (1 - cth) - Tt2 * cth) / (12 * sth);
    const double o13 = (Rr2 * cth - (1 - cth) * (1 - cth) + Tt2 * cth) / (12 * sth);
    const double o23 = (1 + cth * cth) / (12 * sth);
    auto ddir = [&](double vx, double vy) {
      const double n = std::hypot(vx, vy);
      if (n < 1e-30) return Dbend;
      const double nx = -vy / n, ny = vx / n;
      const double w[3] = {nx * nx, ny * ny, 2 * nx * ny};
      double d = 0;
      for (int ii = 0; ii < 3; ++ii)
        for (int jj = 0; jj < 3; ++jj) d += w[ii] * Db[ii + 3 * jj] * w[jj];
      return std::fabs(d) > 1e-30 ? d : Dbend;
    };
    const double Dn12 = dir_pair ? ddir(x2 - x1, y2 - y1) : Dbend;
    const double Dn13 = dir_pair ? ddir(x3 - x1, y3 - y1) : Dbend;
    const double Dn23 = dir_pair ? ddir(x3 - x2, y3 - y2) : Dbend;
    const double Gd = dir_pair ? std::sqrt(D11e * D22e) : Dbend;
    const double c11 = dir_pair ? s6 / Gd + fr / Dn12 + w13 / Dn13 + w23 / Dn23 : a11 / Dbend;
    const double c22 = dir_pair ? s6 / Gd + w12 / Dn12 + fri / Dn13 + w23 / Dn23 : a22 / Dbend;
    const double c12 = dir_pair ? -s6 / Gd + o12 / Dn12 + o13 / Dn13 + o23 / Dn23 : a12 / Dbend;
    double Zb[9];
    Zb[0] = c11 * S1 * S1; Zb[3] = c12 * S1 * S2;
    Zb[1] = Zb[3]; Zb[4] = c22 * S2 * S2;
    Zb[6] = -s6 / Gd * S1 * S3; Zb[2] = Zb[6];
    Zb[7] = s6 / Gd * S2 * S3; Zb[5] = Zb[7];
    Zb[8] = s6 / Gd * S3 * S3;
    if (or_tria3_guard(Zb, La, Lb, cth, sth, dir_pair ? Dn12 : Dbend) < 0) return 111;
    double Wi[9], Zt[9], Zs[9];
    if (!inv_small(W, 3, Wi)) return 111;
    for (int k = 0; k < 9; ++k) Zt[k] = Wi[k] + Zb[k];
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) Zs[i + 3 * j] = 0.5 * (Zt[i + 3 * j] + Zt[j + 3 * i]);
    if (!inv_small(Zs, 3, W)) return 111;
  }
  // Ks = D3' W D3, D3 = [grA; gsB; c] (:9758-9760)
  double D3[27];
  for (int k = 0; k < 9; ++k) { D3[3 * k] = grA[k]; D3[3 * k + 1] = gsB[k]; D3[3 * k + 2] = cvec[k]; }
  double WD[27], Kp[81];
  std::memcpy(Kp, Kb, sizeof Kp);
  mul(WD, 3, 9, W, 3, D3);
  mul_At_add(Kp, 9, 9, D3, 3, WD, 1.0);
  const int b_idx[9] = {2, 3, 4, 8, 9, 10, 14, 15, 16};
  for (int j = 0; j < 9; ++j)
    for (int i = 0; i < 9; ++i) at(Ke, 18, b_idx[i], b_idx[j]) += at(Kp, 9, i, j);
  // lumped drilling: alpha_L = K6ROT 1e-6 Dm[3,3] (2A) per node (:9800-9815)
  const double alpha_L = (k6rot * 1e-6) * Dm[8] * (2 * A);
  for (int i = 0; i < 3; ++i) {
    double Bd[18] = {0};
    for (int j = 0; j < 3; ++j) {
      Bd[6 * j] = 0.5 * cv[j];
      Bd[6 * j + 1] = -0.5 * bv[j];
    }
    Bd[6 * i + 5] = 1.0;
    for (int c = 0; c < 18; ++c)
      for (int r = 0; r < 18; ++r) at(Ke, 18, r, c) += alpha_L * (Bd[r] * Bd[c]);
  }
  return 0;
}

// Global-frame CTRIA3 stiffness (assembly.jl:5395-5503 without SNORM, offsets
// or material rotation): frame helpers.jl:1487-1490 (v1 along G1G2, v3 the
// normal of G1G2 x G1G3), local coordinates about the centroid (:5467-5470),
// T = blockdiag(Rel node_R) (:5483-5493), Ke = T' Ke_loc T.  xyz: 3 rows x 3;
// nodeR: 3 x 9; sect: the CQUAD4 section record (Cm Cb Cs h Eref k6rot flags).
int or_t3_element(const double* xyz, const double* nodeR, const double* sect, double* Ke_global) {
  double p[3][3];
  for (int k = 0; k < 3; ++k)
    for (int a = 0; a < 3; ++a) p[k][a] = xyz[3 * k + a];
  double v1[3], e13[3], v3[3], v2[3];
  for (int a = 0; a < 3; ++a) { v1[a] = p[1][a] - p[0][a]; e13[a] = p[2][a] - p[0][a]; }
  double l1 = std::sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
  for (int a = 0; a < 3; ++a) v1[a] /= l1;
  v3[0] = v1[1] * e13[2] - v1[2] * e13[1];
  v3[1] = v1[2] * e13[0] - v1[0] * e13[2];
  v3[2] = v1[0] * e13[1] - v1[1] * e13[0];
  double l3 = std::sqrt(v3[0] * v3[0] + v3[1] * v3[1] + v3[2] * v3[2]);
  for (int a = 0; a < 3; ++a) v3[a] /= l3;
  v2[0] = v3[1] * v1[2] - v3[2] * v1[1];
  v2[1] = v3[2] * v1[0] - v3[0] * v1[2];
  v2[2] = v3[0] * v1[1] - v3[1] * v1[0];
  double c[3];
  for (int a = 0; a < 3; ++a) c[a] = (p[0][a] + p[1][a] + p[2][a]) / 3.0;
  double lc[6];
  for (int k = 0; k < 3; ++k) {
    double d[3] = {p[k][0] - c[0], p[k][1] - c[1], p[k][2] - c[2]};
    lc[k] = d[0] * v1[0] + d[1] * v1[1] + d[2] * v1[2];
    lc[k + 3] = d[0] * v2[0] + d[1] * v2[1] + d[2] * v2[2];
  }
  double Ke[324];
  int st = or_tria3_local(lc, sect, sect + 9, sect + 18, sect[24], Ke);
  if (st) return st;
  double T[324] = {0};
  const double Rel[3][3] = {{v1[0], v1[1], v1[2]}, {v2[0], v2[1], v2[2]}, {v3[0], v3[1], v3[2]}};
  for (int k = 0; k < 3; ++k) {
    const double* R = nodeR + 9 * k;
    for (int rr = 0; rr < 3; ++rr)
      for (int cc = 0; cc < 3; ++cc) {
        double v = Rel[rr][0] * R[0 + 3 * cc] + Rel[rr][1] * R[1 + 3 * cc] + Rel[rr][2] * R[2 + 3 * cc];
        T[(6 * k + rr) + 18 * (6 * k + cc)] = v;
        T[(6 * k + 3 + rr) + 18 * (6 * k + 3 + cc)] = v;
      }
  }
  double tmp[324] = {0};
  for (int jj = 0; jj < 18; ++jj)
    for (int ll = 0; ll < 18; ++ll) {
      double v = T[ll + 18 * jj];
      if (v != 0.0)
        for (int ii = 0; ii < 18; ++ii) tmp[ii + 18 * jj] += Ke[ii + 18 * ll] * v;
    }
  std::memset(Ke_global, 0, sizeof(double) * 324);
  for (int jj = 0; jj < 18; ++jj)
    for (int ll = 0; ll < 18; ++ll) {
      double v = tmp[ll + 18 * jj];
      if (v != 0.0)
        for (int ii = 0; ii < 18; ++ii) Ke_global[ii + 18 * jj] += T[ll + 18 * ii] * v;
    }
  return 0;
}

// ---------------------------------------------------------------------------
// Triplet emission in the reference's order and Julia's sparse() semantics.
//   Q4: positional slots (ei-1)*576, col-major (assembly.jl:3506-3508, :433-439)
//   CTRIA3: 324 per element col-major (:5505-5507)
//   solids: 900 per element col-major (:5882-5884)
//   Q8: col-major, exact zeros skipped (:5912-5916)
// Counts triplets first (n_q8 contribution depends on values).
int64_t or_assemble_triplets(int64_t n_nodes, const double* xyz, const double* node_R,
                             int64_t n_q4, const int32_t* q4_nodes, const double* q4_sect,
                             int64_t n_t3, const int32_t* t3_nodes, const double* t3_sect,
                             int64_t n_q8, const int32_t* q8_nodes, const double* q8_sect,
                             int64_t n_t10, const int32_t* t10_nodes, const double* t10_mat,
                             int64_t cap, int64_t* I, int64_t* J, double* V, int32_t* err_elem) {
  int64_t cnt = 0;
  *err_elem = -1;
  std::vector<double> Ke(48 * 48);
  double exyz[30], eR[90];
  // positional slots (e*576): the element loop is parallel like the
  // reference's Threads.@threads :static loop (assembly.jl:3603)
  int64_t q4_err = -1;
  int q4_st = 0;
#pragma omp parallel
  {
    std::vector<double> Kt(576);
    double xy[12], Rr[36];
#pragma omp for schedule(static)
    for (int64_t e = 0; e < n_q4; ++e) {
      for (int k = 0; k < 4; ++k) {
        int n = q4_nodes[4 * e + k];
        for (int a = 0; a < 3; ++a) xy[3 * k + a] = xyz[3 * n + a];
        for (int a = 0; a < 9; ++a) Rr[9 * k + a] = node_R[9 * n + a];
      }
      int st = or_q4_element(xy, Rr, q4_sect + 26 * e, Kt.data());
      if (st) {
#pragma omp critical
        { if (q4_err < 0 || e < q4_err) { q4_err = e; q4_st = st; } }
        continue;
      }
      int64_t base = 576 * e;
      if (base + 576 <= cap)
        for (int cc = 0; cc < 24; ++cc)
          for (int rr = 0; rr < 24; ++rr) {
            int64_t t = base + rr + 24 * cc;
            I[t] = 6 * (int64_t)q4_nodes[4 * e + rr / 6] + rr % 6;
            J[t] = 6 * (int64_t)q4_nodes[4 * e + cc / 6] + cc % 6;
            V[t] = Kt[rr + 24 * cc];
          }
    }
  }
  if (q4_err >= 0) { *err_elem = (int32_t)q4_err; return -q4_st; }
  cnt = 576 * n_q4;
  // CTRIA3: all 324 entries, column-major, after the CQUAD4 (:5386-5510)
  for (int64_t e = 0; e < n_t3; ++e) {
    for (int k = 0; k < 3; ++k) {
      int n = t3_nodes[3 * e + k];
      for (int a = 0; a < 3; ++a) exyz[3 * k + a] = xyz[3 * n + a];
      for (int a = 0; a < 9; ++a) eR[9 * k + a] = node_R[9 * n + a];
    }
    int st = or_t3_element(exyz, eR, t3_sect + 26 * e, Ke.data());
    if (st) { *err_elem = (int32_t)(n_q4 + e); return -st; }
    for (int cc = 0; cc < 18; ++cc)
      for (int rr = 0; rr < 18; ++rr) {
        if (cnt < cap) {
          I[cnt] = 6 * (int64_t)t3_nodes[3 * e + rr / 6] + rr % 6;
          J[cnt] = 6 * (int64_t)t3_nodes[3 * e + cc / 6] + cc % 6;
          V[cnt] = Ke[rr + 18 * cc];
        }
        ++cnt;
      }
  }
  for (int64_t e = 0; e < n_t10; ++e) {
    for (int k = 0; k < 10; ++k) {
      int n = t10_nodes[10 * e + k];
      for (int a = 0; a < 3; ++a) exyz[3 * k + a] = xyz[3 * n + a];
      for (int a = 0; a < 9; ++a) eR[9 * k + a] = node_R[9 * n + a];
    }
    int st = or_t10_element(exyz, eR, t10_mat[2 * e], t10_mat[2 * e + 1], Ke.data());
    if (st) { *err_elem = (int32_t)(n_q4 + n_t3 + e); return -st; }
    for (int cc = 0; cc < 30; ++cc)
      for (int rr = 0; rr < 30; ++rr) {
        if (cnt < cap) {
          I[cnt] = 6 * (int64_t)t10_nodes[10 * e + rr / 3] + rr % 3;
          J[cnt] = 6 * (int64_t)t10_nodes[10 * e + cc / 3] + cc % 3;
          V[cnt] = Ke[rr + 30 * cc];
        }
        ++cnt;
      }
  }
  std::vector<double> x8(24), R8(72);
  for (int64_t e = 0; e < n_q8; ++e) {
    for (int k = 0; k < 8; ++k) {
      int n = q8_nodes[8 * e + k];
      for (int a = 0; a < 3; ++a) x8[3 * k + a] = xyz[3 * n + a];
      for (int a = 0; a < 9; ++a) R8[9 * k + a] = node_R[9 * n + a];
    }
    int st = or_q8_element(x8.data(), R8.data(), q8_sect + 22 * e, Ke.data());
    if (st) { *err_elem = (int32_t)(n_q4 + n_t3 + n_t10 + e); return -st; }
    for (int cc = 0; cc < 48; ++cc)
      for (int rr = 0; rr < 48; ++rr) {
        double v = Ke[rr + 48 * cc];
        if (v == 0.0) continue;
        if (cnt < cap) {
          I[cnt] = 6 * (int64_t)q8_nodes[8 * e + rr / 6] + rr % 6;
          J[cnt] = 6 * (int64_t)q8_nodes[8 * e + cc / 6] + cc % 6;
          V[cnt] = v;
        }
        ++cnt;
      }
  }
  (void)n_nodes;
  return cnt;
}

// Julia sparse(I,J,V,n,n) semantics (SparseArrays sparse!: row bucketing in
// triplet order, duplicate combine left-to-right, transpose to CSC) plus the
// triplet -> nzval slot map of _sparse_from_triplets_cached
// (assembly.jl:6008-6033).  colptr: n+1, rowval/nzval: nnz (<= nt).  Returns nnz.
int64_t or_build_csc(int64_t n, int64_t nt, const int64_t* I, const int64_t* J,
                     const double* V, int64_t* colptr, int32_t* rowval, double* nzval,
                     int64_t* slot) {
  // bucket triplets by column (stable), then rows within a column; combine in
  // triplet order.
  std::vector<int64_t> cnt(n + 1, 0);
  for (int64_t t = 0; t < nt; ++t) cnt[J[t] + 1]++;
  for (int64_t j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
  std::vector<int64_t> order(nt);
  {
    std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
    for (int64_t t = 0; t < nt; ++t) order[pos[J[t]]++] = t;
  }
  std::vector<int64_t> last(n, -1);
  int64_t nnz = 0;
  colptr[0] = 0;
  std::vector<std::pair<int64_t, int64_t>> rows;  // (row, first triplet)
  for (int64_t j = 0; j < n; ++j) {
    rows.clear();
    for (int64_t q = cnt[j]; q < cnt[j + 1]; ++q) {
      int64_t t = order[q];
      int64_t r = I[t];
      if (last[r] < 0) { last[r] = (int64_t)rows.size(); rows.push_back({r, t}); }
    }
    std::sort(rows.begin(), rows.end());
    for (size_t k = 0; k < rows.size(); ++k) last[rows[k].first] = nnz + (int64_t)k;
    for (size_t k = 0; k < rows.size(); ++k) {
      rowval[nnz + k] = (int32_t)rows[k].first;
      nzval[nnz + k] = 0.0;
    }
    std::vector<char> seen(rows.size(), 0);
    for (int64_t q = cnt[j]; q < cnt[j + 1]; ++q) {
      int64_t t = order[q];
      int64_t p = last[I[t]];
      slot[t] = p;
      if (!seen[p - nnz]) { nzval[p] = V[t]; seen[p - nnz] = 1; }
      else nzval[p] = nzval[p] + V[t];
    }
    for (auto& rr : rows) last[rr.first] = -1;
    nnz += (int64_t)rows.size();
    colptr[j + 1] = nnz;
  }
  return nnz;
}

// y = K x for CSC K (ndof x ndof), x/y column-major with nrhs columns.
// CTETRA10 centroid stress and strain (recover_solid_stresses!,
// src/solver/stress_recovery.jl:1823-1960, with solid_centroid_B_tetra10,
// src/tetra10.jl:110-115, and stress_solid_3d, src/FEMKernels.jl:13067-13074):
// element displacements are the nodes' translations rotated to the basic
// frame (u = node_R * u_node); B at the centroid (r = s = t = 1/4);
// strain = B u (engineering shears xy, yz, zx), stress = D strain,
// von Mises from the six stress components.  xyz: 10 x 3 (row per node),
// nodeR: 10 x 9 col-major blocks, u_node: 10 x 3 translations in the node
// frames.  out: sxx syy szz txy tyz tzx, exx eyy ezz gxy gyz gzx, von Mises.
int or_t10_stress(const double* xyz, const double* nodeR, double E, double nu, const double* u_node,
                  double* out) {
  if (!(std::isfinite(E) && E > 0 && std::isfinite(nu) && nu > -1 && nu < 0.5)) return 2;
  const int edges[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
  const double dL[3][4] = {{-1, 1, 0, 0}, {-1, 0, 1, 0}, {-1, 0, 0, 1}};
  const double L[4] = {0.25, 0.25, 0.25, 0.25};
  double dN[3][10];
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 3; ++k) dN[k][i] = (4.0 * L[i] - 1.0) * dL[k][i];
  for (int e = 0; e < 6; ++e) {
    int i = edges[e][0], j = edges[e][1];
    for (int k = 0; k < 3; ++k) dN[k][e + 4] = 4.0 * (L[j] * dL[k][i] + L[i] * dL[k][j]);
  }
  double J[9];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double sm = 0;
      for (int k = 0; k < 10; ++k) sm += dN[a][k] * xyz[3 * k + b];
      J[a + 3 * b] = sm;
    }
  double det = J[0] * (J[4] * J[8] - J[7] * J[5]) - J[3] * (J[1] * J[8] - J[7] * J[2]) +
               J[6] * (J[1] * J[5] - J[4] * J[2]);
  if (!(std::isfinite(det) && det > 0.0)) return 1;
  double Ji[9];
  if (!inv_small(J, 3, Ji)) return 1;
  double u[30];
  for (int k = 0; k < 10; ++k)
    for (int a = 0; a < 3; ++a) {
      double sm = 0;
      for (int b = 0; b < 3; ++b) sm += nodeR[9 * k + a + 3 * b] * u_node[3 * k + b];
      u[3 * k + a] = sm;
    }
  double eps[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 10; ++i) {
    double gx = Ji[0] * dN[0][i] + Ji[3] * dN[1][i] + Ji[6] * dN[2][i];
    double gy = Ji[1] * dN[0][i] + Ji[4] * dN[1][i] + Ji[7] * dN[2][i];
    double gz = Ji[2] * dN[0][i] + Ji[5] * dN[1][i] + Ji[8] * dN[2][i];
    const double ux = u[3 * i], uy = u[3 * i + 1], uz = u[3 * i + 2];
    eps[0] += gx * ux;
    eps[1] += gy * uy;
    eps[2] += gz * uz;
    eps[3] += gy * ux + gx * uy;
    eps[4] += gz * uy + gy * uz;
    eps[5] += gz * ux + gx * uz;
  }
  double c = E / ((1.0 + nu) * (1.0 - 2.0 * nu)), d = 1.0 - nu, sh = (1.0 - 2.0 * nu) / 2.0;
  double sig[6];
  for (int i = 0; i < 3; ++i) {
    double sm = 0;
    for (int j = 0; j < 3; ++j) sm += (i == j ? c * d : c * nu) * eps[j];
    sig[i] = sm;
  }
  for (int i = 3; i < 6; ++i) sig[i] = c * sh * eps[i];
  double vm = sig[0] * sig[0] + sig[1] * sig[1] + sig[2] * sig[2] - sig[0] * sig[1] - sig[1] * sig[2] -
              sig[2] * sig[0] + 3.0 * (sig[3] * sig[3] + sig[4] * sig[4] + sig[5] * sig[5]);
  for (int i = 0; i < 6; ++i) { out[i] = sig[i]; out[6 + i] = eps[i]; }
  out[12] = std::sqrt(std::max(0.0, vm));
  return 0;
}

// r = f - A x in double-double arithmetic (Knuth two-sum, FMA two-product)
// per row: the checker's refinement residual carries only the final rounding,
// so refinement can reach the accuracy of the FP64 data even where the row
// sums of a stiffness matrix cancel.  A is m x n in CSC; f, r: m x nrhs.
void or_csc_residual_dd(int64_t m, int64_t n, const int64_t* colptr, const int32_t* rowval,
                        const double* nzval, int32_t nrhs, const double* x, const double* f, double* r) {
  std::vector<double> hi(m), lo(m);
  for (int32_t c = 0; c < nrhs; ++c) {
    const double* xc = x + (int64_t)c * n;
    const double* fc = f + (int64_t)c * m;
    for (int64_t i = 0; i < m; ++i) { hi[i] = -fc[i]; lo[i] = 0.0; }
    for (int64_t j = 0; j < n; ++j) {
      const double xj = xc[j];
      for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) {
        const int64_t i = rowval[p];
        const double prod = nzval[p] * xj;
        const double perr = std::fma(nzval[p], xj, -prod);
        const double s = hi[i] + prod;
        const double bp = s - hi[i];
        const double serr = (hi[i] - (s - bp)) + (prod - bp);
        hi[i] = s;
        lo[i] += serr + perr;
      }
    }
    double* rc = r + (int64_t)c * m;
    for (int64_t i = 0; i < m; ++i) rc[i] = -(hi[i] + lo[i]);
  }
}

void or_csc_matvec(int64_t n, const int64_t* colptr, const int32_t* rowval,
                   const double* nzval, int32_t nrhs, const double* x, double* y) {
  for (int32_t c = 0; c < nrhs; ++c) {
    double* yc = y + (int64_t)c * n;
    const double* xc = x + (int64_t)c * n;
    for (int64_t i = 0; i < n; ++i) yc[i] = 0.0;
    for (int64_t j = 0; j < n; ++j) {
      double xj = xc[j];
      for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) yc[rowval[p]] += nzval[p] * xj;
    }
  }
}

}  // extern "C"
