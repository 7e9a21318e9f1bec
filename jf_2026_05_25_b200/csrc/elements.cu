// elements.cu -- element stiffness kernels (FP64), one warp per element.
//
// CQUAD4: default SOL101 kernel of FEMKernels.jl:2874-4166 for flat elements
//   (MacNeal natural-shear block :4223-4339 / :4599-4783 / :6187-6285,
//    Wilson membrane modes with the patch-consistent Jacobian :1847-1895,
//    A-derived bending enrichment :1989-2024, lumped K6ROT drilling
//    :3749-3818), element frame helpers.jl:1422-1481, PSHELL material angle
//    assembly.jl:4392-4420, transform+emit assembly.jl:359-440.
// CTETRA10: tetra10.jl:6-79 (four-point rule, Symmetric upper copy),
//   node_R congruence assembly.jl:5858-5870.
// CQUAD8: quad8_shell.jl:96-204, node_R congruence assembly.jl:5899-5911.
// CTRIA3: tria3.cu.
//
// Each lane owns a strided subset of the output entries and accumulates them
// in registers; small shared quantities (condensation blocks, the MacNeal
// operator) are exchanged through a per-warp shared-memory slab.  Every
// element writes its full matrix, column-major, to its slot of the element
// value buffer, so consecutive lanes write consecutive addresses.
#include "jfg_internal.h"

namespace jfg {
namespace {

constexpr int WARPS = 4;
constexpr double EPS64 = 2.220446049250313e-16;

__device__ inline void record_error(DevError* err, int32_t code, int64_t idx) {
  if (atomicCAS(&err->code, 0, code) == 0) err->index = idx;
}

__device__ inline double qf3(const double u[3], const double* C, const double v[3]) {
  // u^T C v, C column-major 3x3
  double s = 0.0;
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    double cv = C[0 + 3 * b] * u[0] + C[1 + 3 * b] * u[1] + C[2 + 3 * b] * u[2];
    s += cv * v[b];
  }
  return s;
}

__device__ inline void shape_d(double xi, double eta, double dNr[4], double dNs[4]) {
  dNr[0] = -0.25 * (1 - eta); dNr[1] = 0.25 * (1 - eta);
  dNr[2] = 0.25 * (1 + eta);  dNr[3] = -0.25 * (1 + eta);
  dNs[0] = -0.25 * (1 - xi);  dNs[1] = -0.25 * (1 + xi);
  dNs[2] = 0.25 * (1 + xi);   dNs[3] = 0.25 * (1 - xi);
}
__device__ inline void shape_n(double xi, double eta, double N[4]) {
  N[0] = 0.25 * (1 - xi) * (1 - eta); N[1] = 0.25 * (1 + xi) * (1 - eta);
  N[2] = 0.25 * (1 + xi) * (1 + eta); N[3] = 0.25 * (1 - xi) * (1 + eta);
}
__device__ inline void jac4(const double lc[8], const double dNr[4], const double dNs[4],
                            double& J11, double& J12, double& J21, double& J22) {
  J11 = J12 = J21 = J22 = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    J11 += dNr[k] * lc[k]; J12 += dNr[k] * lc[4 + k];
    J21 += dNs[k] * lc[k]; J22 += dNs[k] * lc[4 + k];
  }
}
__device__ inline bool jac_ok(double d, double a, double b, double c, double e) {
  double scale = fabs(a * e) + fabs(b * c);
  return isfinite(d) && isfinite(scale) && fabs(d) > 64.0 * EPS64 * scale;
}

// Gauss-Jordan inverse with partial pivoting of a column-major n x n matrix.
template <int N>
__device__ bool inv_small(const double* A, double* Ai) {
  double M[N * N];
#pragma unroll
  for (int i = 0; i < N * N; ++i) { M[i] = A[i]; Ai[i] = 0.0; }
#pragma unroll
  for (int i = 0; i < N; ++i) Ai[i + N * i] = 1.0;
  for (int k = 0; k < N; ++k) {
    int p = k;
    double best = fabs(M[k + N * k]);
    for (int i = k + 1; i < N; ++i)
      if (fabs(M[i + N * k]) > best) { best = fabs(M[i + N * k]); p = i; }
    if (!(best > 0.0) || !isfinite(best)) return false;
    if (p != k)
      for (int j = 0; j < N; ++j) {
        double t = M[k + N * j]; M[k + N * j] = M[p + N * j]; M[p + N * j] = t;
        t = Ai[k + N * j]; Ai[k + N * j] = Ai[p + N * j]; Ai[p + N * j] = t;
      }
    double piv = M[k + N * k];
    for (int j = 0; j < N; ++j) { M[k + N * j] /= piv; Ai[k + N * j] /= piv; }
    for (int i = 0; i < N; ++i) {
      if (i == k) continue;
      double f = M[i + N * k];
      if (f == 0.0) continue;
      for (int j = 0; j < N; ++j) {
        M[i + N * j] -= f * M[k + N * j];
        Ai[i + N * j] -= f * Ai[k + N * j];
      }
    }
  }
  return true;
}


// MacNeal shear operator D (4 x 12) and sol = Z^-1 D (one thread).
__device__ int macneal_operator(const double lc[8], const double* Cb, const double* Cs, double* D, double* sol) {
  const double pt = 0.57735026918962573;  // 1/sqrt(3)
  const double sxi[4] = {0.0, 0.0, -pt, pt}, seta[4] = {-pt, pt, 0.0, 0.0};
  double Ce[4][12], Je[4][4];
  for (int sp = 0; sp < 4; ++sp) {
    double xr = sxi[sp] == 0.0 ? 0.0 : copysign(1.0, sxi[sp]);
    double er = seta[sp] == 0.0 ? 0.0 : copysign(1.0, seta[sp]);
    double dNr[4], dNs[4], N[4];
    shape_d(xr, er, dNr, dNs);
    shape_n(xr, er, N);
    double J11, J12, J21, J22;
    jac4(lc, dNr, dNs, J11, J12, J21, J22);
    Je[sp][0] = J11; Je[sp][1] = J12; Je[sp][2] = J21; Je[sp][3] = J22;
    bool c1 = sp < 2;
    double tx = c1 ? J11 : J21, ty = c1 ? J12 : J22;
    for (int k = 0; k < 4; ++k) {
      Ce[sp][3 * k + 0] = c1 ? dNr[k] : dNs[k];
      Ce[sp][3 * k + 1] = -N[k] * ty;
      Ce[sp][3 * k + 2] = N[k] * tx;
    }
  }
  for (int sp = 0; sp < 4; ++sp) {
    double J11 = Je[sp][0], J12 = Je[sp][1], J21 = Je[sp][2], J22 = Je[sp][3];
    double det = J11 * J22 - J12 * J21;
    double adet = fabs(det) < 1e-14 ? (det < 0 ? -1e-14 : 1e-14) : det;
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
  double tr[16];
  for (int i = 0; i < 16; ++i) tr[i] = 0.0;
  const double rn[4] = {-1, 1, 1, -1}, sn[4] = {-1, -1, 1, 1};
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 4; ++k) {
      int b = 3 * k;
      tr[i + 0] += D[i + 4 * (b + 2)];
      tr[i + 4] += sn[k] * D[i + 4 * (b + 2)];
      tr[i + 8] -= D[i + 4 * (b + 1)];
      tr[i + 12] -= rn[k] * D[i + 4 * (b + 1)];
    }
  const double* x = lc; const double* y = lc + 4;
  double ax = 0.25 * (-x[0] + x[1] + x[2] - x[3]), ay = 0.25 * (-y[0] + y[1] + y[2] - y[3]);
  double bx = 0.25 * (-x[0] - x[1] + x[2] + x[3]), by = 0.25 * (-y[0] - y[1] + y[2] + y[3]);
  double cx = 0.25 * (x[0] - x[1] + x[2] - x[3]), cy = 0.25 * (y[0] - y[1] + y[2] - y[3]);
  double det0 = ax * by - ay * bx;
  double det_scale = fmax(hypot(ax, ay) * hypot(bx, by), EPS64);
  if (!(fabs(det0) > 64 * EPS64 * det_scale)) return 2;
  double area = 4.0 * fabs(det0);
  double dx2 = (2 * ax) * (2 * ax), dy2 = (2 * by) * (2 * by);
  double fxx = fabs(2 * ax) > 1e-30 ? (cx / (2 * ax)) * (cx / (2 * ax)) : 0.0;
  double fyy = fabs(2 * by) > 1e-30 ? (cy / (2 * by)) * (cy / (2 * by)) : 0.0;
  if (fxx + fyy > 1e-24 && ((Cb[0] == 0.0) != (Cb[4] == 0.0))) return 3;
  double ux = dx2 / (12 * area * fmax(fabs(Cb[0]), 1e-30));
  double uy = dy2 / (12 * area * fmax(fabs(Cb[4]), 1e-30));
  double zb[4] = {ux, 3 * dy2 / (dy2 + 39 * dx2) * ux, uy, 3 * dx2 / (dx2 + 39 * dy2) * uy};
  double Z[16];
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k) s += tr[i + 4 * k] * zb[k] * tr[j + 4 * k];
      Z[i + 4 * j] = s;
    }
  const double gp = pt;
  auto jacf = [&](double r, double s) {
    return fabs((ax + cx * s) * (by + cy * r) - (ay + cy * s) * (bx + cx * r));
  };
  double va = sqrt(2 * jacf(0.0, -gp)), vb = sqrt(2 * jacf(0.0, gp));
  double vc = sqrt(2 * jacf(-gp, 0.0)), vd = sqrt(2 * jacf(gp, 0.0));
  double pxa[4] = {va, -gp * va, 0, 0}, pxb[4] = {vb, gp * vb, 0, 0};
  double pyc[4] = {0, 0, vc, -gp * vc}, pyd[4] = {0, 0, vd, gp * vd};
  double H[16], Hi[16];
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i)
      H[i + 4 * j] = Cs[0] * (pxa[i] * pxa[j] + pxb[i] * pxb[j]) +
                     Cs[3] * (pyc[i] * pyc[j] + pyd[i] * pyd[j]) +
                     Cs[2] * (pxa[i] + pxb[i]) * (pyc[j] + pyd[j]) / 2 +
                     Cs[1] * (pyc[i] + pyd[i]) * (pxa[j] + pxb[j]) / 2;
  if (!inv_small<4>(H, Hi)) return 4;
  double t4[16];
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k) s += tr[i + 4 * k] * Hi[k + 4 * j];
      t4[i + 4 * j] = s;
    }
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k) s += t4[i + 4 * k] * tr[j + 4 * k];
      Z[i + 4 * j] += s;
    }
  double Zi[16];
  if (!inv_small<4>(Z, Zi)) return 5;
  for (int j = 0; j < 12; ++j)
    for (int i = 0; i < 4; ++i) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k) s += Zi[i + 4 * k] * D[k + 4 * j];
      sol[i + 4 * j] = s;
    }
  return 0;
}

// CQUAD4 in two passes.  k_q4_prep, one thread per element, does the scalar
// work: element frame and local coordinates, the PSHELL material rotation,
// the MacNeal shear operator D and Z^{-1} D, and the 4 x 4 internal-mode
// blocks with their inverses.  k_q4, one warp per element, then accumulates
// the 24 x 24 stiffness with every lane busy (18 entries each): Gauss-point
// membrane and bending, the shear term, lumped drilling, the
// section-kinematic enrichment and the node-frame transform.  The prep record
// per element is Q4P doubles of scratch.
constexpr int Q4P = Q4_PREP_STRIDE;

__global__ void __launch_bounds__(128)
k_q4_prep(int64_t n, const int32_t* __restrict__ nodes, const double* __restrict__ sect,
          const double* __restrict__ xyz, double* __restrict__ prep, DevError* err) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double* out = prep + Q4P * e;
  out[Q4P_STATUS] = 0.0;
  int nd[4];
  double p[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    nd[k] = nodes[4 * e + k];
#pragma unroll
    for (int a = 0; a < 3; ++a) p[k][a] = xyz[3 * (int64_t)nd[k] + a];
  }
  // ---- element frame (diag mode) and local coordinates
  double gxi[3], geta[3], v3[3], d13[3], d24[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    gxi[a] = 0.25 * (-p[0][a] + p[1][a] + p[2][a] - p[3][a]);
    geta[a] = 0.25 * (-p[0][a] - p[1][a] + p[2][a] + p[3][a]);
    d13[a] = p[2][a] - p[0][a];
    d24[a] = p[3][a] - p[1][a];
  }
  auto cross = [](const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1]; o[1] = a[2] * b[0] - a[0] * b[2]; o[2] = a[0] * b[1] - a[1] * b[0];
  };
  auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  cross(gxi, geta, v3);
  if (dot(v3, v3) <= 1e-24) cross(d13, d24, v3);
  {
    double l = sqrt(dot(v3, v3));
    v3[0] /= l; v3[1] /= l; v3[2] /= l;
  }
  double d13n[3], d24n[3];
  {
    double l1 = sqrt(dot(d13, d13)), l2 = sqrt(dot(d24, d24));
#pragma unroll
    for (int a = 0; a < 3; ++a) { d13n[a] = d13[a] / l1; d24n[a] = d24[a] / l2; }
  }
  double xr[3] = {d13n[0] - d24n[0], d13n[1] - d24n[1], d13n[2] - d24n[2]};
  if (dot(xr, xr) < 1e-20)
    for (int a = 0; a < 3; ++a) xr[a] = d13n[a] + d24n[a];
  double dv = dot(xr, v3);
  double v1[3] = {xr[0] - dv * v3[0], xr[1] - dv * v3[1], xr[2] - dv * v3[2]};
  if (dot(v1, v1) <= 1e-24) {
    double ge = dot(geta, v3);
    for (int a = 0; a < 3; ++a) v1[a] = geta[a] - ge * v3[a];
    if (dot(v1, v1) <= 1e-24) {
      double e12[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
      double de = dot(e12, v3);
      for (int a = 0; a < 3; ++a) v1[a] = e12[a] - de * v3[a];
    }
  }
  {
    double l = sqrt(dot(v1, v1));
    v1[0] /= l; v1[1] /= l; v1[2] /= l;
  }
  double v2[3];
  cross(v3, v1, v2);
  double c[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) c[a] = (p[0][a] + p[1][a] + p[2][a] + p[3][a]) / 4.0;
  double lc[8], zmax = 0.0, xmax = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double d[3] = {p[k][0] - c[0], p[k][1] - c[1], p[k][2] - c[2]};
    lc[k] = dot(d, v1);
    lc[4 + k] = dot(d, v2);
    zmax = fmax(zmax, fabs(dot(d, v3)));
    xmax = fmax(xmax, fabs(lc[k]));
  }
  const double* sc = sect + 26 * e;
  if (!(zmax <= 1e-12 * fmax(xmax, 1e-30))) {
    record_error(err, EE_NOT_FLAT, e);
    out[Q4P_STATUS] = 1.0;
    return;
  }
  if (sc[25] != 0.0) {
    record_error(err, EE_FLAGS, e);
    out[Q4P_STATUS] = 1.0;
    return;
  }
  double Cm[9], Cb[9], Cs[4];
#pragma unroll
  for (int i = 0; i < 9; ++i) { Cm[i] = sc[i]; Cb[i] = sc[9 + i]; }
#pragma unroll
  for (int i = 0; i < 4; ++i) Cs[i] = sc[18 + i];
  const double h = sc[22], k6rot = sc[24];
  // PSHELL material angle: projected edge G1-G2 measured from v1
  {
    double e12[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    double de = dot(e12, v3);
    double e12p[3] = {e12[0] - de * v3[0], e12[1] - de * v3[1], e12[2] - de * v3[2]};
    double l2 = dot(e12p, e12p);
    double beta = 0.0;
    if (l2 > 1e-24) {
      double lx = sqrt(l2);
      double xm[3] = {e12p[0] / lx, e12p[1] / lx, e12p[2] / lx};
      beta = atan2(dot(xm, v2), dot(xm, v1));
    }
    if (fabs(beta) > 1e-10) {
      double cb = cos(beta), sb = sin(beta);
      double c2 = cb * cb, s2 = sb * sb, cs = cb * sb;
      double T[9] = {c2, s2, -2 * cs, s2, c2, 2 * cs, cs, -cs, c2 - s2};
      double* Cs3[2] = {Cm, Cb};
      for (int q = 0; q < 2; ++q) {
        double* C = Cs3[q];
        double t[9], o[9];
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i)
            t[i + 3 * j] = C[i] * T[3 * j] + C[i + 3] * T[1 + 3 * j] + C[i + 6] * T[2 + 3 * j];
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i)
            o[i + 3 * j] = T[3 * i] * t[3 * j] + T[1 + 3 * i] * t[1 + 3 * j] + T[2 + 3 * i] * t[2 + 3 * j];
        for (int i = 0; i < 9; ++i) C[i] = o[i];
      }
      double a11 = Cs[0], a12 = Cs[2], a22 = Cs[3];
      Cs[0] = cb * cb * a11 - 2 * cb * sb * a12 + sb * sb * a22;
      Cs[2] = cb * sb * a11 + (cb * cb - sb * sb) * a12 - cb * sb * a22;
      Cs[1] = Cs[2];
      Cs[3] = sb * sb * a11 + 2 * cb * sb * a12 + cb * cb * a22;
    }
  }
  double cmmax = 0.0;
#pragma unroll
  for (int i = 0; i < 9; ++i) cmmax = fmax(cmmax, fabs(Cm[i]));
  const double* shp = cmmax > 0 ? Cm : Cb;
  const double dNr_c[4] = {-0.25, 0.25, 0.25, -0.25}, dNs_c[4] = {-0.25, -0.25, 0.25, 0.25};
  double J11c, J12c, J21c, J22c;
  jac4(lc, dNr_c, dNs_c, J11c, J12c, J21c, J22c);
  const double detJc = J11c * J22c - J12c * J21c;
  const double idc = 1.0 / detJc;
  const double iJ11c = J22c * idc, iJ12c = -J12c * idc, iJ21c = -J21c * idc, iJ22c = J11c * idc;
  // internal-mode blocks over the 2 x 2 Gauss points
  double kbb[16], kbbs[16], kbbb[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) kbb[q] = kbbs[q] = kbbb[q] = 0.0;
  const double pt = 0.57735026918962573;
  const double gr[4] = {-pt, pt, pt, -pt}, gs[4] = {-pt, -pt, pt, pt};
  bool ok = true;
  for (int g = 0; g < 4; ++g) {
    double r = gr[g], sv = gs[g];
    double dNr[4], dNs[4];
    shape_d(r, sv, dNr, dNs);
    double J11, J12, J21, J22;
    jac4(lc, dNr, dNs, J11, J12, J21, J22);
    double detJ = J11 * J22 - J12 * J21;
    if (!jac_ok(detJ, J11, J12, J21, J22)) ok = false;
    double wgt = fabs(detJ), id = 1.0 / detJ;
    double iJ11 = J22 * id, iJ12 = -J12 * id, iJ21 = -J21 * id, iJ22 = J11 * id;
    double ratio = (iJ11 * iJ22 - iJ12 * iJ21) / (iJ11c * iJ22c - iJ12c * iJ21c);
    double p1x = ratio * iJ11c * (-2 * r), p1y = ratio * iJ21c * (-2 * r);
    double p2x = ratio * iJ12c * (-2 * sv), p2y = ratio * iJ22c * (-2 * sv);
    double gq = detJc / detJ;
    double b1x = (iJ11c * (-2 * r)) * gq, b1y = (iJ21c * (-2 * r)) * gq;
    double b2x = (iJ12c * (-2 * sv)) * gq, b2y = (iJ22c * (-2 * sv)) * gq;
    auto bi = [&](int q, double o[3]) {
      if (q == 0) { o[0] = p1x; o[1] = 0; o[2] = p1y; }
      else if (q == 1) { o[0] = 0; o[1] = p1y; o[2] = p1x; }
      else if (q == 2) { o[0] = p2x; o[1] = 0; o[2] = p2y; }
      else { o[0] = 0; o[1] = p2y; o[2] = p2x; }
    };
    auto bib = [&](int q, double o[3]) {
      if (q == 0) { o[0] = 0; o[1] = -b1y; o[2] = -b1x; }
      else if (q == 1) { o[0] = 0; o[1] = -b2y; o[2] = -b2x; }
      else if (q == 2) { o[0] = b1x; o[1] = 0; o[2] = b1y; }
      else { o[0] = b2x; o[1] = 0; o[2] = b2y; }
    };
    for (int l = 0; l < 16; ++l) {
      int i = l % 4, q = l / 4;
      double u[3], v[3];
      bi(i, u); bi(q, v);
      kbb[l] += wgt * qf3(u, Cm, v);
      bib(i, u); bib(q, v);
      kbbs[l] += wgt * qf3(u, shp, v);
      kbbb[l] += wgt * qf3(u, Cb, v);
    }
  }
  if (!ok) {
    record_error(err, EE_JACOBIAN, e);
    out[Q4P_STATUS] = 1.0;
    return;
  }
  double csmax = fmax(fmax(fabs(Cs[0]), fabs(Cs[1])), fmax(fabs(Cs[2]), fabs(Cs[3])));
  bool do_shear = !(h < 1e-30 || csmax < 1e-30);
  if (do_shear) {
    int st = macneal_operator(lc, Cb, Cs, out + Q4P_D, out + Q4P_SOL);
    if (st != 0) {
      record_error(err, EE_SHEAR + st, e);
      out[Q4P_STATUS] = 1.0;
      return;
    }
  }
  // drilling corners must have valid Jacobians
  const double alphaL = (k6rot * 1e-6) * Cm[8] * (4.0 * fabs(detJc));
  if (alphaL != 0.0) {
    const double cr[4] = {-1, 1, 1, -1}, cs4[4] = {-1, -1, 1, 1};
    for (int corner = 0; corner < 4; ++corner) {
      double dNr[4], dNs[4];
      shape_d(cr[corner], cs4[corner], dNr, dNs);
      double J11, J12, J21, J22;
      jac4(lc, dNr, dNs, J11, J12, J21, J22);
      if (!jac_ok(J11 * J22 - J12 * J21, J11, J12, J21, J22)) ok = false;
    }
    if (!ok) {
      record_error(err, EE_JACOBIAN, e);
      out[Q4P_STATUS] = 1.0;
      return;
    }
  }
  // enrichment inverses
  {
    double mx = 0, mb = 0;
    for (int i = 0; i < 16; ++i) { mx = fmax(mx, fabs(kbb[i])); mb = fmax(mb, fabs(kbbs[i])); }
    bool good = true;
    if (mx > 0) { if (!inv_small<4>(kbb, out + Q4P_CI)) good = false; }
    else for (int i = 0; i < 16; ++i) out[Q4P_CI + i] = 0.0;
    if (mb > 0) { if (!inv_small<4>(kbbs, out + Q4P_CI + 16)) good = false; }
    else for (int i = 0; i < 16; ++i) out[Q4P_CI + 16 + i] = 0.0;
    if (!good) {
      record_error(err, EE_ENRICH, e);
      out[Q4P_STATUS] = 1.0;
      return;
    }
  }
  for (int i = 0; i < 8; ++i) out[Q4P_LC + i] = lc[i];
  for (int a = 0; a < 3; ++a) { out[Q4P_V + a] = v1[a]; out[Q4P_V + 3 + a] = v2[a]; out[Q4P_V + 6 + a] = v3[a]; }
  for (int i = 0; i < 9; ++i) { out[Q4P_CM + i] = Cm[i]; out[Q4P_CB + i] = Cb[i]; }
  for (int i = 0; i < 4; ++i) out[Q4P_CS + i] = Cs[i];
  out[Q4P_SHP] = cmmax > 0 ? 1.0 : 0.0;
  out[Q4P_DETJC] = detJc;
  out[Q4P_IJC] = iJ11c; out[Q4P_IJC + 1] = iJ12c; out[Q4P_IJC + 2] = iJ21c; out[Q4P_IJC + 3] = iJ22c;
  out[Q4P_K6] = k6rot;
  out[Q4P_H] = h;
  out[Q4P_SHEAR] = do_shear ? 1.0 : 0.0;
  for (int i = 0; i < 16; ++i) { out[Q4P_KBB + i] = kbb[i]; out[Q4P_KBBB + i] = kbbb[i]; }
}

struct Q4Slab {
  double P[Q4P];
  double Kab[96], Kabs[96], Kabb[96];
  double Pm[96], Pb[96];
  double Ke[576];   // the element matrix, accumulated phase by phase (entry lane + 32 t owned by one lane)
  double T[36];
  double W[368];    // Gauss-point derivatives and right columns of the B matrices
};

__global__ void __launch_bounds__(WARPS * 32)
k_q4(int64_t n, const int32_t* __restrict__ nodes, const double* __restrict__ prep,
     const double* __restrict__ nodeR, double* __restrict__ ev) {
  extern __shared__ __align__(16) unsigned char q4smem[];   // WARPS slabs (above the 48 KB static limit)
  Q4Slab* slabs = reinterpret_cast<Q4Slab*>(q4smem);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t e = (int64_t)blockIdx.x * WARPS + w;
  if (e >= n) return;
  Q4Slab& S = slabs[w];
  const double* src = prep + Q4P * e;
  for (int i = lane; i < Q4P; i += 32) S.P[i] = src[i];
  __syncwarp();
  if (S.P[Q4P_STATUS] != 0.0) return;
  const double* lc = S.P + Q4P_LC;
  const double* Cm = S.P + Q4P_CM;
  const double* Cb = S.P + Q4P_CB;
  const double* shp = S.P[Q4P_SHP] != 0.0 ? Cm : Cb;
  const double detJc = S.P[Q4P_DETJC];
  const double iJ11c = S.P[Q4P_IJC], iJ12c = S.P[Q4P_IJC + 1], iJ21c = S.P[Q4P_IJC + 2], iJ22c = S.P[Q4P_IJC + 3];
  const double k6rot = S.P[Q4P_K6];
  // ---- membrane, bending and the incompatible-mode couplings at the four
  // Gauss points.  Lanes 0-3 prepare one point each: the shape derivatives
  // (dx, dy per node) and, for every column of the B matrices, w = wgt * C b
  // (membrane / bending columns of the 24 DOFs, the four incompatible modes);
  // an entry is then u_i . w_j summed over the points, u_i the left B column
  // (two nonzeros).
  double* GD = S.W;               // [g][8]: dx[4], dy[4]
  double* WM = S.W + 32;          // [g][8][3]: membrane column (node k, u/v) = 2k + c
  double* WB = WM + 96;           // [g][8][3]: bending column (node k, rx/ry) = 2k + c
  double* WI = WB + 96;           // [g][4][3]: Cm bi(q)
  double* WIS = WI + 48;          // [g][4][3]: shp bib(q)
  double* WIB = WIS + 48;         // [g][4][3]: Cb bib(q)
  if (lane < 4) {
    const double pt = 0.57735026918962573;
    const int g = lane;
    const double r = (g == 1 || g == 2) ? pt : -pt, s = (g >= 2) ? pt : -pt;
    double dNr[4], dNs[4];
    shape_d(r, s, dNr, dNs);
    double J11, J12, J21, J22;
    jac4(lc, dNr, dNs, J11, J12, J21, J22);
    const double detJ = J11 * J22 - J12 * J21;
    const double wgt = fabs(detJ), id = 1.0 / detJ;
    const double iJ11 = J22 * id, iJ12 = -J12 * id, iJ21 = -J21 * id, iJ22 = J11 * id;
    double dx[4], dy[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      dx[k] = iJ11 * dNr[k] + iJ12 * dNs[k];
      dy[k] = iJ21 * dNr[k] + iJ22 * dNs[k];
      GD[8 * g + k] = dx[k];
      GD[8 * g + 4 + k] = dy[k];
    }
    const double ratio = (iJ11 * iJ22 - iJ12 * iJ21) / (iJ11c * iJ22c - iJ12c * iJ21c);
    const double p1x = ratio * iJ11c * (-2 * r), p1y = ratio * iJ21c * (-2 * r);
    const double p2x = ratio * iJ12c * (-2 * s), p2y = ratio * iJ22c * (-2 * s);
    const double gq = detJc / detJ;
    const double b1x = (iJ11c * (-2 * r)) * gq, b1y = (iJ21c * (-2 * r)) * gq;
    const double b2x = (iJ12c * (-2 * s)) * gq, b2y = (iJ22c * (-2 * s)) * gq;
    // w = wgt * C v for a right column v
    auto cv = [&](const double* C, double v0, double v1, double v2, double* w) {
      w[0] = wgt * (C[0] * v0 + C[3] * v1 + C[6] * v2);
      w[1] = wgt * (C[1] * v0 + C[4] * v1 + C[7] * v2);
      w[2] = wgt * (C[2] * v0 + C[5] * v1 + C[8] * v2);
    };
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      cv(Cm, dx[k], 0.0, dy[k], WM + 24 * g + 3 * (2 * k));          // u
      cv(Cm, 0.0, dy[k], dx[k], WM + 24 * g + 3 * (2 * k + 1));      // v
      cv(Cb, 0.0, -dy[k], -dx[k], WB + 24 * g + 3 * (2 * k));        // rx
      cv(Cb, dx[k], 0.0, dy[k], WB + 24 * g + 3 * (2 * k + 1));      // ry
    }
    cv(Cm, p1x, 0.0, p1y, WI + 12 * g + 0);
    cv(Cm, 0.0, p1y, p1x, WI + 12 * g + 3);
    cv(Cm, p2x, 0.0, p2y, WI + 12 * g + 6);
    cv(Cm, 0.0, p2y, p2x, WI + 12 * g + 9);
    const double bib[4][3] = {{0.0, -b1y, -b1x}, {0.0, -b2y, -b2x}, {b1x, 0.0, b1y}, {b2x, 0.0, b2y}};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      cv(shp, bib[q][0], bib[q][1], bib[q][2], WIS + 12 * g + 3 * q);
      cv(Cb, bib[q][0], bib[q][1], bib[q][2], WIB + 12 * g + 3 * q);
    }
  }
  __syncwarp();
  // u_i . w over the four points; u_i of a membrane / bending row with two
  // nonzeros: u (dx, 0, dy), v (0, dy, dx), rx (0, -dy, -dx), ry (dx, 0, dy)
  auto udot = [&](int ci, int ki, const double* W, int stride) {
    double acc = 0.0;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      const double dxk = GD[8 * g + ki], dyk = GD[8 * g + 4 + ki];
      const double* w = W + stride * g;
      if (ci == 0 || ci == 4) acc += dxk * w[0] + dyk * w[2];
      else if (ci == 1) acc += dyk * w[1] + dxk * w[2];
      else acc -= dyk * w[1] + dxk * w[2];   // ci == 3
    }
    return acc;
  };
#pragma unroll 2
  for (int t = 0; t < 18; ++t) {
    const int idx = lane + 32 * t;
    const int i = idx % 24, j = idx / 24;
    const int ci = i % 6, cj = j % 6, ki = i / 6, kj = j / 6;
    double acc = 0.0;
    if (ci < 2 && cj < 2) acc = udot(ci, ki, WM + 3 * (2 * kj + cj), 24);
    else if ((ci == 3 || ci == 4) && (cj == 3 || cj == 4)) acc = udot(ci, ki, WB + 3 * (2 * kj + cj - 3), 24);
    S.Ke[idx] = acc;
  }
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    const int idx = lane + 32 * t;
    const int i = idx % 24, q = idx / 24;
    const int ci = i % 6, ki = i / 6;
    double kab = 0.0, kabs = 0.0, kabb = 0.0;
    if (ci < 2) kab = udot(ci, ki, WI + 3 * q, 12);
    if (ci == 3 || ci == 4) {
      kabs = udot(ci, ki, WIS + 3 * q, 12);
      kabb = udot(ci, ki, WIB + 3 * q, 12);
    }
    S.Kab[idx] = kab;
    S.Kabs[idx] = kabs;
    S.Kabb[idx] = kabb;
  }
  // ---- MacNeal shear term
  if (S.P[Q4P_SHEAR] != 0.0) {
    const double* D = S.P + Q4P_D;
    const double* sol = S.P + Q4P_SOL;
#pragma unroll 2
    for (int t = 0; t < 18; ++t) {
      int idx = lane + 32 * t;
      int i = idx % 24, j = idx / 24;
      int ci = i % 6, cj = j % 6;
      if (ci >= 2 && ci <= 4 && cj >= 2 && cj <= 4) {
        int ii = 3 * (i / 6) + ci - 2, jj = 3 * (j / 6) + cj - 2;
        double a = 0.0, b = 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          a += D[q + 4 * ii] * sol[q + 4 * jj];
          b += D[q + 4 * jj] * sol[q + 4 * ii];
        }
        S.Ke[idx] += 0.5 * (a + b);
      }
    }
  }
  // ---- lumped reference drilling
  const double alphaL = (k6rot * 1e-6) * Cm[8] * (4.0 * fabs(detJc));
  if (alphaL != 0.0) {
    const double cr[4] = {-1, 1, 1, -1}, cs[4] = {-1, -1, 1, 1};
    for (int corner = 0; corner < 4; ++corner) {
      double dNr[4], dNs[4];
      shape_d(cr[corner], cs[corner], dNr, dNs);
      double J11, J12, J21, J22;
      jac4(lc, dNr, dNs, J11, J12, J21, J22);
      double detJ = J11 * J22 - J12 * J21;
      double id = 1.0 / detJ;
      double iJ11 = J22 * id, iJ12 = -J12 * id, iJ21 = -J21 * id, iJ22 = J11 * id;
      double wc = alphaL * (fabs(detJ) / fmax(fabs(detJc), 1e-30));
      auto bd = [&](int i) {
        int k = i / 6, cc = i % 6;
        if (cc == 0) return 0.5 * (iJ21 * dNr[k] + iJ22 * dNs[k]);
        if (cc == 1) return -0.5 * (iJ11 * dNr[k] + iJ12 * dNs[k]);
        if (cc == 5 && k == corner) return 1.0;
        return 0.0;
      };
#pragma unroll 2
      for (int t = 0; t < 18; ++t) {
        int idx = lane + 32 * t;
        int i = idx % 24, j = idx / 24;
        double bi_ = bd(i);
        if (bi_ != 0.0) S.Ke[idx] += wc * (bi_ * bd(j));
      }
    }
  }
  // ---- section-kinematic enrichment
  __syncwarp();
  const double* Ci = S.P + Q4P_CI;
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    int idx = lane + 32 * t;      // (q, j) of a 4 x 24 map
    int q = idx % 4, j = idx / 4;
    double pm = 0.0, pb = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      pm -= Ci[q + 4 * k] * S.Kab[j + 24 * k];
      pb -= Ci[16 + q + 4 * k] * S.Kabs[j + 24 * k];
    }
    S.Pm[idx] = pm;
    S.Pb[idx] = pb;
  }
  __syncwarp();
  const double* Kbb = S.P + Q4P_KBB;
  const double* Kbbb = S.P + Q4P_KBBB;
#pragma unroll 1
  for (int t = 0; t < 18; ++t) {
    int idx = lane + 32 * t;
    int i = idx % 24, j = idx / 24;
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v += S.Kab[i + 24 * k] * S.Pm[k + 4 * j] + S.Pm[k + 4 * i] * S.Kab[j + 24 * k] +
           S.Kabb[i + 24 * k] * S.Pb[k + 4 * j] + S.Pb[k + 4 * i] * S.Kabb[j + 24 * k];
#pragma unroll
      for (int l = 0; l < 4; ++l)
        v += S.Pm[k + 4 * i] * Kbb[k + 4 * l] * S.Pm[l + 4 * j] +
             S.Pb[k + 4 * i] * Kbbb[k + 4 * l] * S.Pb[l + 4 * j];
    }
    S.Ke[idx] += v;
  }
  // ---- transform to the node DOF frames and emit
  if (lane < 4) {
    const double* R = nodeR + 9 * (int64_t)nodes[4 * e + lane];
    const double* V = S.P + Q4P_V;
    const double Rel[3][3] = {{V[0], V[1], V[2]}, {V[3], V[4], V[5]}, {V[6], V[7], V[8]}};
    for (int rr = 0; rr < 3; ++rr)
      for (int cc = 0; cc < 3; ++cc)
        S.T[9 * lane + rr + 3 * cc] =
            Rel[rr][0] * R[0 + 3 * cc] + Rel[rr][1] * R[1 + 3 * cc] + Rel[rr][2] * R[2 + 3 * cc];
  }
  __syncwarp();
  double* out = ev + 576 * e;
#pragma unroll
  for (int t = 0; t < 18; ++t) {
    int idx = lane + 32 * t;
    int I = idx % 24, J = idx / 24;
    int a = I / 6, pp = I % 6, sI = pp / 3, ip = pp % 3;
    int b = J / 6, qq = J % 6, sJ = qq / 3, jq = qq % 3;
    const double* Ta = S.T + 9 * a;
    const double* Tb = S.T + 9 * b;
    int r0 = 6 * a + 3 * sI, c0 = 6 * b + 3 * sJ;
    double sum = 0.0;
#pragma unroll
    for (int kk = 0; kk < 3; ++kk) {
      double tk = Ta[kk + 3 * ip];
      if (tk == 0.0) continue;
      double inner = 0.0;
#pragma unroll
      for (int ll = 0; ll < 3; ++ll) inner += S.Ke[(r0 + kk) + 24 * (c0 + ll)] * Tb[ll + 3 * jq];
      sum += tk * inner;
    }
    out[idx] = sum;
  }
}

constexpr size_t Q4_SMEM = WARPS * sizeof(Q4Slab);

// the warp pass's dynamic shared-memory limit, set once per device
jfg_status q4_attributes() {
  static bool done[64] = {};
  int dev = 0;
  JFG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return JFG_OK;
  if (!done[dev]) {
    JFG_CUDA(cudaFuncSetAttribute(k_q4, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Q4_SMEM));
    done[dev] = true;
  }
  return JFG_OK;
}

struct T10Slab {
  double K[900];
};

__global__ void __launch_bounds__(WARPS * 32)
k_t10(int64_t n, const int32_t* __restrict__ nodes, const double* __restrict__ mat,
      const double* __restrict__ xyz, const double* __restrict__ nodeR, int identity_R,
      double* __restrict__ ev, DevError* err) {
  __shared__ T10Slab slabs[WARPS];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t e = (int64_t)blockIdx.x * WARPS + w;
  if (e >= n) return;
  int nd[10];
  double X[10][3];
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    nd[k] = nodes[10 * e + k];
#pragma unroll
    for (int a = 0; a < 3; ++a) X[k][a] = xyz[3 * (int64_t)nd[k] + a];
  }
  const double E = mat[2 * e], nu = mat[2 * e + 1];
  if (!(isfinite(E) && E > 0 && isfinite(nu) && nu > -1 && nu < 0.5)) {
    if (lane == 0) record_error(err, EE_T10_MAT, e);
    return;
  }
  const double c = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
  const double lam = c * nu, mu = c * ((1.0 - 2.0 * nu) / 2.0);
  const double A = (5.0 + 3.0 * 2.23606797749978969) / 20.0, B = (5.0 - 2.23606797749978969) / 20.0;
  double acc[29];
#pragma unroll
  for (int t = 0; t < 29; ++t) acc[t] = 0.0;
  bool ok = true;
  for (int q = 0; q < 4; ++q) {
    double L1 = q == 1 ? A : B, L2 = q == 2 ? A : B, L3 = q == 3 ? A : B;
    double L[4] = {1.0 - L1 - L2 - L3, L1, L2, L3};
    const double dL[3][4] = {{-1, 1, 0, 0}, {-1, 0, 1, 0}, {-1, 0, 0, 1}};
    double dN[3][10];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int k = 0; k < 3; ++k) dN[k][i] = (4.0 * L[i] - 1.0) * dL[k][i];
    const int ed[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      int i = ed[m][0], j = ed[m][1];
#pragma unroll
      for (int k = 0; k < 3; ++k) dN[k][m + 4] = 4.0 * (L[j] * dL[k][i] + L[i] * dL[k][j]);
    }
    double J[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 10; ++k) s += dN[a][k] * X[k][b];
        J[a + 3 * b] = s;
      }
    double det = J[0] * (J[4] * J[8] - J[7] * J[5]) - J[3] * (J[1] * J[8] - J[7] * J[2]) +
                 J[6] * (J[1] * J[5] - J[4] * J[2]);
    if (!(isfinite(det) && det > 0.0)) { ok = false; break; }
    double id = 1.0 / det;
    double Ji[9];
    Ji[0] = (J[4] * J[8] - J[7] * J[5]) * id;
    Ji[3] = -(J[3] * J[8] - J[6] * J[5]) * id;
    Ji[6] = (J[3] * J[7] - J[6] * J[4]) * id;
    Ji[1] = -(J[1] * J[8] - J[7] * J[2]) * id;
    Ji[4] = (J[0] * J[8] - J[6] * J[2]) * id;
    Ji[7] = -(J[0] * J[7] - J[6] * J[1]) * id;
    Ji[2] = (J[1] * J[5] - J[4] * J[2]) * id;
    Ji[5] = -(J[0] * J[5] - J[3] * J[2]) * id;
    Ji[8] = (J[0] * J[4] - J[3] * J[1]) * id;
    double g[3][10];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int k = 0; k < 10; ++k) g[a][k] = Ji[a] * dN[0][k] + Ji[a + 3] * dN[1][k] + Ji[a + 6] * dN[2][k];
    double wgt = det / 24.0;
#pragma unroll
    for (int t = 0; t < 29; ++t) {
      int idx = lane + 32 * t;
      if (idx >= 900) break;
      int i = idx % 30, j = idx / 30;
      if (i > j) { int tt = i; i = j; j = tt; }   // Symmetric(K): upper triangle
      int I = i / 3, al = i % 3, Jn = j / 3, be = j % 3;
      double gg = g[0][I] * g[0][Jn] + g[1][I] * g[1][Jn] + g[2][I] * g[2][Jn];
      double v = lam * g[al][I] * g[be][Jn] + mu * ((al == be ? gg : 0.0) + g[be][I] * g[al][Jn]);
      acc[t] += wgt * v;
    }
  }
  if (!ok) {
    if (lane == 0) record_error(err, EE_T10_JAC, e);
    return;
  }
  double* out = ev + 900 * e;
  if (identity_R) {
#pragma unroll
    for (int t = 0; t < 29; ++t) {
      int idx = lane + 32 * t;
      if (idx < 900) out[idx] = acc[t];
    }
    return;
  }
  T10Slab& S = slabs[w];
#pragma unroll
  for (int t = 0; t < 29; ++t) {
    int idx = lane + 32 * t;
    if (idx < 900) S.K[idx] = acc[t];
  }
  __syncwarp();
#pragma unroll
  for (int t = 0; t < 29; ++t) {
    int idx = lane + 32 * t;
    if (idx >= 900) break;
    int I = idx % 30, J = idx / 30;
    int a = I / 3, ip = I % 3, b = J / 3, jq = J % 3;
    const double* Ra = nodeR + 9 * (int64_t)nd[a];
    const double* Rb = nodeR + 9 * (int64_t)nd[b];
    double sum = 0.0;
    for (int kk = 0; kk < 3; ++kk) {
      double inner = 0.0;
      for (int ll = 0; ll < 3; ++ll) inner += S.K[(3 * a + kk) + 30 * (3 * b + ll)] * Rb[ll + 3 * jq];
      sum += Ra[kk + 3 * ip] * inner;
    }
    out[idx] = sum;
  }
}


// ---------------------------------------------------------------------------
// CQUAD8 native shell (quad8_shell.jl:34-204; frame and congruences
// assembly.jl:5893-5915).  One CTA of 128 threads per element:
//   * thread 0: flat-parallelogram test, element frame, local coordinates;
//   * threads 0..24: shape functions, derivatives and Jacobians at the 25
//     points of the 2- and 3-point Gauss abscissas (every integration point
//     of the element is one of them);
//   * every thread owns 18 of the 48 x 48 entries and accumulates membrane
//     (2x2 plus the 3-point excess corrections), bending (2x2 with the twist
//     split and the 2x3 / 3x2 twist passes) and the shear term
//     Bs^T F^{-1} Bs (F: 8 x 8 sampled flexibility, inverted by thread 0);
//   * T^T K T with the element frame, symmetrisation, then the node_R
//     congruence, each as 9-term block sums out of shared memory.
// Section record: A (9), D (9), shear = G3 TS/T t, dref = D11, hasA, hasD.
constexpr int Q8_THREADS = 128;

__device__ __forceinline__ void q8_shape(double r, double s, double N[8], double dr[8], double ds[8]) {
  const double rc[4] = {-1, 1, 1, -1}, sc[4] = {-1, -1, 1, 1};
#pragma unroll
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

__device__ __forceinline__ double q8_norm3(const double* a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

struct Q8Point {
  double N[8], dx[8], dy[8], det, jac[4];
};

// membrane / curvature strain-displacement column p (3 components)
__device__ __forceinline__ void q8_bm(const Q8Point& P, int p, double b[3]) {
  int k = p / 6, c = p % 6;
  b[0] = (c == 0) ? P.dx[k] : 0.0;
  b[1] = (c == 1) ? P.dy[k] : 0.0;
  b[2] = (c == 0) ? P.dy[k] : (c == 1 ? P.dx[k] : 0.0);
}
__device__ __forceinline__ void q8_bb(const Q8Point& P, int p, double b[3]) {
  int k = p / 6, c = p % 6;
  b[0] = (c == 4) ? P.dx[k] : 0.0;
  b[1] = (c == 3) ? -P.dy[k] : 0.0;
  b[2] = (c == 4) ? P.dy[k] : (c == 3 ? -P.dx[k] : 0.0);
}
// b_p^T D b_q, D 3 x 3 column-major
__device__ __forceinline__ double q8_bdb(const double bp[3], const double* D, const double bq[3]) {
  double v = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double t = D[a] * bq[0] + D[a + 3] * bq[1] + D[a + 6] * bq[2];
    v += bp[a] * t;
  }
  return v;
}

__global__ void __launch_bounds__(Q8_THREADS)
k_q8(int64_t n, const int32_t* __restrict__ q8n, const double* __restrict__ q8s, const double* __restrict__ xyz,
     const double* __restrict__ nodeR, double* __restrict__ ev, DevError* __restrict__ err) {
  const int64_t e = blockIdx.x;
  if (e >= n) return;
  const int t = threadIdx.x;
  __shared__ double X[24], RN[72], S[22], xy[16], Rf[9];
  __shared__ Q8Point PT[25];
  __shared__ double Kl[48 * 48], W[48 * 48];
  __shared__ double Bs[8][48], Fi[64];
  double (*Y)[48] = reinterpret_cast<double (*)[48]>(W);   // W is free until the frame transform
  __shared__ int status;
  if (t < 24) X[t] = xyz[3 * (int64_t)q8n[8 * e + t / 3] + t % 3];
  if (t < 72) RN[t] = nodeR[9 * (int64_t)q8n[8 * e + t / 9] + t % 9];
  if (t < 22) S[t] = q8s[22 * e + t];
  if (t == 0) status = 0;
  __syncthreads();
  if (t == 0) {
    // flat parallelogram with mid-side nodes at the edge midpoints
    auto P = [&](int k, int a) { return X[3 * k + a]; };
    double d21[3], d41[3], tv[3];
    for (int a = 0; a < 3; ++a) { d21[a] = P(1, a) - P(0, a); d41[a] = P(3, a) - P(0, a); }
    double scale = fmax(q8_norm3(d21), q8_norm3(d41));
    bool ok = scale > 0;
    double lim = 1e-6 * scale;
    for (int a = 0; a < 3; ++a) tv[a] = P(0, a) + P(2, a) - P(1, a) - P(3, a);
    if (q8_norm3(tv) > lim) ok = false;
    const int mab[4][3] = {{4, 0, 1}, {5, 1, 2}, {6, 2, 3}, {7, 3, 0}};
    for (int q = 0; q < 4; ++q) {
      for (int a = 0; a < 3; ++a) tv[a] = P(mab[q][0], a) - (P(mab[q][1], a) + P(mab[q][2], a)) / 2;
      if (q8_norm3(tv) > lim) ok = false;
    }
    double nn[3] = {d21[1] * d41[2] - d21[2] * d41[1], d21[2] * d41[0] - d21[0] * d41[2],
                    d21[0] * d41[1] - d21[1] * d41[0]};
    if (!(q8_norm3(nn) > 1e-12 * scale * scale)) ok = false;
    if (!ok) {
      status = EE_Q8_SHAPE;
    } else {
      double gxi[3], geta[3], cen[3], ez[3], av[3], bv[3], ex[3], ey[3];
      for (int q = 0; q < 3; ++q) {
        gxi[q] = (P(1, q) + P(2, q) - P(0, q) - P(3, q)) / 4;
        geta[q] = (P(2, q) + P(3, q) - P(0, q) - P(1, q)) / 4;
        cen[q] = (P(0, q) + P(1, q) + P(2, q) + P(3, q)) / 4;
      }
      ez[0] = gxi[1] * geta[2] - gxi[2] * geta[1];
      ez[1] = gxi[2] * geta[0] - gxi[0] * geta[2];
      ez[2] = gxi[0] * geta[1] - gxi[1] * geta[0];
      double l = q8_norm3(ez);
      for (int q = 0; q < 3; ++q) ez[q] /= l;
      double lg = q8_norm3(gxi), le = q8_norm3(geta);
      for (int q = 0; q < 3; ++q) av[q] = gxi[q] / lg + geta[q] / le;
      l = q8_norm3(av);
      for (int q = 0; q < 3; ++q) av[q] /= l;
      bv[0] = ez[1] * av[2] - ez[2] * av[1];
      bv[1] = ez[2] * av[0] - ez[0] * av[2];
      bv[2] = ez[0] * av[1] - ez[1] * av[0];
      const double rs2 = sqrt(2.0);
      for (int q = 0; q < 3; ++q) { ex[q] = (av[q] - bv[q]) / rs2; ey[q] = (av[q] + bv[q]) / rs2; }
      for (int q = 0; q < 3; ++q) { Rf[q] = ex[q]; Rf[3 + q] = ey[q]; Rf[6 + q] = ez[q]; }
      for (int k = 0; k < 8; ++k) {
        double d[3] = {P(k, 0) - cen[0], P(k, 1) - cen[1], P(k, 2) - cen[2]};
        xy[k] = d[0] * ex[0] + d[1] * ex[1] + d[2] * ex[2];
        xy[k + 8] = d[0] * ey[0] + d[1] * ey[1] + d[2] * ey[2];
      }
    }
  }
  __syncthreads();
  if (status) {
    if (t == 0 && atomicCAS(&err->code, 0, status) == 0) err->index = e;
    return;
  }
  // shape data at the 25 points: abscissas {-1/sqrt3, 1/sqrt3, -sqrt0.6, 0, sqrt0.6}
  const double g5[5] = {-1.0 / sqrt(3.0), 1.0 / sqrt(3.0), -sqrt(0.6), 0.0, sqrt(0.6)};
  if (t < 25) {
    double r = g5[t / 5], sv = g5[t % 5];
    Q8Point& P = PT[t];
    double dr[8], ds[8];
    q8_shape(r, sv, P.N, dr, ds);
    double j11 = 0, j12 = 0, j21 = 0, j22 = 0;
    for (int k = 0; k < 8; ++k) {
      j11 += dr[k] * xy[k]; j12 += dr[k] * xy[k + 8];
      j21 += ds[k] * xy[k]; j22 += ds[k] * xy[k + 8];
    }
    double det = j11 * j22 - j12 * j21;
    for (int k = 0; k < 8; ++k) {
      P.dx[k] = (j22 * dr[k] - j12 * ds[k]) / det;
      P.dy[k] = (-j21 * dr[k] + j11 * ds[k]) / det;
    }
    P.det = det;
    P.jac[0] = j11; P.jac[1] = j12; P.jac[2] = j21; P.jac[3] = j22;
  }
  __syncthreads();
  const double* A = S;
  const double* Dm = S + 9;
  const double shear = S[18], dref = S[19];
  const bool hasA = S[20] != 0.0, hasD = S[21] != 0.0;
  const double w3[3] = {5.0 / 9, 8.0 / 9, 5.0 / 9};
  double acc[18];
#pragma unroll
  for (int u = 0; u < 18; ++u) acc[u] = 0.0;
  if (hasA) {
    for (int ir = 0; ir < 2; ++ir)
      for (int is = 0; is < 2; ++is) {
        const Q8Point& P = PT[ir * 5 + is];
#pragma unroll
        for (int u = 0; u < 18; ++u) {
          int ent = t + Q8_THREADS * u, p = ent % 48, q = ent / 48;
          double bp[3], bq[3];
          q8_bm(P, p, bp); q8_bm(P, q, bq);
          acc[u] += P.det * q8_bdb(bp, A, bq);
        }
      }
    // 3-point excess corrections of the normal membrane strains
    for (int row = 1; row <= 2; ++row) {
      const double modulus = row == 1 ? A[0] : A[4];
      for (int pass = 0; pass < 2; ++pass) {
        const double sign = pass == 0 ? 1.0 : -1.0;
        // row 1: r on 2 points, s on 3 (pass 0) or 2; row 2: r on 3 (pass 0) or 2, s on 2
        const bool r3 = (row == 2 && pass == 0), s3 = (row == 1 && pass == 0);
        const int nr = r3 ? 3 : 2, ns = s3 ? 3 : 2;
        for (int i = 0; i < nr; ++i)
          for (int j = 0; j < ns; ++j) {
            const int pr = r3 ? 2 + i : i, ps = s3 ? 2 + j : j;
            const double wr = r3 ? w3[i] : 1.0, ws = s3 ? w3[j] : 1.0;
            const Q8Point& P = PT[pr * 5 + ps];
            const double f = 0.25 * sign * wr * ws * P.det * modulus;
#pragma unroll
            for (int u = 0; u < 18; ++u) {
              int ent = t + Q8_THREADS * u, p = ent % 48, q = ent / 48;
              double vp = (p % 6 == row - 1) ? (row == 1 ? P.dx[p / 6] : P.dy[p / 6]) : 0.0;
              double vq = (q % 6 == row - 1) ? (row == 1 ? P.dx[q / 6] : P.dy[q / 6]) : 0.0;
              acc[u] += f * (vp * vq);
            }
          }
      }
    }
  }
  if (hasD) {
    double Dx[9] = {Dm[0], Dm[3], 0.0, Dm[3], Dm[4], 0.0, 0.0, 0.0, 4 * Dm[8]};
    for (int ir = 0; ir < 2; ++ir)
      for (int is = 0; is < 2; ++is) {
        const Q8Point& P = PT[ir * 5 + is];
#pragma unroll
        for (int u = 0; u < 18; ++u) {
          int ent = t + Q8_THREADS * u, p = ent % 48, q = ent / 48;
          double bp[3], bq[3];
          q8_bb(P, p, bp); q8_bb(P, q, bq);
          acc[u] += P.det * q8_bdb(bp, Dm, bq) - (2 * P.det) * q8_bdb(bp, Dx, bq);
        }
      }
    for (int pass = 0; pass < 2; ++pass) {
      const int nr = pass == 0 ? 2 : 3, ns = pass == 0 ? 3 : 2;
      for (int i = 0; i < nr; ++i)
        for (int j = 0; j < ns; ++j) {
          const int pr = pass == 0 ? i : 2 + i, ps = pass == 0 ? 2 + j : j;
          const double wr = pass == 0 ? 1.0 : w3[i], ws = pass == 0 ? w3[j] : 1.0;
          const Q8Point& P = PT[pr * 5 + ps];
          const double f = wr * ws * P.det;
#pragma unroll
          for (int u = 0; u < 18; ++u) {
            int ent = t + Q8_THREADS * u, p = ent % 48, q = ent / 48;
            double bp[3], bq[3];
            q8_bb(P, p, bp); q8_bb(P, q, bq);
            acc[u] += f * q8_bdb(bp, Dx, bq);
          }
        }
    }
    // transverse shear: sampled at the 2x2 points; flexibility from the last
    if (t == 0) {
      int st = 0;
      if (!(dref > 0)) st = EE_Q8_DREF;
      const Q8Point& P0 = PT[1 * 5 + 1];
      const double detJ0 = P0.det;
      const double rx = detJ0 / (P0.jac[0] * P0.jac[0]), ry = detJ0 / (P0.jac[3] * P0.jac[3]);
      const double pat[4][4] = {{1, 1, 1, 1}, {-1, -1, 1, 1}, {-1, 1, -1, 1}, {1, -1, -1, 1}};
      const double sx[4] = {12 * rx + 1200 * ry, 9.6 * rx, 12 * rx + 400 * ry, 12 * rx + 120 * ry};
      const double sy[4] = {12 * ry + 1200 * rx, 12 * ry + 400 * rx, 9.6 * ry, 12 * ry + 120 * rx};
      double F[64], M[64];
      for (int q = 0; q < 64; ++q) F[q] = 0.0;
      const double base = isfinite(shear) ? 1 / (shear * detJ0) : 0.0;
      for (int q = 0; q < 8; ++q) F[q + 8 * q] = base;
      for (int comp = 1; comp <= 2; ++comp)
        for (int k = 0; k < 4; ++k) {
          double stiff = comp == 1 ? sx[k] : sy[k];
          double f = 1 / (stiff * dref) / 4;
          for (int aa = 0; aa < 4; ++aa)
            for (int cc = 0; cc < 4; ++cc)
              F[(2 * aa + comp - 1) + 8 * (2 * cc + comp - 1)] += f * pat[k][aa] * pat[k][cc];
        }
      // Gauss-Jordan with partial pivoting
      for (int q = 0; q < 64; ++q) { M[q] = F[q]; Fi[q] = (q % 9 == 0) ? 1.0 : 0.0; }
      for (int k = 0; k < 8 && !st; ++k) {
        int pv = k;
        double best = fabs(M[k + 8 * k]);
        for (int i = k + 1; i < 8; ++i)
          if (fabs(M[i + 8 * k]) > best) { best = fabs(M[i + 8 * k]); pv = i; }
        if (best == 0.0 || !isfinite(best)) { st = EE_Q8_SINGULAR; break; }
        if (pv != k)
          for (int j = 0; j < 8; ++j) {
            double a = M[k + 8 * j]; M[k + 8 * j] = M[pv + 8 * j]; M[pv + 8 * j] = a;
            double b = Fi[k + 8 * j]; Fi[k + 8 * j] = Fi[pv + 8 * j]; Fi[pv + 8 * j] = b;
          }
        double piv = M[k + 8 * k];
        for (int j = 0; j < 8; ++j) { M[k + 8 * j] /= piv; Fi[k + 8 * j] /= piv; }
        for (int i = 0; i < 8; ++i) {
          if (i == k) continue;
          double f = M[i + 8 * k];
          if (f == 0.0) continue;
          for (int j = 0; j < 8; ++j) { M[i + 8 * j] -= f * M[k + 8 * j]; Fi[i + 8 * j] -= f * Fi[k + 8 * j]; }
        }
      }
      status = st;
    }
    // Bs (8 x 48): sample s = 2 ir + is, rows 2s (dx, N on w, theta_y) and 2s+1 (dy, -N on theta_x)
    for (int q = t; q < 8 * 48; q += Q8_THREADS) {
      int a = q / 48, col = q % 48, smp = a / 2, k = col / 6, c = col % 6;
      const Q8Point& P = PT[(smp / 2) * 5 + (smp % 2)];
      double v = 0.0;
      if (a % 2 == 0) v = (c == 2) ? P.dx[k] : (c == 4 ? P.N[k] : 0.0);
      else v = (c == 2) ? P.dy[k] : (c == 3 ? -P.N[k] : 0.0);
      Bs[a][col] = v;
    }
    __syncthreads();
    if (status) {
      if (t == 0 && atomicCAS(&err->code, 0, status) == 0) err->index = e;
      return;
    }
    for (int q = t; q < 8 * 48; q += Q8_THREADS) {
      int a = q / 48, col = q % 48;
      double v = 0.0;
      for (int b = 0; b < 8; ++b) v += Fi[a + 8 * b] * Bs[b][col];
      Y[a][col] = v;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 18; ++u) {
      int ent = t + Q8_THREADS * u, p = ent % 48, q = ent / 48;
      double v = 0.0;
      for (int a = 0; a < 8; ++a) v += Bs[a][p] * Y[a][q];
      acc[u] += v;
    }
  }
#pragma unroll
  for (int u = 0; u < 18; ++u) Kl[t + Q8_THREADS * u] = acc[u];
  __syncthreads();
  // K = T^T Kl T, T block-diagonal with T(c + a, c + b) = e_a[b] (element axes)
#pragma unroll
  for (int u = 0; u < 18; ++u) {
    int ent = t + Q8_THREADS * u, i = ent % 48, j = ent / 48;
    int ci = i - i % 3, cj = j - j % 3;
    double v = 0.0;
    for (int a = 0; a < 3; ++a) {
      double ta = Rf[(i - ci) + 3 * a];
      double row = 0.0;
      for (int b = 0; b < 3; ++b) row += Kl[(ci + a) + 48 * (cj + b)] * Rf[(j - cj) + 3 * b];
      v += ta * row;
    }
    W[ent] = v;
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < 18; ++u) {
    int ent = t + Q8_THREADS * u, i = ent % 48, j = ent / 48;
    Kl[ent] = (W[i + 48 * j] + W[j + 48 * i]) / 2;
  }
  __syncthreads();
  // node_R congruence: Tn(r0 + a, r0 + b) = R_node(a, b)
  double* out = ev + 2304 * e;
#pragma unroll
  for (int u = 0; u < 18; ++u) {
    int ent = t + Q8_THREADS * u, i = ent % 48, j = ent / 48;
    int ci = i - i % 3, cj = j - j % 3;
    const double* Ri = RN + 9 * (i / 6);
    const double* Rj = RN + 9 * (j / 6);
    double v = 0.0;
    for (int a = 0; a < 3; ++a) {
      double ta = Ri[a + 3 * (i - ci)];
      double row = 0.0;
      for (int b = 0; b < 3; ++b) row += Kl[(ci + a) + 48 * (cj + b)] * Rj[b + 3 * (j - cj)];
      v += ta * row;
    }
    out[ent] = v;
  }
}

}  // namespace

jfg_status launch_q4_prep(const jfg_model* m, cudaStream_t st) {
  if (m->n_q4 == 0) return JFG_OK;
  k_q4_prep<<<(unsigned)((m->n_q4 + 127) / 128), 128, 0, st>>>(m->n_q4, m->d_q4n, m->d_q4s, m->d_xyz, m->d_q4prep,
                                                                m->d_err);
  count_launch();
  JFG_CUDA(cudaGetLastError());
  return JFG_OK;
}

jfg_status launch_elements(jfg_model* m, cudaStream_t st) {
  if (m->n_q4 > 0) {
    JFG_TRY(q4_attributes());
    int64_t blocks = (m->n_q4 + WARPS - 1) / WARPS;
    int ps = prof_start(st);
    { k_q4_prep<<<(unsigned)((m->n_q4 + 127) / 128), 128, 0, st>>>(m->n_q4, m->d_q4n, m->d_q4s, m->d_xyz,
                                                                 m->d_q4prep, m->d_err); count_launch(); }
    { k_q4<<<(unsigned)blocks, WARPS * 32, Q4_SMEM, st>>>(m->n_q4, m->d_q4n, m->d_q4prep, m->d_R, m->d_ev);
      count_launch(); }
    // algorithmic bytes: connectivity + section in, matrix out, coordinates once
    prof_end(ps, st, KS_Q4, (double)m->n_q4 * (16 + 8 * 26 + 8 * 576) + 24.0 * m->n_nodes);
    JFG_CUDA(cudaGetLastError());
  }
  if (m->n_t10 > 0) {
    bool ident = true;
    for (int64_t i = 0; i < m->n_nodes && ident; ++i) {
      const double* R = m->h_R.data() + 9 * i;
      ident = R[0] == 1 && R[4] == 1 && R[8] == 1 && R[1] == 0 && R[2] == 0 && R[3] == 0 &&
              R[5] == 0 && R[6] == 0 && R[7] == 0;
    }
    int ps = prof_start(st);
    int64_t blocks = (m->n_t10 + WARPS - 1) / WARPS;
    { k_t10<<<(unsigned)blocks, WARPS * 32, 0, st>>>(m->n_t10, m->d_t10n, m->d_t10m, m->d_xyz, m->d_R,
                                                  ident ? 1 : 0, m->d_ev + m->ev_t10_off, m->d_err); count_launch(); }
    prof_end(ps, st, KS_T10, (double)m->n_t10 * (40 + 16 + 8 * 900) + 24.0 * m->n_nodes);
    JFG_CUDA(cudaGetLastError());
  }
  if (m->n_q8 > 0) {
    int ps = prof_start(st);
    { k_q8<<<(unsigned)m->n_q8, Q8_THREADS, 0, st>>>(m->n_q8, m->d_q8n, m->d_q8s, m->d_xyz, m->d_R,
                                                   m->d_ev + m->ev_q8_off, m->d_err); count_launch(); }
    prof_end(ps, st, KS_T10, (double)m->n_q8 * (32 + 8 * 22 + 8 * 2304) + 24.0 * m->n_nodes);
    JFG_CUDA(cudaGetLastError());
  }
  if (m->n_t3 > 0) {
    int ps = prof_start(st);
    JFG_TRY(launch_t3(m, st, m->d_ev + m->ev_t3_off, m->d_err));
    prof_end(ps, st, KS_Q4, (double)m->n_t3 * (12 + 8 * 26 + 8 * 324) + 24.0 * m->n_nodes);
  }
  return JFG_OK;
}

// Same element kernels as launch_elements, writing the element matrices to
// `ev` (n_ev doubles), the CQUAD4 prep records to `q4prep` (n_q4 x
// Q4_PREP_STRIDE doubles) and the first element error to `err` instead of
// the model's own buffers; no profiling events.
jfg_status launch_elements_into(const jfg_model* m, cudaStream_t st, double* ev, double* q4prep, DevError* err) {
  if (m->n_q4 > 0) {
    JFG_TRY(q4_attributes());
    int64_t blocks = (m->n_q4 + WARPS - 1) / WARPS;
    { k_q4_prep<<<(unsigned)((m->n_q4 + 127) / 128), 128, 0, st>>>(m->n_q4, m->d_q4n, m->d_q4s, m->d_xyz, q4prep,
                                                                 err); count_launch(); }
    { k_q4<<<(unsigned)blocks, WARPS * 32, Q4_SMEM, st>>>(m->n_q4, m->d_q4n, q4prep, m->d_R, ev); count_launch(); }
    JFG_CUDA(cudaGetLastError());
  }
  if (m->n_t10 > 0) {
    bool ident = true;
    for (int64_t i = 0; i < m->n_nodes && ident; ++i) {
      const double* R = m->h_R.data() + 9 * i;
      ident = R[0] == 1 && R[4] == 1 && R[8] == 1 && R[1] == 0 && R[2] == 0 && R[3] == 0 &&
              R[5] == 0 && R[6] == 0 && R[7] == 0;
    }
    int64_t blocks = (m->n_t10 + WARPS - 1) / WARPS;
    { k_t10<<<(unsigned)blocks, WARPS * 32, 0, st>>>(m->n_t10, m->d_t10n, m->d_t10m, m->d_xyz, m->d_R,
                                                  ident ? 1 : 0, ev + m->ev_t10_off, err);
      count_launch(); }
    JFG_CUDA(cudaGetLastError());
  }
  if (m->n_q8 > 0) {
    { k_q8<<<(unsigned)m->n_q8, Q8_THREADS, 0, st>>>(m->n_q8, m->d_q8n, m->d_q8s, m->d_xyz, m->d_R,
                                                   ev + m->ev_q8_off, err); count_launch(); }
    JFG_CUDA(cudaGetLastError());
  }
  JFG_TRY(launch_t3(m, st, ev + m->ev_t3_off, err));
  return JFG_OK;
}

}  // namespace jfg
