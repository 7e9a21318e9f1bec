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

struct Q4Slab {
  double Kab[96], Kbb[16], Kabs[96], Kbbs[16], Kabb[96], Kbbb[16];
  double D[48], sol[48], Ci[32];
  double Pm[96], Pb[96];
  double Ke[576];
  double T[36];
  int status;
};

// MacNeal shear operator D (4 x 12) and sol = Z^-1 D; single lane.
__device__ int macneal_operator(const double lc[8], const double* Cb, const double* Cs, Q4Slab& S) {
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
  double* D = S.D;
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
      S.sol[i + 4 * j] = s;
    }
  return 0;
}

__global__ void __launch_bounds__(WARPS * 32)
k_q4(int64_t n, const int32_t* __restrict__ nodes, const double* __restrict__ sect,
     const double* __restrict__ xyz, const double* __restrict__ nodeR, double* __restrict__ ev,
     DevError* err) {
  __shared__ Q4Slab slabs[WARPS];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t e = (int64_t)blockIdx.x * WARPS + w;
  if (e >= n) return;
  Q4Slab& S = slabs[w];
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
    if (lane == 0) record_error(err, EE_NOT_FLAT, e);
    return;
  }
  if (sc[25] != 0.0) {
    if (lane == 0) record_error(err, EE_FLAGS, e);
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
  // ---- center Jacobian
  const double dNr_c[4] = {-0.25, 0.25, 0.25, -0.25}, dNs_c[4] = {-0.25, -0.25, 0.25, 0.25};
  double J11c, J12c, J21c, J22c;
  jac4(lc, dNr_c, dNs_c, J11c, J12c, J21c, J22c);
  const double detJc = J11c * J22c - J12c * J21c;
  const double idc = 1.0 / detJc;
  const double iJ11c = J22c * idc, iJ12c = -J12c * idc, iJ21c = -J21c * idc, iJ22c = J11c * idc;
  // ---- owned accumulators
  double ke[18], kab[3], kabs[3], kabb[3], kbb = 0, kbbs = 0, kbbb = 0;
#pragma unroll
  for (int t = 0; t < 18; ++t) ke[t] = 0.0;
#pragma unroll
  for (int t = 0; t < 3; ++t) { kab[t] = 0.0; kabs[t] = 0.0; kabb[t] = 0.0; }
  const double pt = 0.57735026918962573;
  const double gr[4] = {-pt, pt, pt, -pt}, gs[4] = {-pt, -pt, pt, pt};
  bool ok = true;
  for (int g = 0; g < 4; ++g) {
    double r = gr[g], s = gs[g];
    double dNr[4], dNs[4];
    shape_d(r, s, dNr, dNs);
    double J11, J12, J21, J22;
    jac4(lc, dNr, dNs, J11, J12, J21, J22);
    double detJ = J11 * J22 - J12 * J21;
    if (!jac_ok(detJ, J11, J12, J21, J22)) ok = false;
    double wgt = fabs(detJ), id = 1.0 / detJ;
    double iJ11 = J22 * id, iJ12 = -J12 * id, iJ21 = -J21 * id, iJ22 = J11 * id;
    double dx[4], dy[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      dx[k] = iJ11 * dNr[k] + iJ12 * dNs[k];
      dy[k] = iJ21 * dNr[k] + iJ22 * dNs[k];
    }
    double ratio = (iJ11 * iJ22 - iJ12 * iJ21) / (iJ11c * iJ22c - iJ12c * iJ21c);
    double p1x = ratio * iJ11c * (-2 * r), p1y = ratio * iJ21c * (-2 * r);
    double p2x = ratio * iJ12c * (-2 * s), p2y = ratio * iJ22c * (-2 * s);
    double gq = detJc / detJ;
    double b1x = (iJ11c * (-2 * r)) * gq, b1y = (iJ21c * (-2 * r)) * gq;
    double b2x = (iJ12c * (-2 * s)) * gq, b2y = (iJ22c * (-2 * s)) * gq;
    auto bm = [&](int i, double o[3]) {
      int k = i / 6, cc = i % 6;
      o[0] = o[1] = o[2] = 0.0;
      if (cc == 0) { o[0] = dx[k]; o[2] = dy[k]; }
      else if (cc == 1) { o[1] = dy[k]; o[2] = dx[k]; }
    };
    auto bb = [&](int i, double o[3]) {
      int k = i / 6, cc = i % 6;
      o[0] = o[1] = o[2] = 0.0;
      if (cc == 4) { o[0] = dx[k]; o[2] = dy[k]; }
      else if (cc == 3) { o[1] = -dy[k]; o[2] = -dx[k]; }
    };
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
#pragma unroll
    for (int t = 0; t < 18; ++t) {
      int idx = lane + 32 * t;
      int i = idx % 24, j = idx / 24;
      int ci = i % 6, cj = j % 6;
      double acc = 0.0;
      if (ci < 2 && cj < 2) {
        double u[3], v[3];
        bm(i, u); bm(j, v);
        acc += qf3(u, Cm, v);
      }
      if ((ci == 3 || ci == 4) && (cj == 3 || cj == 4)) {
        double u[3], v[3];
        bb(i, u); bb(j, v);
        acc += qf3(u, Cb, v);
      }
      ke[t] += wgt * acc;
    }
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      int idx = lane + 32 * t;
      int i = idx % 24, q = idx / 24;
      int ci = i % 6;
      double u[3], v[3];
      if (ci < 2) { bm(i, u); bi(q, v); kab[t] += wgt * qf3(u, Cm, v); }
      if (ci == 3 || ci == 4) {
        bb(i, u); bib(q, v);
        kabs[t] += wgt * qf3(u, shp, v);
        kabb[t] += wgt * qf3(u, Cb, v);
      }
    }
    if (lane < 16) {
      int i = lane % 4, q = lane / 4;
      double u[3], v[3];
      bi(i, u); bi(q, v);
      kbb += wgt * qf3(u, Cm, v);
      bib(i, u); bib(q, v);
      kbbs += wgt * qf3(u, shp, v);
      kbbb += wgt * qf3(u, Cb, v);
    }
  }
  if (!ok) {
    if (lane == 0) record_error(err, EE_JACOBIAN, e);
    return;
  }
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    S.Kab[lane + 32 * t] = kab[t];
    S.Kabs[lane + 32 * t] = kabs[t];
    S.Kabb[lane + 32 * t] = kabb[t];
  }
  if (lane < 16) { S.Kbb[lane] = kbb; S.Kbbs[lane] = kbbs; S.Kbbb[lane] = kbbb; }
  // ---- MacNeal shear operator (lane 0), needs only lc/Cb/Cs
  double csmax = fmax(fmax(fabs(Cs[0]), fabs(Cs[1])), fmax(fabs(Cs[2]), fabs(Cs[3])));
  bool do_shear = !(h < 1e-30 || csmax < 1e-30);
  if (lane == 0) S.status = do_shear ? macneal_operator(lc, Cb, Cs, S) : 0;
  __syncwarp();
  if (S.status != 0) {
    if (lane == 0) record_error(err, EE_SHEAR + S.status, e);
    return;
  }
  if (do_shear) {
#pragma unroll
    for (int t = 0; t < 18; ++t) {
      int idx = lane + 32 * t;
      int i = idx % 24, j = idx / 24;
      int ci = i % 6, cj = j % 6;
      if (ci >= 2 && ci <= 4 && cj >= 2 && cj <= 4) {
        int ii = 3 * (i / 6) + ci - 2, jj = 3 * (j / 6) + cj - 2;
        double a = 0.0, b = 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          a += S.D[q + 4 * ii] * S.sol[q + 4 * jj];
          b += S.D[q + 4 * jj] * S.sol[q + 4 * ii];
        }
        ke[t] += 0.5 * (a + b);
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
      if (!jac_ok(detJ, J11, J12, J21, J22)) ok = false;
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
#pragma unroll
      for (int t = 0; t < 18; ++t) {
        int idx = lane + 32 * t;
        int i = idx % 24, j = idx / 24;
        double bi_ = bd(i);
        if (bi_ != 0.0) ke[t] += wc * (bi_ * bd(j));
      }
    }
    if (!ok) {
      if (lane == 0) record_error(err, EE_JACOBIAN, e);
      return;
    }
  }
  // ---- section-kinematic enrichment
  __syncwarp();
  if (lane == 0) {
    double mx = 0, mb = 0;
    for (int i = 0; i < 16; ++i) { mx = fmax(mx, fabs(S.Kbb[i])); mb = fmax(mb, fabs(S.Kbbs[i])); }
    int st = 0;
    if (mx > 0) { if (!inv_small<4>(S.Kbb, S.Ci)) st = 1; }
    else for (int i = 0; i < 16; ++i) S.Ci[i] = 0.0;
    if (mb > 0) { if (!inv_small<4>(S.Kbbs, S.Ci + 16)) st = 1; }
    else for (int i = 0; i < 16; ++i) S.Ci[16 + i] = 0.0;
    S.status = st;
  }
  __syncwarp();
  if (S.status != 0) {
    if (lane == 0) record_error(err, EE_ENRICH, e);
    return;
  }
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    int idx = lane + 32 * t;      // (q, j) of a 4 x 24 map
    int q = idx % 4, j = idx / 4;
    double pm = 0.0, pb = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      pm -= S.Ci[q + 4 * k] * S.Kab[j + 24 * k];
      pb -= S.Ci[16 + q + 4 * k] * S.Kabs[j + 24 * k];
    }
    S.Pm[idx] = pm;
    S.Pb[idx] = pb;
  }
  __syncwarp();
#pragma unroll
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
        v += S.Pm[k + 4 * i] * S.Kbb[k + 4 * l] * S.Pm[l + 4 * j] +
             S.Pb[k + 4 * i] * S.Kbbb[k + 4 * l] * S.Pb[l + 4 * j];
    }
    ke[t] += v;
  }
  // ---- transform to the node DOF frames and emit
#pragma unroll
  for (int t = 0; t < 18; ++t) S.Ke[lane + 32 * t] = ke[t];
  if (lane < 4) {
    const double* R = nodeR + 9 * (int64_t)nd[lane];
    const double Rel[3][3] = {{v1[0], v1[1], v1[2]}, {v2[0], v2[1], v2[2]}, {v3[0], v3[1], v3[2]}};
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

}  // namespace

jfg_status launch_elements(jfg_model* m, cudaStream_t st) {
  if (m->n_q4 > 0) {
    int64_t blocks = (m->n_q4 + WARPS - 1) / WARPS;
    int ps = prof_start(st);
    { k_q4<<<(unsigned)blocks, WARPS * 32, 0, st>>>(m->n_q4, m->d_q4n, m->d_q4s, m->d_xyz, m->d_R,
                                                 m->d_ev, m->d_err); count_launch(); }
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
    set_error("CQUAD8 device kernel not built into this library version");
    return JFG_UNSUPPORTED;
  }
  return JFG_OK;
}

// Same element kernels as launch_elements, writing the element matrices to
// `ev` (n_ev doubles) and the first element error to `err` instead of the
// model's own buffers; no profiling events.
jfg_status launch_elements_into(const jfg_model* m, cudaStream_t st, double* ev, DevError* err) {
  if (m->n_q8 > 0) {
    set_error("CQUAD8 device kernel not built into this library version");
    return JFG_UNSUPPORTED;
  }
  if (m->n_q4 > 0) {
    int64_t blocks = (m->n_q4 + WARPS - 1) / WARPS;
    { k_q4<<<(unsigned)blocks, WARPS * 32, 0, st>>>(m->n_q4, m->d_q4n, m->d_q4s, m->d_xyz, m->d_R, ev, err);
      count_launch(); }
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
  return JFG_OK;
}

}  // namespace jfg
