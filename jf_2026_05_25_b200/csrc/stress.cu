// stress.cu -- element stress and strain recovery from the displacement
// fields of a solve (the recovery step of _build_results_from_state,
// src/solver/solve_case.jl:182-303).
//
// CTETRA10 (recover_solid_stresses!, src/solver/stress_recovery.jl:1823-1960):
// one thread per element and load case.  The element's displacements are its
// nodes' translations rotated to the basic frame (node_R * u); B is taken at
// the centroid (solid_centroid_B_tetra10, src/tetra10.jl:110-115); strain =
// B u with engineering shears (xy, yz, zx), stress = D strain for the
// isotropic law, von Mises from the six components (stress_solid_3d,
// src/FEMKernels.jl:13067-13074).  Output per element and load case: 13
// doubles, stored load-case major so that the threads of a warp write one
// contiguous run.
//
// CQUAD4 (recover_shell_stresses!, stress_recovery.jl:505-1237 with n == 4,
// on the default isotropic PSHELL path: flat, no offset, no SNORM, no
// thermal load): one thread per element and load case.  The element frame,
// corner coordinates and MacNeal shear operator come from the element's
// prep record (k_q4_prep, refreshed first); the displacements are rotated
// to the element frame ((Rel * node_R) u, :774-781).  Centre fields follow
// stress_strain_quad4's default branch (FEMKernels.jl:6794-6978): the four
// Wilson membrane modes (patch-consistent Jacobian, FEMKernels.jl:1847-1895)
// are condensed with Cm, alpha = -K_bb^-1 sum_g w_g Bi_g^T Cm (Bm_g u), and
// eps and kappa are the area-weighted means over the 2 x 2 Gauss points;
// N = Cm eps, M = -Cb kappa, fibre stresses D (eps -+ h/2 kappa) with
// D = Cm / h.  Q is the area-mean MacNeal shear resultant
// (FEMKernels.jl:6623-6646: rows theta_y and theta_x of D^T Z^-1 D u summed
// over the corners, over 4 |det J(0)|), which replaces the centre shear on
// this path (stress_recovery.jl:248-292, :917-927).  Output per element and
// load case: 31 doubles (fx fy fxy mx my mxy qx qy; fibre -h/2 and +h/2:
// sx sy txy von Mises major minor; membrane strain ex ey gxy major minor;
// -kappa, same layout; the major principal stress at -h/2).  Elements the
// stiffness pass refused get NaN records.
#include "jfg_internal.h"

namespace jfg {
namespace {

constexpr int T10_REC = 13;

__global__ void __launch_bounds__(256)
k_t10_stress(int64_t n, int nrhs, const int32_t* __restrict__ nodes, const double* __restrict__ mat,
             const double* __restrict__ xyz, const double* __restrict__ nodeR, const double* __restrict__ U,
             int64_t ldu, double* __restrict__ out, DevError* err) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nrhs) return;
  const int64_t e = t % n;
  const int k = (int)(t / n);
  int nd[10];
#pragma unroll
  for (int i = 0; i < 10; ++i) nd[i] = nodes[10 * e + i];
  const double E = mat[2 * e], nu = mat[2 * e + 1];
  if (!(isfinite(E) && E > 0 && isfinite(nu) && nu > -1 && nu < 0.5)) {
    if (atomicCAS(&err->code, 0, (int32_t)EE_T10_MAT) == 0) err->index = e;
    return;
  }
  // shape-function derivatives at the centroid: L_i = 1/4, so the corner
  // terms (4 L_i - 1) vanish and every edge term is 4 (L_j dL_i + L_i dL_j)
  const double dL[3][4] = {{-1, 1, 0, 0}, {-1, 0, 1, 0}, {-1, 0, 0, 1}};
  const int ed[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
  double dN[3][10];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int a = 0; a < 3; ++a) dN[a][i] = (4.0 * 0.25 - 1.0) * dL[a][i];
#pragma unroll
  for (int q = 0; q < 6; ++q)
#pragma unroll
    for (int a = 0; a < 3; ++a) dN[a][q + 4] = 4.0 * (0.25 * dL[a][ed[q][0]] + 0.25 * dL[a][ed[q][1]]);
  double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double u[10][3];
  const double* Uk = U + ldu * k;
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const int64_t g = nd[i];
    const double x0 = xyz[3 * g], x1 = xyz[3 * g + 1], x2 = xyz[3 * g + 2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      J[a] += dN[a][i] * x0;
      J[a + 3] += dN[a][i] * x1;
      J[a + 6] += dN[a][i] * x2;
    }
    const double* R = nodeR + 9 * g;
    const double v0 = Uk[6 * g], v1 = Uk[6 * g + 1], v2 = Uk[6 * g + 2];
#pragma unroll
    for (int a = 0; a < 3; ++a) u[i][a] = R[a] * v0 + R[a + 3] * v1 + R[a + 6] * v2;
  }
  const double det = J[0] * (J[4] * J[8] - J[7] * J[5]) - J[3] * (J[1] * J[8] - J[7] * J[2]) +
                     J[6] * (J[1] * J[5] - J[4] * J[2]);
  if (!(isfinite(det) && det > 0.0)) {
    if (atomicCAS(&err->code, 0, (int32_t)EE_T10_JAC) == 0) err->index = e;
    return;
  }
  const double id = 1.0 / det;
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
  double eps[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const double gx = Ji[0] * dN[0][i] + Ji[3] * dN[1][i] + Ji[6] * dN[2][i];
    const double gy = Ji[1] * dN[0][i] + Ji[4] * dN[1][i] + Ji[7] * dN[2][i];
    const double gz = Ji[2] * dN[0][i] + Ji[5] * dN[1][i] + Ji[8] * dN[2][i];
    eps[0] += gx * u[i][0];
    eps[1] += gy * u[i][1];
    eps[2] += gz * u[i][2];
    eps[3] += gy * u[i][0] + gx * u[i][1];
    eps[4] += gz * u[i][1] + gy * u[i][2];
    eps[5] += gz * u[i][0] + gx * u[i][2];
  }
  const double c = E / ((1.0 + nu) * (1.0 - 2.0 * nu)), d = 1.0 - nu, sh = (1.0 - 2.0 * nu) / 2.0;
  double sg[6];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) s += (i == j ? c * d : c * nu) * eps[j];
    sg[i] = s;
  }
#pragma unroll
  for (int i = 3; i < 6; ++i) sg[i] = c * sh * eps[i];
  const double vm = sg[0] * sg[0] + sg[1] * sg[1] + sg[2] * sg[2] - sg[0] * sg[1] - sg[1] * sg[2] -
                    sg[2] * sg[0] + 3.0 * (sg[3] * sg[3] + sg[4] * sg[4] + sg[5] * sg[5]);
  double* o = out + T10_REC * t;
#pragma unroll
  for (int i = 0; i < 6; ++i) { o[i] = sg[i]; o[6 + i] = eps[i]; }
  o[12] = sqrt(fmax(0.0, vm));
}

constexpr int Q4_REC = 31;

// principal values of a 2-D symmetric tensor without cancellation
// (_recovery_principal_2d, stress_recovery.jl:17-34)
__device__ void principal2(double xx, double yy, double xy, double& major, double& minor) {
  if (xy == 0.0) {
    major = fmax(xx, yy);
    minor = fmin(xx, yy);
    return;
  }
  const double scale = fmax(fmax(fabs(xx), fabs(yy)), fabs(xy));
  const double a = xx / scale, b = yy / scale, c = xy / scale;
  const double mean = (a + b) / 2, radius = hypot((a - b) / 2, c);
  const double large = (mean + copysign(radius, mean)) * scale;
  if (!isfinite(large)) {
    major = (mean + radius) * scale;
    minor = (mean - radius) * scale;
    return;
  }
  const bool xbig = fabs(xx) >= fabs(yy);
  const double hi = xbig ? xx : yy, lo = xbig ? yy : xx;
  const double small = (hi / large) * lo - (xy / large) * xy;
  major = fmax(large, small);
  minor = fmin(large, small);
}

// Gauss-point operators of the flat quadrilateral: physical shape
// derivatives dx, dy, the Jacobian measure w and the Wilson mode gradients
// (p1x, p1y, p2x, p2y) with the patch-consistent Jacobian
__device__ void q4_gauss_point(const double lc[8], double r, double s, double iJ11c, double iJ12c, double iJ21c,
                               double iJ22c, double dx[4], double dy[4], double& w, double pm[4]) {
  const double dNr[4] = {-0.25 * (1 - s), 0.25 * (1 - s), 0.25 * (1 + s), -0.25 * (1 + s)};
  const double dNs[4] = {-0.25 * (1 - r), -0.25 * (1 + r), 0.25 * (1 + r), 0.25 * (1 - r)};
  double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    J11 += dNr[a] * lc[a];
    J12 += dNr[a] * lc[4 + a];
    J21 += dNs[a] * lc[a];
    J22 += dNs[a] * lc[4 + a];
  }
  const double det = J11 * J22 - J12 * J21;
  w = fabs(det);
  const double id = 1.0 / det;
  const double iJ11 = J22 * id, iJ12 = -J12 * id, iJ21 = -J21 * id, iJ22 = J11 * id;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    dx[a] = iJ11 * dNr[a] + iJ12 * dNs[a];
    dy[a] = iJ21 * dNr[a] + iJ22 * dNs[a];
  }
  const double ratio = (iJ11 * iJ22 - iJ12 * iJ21) / (iJ11c * iJ22c - iJ12c * iJ21c);
  pm[0] = ratio * iJ11c * (-2 * r);
  pm[1] = ratio * iJ21c * (-2 * r);
  pm[2] = ratio * iJ12c * (-2 * s);
  pm[3] = ratio * iJ22c * (-2 * s);
}

__global__ void __launch_bounds__(128)
k_q4_stress(int64_t n, int nrhs, const int32_t* __restrict__ nodes, const double* __restrict__ prep,
            const double* __restrict__ sect, const double* __restrict__ nodeR, const double* __restrict__ U,
            int64_t ldu, double* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nrhs) return;
  const int64_t e = t % n;
  const int k = (int)(t / n);
  const double* P = prep + (int64_t)Q4_PREP_STRIDE * e;
  double* o = out + Q4_REC * t;
  if (P[Q4P_STATUS] != 0.0) {
    for (int i = 0; i < Q4_REC; ++i) o[i] = nan("");
    return;
  }
  double lc[8], Rel[9];
#pragma unroll
  for (int i = 0; i < 8; ++i) lc[i] = P[Q4P_LC + i];
#pragma unroll
  for (int i = 0; i < 9; ++i) Rel[i] = P[Q4P_V + i];   // rows v1, v2, v3
  const double* sc = sect + (int64_t)JFG_Q4_SECT_STRIDE * e;
  double Cm[9], Cb[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) { Cm[i] = sc[i]; Cb[i] = sc[9 + i]; }
  const double h = sc[22];
  // element-frame displacements
  double ue[24];
  const double* Uk = U + ldu * k;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int64_t g = nodes[4 * e + a];
    const double* R = nodeR + 9 * g;
    double ut[3], ur[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) { ut[c] = Uk[6 * g + c]; ur[c] = Uk[6 * g + 3 + c]; }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      double x = 0, y = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double tn = Rel[3 * r] * R[3 * c] + Rel[3 * r + 1] * R[1 + 3 * c] + Rel[3 * r + 2] * R[2 + 3 * c];
        x += tn * ut[c];
        y += tn * ur[c];
      }
      ue[6 * a + r] = x;
      ue[6 * a + 3 + r] = y;
    }
  }
  // centre inverse Jacobian
  const double dNr_c[4] = {-0.25, 0.25, 0.25, -0.25}, dNs_c[4] = {-0.25, -0.25, 0.25, 0.25};
  double J11c = 0, J12c = 0, J21c = 0, J22c = 0;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    J11c += dNr_c[a] * lc[a];
    J12c += dNr_c[a] * lc[4 + a];
    J21c += dNs_c[a] * lc[a];
    J22c += dNs_c[a] * lc[4 + a];
  }
  const double idc = 1.0 / (J11c * J22c - J12c * J21c);
  const double iJ11c = J22c * idc, iJ12c = -J12c * idc, iJ21c = -J21c * idc, iJ22c = J11c * idc;
  const double pt = 0.57735026918962573;   // 1/sqrt(3)
  const double gr[4] = {-pt, pt, pt, -pt}, gs[4] = {-pt, -pt, pt, pt};
  // Wilson modes: K_bb and K_ab^T u = sum_g w Bi^T Cm (Bm u)
  double Kbb[16], rhs[4] = {0, 0, 0, 0};
#pragma unroll
  for (int i = 0; i < 16; ++i) Kbb[i] = 0.0;
  for (int g = 0; g < 4; ++g) {
    double dx[4], dy[4], w, pm[4];
    q4_gauss_point(lc, gr[g], gs[g], iJ11c, iJ12c, iJ21c, iJ22c, dx, dy, w, pm);
    double ec[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      ec[0] += dx[a] * ue[6 * a];
      ec[1] += dy[a] * ue[6 * a + 1];
      ec[2] += dy[a] * ue[6 * a] + dx[a] * ue[6 * a + 1];
    }
    // the four mode columns of Bi (3 x 4)
    const double bi[4][3] = {{pm[0], 0.0, pm[1]}, {0.0, pm[1], pm[0]}, {pm[2], 0.0, pm[3]}, {0.0, pm[3], pm[2]}};
    double cb[4][3];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 3; ++r) cb[j][r] = Cm[r] * bi[j][0] + Cm[r + 3] * bi[j][1] + Cm[r + 6] * bi[j][2];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      rhs[j] += w * (ec[0] * cb[j][0] + ec[1] * cb[j][1] + ec[2] * cb[j][2]);
#pragma unroll
      for (int i = 0; i < 4; ++i) Kbb[i + 4 * j] += w * (bi[i][0] * cb[j][0] + bi[i][1] * cb[j][1] + bi[i][2] * cb[j][2]);
    }
  }
  // alpha = -(K_bb \ rhs): Gaussian elimination with partial pivoting
  double alpha[4];
  {
    double A[4][5];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
#pragma unroll
      for (int j = 0; j < 4; ++j) A[i][j] = Kbb[i + 4 * j];
      A[i][4] = rhs[i];
    }
    for (int c = 0; c < 4; ++c) {
      int pv = c;
      for (int i = c + 1; i < 4; ++i)
        if (fabs(A[i][c]) > fabs(A[pv][c])) pv = i;
      if (pv != c)
        for (int j = 0; j < 5; ++j) { double tmp = A[c][j]; A[c][j] = A[pv][j]; A[pv][j] = tmp; }
      for (int i = c + 1; i < 4; ++i) {
        const double f = A[i][c] / A[c][c];
        for (int j = c; j < 5; ++j) A[i][j] -= f * A[c][j];
      }
    }
    for (int i = 3; i >= 0; --i) {
      double v = A[i][4];
      for (int j = i + 1; j < 4; ++j) v -= A[i][j] * alpha[j];
      alpha[i] = v / A[i][i];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) alpha[i] = -alpha[i];
  }
  // area-weighted means of the membrane strain and the curvature
  double eps[3] = {0, 0, 0}, kap[3] = {0, 0, 0}, area = 0.0;
  for (int g = 0; g < 4; ++g) {
    double dx[4], dy[4], w, pm[4];
    q4_gauss_point(lc, gr[g], gs[g], iJ11c, iJ12c, iJ21c, iJ22c, dx, dy, w, pm);
    double ep[3] = {pm[0] * alpha[0] + pm[2] * alpha[2], pm[1] * alpha[1] + pm[3] * alpha[3],
                    pm[1] * alpha[0] + pm[0] * alpha[1] + pm[3] * alpha[2] + pm[2] * alpha[3]};
    double kp[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const double u = ue[6 * a], v = ue[6 * a + 1], tx = ue[6 * a + 3], ty = ue[6 * a + 4];
      ep[0] += dx[a] * u;
      ep[1] += dy[a] * v;
      ep[2] += dy[a] * u + dx[a] * v;
      kp[0] += dx[a] * ty;
      kp[1] -= dy[a] * tx;
      kp[2] += dy[a] * ty - dx[a] * tx;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) { eps[r] += ep[r] * w; kap[r] += kp[r] * w; }
    area += w;
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) { eps[r] /= area; kap[r] /= area; }
  double N[3], M[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    N[r] = Cm[r] * eps[0] + Cm[r + 3] * eps[1] + Cm[r + 6] * eps[2];
    M[r] = -(Cb[r] * kap[0] + Cb[r + 3] * kap[1] + Cb[r + 6] * kap[2]);
  }
  // area-mean MacNeal shear resultant
  double qx = 0.0, qy = 0.0;
  if (P[Q4P_SHEAR] != 0.0) {
    double up[12];
#pragma unroll
    for (int a = 0; a < 4; ++a) { up[3 * a] = ue[6 * a + 2]; up[3 * a + 1] = ue[6 * a + 3]; up[3 * a + 2] = ue[6 * a + 4]; }
    double tv[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < 12; ++j) acc += P[Q4P_SOL + i + 4 * j] * up[j];
      tv[i] = acc;
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      double ry = 0.0, rx = 0.0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        ry += P[Q4P_D + i + 4 * (3 * a + 2)] * tv[i];
        rx += P[Q4P_D + i + 4 * (3 * a + 1)] * tv[i];
      }
      qx += ry;
      qy -= rx;
    }
    const double a4 = 4.0 * fabs(P[Q4P_DETJC]);
    qx /= a4;
    qy /= a4;
  }
  double ez1[3], ez2[3], sz1[3], sz2[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    ez1[r] = eps[r] + (-h / 2.0) * kap[r];
    ez2[r] = eps[r] + (h / 2.0) * kap[r];
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    sz1[r] = (Cm[r] * ez1[0] + Cm[r + 3] * ez1[1] + Cm[r + 6] * ez1[2]) / h;
    sz2[r] = (Cm[r] * ez2[0] + Cm[r + 3] * ez2[1] + Cm[r + 6] * ez2[2]) / h;
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) { o[r] = N[r]; o[3 + r] = M[r]; }
  o[6] = qx;
  o[7] = qy;
  const double* fib[2] = {sz1, sz2};
#pragma unroll
  for (int f = 0; f < 2; ++f) {
    const double* sg = fib[f];
    double* of = o + 8 + 6 * f;
    of[0] = sg[0];
    of[1] = sg[1];
    of[2] = sg[2];
    of[3] = sqrt(sg[0] * sg[0] - sg[0] * sg[1] + sg[1] * sg[1] + 3 * sg[2] * sg[2]);
    principal2(sg[0], sg[1], sg[2], of[4], of[5]);
  }
  double em[3], kn[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    em[r] = (ez1[r] + ez2[r]) / 2.0;
    kn[r] = (ez1[r] - ez2[r]) / h;
  }
  const double* st[2] = {em, kn};
#pragma unroll
  for (int f = 0; f < 2; ++f) {
    double* of = o + 20 + 5 * f;
    of[0] = st[f][0];
    of[1] = st[f][1];
    of[2] = st[f][2];
    principal2(st[f][0], st[f][1], st[f][2] / 2, of[3], of[4]);
  }
  const double savg = (sz1[0] + sz1[1]) / 2.0, hd = (sz1[0] - sz1[1]) / 2.0;
  o[30] = savg + sqrt(hd * hd + sz1[2] * sz1[2]);
}

}  // namespace

jfg_status recover_q4_stresses(jfg_model* m, int nrhs, const double* U_dev, double* out_dev, cudaStream_t st) {
  const int64_t total = m->n_q4 * (int64_t)nrhs;
  if (total == 0) return JFG_OK;
  JFG_TRY(launch_q4_prep(m, st));
  k_q4_stress<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(m->n_q4, nrhs, m->d_q4n, m->d_q4prep, m->d_q4s,
                                                               m->d_R, U_dev, m->ndof, out_dev);
  count_launch();
  JFG_CUDA(cudaGetLastError());
  return JFG_OK;
}

jfg_status recover_t10_stresses(jfg_model* m, int nrhs, const double* U_dev, double* out_dev, cudaStream_t st) {
  const int64_t total = m->n_t10 * (int64_t)nrhs;
  if (total == 0) return JFG_OK;
  const unsigned blocks = (unsigned)((total + 255) / 256);
  k_t10_stress<<<blocks, 256, 0, st>>>(m->n_t10, nrhs, m->d_t10n, m->d_t10m, m->d_xyz, m->d_R, U_dev, m->ndof,
                                       out_dev, m->d_err);
  count_launch();
  JFG_CUDA(cudaGetLastError());
  return JFG_OK;
}

}  // namespace jfg
