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

}  // namespace

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
