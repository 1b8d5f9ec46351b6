// ANM Hessian assembly into the rank-one block store.
//
// Reference: InchingLiteInteger/Fuel/T1.py:276-455 builds, per row batch, the
// dense (m, w, 3, 3) tensor x_ij x_ij^T * (-1/d^2) (zero when d^2 > rc^2 or
// d^2 == 0), writes -(row sum) + PlusI*I into the diagonal blocks and keeps the
// lower triangle as CSR.  Every off-diagonal block is rank one, so this kernel
// stores only w = x/d per adjacency entry (block = -w w^T) and the symmetric
// diagonal block, computed in FP64 and optionally rounded to FP32 for the
// mixed-precision operator.  One warp per atom row; entries in adjacency order.
#include "common.cuh"

namespace inch {
namespace {

constexpr int kWarps = 8;

__global__ void __launch_bounds__(kWarps * 32)
k_assemble(const double* __restrict__ X, int64_t n, double r2, double plus_i, const int64_t* __restrict__ rowptr,
           const int* __restrict__ cols, double2* __restrict__ ent64, double* __restrict__ diag64,
           float4* __restrict__ ent32, float* __restrict__ diag32, const double* __restrict__ pair_w,
           const int8_t* __restrict__ image, double bx, double by) {
  const int lane = threadIdx.x & 31;
  for (int64_t i = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5); i < n; i += (int64_t)gridDim.x * kWarps) {
    const double xi = X[3 * i], yi = X[3 * i + 1], zi = X[3 * i + 2];
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t e = rowptr[i] + lane; e < rowptr[i + 1]; e += 32) {
      const int j = cols[e];
      double xj = X[3 * (int64_t)j], yj = X[3 * (int64_t)j + 1];
      if (image != nullptr) {
        // periodic xy image: entry e was found with the query x_i + s (s = image
        // code e's shift); the reference's assembly forms (x_j + box * instr) - x_i
        // for every instruction (Fuel/T1.py:332-334), and this pair is its
        // instruction -s, so d = (x_j - s) - x_i in that operation order
        const int k = image[e];
        const int ix = (k == 1 || k == 5 || k == 6) ? 1 : ((k == 2 || k == 7 || k == 8) ? -1 : 0);
        const int iy = (k == 3 || k == 5 || k == 7) ? 1 : ((k == 4 || k == 6 || k == 8) ? -1 : 0);
        if (ix) xj = __dadd_rn(xj, ix > 0 ? -bx : bx);
        if (iy) yj = __dadd_rn(yj, iy > 0 ? -by : by);
      }
      const double dx = xj - xi, dy = yj - yi, dz = X[3 * (int64_t)j + 2] - zi;
      // Same rounding as the neighbour test, so the pair set matches the adjacency.
      const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
      const bool ok = d2 > 0.0 && d2 <= r2;
      double inv = ok ? 1.0 / sqrt(d2) : 0.0;
      if (pair_w != nullptr) inv *= sqrt(pair_w[e]);   // spring constant gamma_e: block = -gamma u u^T
      const double wx = dx * inv, wy = dy * inv, wz = dz * inv;
      s[0] += wx * wx;
      s[1] += wy * wy;
      s[2] += wz * wz;
      s[3] += wx * wy;
      s[4] += wx * wz;
      s[5] += wy * wz;
      if (ent64) {
        ent64[2 * e] = make_double2(wx, wy);
        ent64[2 * e + 1] = make_double2(wz, static_cast<double>(j));
      }
      if (ent32) ent32[e] = make_float4((float)wx, (float)wy, (float)wz, __int_as_float(j));
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = warp_sum(s[k]);
    if (lane < 8) {
      double v = 0.0;
      if (lane < 3) v = s[lane] + plus_i;
      else if (lane < 6) v = s[lane];
      if (diag64) diag64[8 * i + lane] = v;
      if (diag32) diag32[8 * i + lane] = (float)v;
    }
  }
}

}  // namespace
}  // namespace inch

using namespace inch;

extern "C" inch_status inch_hessian_assemble(const double* X, int64_t n, double rc, double plus_i,
                                             const int64_t* rowptr, const int32_t* cols, double* ent64,
                                             double* diag64, float* ent32, float* diag32, cudaStream_t stream) {
  INCH_REQUIRE(X && rowptr && cols, INCH_INVALID_ARG, "inch_hessian_assemble: NULL argument");
  INCH_REQUIRE(n >= 1 && n < (int64_t(1) << 31), INCH_INVALID_ARG, "inch_hessian_assemble: n_atoms out of range");
  INCH_REQUIRE((ent64 != nullptr) == (diag64 != nullptr) && (ent32 != nullptr) == (diag32 != nullptr),
               INCH_INVALID_ARG, "inch_hessian_assemble: entries and diagonal must be given together");
  INCH_REQUIRE(ent64 || ent32, INCH_INVALID_ARG, "inch_hessian_assemble: no output requested");
  INCH_REQUIRE((reinterpret_cast<uintptr_t>(ent64) & 15) == 0 && (reinterpret_cast<uintptr_t>(ent32) & 15) == 0,
               INCH_INVALID_ARG, "inch_hessian_assemble: entry buffers must be 16-byte aligned");
  const int g = grid_for(n, kWarps, 148 * 16);
  k_assemble<<<g, kWarps * 32, 0, stream>>>(X, n, rc * rc, plus_i, rowptr, cols,
                                             reinterpret_cast<double2*>(ent64), diag64,
                                             reinterpret_cast<float4*>(ent32), diag32, nullptr, nullptr, 0.0, 0.0);
  INCH_LAUNCH_CHECK();
  return INCH_OK;
}

extern "C" inch_status inch_hessian_assemble_weighted(const double* X, int64_t n, double rc, double plus_i,
                                                      const int64_t* rowptr, const int32_t* cols,
                                                      const double* pair_weight, double* ent64, double* diag64,
                                                      float* ent32, float* diag32, cudaStream_t stream) {
  INCH_REQUIRE(X && rowptr && cols && pair_weight, INCH_INVALID_ARG, "inch_hessian_assemble_weighted: NULL argument");
  INCH_REQUIRE(n >= 1 && n < (int64_t(1) << 31), INCH_INVALID_ARG, "inch_hessian_assemble_weighted: bad n_atoms");
  INCH_REQUIRE((ent64 != nullptr) == (diag64 != nullptr) && (ent32 != nullptr) == (diag32 != nullptr) &&
                   (ent64 || ent32),
               INCH_INVALID_ARG, "inch_hessian_assemble_weighted: bad outputs");
  INCH_REQUIRE((reinterpret_cast<uintptr_t>(ent64) & 15) == 0 && (reinterpret_cast<uintptr_t>(ent32) & 15) == 0,
               INCH_INVALID_ARG, "inch_hessian_assemble_weighted: entry buffers must be 16-byte aligned");
  const int g = grid_for(n, kWarps, 148 * 16);
  k_assemble<<<g, kWarps * 32, 0, stream>>>(X, n, rc * rc, plus_i, rowptr, cols, reinterpret_cast<double2*>(ent64),
                                             diag64, reinterpret_cast<float4*>(ent32), diag32, pair_weight, nullptr,
                                             0.0, 0.0);
  INCH_LAUNCH_CHECK();
  return INCH_OK;
}

extern "C" inch_status inch_hessian_assemble_pbc_xy(const double* X, int64_t n, double rc, double plus_i,
                                                    const int64_t* rowptr, const int32_t* cols, const int8_t* image,
                                                    double box_x, double box_y, double* ent64, double* diag64,
                                                    float* ent32, float* diag32, cudaStream_t stream) {
  INCH_REQUIRE(X && rowptr && cols && image, INCH_INVALID_ARG, "inch_hessian_assemble_pbc_xy: NULL argument");
  INCH_REQUIRE(n >= 1 && n < (int64_t(1) << 31), INCH_INVALID_ARG, "inch_hessian_assemble_pbc_xy: bad n_atoms");
  INCH_REQUIRE(box_x > rc, INCH_INVALID_ARG, "ABORTED. The PBC box size X is smaller than rc gamma.");
  INCH_REQUIRE(box_y > rc, INCH_INVALID_ARG, "ABORTED. The PBC box size Y is smaller than rc gamma.");
  INCH_REQUIRE((ent64 != nullptr) == (diag64 != nullptr) && (ent32 != nullptr) == (diag32 != nullptr) &&
                   (ent64 || ent32),
               INCH_INVALID_ARG, "inch_hessian_assemble_pbc_xy: bad outputs");
  INCH_REQUIRE((reinterpret_cast<uintptr_t>(ent64) & 15) == 0 && (reinterpret_cast<uintptr_t>(ent32) & 15) == 0,
               INCH_INVALID_ARG, "inch_hessian_assemble_pbc_xy: entry buffers must be 16-byte aligned");
  const int g = grid_for(n, kWarps, 148 * 16);
  k_assemble<<<g, kWarps * 32, 0, stream>>>(X, n, rc * rc, plus_i, rowptr, cols, reinterpret_cast<double2*>(ent64),
                                             diag64, reinterpret_cast<float4*>(ent32), diag32, nullptr, image, box_x,
                                             box_y);
  INCH_LAUNCH_CHECK();
  return INCH_OK;
}
