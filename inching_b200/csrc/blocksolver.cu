// Dense building blocks of the block eigensolvers, for hosts that drive a solver
// iteration through the C ABI: explicit deflation + Cholesky-QR orthonormalisation
// of a tall block, the Rayleigh-Ritz projection G = Y^T (H Y), the rotation by the
// small eigenvector matrix, and FP64 residual norms ||H y - theta y||.
//
// Reference counterparts (one vector at a time there): the classical / modified
// Gram-Schmidt of Burn/Orthogonalization/T1.py:56-64 and T2.py:64-137, the
// projected matrix G = V^T A V of JacobiDavidsonHotellingDeflation/T1.py:440-451,
// the Ritz residual r = A u - theta u of T1.py:543-560.
//
// Layout: every tall block is row-major (n rows, b columns, leading dimension ld
// >= b), i.e. column-major (b x n) for cuBLAS, which runs the tall-skinny GEMMs
// and the triangular solve.  One cuBLAS handle per device is created on the first
// call (cuBLAS keeps a small allocation of its own for it); its GEMM workspace is
// set from the caller's workspace on every call.  Calls on one device are
// serialised by a mutex while they enqueue work.
#include <cublas_v2.h>

#include <cmath>
#include <mutex>

#include "common.cuh"

namespace inch {
namespace {

constexpr size_t kCublasWs = size_t(4) << 20;   // GEMM workspace handed to cuBLAS

std::mutex g_mu;
cublasHandle_t g_handle[64] = {};

// Handle of the current device (created once, under g_mu held by the caller).
cublasHandle_t handle_for_current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  if (g_handle[dev] == nullptr) {
    cublasHandle_t h = nullptr;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return nullptr;
    g_handle[dev] = h;
  }
  return g_handle[dev];
}

#define INCH_CUBLAS(call)                                                              \
  do {                                                                                 \
    cublasStatus_t _s = (call);                                                        \
    if (_s != CUBLAS_STATUS_SUCCESS) {                                                 \
      ::inch::set_error("%s:%d %s: cuBLAS status %d", __FILE__, __LINE__, #call, (int)_s); \
      return INCH_CUDA_ERROR;                                                          \
    }                                                                                  \
  } while (0)

// In-place lower Cholesky of the symmetric column-major b x b matrix G + shift*I
// (one CTA).  info = 0 on success, j + 1 if the j-th pivot is not positive.
__global__ void k_potrf_lower(double* __restrict__ G, int b, double shift, int* __restrict__ info) {
  __shared__ double piv;
  for (int j = 0; j < b; ++j) {
    if (threadIdx.x == 0) {
      double s = G[j + (int64_t)j * b] + shift;
      for (int k = 0; k < j; ++k) s -= G[j + (int64_t)k * b] * G[j + (int64_t)k * b];
      if (!(s > 0.0) || !isfinite(s)) {
        *info = j + 1;
        piv = 0.0;
      } else {
        piv = sqrt(s);
        G[j + (int64_t)j * b] = piv;
      }
    }
    __syncthreads();
    const double p = piv;
    if (p == 0.0) return;    // every thread sees the same value: all leave together
    for (int i = j + 1 + threadIdx.x; i < b; i += blockDim.x) {
      double s = G[i + (int64_t)j * b];
      for (int k = 0; k < j; ++k) s -= G[i + (int64_t)k * b] * G[j + (int64_t)k * b];
      G[i + (int64_t)j * b] = s / p;
    }
    __syncthreads();
  }
}

// G <- (G + G^T) / 2 for a column-major b x b matrix; maxdiag[0] = max_i G_ii.
__global__ void k_symmetrize(double* __restrict__ G, int b) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)b * b;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int r = static_cast<int>(t % b), c = static_cast<int>(t / b);
    if (r < c) {
      const double v = 0.5 * (G[r + (int64_t)c * b] + G[c + (int64_t)r * b]);
      G[r + (int64_t)c * b] = v;
      G[c + (int64_t)r * b] = v;
    }
  }
}

__global__ void k_maxdiag(const double* __restrict__ G, int b, double* __restrict__ out) {
  __shared__ double s[256];
  double m = 0.0;
  for (int i = threadIdx.x; i < b; i += blockDim.x) m = fmax(m, fabs(G[i + (int64_t)i * b]));
  s[threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = s[0];
}

// Column norms of HY - Y * diag(theta) (row-major n x b blocks): per-block partial
// sums of squares for a slab of rows, then a deterministic second pass.
constexpr int kResBlocks = 296;
__global__ void k_resid_partial(const double* __restrict__ HY, int64_t ldh, const double* __restrict__ Y,
                                int64_t ldy, const double* __restrict__ theta, int64_t n, int b,
                                double* __restrict__ partial) {
  for (int c0 = 0; c0 < b; c0 += blockDim.x) {
    const int c = c0 + threadIdx.x;
    double s = 0.0;
    if (c < b) {
      const double th = theta[c];
      for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
        const double r = HY[i * ldh + c] - th * Y[i * ldy + c];
        s += r * r;
      }
      partial[(int64_t)blockIdx.x * b + c] = s;
    }
  }
}

__global__ void k_resid_final(const double* __restrict__ partial, int P, int b, double* __restrict__ out) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < b; c += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int p = 0; p < P; ++p) s += partial[(int64_t)p * b + c];
    out[c] = sqrt(s);
  }
}

// Y <- Y - B^T (B Y) for the r rows of B (row-major r x n, leading dimension ldb).
inch_status project_out(cublasHandle_t h, int64_t n, int b, double* Y, int64_t ldy, const double* B, int64_t r,
                        int64_t ldb, double* C) {
  const double one = 1.0, zero = 0.0, mone = -1.0;
  // C (col-major b x r) = Yc (b x n) * Bc (n x r)
  INCH_CUBLAS(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, b, (int)r, (int)n, &one, Y, (int)ldy, B, (int)ldb, &zero, C,
                          b));
  // Yc -= C * Bc^T
  INCH_CUBLAS(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, b, (int)n, (int)r, &mone, C, b, B, (int)ldb, &one, Y,
                          (int)ldy));
  return INCH_OK;
}

}  // namespace
}  // namespace inch

using namespace inch;

extern "C" size_t inch_block_orth_workspace_size(int32_t b, int64_t r_max) {
  Sizer s;
  s.take<double>((size_t)b * b);                            // Gram matrix / Cholesky factor
  s.take<double>((size_t)b * (r_max > 0 ? r_max : 1));      // projection coefficients
  s.take<int>(4);
  s.take<double>(4);
  s.take<char>(kCublasWs);
  return s.bytes();
}

extern "C" inch_status inch_block_orth(int64_t n, int32_t b, double* Y, int64_t ldy, const double* B1, int64_t r1,
                                       int64_t ldb1, const double* B2, int64_t r2, int64_t ldb2, int32_t passes,
                                       void* ws, size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(Y != nullptr && n >= 1 && b >= 1 && ldy >= b, INCH_INVALID_ARG, "inch_block_orth: bad block");
  INCH_REQUIRE(n < (int64_t(1) << 31) && (int64_t)b <= n, INCH_INVALID_ARG, "inch_block_orth: n must be in [b, 2^31)");
  INCH_REQUIRE((r1 == 0 || (B1 && ldb1 >= n)) && (r2 == 0 || (B2 && ldb2 >= n)) && r1 >= 0 && r2 >= 0,
               INCH_INVALID_ARG, "inch_block_orth: bad deflation basis");
  INCH_REQUIRE(passes >= 1 && passes <= 4, INCH_INVALID_ARG, "inch_block_orth: passes in 1..4");
  const int64_t rmax = r1 > r2 ? r1 : r2;
  Carver c(ws, ws_bytes);
  double* G = c.take<double>((size_t)b * b);
  double* C = c.take<double>((size_t)b * (rmax > 0 ? rmax : 1));
  int* info = c.take<int>(4);
  double* md = c.take<double>(4);
  void* cws = c.take<char>(kCublasWs);
  INCH_REQUIRE(c.ok, INCH_OOM, "inch_block_orth: workspace of %zu bytes, need %zu", ws_bytes,
               inch_block_orth_workspace_size(b, rmax));
  std::lock_guard<std::mutex> lock(g_mu);
  cublasHandle_t h = handle_for_current_device();
  INCH_REQUIRE(h != nullptr, INCH_CUDA_ERROR, "inch_block_orth: cannot create the cuBLAS handle");
  INCH_CUBLAS(cublasSetStream(h, stream));
  INCH_CUBLAS(cublasSetWorkspace(h, cws, kCublasWs));
  const double one = 1.0, zero = 0.0;
  // explicit deflation: two classical passes against each basis
  for (int t = 0; t < 2; ++t) {
    if (r1 > 0 && project_out(h, n, b, Y, ldy, B1, r1, ldb1, C) != INCH_OK) return INCH_CUDA_ERROR;
    if (r2 > 0 && project_out(h, n, b, Y, ldy, B2, r2, ldb2, C) != INCH_OK) return INCH_CUDA_ERROR;
  }
  // Cholesky-QR passes: G = Y^T Y = L L^T, Y <- Y L^{-T} (a left triangular solve
  // on the column-major view, in place).  A Gram matrix that is not numerically
  // positive gets a shift of 1e-12 * max diag (shifted Cholesky-QR; the next pass
  // restores orthonormality).
  for (int p = 0; p < passes; ++p) {
    for (int attempt = 0; attempt < 2; ++attempt) {
      INCH_CUBLAS(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, b, b, (int)n, &one, Y, (int)ldy, Y, (int)ldy, &zero, G, b));
      k_symmetrize<<<grid_for((int64_t)b * b, 256, 148 * 4), 256, 0, stream>>>(G, b);
      INCH_LAUNCH_CHECK();
      double shift = 0.0;
      if (attempt == 1) {
        k_maxdiag<<<1, 256, 0, stream>>>(G, b, md);
        INCH_LAUNCH_CHECK();
        double hmd = 0.0;
        INCH_CUDA(cudaMemcpyAsync(&hmd, md, sizeof(double), cudaMemcpyDeviceToHost, stream));
        INCH_CUDA(cudaStreamSynchronize(stream));
        shift = 1e-12 * hmd;
      }
      INCH_CUDA(cudaMemsetAsync(info, 0, sizeof(int), stream));
      k_potrf_lower<<<1, 256, 0, stream>>>(G, b, shift, info);
      INCH_LAUNCH_CHECK();
      int hinfo = 0;
      INCH_CUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, stream));
      INCH_CUDA(cudaStreamSynchronize(stream));
      if (hinfo == 0) break;
      INCH_REQUIRE(attempt == 0, INCH_INVALID_ARG,
                   "inch_block_orth: the block is rank deficient (pivot %d not positive after a shift)", hinfo);
    }
    INCH_CUBLAS(cublasDtrsm(h, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, b,
                            (int)n, &one, G, b, Y, (int)ldy));
  }
  return INCH_OK;
}

extern "C" size_t inch_rr_workspace_size(void) {
  Sizer s;
  s.take<char>(kCublasWs);
  return s.bytes();
}

extern "C" inch_status inch_rr_project(int64_t n, int32_t b, const double* Y, int64_t ldy, const double* HY,
                                       int64_t ldh, double* G, void* ws, size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(Y && HY && G && n >= 1 && b >= 1 && ldy >= b && ldh >= b && n < (int64_t(1) << 31), INCH_INVALID_ARG,
               "inch_rr_project: bad arguments");
  Carver c(ws, ws_bytes);
  void* cws = c.take<char>(kCublasWs);
  INCH_REQUIRE(c.ok, INCH_OOM, "inch_rr_project: workspace of %zu bytes, need %zu", ws_bytes, inch_rr_workspace_size());
  std::lock_guard<std::mutex> lock(g_mu);
  cublasHandle_t h = handle_for_current_device();
  INCH_REQUIRE(h != nullptr, INCH_CUDA_ERROR, "inch_rr_project: cannot create the cuBLAS handle");
  INCH_CUBLAS(cublasSetStream(h, stream));
  INCH_CUBLAS(cublasSetWorkspace(h, cws, kCublasWs));
  const double one = 1.0, zero = 0.0;
  INCH_CUBLAS(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, b, b, (int)n, &one, Y, (int)ldy, HY, (int)ldh, &zero, G, b));
  k_symmetrize<<<grid_for((int64_t)b * b, 256, 148 * 4), 256, 0, stream>>>(G, b);
  INCH_LAUNCH_CHECK();
  return INCH_OK;
}

extern "C" inch_status inch_rr_rotate(int64_t n, int32_t b, int32_t m, const double* Y, int64_t ldy, const double* W,
                                      double* Z, int64_t ldz, void* ws, size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(Y && W && Z && Y != Z && n >= 1 && b >= 1 && m >= 1 && m <= b && ldy >= b && ldz >= m &&
                   n < (int64_t(1) << 31),
               INCH_INVALID_ARG, "inch_rr_rotate: bad arguments");
  Carver c(ws, ws_bytes);
  void* cws = c.take<char>(kCublasWs);
  INCH_REQUIRE(c.ok, INCH_OOM, "inch_rr_rotate: workspace of %zu bytes, need %zu", ws_bytes, inch_rr_workspace_size());
  std::lock_guard<std::mutex> lock(g_mu);
  cublasHandle_t h = handle_for_current_device();
  INCH_REQUIRE(h != nullptr, INCH_CUDA_ERROR, "inch_rr_rotate: cannot create the cuBLAS handle");
  INCH_CUBLAS(cublasSetStream(h, stream));
  INCH_CUBLAS(cublasSetWorkspace(h, cws, kCublasWs));
  const double one = 1.0, zero = 0.0;
  // Z (n x m) = Y (n x b) W (b x m, column-major: eigenvector t in column t)
  // column-major view: Zc (m x n) = W^T (m x b) * Yc (b x n)
  INCH_CUBLAS(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, m, (int)n, b, &one, W, b, Y, (int)ldy, &zero, Z, (int)ldz));
  return INCH_OK;
}

extern "C" size_t inch_residual_workspace_size(int32_t b) {
  Sizer s;
  s.take<double>((size_t)kResBlocks * b);
  return s.bytes();
}

extern "C" inch_status inch_residual_fp64(int64_t n, int32_t b, const double* HY, int64_t ldh, const double* Y,
                                          int64_t ldy, const double* theta_dev, double* res_dev, void* ws,
                                          size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(HY && Y && theta_dev && res_dev && n >= 1 && b >= 1 && ldh >= b && ldy >= b, INCH_INVALID_ARG,
               "inch_residual_fp64: bad arguments");
  Carver c(ws, ws_bytes);
  double* partial = c.take<double>((size_t)kResBlocks * b);
  INCH_REQUIRE(c.ok, INCH_OOM, "inch_residual_fp64: workspace of %zu bytes, need %zu", ws_bytes,
               inch_residual_workspace_size(b));
  const int threads = b >= 256 ? 256 : ((b + 31) / 32) * 32;
  k_resid_partial<<<kResBlocks, threads, 0, stream>>>(HY, ldh, Y, ldy, theta_dev, n, b, partial);
  INCH_LAUNCH_CHECK();
  k_resid_final<<<(b + 255) / 256, 256, 0, stream>>>(partial, kResBlocks, b, res_dev);
  INCH_LAUNCH_CHECK();
  return INCH_OK;
}
