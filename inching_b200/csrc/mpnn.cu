// Kernels of the learned warm start: a message-passing network on the coarse
// bead graph that predicts the bead model's spring constants (no reference
// counterpart).  Dense layers are GEMMs done by the caller; these kernels do the
// graph-structured and element-wise parts of the forward and backward passes,
// the eigenvalue gradient of the bead Hessian and the optimiser step.
//
// Graph layout: directed edges in CSR by destination (rowptr over nodes, src per
// edge), both directions of every bead pair present, no self edges.
#include "common.cuh"

namespace inch {
namespace {

constexpr int kT = 256;

// Z[e, :F] = H[src[e], :], Z[e, F:F+G] = EF[e, :]  (message-MLP input)
__global__ void k_edge_concat(const float* __restrict__ H, const float* __restrict__ EF, const int* __restrict__ src,
                              int64_t E, int F, int G, float* __restrict__ Z) {
  const int W = F + G;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < E * W; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / W;
    const int c = static_cast<int>(t % W);
    Z[t] = c < F ? H[(int64_t)src[e] * F + c] : EF[e * G + (c - F)];
  }
}

// dH[src[e], :] += dZ[e, :F]  (backward of the gather; atomic, FP32)
__global__ void k_edge_concat_bwd(const float* __restrict__ dZ, const int* __restrict__ src, int64_t E, int F, int G,
                                  float* __restrict__ dH) {
  const int W = F + G;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < E * F; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / F;
    const int c = static_cast<int>(t % F);
    atomicAdd(&dH[(int64_t)src[e] * F + c], dZ[e * W + c]);
  }
}

// M[i, :] = mean over the edges e of row i of A[e, :]   (deterministic per node)
__global__ void k_segment_sum(const float* __restrict__ A, const int64_t* __restrict__ rowptr, int64_t N, int F,
                              float* __restrict__ M) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N * F; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / F;
    const int c = static_cast<int>(t % F);
    float s = 0.f;
    for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) s += A[e * F + c];
    const int64_t d = rowptr[i + 1] - rowptr[i];
    M[t] = d > 0 ? s / (float)d : 0.f;
  }
}

// dA[e, :] = dM[dst(e), :] / deg(dst(e))   (backward of the neighbour mean)
__global__ void k_segment_sum_bwd(const float* __restrict__ dM, const int64_t* __restrict__ rowptr,
                                  const int* __restrict__ dst, int64_t E, int F, float* __restrict__ dA) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < E * F; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / F;
    const int c = static_cast<int>(t % F);
    const int64_t i = dst[e];
    dA[t] = dM[i * F + c] / (float)(rowptr[i + 1] - rowptr[i]);
  }
}

// Y = relu(Y + b) in place (b broadcast over rows); mask kept implicitly in Y > 0
__global__ void k_bias_relu(float* __restrict__ Y, const float* __restrict__ b, int64_t R, int F) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < R * F; t += (int64_t)gridDim.x * blockDim.x) {
    const float v = Y[t] + b[t % F];
    Y[t] = v > 0.f ? v : 0.f;
  }
}

// dY *= (Y > 0)   (backward of relu given its output)
__global__ void k_relu_bwd(float* __restrict__ dY, const float* __restrict__ Y, int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    if (!(Y[t] > 0.f)) dY[t] = 0.f;
}

// R[e, :F] = H[i(e)] + H[src(e)], R[e, F:] = EF[e]   (symmetric edge readout input)
__global__ void k_edge_pair(const float* __restrict__ H, const float* __restrict__ EF, const int* __restrict__ src,
                            const int* __restrict__ dst, int64_t E, int F, int G, float* __restrict__ Rz) {
  const int W = F + G;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < E * W; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / W;
    const int c = static_cast<int>(t % W);
    Rz[t] = c < F ? H[(int64_t)dst[e] * F + c] + H[(int64_t)src[e] * F + c] : EF[e * G + (c - F)];
  }
}

__global__ void k_edge_pair_bwd(const float* __restrict__ dR, const int* __restrict__ src, const int* __restrict__ dst,
                                int64_t E, int F, int G, float* __restrict__ dH) {
  const int W = F + G;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < E * F; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / F;
    const int c = static_cast<int>(t % F);
    const float g = dR[e * W + c];
    atomicAdd(&dH[(int64_t)dst[e] * F + c], g);
    atomicAdd(&dH[(int64_t)src[e] * F + c], g);
  }
}

// gamma = softplus(s) + floor ; ds_out = softplus'(s) * dgamma (if dgamma given)
__global__ void k_softplus(const float* __restrict__ s, int64_t E, float floor_v, double* __restrict__ gamma,
                           const double* __restrict__ dgamma, float* __restrict__ ds) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    const float x = s[e];
    const float sp = x > 20.f ? x : log1pf(expf(x));
    if (gamma) gamma[e] = (double)sp + (double)floor_v;
    if (dgamma) ds[e] = (float)(dgamma[e] / (1.0 + exp(-(double)x)));
  }
}

// Eigenvalue gradient of the bead Hessian (Hellmann-Feynman): for lambda_t with
// unit eigenvector v_t, d lambda_t / d gamma_e = (u_e . (v_t[a] - v_t[b]))^2 over
// the pair e = (a, b) (both directions stored: each carries half).
// out[e] = sum_t c[t] * that.   V: (3 * nodes, m) row-major FP64.
__global__ void k_hf_grad(const double* __restrict__ P, const int64_t* __restrict__ rowptr,
                          const int* __restrict__ src, const int* __restrict__ dst, const double* __restrict__ V,
                          int m, const double* __restrict__ c, int64_t E, double* __restrict__ out) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = dst[e], b = src[e];
    double ux = P[3 * b] - P[3 * a], uy = P[3 * b + 1] - P[3 * a + 1], uz = P[3 * b + 2] - P[3 * a + 2];
    const double d = sqrt(ux * ux + uy * uy + uz * uz);
    ux /= d;
    uy /= d;
    uz /= d;
    double g = 0.0;
    for (int t = 0; t < m; ++t) {
      const double p = ux * (V[(3 * a) * m + t] - V[(3 * b) * m + t]) + uy * (V[(3 * a + 1) * m + t] - V[(3 * b + 1) * m + t]) +
                       uz * (V[(3 * a + 2) * m + t] - V[(3 * b + 2) * m + t]);
      g += c[t] * p * p;
    }
    out[e] = 0.5 * g;
  }
}

// Adam step on a flat parameter vector (bias-corrected).
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, int64_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const float gt = g[t];
    const float a = b1 * m1[t] + (1.f - b1) * gt;
    const float b = b2 * m2[t] + (1.f - b2) * gt * gt;
    m1[t] = a;
    m2[t] = b;
    w[t] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
  }
}

// Dense layers: C = A B (+ beta C) in FP32 with arbitrary element strides, so the
// same kernel serves X W, X^T dY (weight gradients, a reduction over the long
// dimension) and dY W^T.  64 x 64 output tiles, K in chunks of 16 staged in shared
// memory, 4 x 4 outputs per thread.  Small output grids over a long K split K over
// gridDim.z into per-split partial tiles, added in a fixed order by k_gemm_reduce
// (deterministic).
constexpr int kGM = 64, kGN = 64, kGK = 16;

__global__ void __launch_bounds__(256)
k_gemm(int M, int N, int K, const float* __restrict__ A, int64_t sai, int64_t sak, const float* __restrict__ B,
       int64_t sbk, int64_t sbn, float* C, int64_t ldc, float beta, int kchunk, float* __restrict__ part) {
  __shared__ float As[kGK][kGM + 4];
  __shared__ float Bs[kGK][kGN + 4];
  const int bm = blockIdx.y * kGM, bn = blockIdx.x * kGN;
  const int k_beg = blockIdx.z * kchunk;
  const int k_end = (K - k_beg) < kchunk ? K : k_beg + kchunk;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.f;
  for (int k0 = k_beg; k0 < k_end; k0 += kGK) {
    // stage the A and B tiles, consecutive threads along whichever index is unit-stride
    for (int t = threadIdx.x; t < kGM * kGK; t += 256) {
      const int mm = (sak == 1) ? t / kGK : t % kGM;
      const int kk = (sak == 1) ? t % kGK : t / kGM;
      const int gi = bm + mm, gk = k0 + kk;
      As[kk][mm] = (gi < M && gk < k_end) ? A[(int64_t)gi * sai + (int64_t)gk * sak] : 0.f;
    }
    for (int t = threadIdx.x; t < kGN * kGK; t += 256) {
      const int nn = (sbn == 1) ? t % kGN : t / kGK;
      const int kk = (sbn == 1) ? t / kGN : t % kGK;
      const int gj = bn + nn, gk = k0 + kk;
      Bs[kk][nn] = (gj < N && gk < k_end) ? B[(int64_t)gk * sbk + (int64_t)gj * sbn] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = As[kk][ty * 4 + r];
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = Bs[kk][tx * 4 + c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(a[r], b[c], acc[r][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i = bm + ty * 4 + r;
    if (i >= M) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int j = bn + tx * 4 + c;
      if (j >= N) continue;
      if (part != nullptr) {
        part[((int64_t)blockIdx.z * M + i) * N + j] = acc[r][c];
      } else {
        float* cp = C + (int64_t)i * ldc + j;
        *cp = beta != 0.f ? fmaf(beta, *cp, acc[r][c]) : acc[r][c];
      }
    }
  }
}

__global__ void k_gemm_reduce(int M, int N, int splits, const float* __restrict__ part, float* C, int64_t ldc,
                              float beta) {
  const int64_t total = (int64_t)M * N;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / N, j = t % N;
    float sum = 0.f;
    for (int sp = 0; sp < splits; ++sp) sum += part[sp * total + t];
    float* cp = C + i * ldc + j;
    *cp = beta != 0.f ? fmaf(beta, *cp, sum) : sum;
  }
}

// K splits of a (M x N) product over K: enough blocks for the 148 SMs when the
// output grid alone is small and K is long.
int gemm_splits(int M, int N, int K) {
  const int tiles = ((M + kGM - 1) / kGM) * ((N + kGN - 1) / kGN);
  if (tiles >= 148 || K <= 2048) return 1;
  int sp = (2 * 148 + tiles - 1) / tiles;
  const int by_k = (K + 1023) / 1024;
  if (sp > by_k) sp = by_k;
  if (sp > 64) sp = 64;
  return sp < 1 ? 1 : sp;
}

int blocks(int64_t work) { return grid_for(work, kT, 148 * 16); }

}  // namespace
}  // namespace inch

using namespace inch;

#define MP_CHECK() INCH_LAUNCH_CHECK(); return INCH_OK

extern "C" inch_status inch_mp_edge_concat(const float* H, const float* EF, const int32_t* src, int64_t E, int32_t F,
                                           int32_t G, float* Z, cudaStream_t s) {
  INCH_REQUIRE(H && EF && src && Z && E >= 0 && F > 0 && G >= 0, INCH_INVALID_ARG, "inch_mp_edge_concat: bad args");
  k_edge_concat<<<blocks(E * (F + G)), kT, 0, s>>>(H, EF, src, E, F, G, Z);
  MP_CHECK();
}
extern "C" inch_status inch_mp_edge_concat_bwd(const float* dZ, const int32_t* src, int64_t E, int32_t F, int32_t G,
                                               float* dH, cudaStream_t s) {
  INCH_REQUIRE(dZ && src && dH, INCH_INVALID_ARG, "inch_mp_edge_concat_bwd: bad args");
  k_edge_concat_bwd<<<blocks(E * F), kT, 0, s>>>(dZ, src, E, F, G, dH);
  MP_CHECK();
}
extern "C" inch_status inch_mp_segment_sum(const float* A, const int64_t* rowptr, int64_t N, int32_t F, float* M,
                                           cudaStream_t s) {
  INCH_REQUIRE(A && rowptr && M, INCH_INVALID_ARG, "inch_mp_segment_sum: bad args");
  k_segment_sum<<<blocks(N * F), kT, 0, s>>>(A, rowptr, N, F, M);
  MP_CHECK();
}
extern "C" inch_status inch_mp_segment_sum_bwd(const float* dM, const int64_t* rowptr, const int32_t* dst, int64_t E,
                                               int32_t F, float* dA, cudaStream_t s) {
  INCH_REQUIRE(dM && rowptr && dst && dA, INCH_INVALID_ARG, "inch_mp_segment_sum_bwd: bad args");
  k_segment_sum_bwd<<<blocks(E * F), kT, 0, s>>>(dM, rowptr, dst, E, F, dA);
  MP_CHECK();
}
extern "C" inch_status inch_mp_bias_relu(float* Y, const float* b, int64_t R, int32_t F, cudaStream_t s) {
  INCH_REQUIRE(Y && b, INCH_INVALID_ARG, "inch_mp_bias_relu: bad args");
  k_bias_relu<<<blocks(R * F), kT, 0, s>>>(Y, b, R, F);
  MP_CHECK();
}
extern "C" inch_status inch_mp_relu_bwd(float* dY, const float* Y, int64_t n, cudaStream_t s) {
  INCH_REQUIRE(dY && Y, INCH_INVALID_ARG, "inch_mp_relu_bwd: bad args");
  k_relu_bwd<<<blocks(n), kT, 0, s>>>(dY, Y, n);
  MP_CHECK();
}
extern "C" inch_status inch_mp_edge_pair(const float* H, const float* EF, const int32_t* src, const int32_t* dst,
                                         int64_t E, int32_t F, int32_t G, float* R, cudaStream_t s) {
  INCH_REQUIRE(H && EF && src && dst && R, INCH_INVALID_ARG, "inch_mp_edge_pair: bad args");
  k_edge_pair<<<blocks(E * (F + G)), kT, 0, s>>>(H, EF, src, dst, E, F, G, R);
  MP_CHECK();
}
extern "C" inch_status inch_mp_edge_pair_bwd(const float* dR, const int32_t* src, const int32_t* dst, int64_t E,
                                             int32_t F, int32_t G, float* dH, cudaStream_t s) {
  INCH_REQUIRE(dR && src && dst && dH, INCH_INVALID_ARG, "inch_mp_edge_pair_bwd: bad args");
  k_edge_pair_bwd<<<blocks(E * F), kT, 0, s>>>(dR, src, dst, E, F, G, dH);
  MP_CHECK();
}
extern "C" inch_status inch_mp_softplus(const float* sc, int64_t E, float floor_v, double* gamma, const double* dgamma,
                                        float* ds, cudaStream_t s) {
  INCH_REQUIRE(sc && (gamma || (dgamma && ds)), INCH_INVALID_ARG, "inch_mp_softplus: bad args");
  k_softplus<<<blocks(E), kT, 0, s>>>(sc, E, floor_v, gamma, dgamma, ds);
  MP_CHECK();
}
extern "C" inch_status inch_mp_hf_grad(const double* P, const int64_t* rowptr, const int32_t* src, const int32_t* dst,
                                       const double* V, int32_t m, const double* c, int64_t E, double* out,
                                       cudaStream_t s) {
  INCH_REQUIRE(P && rowptr && src && dst && V && c && out && m > 0, INCH_INVALID_ARG, "inch_mp_hf_grad: bad args");
  k_hf_grad<<<blocks(E), kT, 0, s>>>(P, rowptr, src, dst, V, m, c, E, out);
  MP_CHECK();
}
extern "C" inch_status inch_mp_adam(float* w, const float* g, float* m1, float* m2, int64_t n, float lr, float b1,
                                    float b2, float eps, int32_t step, cudaStream_t s) {
  INCH_REQUIRE(w && g && m1 && m2 && step >= 1, INCH_INVALID_ARG, "inch_mp_adam: bad args");
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<blocks(n), kT, 0, s>>>(w, g, m1, m2, n, lr, b1, b2, eps, c1, c2);
  MP_CHECK();
}

extern "C" size_t inch_mp_gemm_workspace_size(int32_t M, int32_t N, int32_t K) {
  const int sp = gemm_splits(M, N, K);
  return sp > 1 ? (size_t)sp * M * N * sizeof(float) + 256 : 256;
}

extern "C" inch_status inch_mp_gemm(int32_t M, int32_t N, int32_t K, const float* A, int64_t sai, int64_t sak,
                                    const float* B, int64_t sbk, int64_t sbn, float* C, int64_t ldc, float beta,
                                    void* ws, size_t ws_bytes, cudaStream_t s) {
  INCH_REQUIRE(A && B && C && M >= 1 && N >= 1 && K >= 1 && ldc >= N, INCH_INVALID_ARG, "inch_mp_gemm: bad args");
  const int sp = gemm_splits(M, N, K);
  float* part = nullptr;
  int kchunk = K;
  if (sp > 1) {
    INCH_REQUIRE(ws != nullptr && ws_bytes >= inch_mp_gemm_workspace_size(M, N, K), INCH_OOM,
                 "inch_mp_gemm: workspace of %zu bytes, need %zu", ws_bytes, inch_mp_gemm_workspace_size(M, N, K));
    part = static_cast<float*>(ws);
    kchunk = ((K + sp - 1) / sp + kGK - 1) / kGK * kGK;
  }
  const int zs = (K + kchunk - 1) / kchunk;
  dim3 g((N + kGN - 1) / kGN, (M + kGM - 1) / kGM, zs);
  k_gemm<<<g, 256, 0, s>>>(M, N, K, A, sai, sak, B, sbk, sbn, C, ldc, beta, kchunk, part);
  INCH_LAUNCH_CHECK();
  if (part != nullptr) {
    k_gemm_reduce<<<blocks((int64_t)M * N), kT, 0, s>>>(M, N, zs, part, C, ldc, beta);
    INCH_LAUNCH_CHECK();
  }
  return INCH_OK;
}
