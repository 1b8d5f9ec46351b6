// Batched symmetric eigensolver for many small matrices (the per-structure
// Rayleigh-Ritz problems of the batched solve: a few dozen columns each, hundreds
// of structures).  No reference counterpart (the reference solves one projected
// matrix at a time on the host, numpy.linalg.eigh).
//
// One CTA per matrix, the matrix and its eigenvector accumulator in shared memory.
// Cyclic Jacobi with the round-robin ("circle") pair ordering: in each of the P-1
// rounds of a sweep the P/2 pairs are disjoint, so their rotations are computed and
// applied in parallel (A <- A J on columns, then A <- J^T A on rows, V <- V J).
// Sweeps stop when the off-diagonal Frobenius norm falls below tol times the
// matrix's, or after max_sweeps (bounded; the number used is reported).  Jacobi
// reaches full FP64 accuracy on small symmetric matrices (Demmel & Veselic 1992).
#include <cmath>

#include "common.cuh"

namespace inch {
namespace {

constexpr int kPMax = 64;
constexpr int kLd = kPMax + 1;       // padded row length in shared memory
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads)
k_jacobi_batched(const double* __restrict__ A, int p, double* __restrict__ W, double* __restrict__ V, int max_sweeps,
                 double tol, int* __restrict__ sweeps_out) {
  extern __shared__ double sm[];
  double* a = sm;                        // P x kLd
  double* v = sm + kPMax * kLd;          // P x kLd
  __shared__ double c_s[kPMax / 2], s_s[kPMax / 2];
  __shared__ int pp_s[kPMax / 2], qq_s[kPMax / 2];
  __shared__ double red[kThreads];
  __shared__ int perm[kPMax];
  const int P = (p + 1) & ~1;            // even size; an odd p gets a decoupled zero row/column
  const int64_t m = blockIdx.x;
  const double* Am = A + m * (int64_t)p * p;
  for (int t = threadIdx.x; t < P * P; t += kThreads) {
    const int r = t / P, c = t % P;
    a[r * kLd + c] = (r < p && c < p) ? 0.5 * (Am[r * p + c] + Am[c * p + r]) : 0.0;
    v[r * kLd + c] = (r == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  // Frobenius norm of the matrix (threshold reference)
  double s = 0.0;
  for (int t = threadIdx.x; t < P * P; t += kThreads) {
    const double x = a[(t / P) * kLd + t % P];
    s += x * x;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  const double fro2 = red[0];
  __syncthreads();
  const int half = P / 2;
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    // off-diagonal norm
    double off = 0.0;
    for (int t = threadIdx.x; t < P * P; t += kThreads) {
      const int r = t / P, c = t % P;
      if (r != c) off += a[r * kLd + c] * a[r * kLd + c];
    }
    red[threadIdx.x] = off;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
      __syncthreads();
    }
    const bool done = !(red[0] > tol * tol * fro2);
    __syncthreads();
    if (done) break;
    for (int round = 0; round < P - 1; ++round) {
      if (threadIdx.x < half) {
        const int k = threadIdx.x;
        int i, j;
        if (k == 0) {
          i = P - 1;
          j = round;
        } else {
          i = (round + k) % (P - 1);
          j = (round - k + (P - 1)) % (P - 1);
        }
        const int pq = i < j ? i : j, qq = i < j ? j : i;
        const double apq = a[pq * kLd + qq];
        double c = 1.0, sn = 0.0;
        if (apq != 0.0) {
          const double theta = (a[qq * kLd + qq] - a[pq * kLd + pq]) / (2.0 * apq);
          const double tt = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
          c = 1.0 / sqrt(tt * tt + 1.0);
          sn = tt * c;
        }
        pp_s[k] = pq;
        qq_s[k] = qq;
        c_s[k] = c;
        s_s[k] = sn;
      }
      __syncthreads();
      // columns: A <- A J, V <- V J (each pair touches its own two columns)
      for (int t = threadIdx.x; t < half * P; t += kThreads) {
        const int k = t / P, r = t % P;
        const int i = pp_s[k], j = qq_s[k];
        const double c = c_s[k], sn = s_s[k];
        const double ai = a[r * kLd + i], aj = a[r * kLd + j];
        a[r * kLd + i] = c * ai - sn * aj;
        a[r * kLd + j] = sn * ai + c * aj;
        const double vi = v[r * kLd + i], vj = v[r * kLd + j];
        v[r * kLd + i] = c * vi - sn * vj;
        v[r * kLd + j] = sn * vi + c * vj;
      }
      __syncthreads();
      // rows: A <- J^T A
      for (int t = threadIdx.x; t < half * P; t += kThreads) {
        const int k = t / P, cc = t % P;
        const int i = pp_s[k], j = qq_s[k];
        const double c = c_s[k], sn = s_s[k];
        const double ai = a[i * kLd + cc], aj = a[j * kLd + cc];
        a[i * kLd + cc] = c * ai - sn * aj;
        a[j * kLd + cc] = sn * ai + c * aj;
      }
      __syncthreads();
    }
  }
  // ascending order of the p real eigenvalues (the padding index, if any, is p)
  if (threadIdx.x == 0) {
    for (int i = 0; i < p; ++i) perm[i] = i;
    for (int i = 1; i < p; ++i) {          // insertion sort, p <= 64
      const int x = perm[i];
      const double key = a[x * kLd + x];
      int j = i - 1;
      while (j >= 0 && a[perm[j] * kLd + perm[j]] > key) {
        perm[j + 1] = perm[j];
        --j;
      }
      perm[j + 1] = x;
    }
    if (sweeps_out) sweeps_out[m] = sweep;
  }
  __syncthreads();
  double* Wm = W + m * (int64_t)p;
  double* Vm = V + m * (int64_t)p * p;
  for (int t = threadIdx.x; t < p * p; t += kThreads) {
    const int r = t / p, k = t % p;
    Vm[r * p + k] = v[r * kLd + perm[k]];      // eigenvector k in column k
  }
  for (int k = threadIdx.x; k < p; k += kThreads) Wm[k] = a[perm[k] * kLd + perm[k]];
}

}  // namespace
}  // namespace inch

using namespace inch;

extern "C" inch_status inch_eigh_batched_small(const double* A, int64_t n_mat, int32_t p, double* W, double* V,
                                               int32_t max_sweeps, double tol, int32_t* sweeps_used,
                                               cudaStream_t stream) {
  INCH_REQUIRE(A && W && V, INCH_INVALID_ARG, "inch_eigh_batched_small: NULL argument");
  INCH_REQUIRE(p >= 1 && p <= kPMax, INCH_LIMIT, "inch_eigh_batched_small: p = %d outside 1..%d", p, kPMax);
  INCH_REQUIRE(n_mat >= 1 && n_mat < (int64_t(1) << 31), INCH_INVALID_ARG, "inch_eigh_batched_small: bad count");
  INCH_REQUIRE(max_sweeps >= 1 && max_sweeps <= 100 && tol > 0.0 && std::isfinite(tol), INCH_INVALID_ARG,
               "inch_eigh_batched_small: max_sweeps in 1..100 and tol > 0");
  const size_t smem = size_t(2) * kPMax * kLd * sizeof(double);
  INCH_CUDA(cudaFuncSetAttribute(k_jacobi_batched, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_jacobi_batched<<<(unsigned)n_mat, kThreads, smem, stream>>>(A, p, W, V, max_sweeps, tol, sweeps_used);
  INCH_LAUNCH_CHECK();
  return INCH_OK;
}
