// Hessian x multivector on the rank-one block store, with a fused epilogue.
//
// Reference operator: InchingLiteInteger/Burn/Krylov/T3.py:54-165 computes
// u = L v + L^T v - diag(A) v with two cuSPARSE CSR SpMVs over the scalar lower
// triangle, one vector at a time.  Here one pass streams the full (both
// triangles) rank-one store once per multivector tile:
//     (H X)_i = D_i X_i - sum_j w_ij (w_ij . X_j)
// and applies, per output element, the epilogue
//     Y = alpha*(H X) + gamma*X + beta*Yin + hot_shift * Q^T (Q X)   [Acc += mu*Y]
// which covers the shift of the JD correction operator (JacobiDavidson.../T1.py:
// 67-331), explicit Hotelling deflation (Orthogonalization/T3.py:62-164) and one
// three-term Chebyshev step with its accumulation (PolynomialFilters/T2.py:59-80).
//
// Thread mapping: a group of G lanes owns one atom row (3 dofs x B columns); the
// lanes of the group stride over the row's entries (one 16-byte load per entry in
// FP32, two in FP64), gather X_j from L1/L2 (rows are banded after Cuthill-McKee
// so neighbouring rows share their X_j), and reduce with xor shuffles.
#include <atomic>

#include <cub/cub.cuh>

#include "common.cuh"

namespace inch {
namespace {

struct Epi {
  double alpha, gamma, beta, mu;
  int r, accumulate, has_yin;
  // optional per-segment (alpha, gamma, beta): atom i uses seg_coef[3 * atom_seg[i] ...]
  const double* seg_coef = nullptr;
  const int* atom_seg = nullptr;
};

template <class T>
struct Ent;
template <>
struct Ent<float> {
  __device__ __forceinline__ static void load(const void* base, int64_t e, float& wx, float& wy, float& wz, int& j) {
    float4 v = __ldg(reinterpret_cast<const float4*>(base) + e);
    wx = v.x;
    wy = v.y;
    wz = v.z;
    j = __float_as_int(v.w);
  }
  // streaming load (evict-first): an entry read once per product should not push
  // the gathered vector rows out of L1
  __device__ __forceinline__ static void load_cs(const void* base, int64_t e, float& wx, float& wy, float& wz,
                                                 int& j) {
    float4 v = __ldcs(reinterpret_cast<const float4*>(base) + e);
    wx = v.x;
    wy = v.y;
    wz = v.z;
    j = __float_as_int(v.w);
  }
};
template <>
struct Ent<double> {
  __device__ __forceinline__ static void load(const void* base, int64_t e, double& wx, double& wy, double& wz,
                                              int& j) {
    const double2* p = reinterpret_cast<const double2*>(base) + 2 * e;
    double2 a = __ldg(p), b = __ldg(p + 1);
    wx = a.x;
    wy = a.y;
    wz = b.x;
    j = static_cast<int>(b.y);
  }
  __device__ __forceinline__ static void load_cs(const void* base, int64_t e, double& wx, double& wy, double& wz,
                                                 int& j) {
    const double2* p = reinterpret_cast<const double2*>(base) + 2 * e;
    double2 a = __ldcs(p), b = __ldcs(p + 1);
    wx = a.x;
    wy = a.y;
    wz = b.x;
    j = static_cast<int>(b.y);
  }
};

constexpr int kThreads = 256;

// Launch shape of the wide-block kernel (threads per block, blocks per SM):
// process-wide, set by inch_spmm_tune (the autotuner's hook).
std::atomic<int> g_cols_threads{256};
std::atomic<int> g_cols_blocks_per_sm{5};
std::atomic<int> g_warp_kernel{0};   // 1: whole-warp rows with batched gathers where B/V >= 32
// Row traversal of the wide-block kernel when a workspace holds a row counter:
// 0 fixed block-interleaved stride, 1 per-warp chunks from the counter, 2 per-block
// chunks from the counter (set by inch_spmm_traversal, the autotuner's hook).
std::atomic<int> g_cols_traversal{1};

template <class T, int B, int G>
__global__ void __launch_bounds__(kThreads)
k_spmm(int64_t n_atoms, const int64_t* __restrict__ rowptr, const void* __restrict__ ent,
       const T* __restrict__ diag, const T* __restrict__ X, int64_t ldx, T* Y, int64_t ldy, const T* Yin,
       int64_t ldyin, T* __restrict__ Acc, int64_t ldacc, int c0, Epi ep, const double* __restrict__ Q,
       int64_t ndof, const double* __restrict__ coef) {
  __shared__ double s_coef[8 * B];
  if (ep.r > 0) {
    for (int t = threadIdx.x; t < ep.r * B; t += kThreads) s_coef[t] = coef[t];
    __syncthreads();
  }
  const int lg = threadIdx.x % G;
  const int64_t groups = (int64_t)gridDim.x * (kThreads / G);
  for (int64_t i = (int64_t)blockIdx.x * (kThreads / G) + threadIdx.x / G; i < n_atoms; i += groups) {
    T acc[3][B];
#pragma unroll
    for (int c = 0; c < B; ++c) acc[0][c] = acc[1][c] = acc[2][c] = T(0);
    const int64_t e1 = rowptr[i + 1];
#pragma unroll 2
    for (int64_t e = rowptr[i] + lg; e < e1; e += G) {
      T wx, wy, wz;
      int j;
      Ent<T>::load_cs(ent, e, wx, wy, wz, j);
      const T* xj = X + 3 * (int64_t)j * ldx + c0;
#pragma unroll
      for (int c = 0; c < B; ++c) {
        T dot = wx * __ldg(xj + c) + wy * __ldg(xj + ldx + c) + wz * __ldg(xj + 2 * ldx + c);
        acc[0][c] -= wx * dot;
        acc[1][c] -= wy * dot;
        acc[2][c] -= wz * dot;
      }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
#pragma unroll
      for (int c = 0; c < B; ++c) {
        acc[0][c] += __shfl_xor_sync(0xffffffffu, acc[0][c], o);
        acc[1][c] += __shfl_xor_sync(0xffffffffu, acc[1][c], o);
        acc[2][c] += __shfl_xor_sync(0xffffffffu, acc[2][c], o);
      }
    }
    const T* d = diag + 8 * i;
    const T dxx = d[0], dyy = d[1], dzz = d[2], dxy = d[3], dxz = d[4], dyz = d[5];
#pragma unroll
    for (int c = 0; c < B; ++c) {
      if ((c % G) != lg) continue;
      const int64_t r0 = 3 * i;
      const T x0 = X[r0 * ldx + c0 + c], x1 = X[(r0 + 1) * ldx + c0 + c], x2 = X[(r0 + 2) * ldx + c0 + c];
      T h[3];
      h[0] = acc[0][c] + dxx * x0 + dxy * x1 + dxz * x2;
      h[1] = acc[1][c] + dxy * x0 + dyy * x1 + dyz * x2;
      h[2] = acc[2][c] + dxz * x0 + dyz * x1 + dzz * x2;
      const T xs[3] = {x0, x1, x2};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int64_t row = r0 + a;
        double al = ep.alpha, ga = ep.gamma, be = ep.beta;
        if (ep.seg_coef != nullptr) {
          const int sg = __ldg(ep.atom_seg + i);
          al = __ldg(ep.seg_coef + 3 * sg);
          ga = __ldg(ep.seg_coef + 3 * sg + 1);
          be = __ldg(ep.seg_coef + 3 * sg + 2);
        }
        double y = al * (double)h[a] + ga * (double)xs[a];
        if (ep.has_yin) y += be * (double)Yin[row * ldyin + c0 + c];
        for (int q = 0; q < ep.r; ++q) y += Q[q * ndof + row] * s_coef[q * B + c];
        Y[row * ldy + c0 + c] = (T)y;
        if (ep.accumulate) Acc[row * ldacc + c0 + c] += (T)(ep.mu * y);
      }
    }
  }
}

// Wide multivectors: lanes map to columns.  A group of LPR lanes owns one row;
// each lane owns V consecutive columns per chunk (V = 2 -> float2/double2 loads).
// Every lane of the group reads the same 16-byte entry (one broadcast
// transaction) and the group reads each X_j row as one coalesced segment.
// Each block walks one contiguous slab of rows (its warps on neighbouring rows at
// the same time), so the X_j rows shared by neighbouring atoms are reused from
// L1.  No shuffles: each lane accumulates its own columns.
template <class T, int V>
struct VecT;
template <>
struct VecT<float, 1> {
  using t = float;
};
template <>
struct VecT<float, 2> {
  using t = float2;
};
template <>
struct VecT<double, 1> {
  using t = double;
};
template <>
struct VecT<float, 4> {
  using t = float4;
};
template <>
struct VecT<double, 2> {
  using t = double2;
};

template <class T, int V>
__device__ __forceinline__ void vld(const T* p, T (&x)[V]) {
  if constexpr (V == 1) {
    x[0] = __ldg(p);
  } else if constexpr (V == 4) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    x[0] = v.x;
    x[1] = v.y;
    x[2] = v.z;
    x[3] = v.w;
  } else {
    const typename VecT<T, 2>::t v = __ldg(reinterpret_cast<const typename VecT<T, 2>::t*>(p));
    x[0] = v.x;
    x[1] = v.y;
  }
}

// Steps of rows a warp takes per grab of the row counter: warps take chunks of
// consecutive rows in order, so all SMs work on one compact frontier and the
// X_j rows they gather stay an L2-sized window, however far blocks would drift
// apart under a fixed grid stride (on the 2.4M-atom cube the fixed stride read
// 11x the algorithmic bytes from DRAM).
constexpr int kRowSteps = 4;

template <class T>
__device__ __forceinline__ T mad(T a, T b, T c);
template <>
__device__ __forceinline__ float mad<float>(float a, float b, float c) {
  return __fmaf_rn(a, b, c);
}
template <>
__device__ __forceinline__ double mad<double>(double a, double b, double c) {
  return __fma_rn(a, b, c);
}

template <int B, int V>
constexpr int lanes_per_row() {
  return (B / V) < 32 ? (B / V) : 32;
}
template <int B, int V>
constexpr int cols_per_lane() {
  return B / (lanes_per_row<B, V>() * V);
}

// Output of atom row i: h = D_i X_i + acc (acc = -sum_j w_ij (w_ij . X_j), or its
// negation when NEG) followed by the fused epilogue.  Columns at or beyond nc (a
// partial last tile) are neither read nor written.
template <class T, int B, int V, bool NEG>
__device__ __forceinline__ void row_out(int64_t i, const T (&acc)[3][cols_per_lane<B, V>()][V], int nc,
                                        const T* __restrict__ diag, const T* __restrict__ X, int64_t ldx, T* Y,
                                        int64_t ldy, const T* Yin, int64_t ldyin, T* __restrict__ Acc,
                                        int64_t ldacc, int c0, const Epi& ep, const double* __restrict__ Q,
                                        int64_t ndof, const double* s_coef, int cl) {
  constexpr int LPR = lanes_per_row<B, V>();
  constexpr int CPL = cols_per_lane<B, V>();
  const T* d = diag + 8 * i;
  const T dxx = d[0], dyy = d[1], dzz = d[2], dxy = d[3], dxz = d[4], dyz = d[5];
  const int64_t r0 = 3 * i;
  double al = ep.alpha, ga = ep.gamma, be = ep.beta;
  if (ep.seg_coef != nullptr) {
    const int sg = __ldg(ep.atom_seg + i);
    al = __ldg(ep.seg_coef + 3 * sg);
    ga = __ldg(ep.seg_coef + 3 * sg + 1);
    be = __ldg(ep.seg_coef + 3 * sg + 2);
  }
#pragma unroll
  for (int t = 0; t < CPL; ++t) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int c = (t * LPR + cl) * V + v;
      if (c >= nc) continue;
      const T x0 = X[r0 * ldx + c0 + c], x1 = X[(r0 + 1) * ldx + c0 + c], x2 = X[(r0 + 2) * ldx + c0 + c];
      const T a0 = NEG ? -acc[0][t][v] : acc[0][t][v];
      const T a1 = NEG ? -acc[1][t][v] : acc[1][t][v];
      const T a2 = NEG ? -acc[2][t][v] : acc[2][t][v];
      T h[3];
      h[0] = mad(dxz, x2, mad(dxy, x1, mad(dxx, x0, a0)));
      h[1] = mad(dyz, x2, mad(dyy, x1, mad(dxy, x0, a1)));
      h[2] = mad(dzz, x2, mad(dyz, x1, mad(dxz, x0, a2)));
      const T xs[3] = {x0, x1, x2};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int64_t row = r0 + a;
        double y = al * (double)h[a] + ga * (double)xs[a];
        if (ep.has_yin) y += be * (double)Yin[row * ldyin + c0 + c];
        for (int q = 0; q < ep.r; ++q) y += Q[q * ndof + row] * s_coef[q * B + c];
        Y[row * ldy + c0 + c] = (T)y;
        if (ep.accumulate) Acc[row * ldacc + c0 + c] += (T)(ep.mu * y);
      }
    }
  }
}

template <class T, int B, int V, int NT>
__device__ __forceinline__ void cols_row(int64_t i, const int64_t* __restrict__ rowptr, const void* __restrict__ ent,
                                         const T* __restrict__ diag, const T* __restrict__ X, int64_t ldx, T* Y,
                                         int64_t ldy, const T* Yin, int64_t ldyin, T* __restrict__ Acc,
                                         int64_t ldacc, int c0, const Epi& ep, const double* __restrict__ Q,
                                         int64_t ndof, const double* s_coef, int cl) {
  constexpr int LPR = lanes_per_row<B, V>();
  constexpr int CPL = cols_per_lane<B, V>();
  T acc[3][CPL][V];
#pragma unroll
  for (int t = 0; t < CPL; ++t)
#pragma unroll
    for (int v = 0; v < V; ++v) acc[0][t][v] = acc[1][t][v] = acc[2][t][v] = T(0);
  const int64_t e1 = rowptr[i + 1];
  const T* Xc = X + c0 + cl * V;
  // 128-column rows (float4 gathers) keep four entries' loads in flight
  constexpr int kUnrollE = B >= 128 ? 4 : 2;
#pragma unroll kUnrollE
  for (int64_t e = rowptr[i]; e < e1; ++e) {
    T wx, wy, wz;
    int j;
    Ent<T>::load(ent, e, wx, wy, wz, j);
    const T* xj = Xc + 3 * (int64_t)j * ldx;
#pragma unroll
    for (int t = 0; t < CPL; ++t) {
      T x0[V], x1[V], x2[V];
      vld<T, V>(xj + t * LPR * V, x0);
      vld<T, V>(xj + ldx + t * LPR * V, x1);
      vld<T, V>(xj + 2 * ldx + t * LPR * V, x2);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        // dot = ((wx x0) + wy x1) + wz x2, each step one rounding (the row-group
        // kernel repeats this order, so both layouts give the same bits)
        const T dot = mad(wz, x2[v], mad(wy, x1[v], wx * x0[v]));
        acc[0][t][v] = mad(-wx, dot, acc[0][t][v]);
        acc[1][t][v] = mad(-wy, dot, acc[1][t][v]);
        acc[2][t][v] = mad(-wz, dot, acc[2][t][v]);
      }
    }
  }
  row_out<T, B, V, false>(i, acc, B, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, ep, Q, ndof, s_coef, cl);
}

template <class T, int B, int V, int NT>
__global__ void __launch_bounds__(NT)
k_spmm_cols(int64_t n_atoms, const int64_t* __restrict__ rowptr, const void* __restrict__ ent,
            const T* __restrict__ diag, const T* __restrict__ X, int64_t ldx, T* Y, int64_t ldy, const T* Yin,
            int64_t ldyin, T* __restrict__ Acc, int64_t ldacc, int c0, Epi ep, const double* __restrict__ Q,
            int64_t ndof, const double* __restrict__ coef, int* __restrict__ row_counter, int traversal) {
  constexpr int LPR = (B / V) < 32 ? (B / V) : 32;
  constexpr int RPW = 32 / LPR;
  constexpr int GPB = (NT / 32) * RPW;
  __shared__ double s_coef[8 * B];
  __shared__ int s_row;
  if (ep.r > 0) {
    for (int t = threadIdx.x; t < ep.r * B; t += NT) s_coef[t] = coef[t];
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const int cl = lane % LPR;
  const int grp = (threadIdx.x >> 5) * RPW + lane / LPR;
  if (row_counter == nullptr || traversal == 0) {
    // fixed block-interleaved stride: the grid starts on one band of consecutive
    // rows, each block's warps on neighbouring rows (their X_j rows shared in L1)
    for (int64_t i = (int64_t)blockIdx.x * GPB + grp; i < n_atoms; i += (int64_t)gridDim.x * GPB)
      cols_row<T, B, V, NT>(i, rowptr, ent, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, ep, Q, ndof, s_coef,
                            cl);
    return;
  }
  if (traversal == 2) {
    // each block takes a chunk of kRowSteps * GPB consecutive rows, its warps on
    // neighbouring rows (compact frontier and L1 sharing, one barrier per chunk)
    for (;;) {
      if (threadIdx.x == 0) s_row = atomicAdd(row_counter, GPB * kRowSteps);
      __syncthreads();
      const int64_t base = s_row;
      __syncthreads();                   // every thread has read s_row before the next grab
      if (base >= n_atoms) break;
#pragma unroll 1
      for (int st = 0; st < kRowSteps; ++st) {
        const int64_t i = base + st * GPB + grp;
        if (i < n_atoms)
          cols_row<T, B, V, NT>(i, rowptr, ent, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, ep, Q, ndof,
                                s_coef, cl);
      }
    }
    return;
  }
  // each warp takes its own chunk of kRowSteps * RPW consecutive rows (no block
  // barrier, so a long row holds back only its own warp)
  const int wg = lane / LPR;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(row_counter, RPW * kRowSteps);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n_atoms) break;
#pragma unroll 1
    for (int st = 0; st < kRowSteps; ++st) {
      const int64_t i = (int64_t)base + st * RPW + wg;
      if (i < n_atoms)
        cols_row<T, B, V, NT>(i, rowptr, ent, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, ep, Q, ndof,
                              s_coef, cl);
    }
  }
}

// Whole-warp rows (B / V >= 32 columns per lane-row): the warp loads 32 entries of
// its row at once (one coalesced 512-byte load), broadcasts them by shuffle and
// issues the X_j gathers of U entries back to back, so U * 3 gathers per warp are
// in flight instead of 3.  Tail slots use w = 0 and j = the row itself.
template <class T, int B, int V, int U>
__global__ void __launch_bounds__(kThreads)
k_spmm_warp(int64_t n_atoms, const int64_t* __restrict__ rowptr, const void* __restrict__ ent,
            const T* __restrict__ diag, const T* __restrict__ X, int64_t ldx, T* Y, int64_t ldy, const T* Yin,
            int64_t ldyin, T* __restrict__ Acc, int64_t ldacc, int c0, Epi ep, const double* __restrict__ Q,
            int64_t ndof, const double* __restrict__ coef) {
  constexpr int CPL = B / (32 * V);
  static_assert(CPL >= 1, "whole-warp rows need B / V >= 32");
  constexpr int WPB = kThreads / 32;
  __shared__ double s_coef[8 * B];
  if (ep.r > 0) {
    for (int t = threadIdx.x; t < ep.r * B; t += kThreads) s_coef[t] = coef[t];
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t per = (n_atoms + gridDim.x - 1) / gridDim.x;
  const int64_t r_beg = (int64_t)blockIdx.x * per;
  const int64_t r_end = r_beg + per < n_atoms ? r_beg + per : n_atoms;
  for (int64_t i = r_beg + warp; i < r_end; i += WPB) {
    T acc[3][CPL][V];
#pragma unroll
    for (int t = 0; t < CPL; ++t)
#pragma unroll
      for (int v = 0; v < V; ++v) acc[0][t][v] = acc[1][t][v] = acc[2][t][v] = T(0);
    const int64_t e0 = rowptr[i], e1 = rowptr[i + 1];
    const T* Xc = X + c0 + lane * V;
    for (int64_t base = e0; base < e1; base += 32) {
      const int cnt = (int)((e1 - base) < 32 ? (e1 - base) : 32);
      T mx = T(0), my = T(0), mz = T(0);
      int mj = static_cast<int>(i);
      if (lane < cnt) Ent<T>::load(ent, base + lane, mx, my, mz, mj);
      for (int k = 0; k < cnt; k += U) {
        T wx[U], wy[U], wz[U];
        T xv[U][3][CPL][V];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          wx[u] = __shfl_sync(0xffffffffu, mx, (k + u) & 31);
          wy[u] = __shfl_sync(0xffffffffu, my, (k + u) & 31);
          wz[u] = __shfl_sync(0xffffffffu, mz, (k + u) & 31);
          const int j = __shfl_sync(0xffffffffu, mj, (k + u) & 31);
          // slots past the end of the row carry w = 0 (lanes >= cnt loaded nothing)
          const T* xj = Xc + 3 * (int64_t)j * ldx;
#pragma unroll
          for (int t = 0; t < CPL; ++t) {
            vld<T, V>(xj + t * 32 * V, xv[u][0][t]);
            vld<T, V>(xj + ldx + t * 32 * V, xv[u][1][t]);
            vld<T, V>(xj + 2 * ldx + t * 32 * V, xv[u][2][t]);
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
          for (int t = 0; t < CPL; ++t)
#pragma unroll
            for (int v = 0; v < V; ++v) {
              const T dot = wx[u] * xv[u][0][t][v] + wy[u] * xv[u][1][t][v] + wz[u] * xv[u][2][t][v];
              acc[0][t][v] -= wx[u] * dot;
              acc[1][t][v] -= wy[u] * dot;
              acc[2][t][v] -= wz[u] * dot;
            }
      }
    }
    const T* d = diag + 8 * i;
    const T dxx = d[0], dyy = d[1], dzz = d[2], dxy = d[3], dxz = d[4], dyz = d[5];
    const int64_t r0 = 3 * i;
#pragma unroll
    for (int t = 0; t < CPL; ++t) {
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int c = (t * 32 + lane) * V + v;
        const T x0 = X[r0 * ldx + c0 + c], x1 = X[(r0 + 1) * ldx + c0 + c], x2 = X[(r0 + 2) * ldx + c0 + c];
        T h[3];
        h[0] = acc[0][t][v] + dxx * x0 + dxy * x1 + dxz * x2;
        h[1] = acc[1][t][v] + dxy * x0 + dyy * x1 + dyz * x2;
        h[2] = acc[2][t][v] + dxz * x0 + dyz * x1 + dzz * x2;
        const T xs[3] = {x0, x1, x2};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int64_t row = r0 + a;
          double al = ep.alpha, ga = ep.gamma, be = ep.beta;
        if (ep.seg_coef != nullptr) {
          const int sg = __ldg(ep.atom_seg + i);
          al = __ldg(ep.seg_coef + 3 * sg);
          ga = __ldg(ep.seg_coef + 3 * sg + 1);
          be = __ldg(ep.seg_coef + 3 * sg + 2);
        }
        double y = al * (double)h[a] + ga * (double)xs[a];
          if (ep.has_yin) y += be * (double)Yin[row * ldyin + c0 + c];
          for (int q = 0; q < ep.r; ++q) y += Q[q * ndof + row] * s_coef[q * B + c];
          Y[row * ldy + c0 + c] = (T)y;
          if (ep.accumulate) Acc[row * ldacc + c0 + c] += (T)(ep.mu * y);
        }
      }
    }
  }
}

// Partial sums of Q X over a dof range (blockIdx.x), one deflation vector per
// blockIdx.y; thread t accumulates column t % B.
template <class T, int B>
__global__ void __launch_bounds__(kThreads)
k_qx_partial(const double* __restrict__ Q, int64_t ndof, const T* __restrict__ X, int64_t ldx, int c0,
             double* __restrict__ partial, int nc = B) {
  const int q = blockIdx.y, r = gridDim.y;
  const double* qr = Q + q * ndof;
  const int c = threadIdx.x % B;
  double acc = 0.0;
  const int64_t total = ndof * B;
  for (int64_t p = (int64_t)blockIdx.x * kThreads + threadIdx.x; p < total; p += (int64_t)gridDim.x * kThreads) {
    const int64_t dof = p / B;
    if (c < nc) acc += qr[dof] * (double)X[dof * ldx + c0 + c];   // columns past nc: outside the tile
  }
  __shared__ double s[kThreads];
  s[threadIdx.x] = acc;
  __syncthreads();
  // tree over the threads of one column (B is a power of two dividing kThreads,
  // so t and t + stride always share a column): log2(kThreads / B) steps
#pragma unroll
  for (int stride = kThreads / 2; stride >= B; stride >>= 1) {
    if (threadIdx.x < stride) s[threadIdx.x] += s[threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x < B) partial[((int64_t)blockIdx.x * r + q) * B + threadIdx.x] = s[threadIdx.x];
}

// coef[t] = shift * sum_p partial[p, t]: one warp per output (vector, column), its
// lanes striding over the P partials, then a fixed shuffle tree (deterministic).
__global__ void __launch_bounds__(kThreads)
k_qx_final(const double* __restrict__ partial, int P, int r, int B, double shift, double* __restrict__ coef) {
  const int t = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (t >= r * B) return;
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int p = lane; p < P; p += 32) s += partial[(int64_t)p * r * B + t];
  s = warp_sum(s);
  if (lane == 0) coef[t] = shift * s;
}

constexpr int kQxBlocks = 296;

template <class T, int B, int G>
cudaError_t launch_tile(int64_t n_atoms, const int64_t* rowptr, const void* ent, const T* diag, const T* X,
                        int64_t ldx, T* Y, int64_t ldy, const T* Yin, int64_t ldyin, T* Acc, int64_t ldacc, int c0,
                        Epi ep, const double* Q, double hot_shift, double* partial, double* coef,
                        cudaStream_t stream, int* row_counter) {
  const int64_t ndof = 3 * n_atoms;
  if (ep.r > 0) {
    dim3 g(kQxBlocks, ep.r);
    k_qx_partial<T, B><<<g, kThreads, 0, stream>>>(Q, ndof, X, ldx, c0, partial);
    k_qx_final<<<(ep.r * B + kThreads / 32 - 1) / (kThreads / 32), kThreads, 0, stream>>>(partial, kQxBlocks,
                                                                                          ep.r, B, hot_shift, coef);
  }
  if constexpr (G == 0) {
    // Vector (V = 2) gathers need X, Y (and Yin / Acc when used) rows aligned to
    // 2 elements: every leading dimension and the column offset even, bases aligned.
    const uintptr_t al = 2 * sizeof(T);
    bool vec = (ldx % 2 == 0) && (ldy % 2 == 0) && (c0 % 2 == 0) && ((uintptr_t)X % al == 0) &&
               ((uintptr_t)Y % al == 0);
    if (ep.has_yin) vec = vec && (ldyin % 2 == 0) && ((uintptr_t)Yin % al == 0);
    if (ep.accumulate) vec = vec && (ldacc % 2 == 0) && ((uintptr_t)Acc % al == 0);
    const int nt = g_cols_threads.load();
    const int bps = g_cols_blocks_per_sm.load();
    const int trav = row_counter != nullptr ? g_cols_traversal.load() : 0;
    if (trav != 0) {
      const cudaError_t me = cudaMemsetAsync(row_counter, 0, sizeof(int), stream);
      if (me != cudaSuccess) return me;
    }
#define COLS_LAUNCH(NTV)                                                                                     \
  {                                                                                                           \
    const int blocks = grid_for(n_atoms, 4 * NTV / 32, 148 * bps);                                            \
    if constexpr (B == 128 && sizeof(T) == 4) {                                                               \
      k_spmm_cols<T, B, 4, NTV><<<blocks, NTV, 0, stream>>>(n_atoms, rowptr, ent, diag, X, ldx, Y, ldy, Yin,   \
                                                            ldyin, Acc, ldacc, c0, ep, Q, ndof, coef,        \
                                                            row_counter, trav);                              \
    } else if (vec)                                                                                           \
      k_spmm_cols<T, B, 2, NTV><<<blocks, NTV, 0, stream>>>(n_atoms, rowptr, ent, diag, X, ldx, Y, ldy, Yin,   \
                                                            ldyin, Acc, ldacc, c0, ep, Q, ndof, coef,        \
                                                            row_counter, trav);                              \
    else                                                                                                      \
      k_spmm_cols<T, B, 1, NTV><<<blocks, NTV, 0, stream>>>(n_atoms, rowptr, ent, diag, X, ldx, Y, ldy, Yin,   \
                                                            ldyin, Acc, ldacc, c0, ep, Q, ndof, coef,        \
                                                            row_counter, trav);                              \
  }
    const int wmode = g_warp_kernel.load();
    if (wmode > 0 && B >= 32 && (vec || B >= 32)) {
      const int blocks = grid_for(n_atoms, kThreads / 32, 148 * bps);
      if constexpr (B >= 64) {
        if (vec)
          k_spmm_warp<T, B, 2, 4><<<blocks, kThreads, 0, stream>>>(n_atoms, rowptr, ent, diag, X, ldx, Y, ldy, Yin,
                                                                    ldyin, Acc, ldacc, c0, ep, Q, ndof, coef);
        else
          k_spmm_warp<T, B, 1, 4><<<blocks, kThreads, 0, stream>>>(n_atoms, rowptr, ent, diag, X, ldx, Y, ldy, Yin,
                                                                    ldyin, Acc, ldacc, c0, ep, Q, ndof, coef);
      } else if constexpr (B >= 32) {
        k_spmm_warp<T, B, 1, 4><<<blocks, kThreads, 0, stream>>>(n_atoms, rowptr, ent, diag, X, ldx, Y, ldy, Yin,
                                                                  ldyin, Acc, ldacc, c0, ep, Q, ndof, coef);
      }
    } else if (nt == 1024) COLS_LAUNCH(1024)
    else if (nt == 512) COLS_LAUNCH(512)
    else COLS_LAUNCH(256)
#undef COLS_LAUNCH
  } else {
    const int rows_per_block = kThreads / G;
    const int blocks = grid_for(n_atoms, rows_per_block, 148 * 16);
    k_spmm<T, B, G><<<blocks, kThreads, 0, stream>>>(n_atoms, rowptr, ent, diag, X, ldx, Y, ldy, Yin, ldyin, Acc,
                                                     ldacc, c0, ep, Q, ndof, coef);
  }
  return cudaGetLastError();
}

template <class T>
cudaError_t run(int64_t n_atoms, const int64_t* rowptr, const void* ent, const void* diag, const void* Xv,
                int64_t ldx, int b, void* Yv, int64_t ldy, const void* Yinv, int64_t ldyin, void* Accv, int64_t ldacc,
                Epi ep, const double* Q, double hot_shift, double* partial, double* coef, cudaStream_t s,
                int* row_counter = nullptr) {
  const T* X = static_cast<const T*>(Xv);
  T* Y = static_cast<T*>(Yv);
  const T* Yin = static_cast<const T*>(Yinv);
  T* Acc = static_cast<T*>(Accv);
  const T* D = static_cast<const T*>(diag);
  int c0 = 0;
  cudaError_t e = cudaSuccess;
  while (c0 < b && e == cudaSuccess) {
    const int rem = b - c0;
#define TILE(BB, GG)                                                                                          \
  e = launch_tile<T, BB, GG>(n_atoms, rowptr, ent, D, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, ep, Q,     \
                             hot_shift, partial, coef, s, row_counter);                                        \
  c0 += BB;
    bool done64 = false;
    if constexpr (sizeof(T) == 4) {
      // 128-column tiles gather float4 rows: every vector row 16-byte aligned
      const bool al16 = (ldx % 4 == 0) && (ldy % 4 == 0) && (c0 % 4 == 0) && ((uintptr_t)X % 16 == 0) &&
                        ((uintptr_t)Y % 16 == 0) && (!ep.has_yin || ((ldyin % 4 == 0) && ((uintptr_t)Yin % 16 == 0))) &&
                        (!ep.accumulate || ((ldacc % 4 == 0) && ((uintptr_t)Acc % 16 == 0)));
      if (rem >= 128 && al16) {
        TILE(128, 0)
        done64 = true;
      } else if (rem >= 64) {
        TILE(64, 0)
        done64 = true;
      }
    }
    if (done64) {
    } else if (rem >= 32) { TILE(32, 0) }
    else if (rem >= 16) { TILE(16, 0) }
    else if (rem >= 8) { TILE(8, 0) }
    else if (rem >= 4) { TILE(4, 8) }
    else if (rem >= 2) { TILE(2, 8) }
    else { TILE(1, 8) }
#undef TILE
  }
  return e;
}

// ---------------------------------------------------------------------------
// Row-group layout (FP32): R consecutive atom rows (R = 2 or 4) merged over their
// sorted neighbour lists.  Group g covers atoms [R g, R g + R); its union column
// u holds R float4 slots, slot r = {wx, wy, wz, .} of row R g + r's entry for that
// column, or zeros when the row has none; slot 0's last field holds the column
// index.  A row's entries keep their order inside the union (the merge is stable
// per row and repeated columns stay separate unions), so each row sums the same
// terms in the same order as in the pair layout, with exact zeros in between.
// One gather of X_j then serves every row of the group that needs it: after
// Cuthill-McKee, consecutive rows share most of their neighbours (100k-atom
// assembly: 1.36 pairs per union for R = 2, 1.87 for R = 4), and the pair
// product is bound by these gathers (L2 -> SM).
// ---------------------------------------------------------------------------
constexpr int kGroupBuildThreads = 256;
constexpr int kGroupSteps = 4;   // groups a warp takes per grab of the counter
// Each group's union count is padded to a multiple of kGroupPad with zero-weight
// unions (column = the group's first atom), so the product walks whole chunks.
constexpr int kGroupPad = 16;

// One thread per group: an R-way merge over the rows' entries.  Pass 0 counts the
// (padded) unions of each group, pass 1 writes them at gptr[g].
template <int PASS, int R>
__global__ void __launch_bounds__(kGroupBuildThreads)
k_group_merge(int64_t n, const int64_t* __restrict__ rowptr, const float4* __restrict__ ent,
              int64_t* __restrict__ count, const int64_t* __restrict__ gptr, float4* __restrict__ gent) {
  const int64_t ng = (n + R - 1) / R;
  for (int64_t g = (int64_t)blockIdx.x * kGroupBuildThreads + threadIdx.x; g < ng;
       g += (int64_t)gridDim.x * kGroupBuildThreads) {
    int64_t e[R], e1[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t i = R * g + r;
      e[r] = i < n ? rowptr[i] : 0;
      e1[r] = i < n ? rowptr[i + 1] : 0;
    }
    const int64_t ubase = PASS == 1 ? gptr[g] : 0;
    int64_t u = ubase;
    for (;;) {
      int head[R];
      int m = 0x7fffffff;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        head[r] = e[r] < e1[r] ? __float_as_int(ent[e[r]].w) : 0x7fffffff;
        m = min(m, head[r]);
      }
      if (m == 0x7fffffff) break;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const bool take = head[r] == m;
        if (PASS == 1) {
          float4 w = take ? ent[e[r]] : make_float4(0.f, 0.f, 0.f, 0.f);
          w.w = r == 0 ? __int_as_float(m) : 0.f;
          gent[R * u + r] = w;
        }
        if (take) ++e[r];
      }
      ++u;
    }
    const int64_t u_end = ubase + (u - ubase + kGroupPad - 1) / kGroupPad * kGroupPad;
    if (PASS == 1) {
      for (; u < u_end; ++u)
#pragma unroll
        for (int r = 0; r < R; ++r)
          gent[R * u + r] = make_float4(0.f, 0.f, 0.f, r == 0 ? __int_as_float((int)(R * g)) : 0.f);
    }
    if (PASS == 0) count[g] = u_end;
  }
}

__global__ void k_set0(int64_t* a) { a[0] = 0; }

// float2 view of V consecutive floats (V = 2 or 4)
template <int V>
struct F2 {
  float2 v[V / 2];
};

template <int V>
__device__ __forceinline__ void vld2(const float* p, F2<V>& x) {
  if constexpr (V == 4) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    x.v[0] = make_float2(t.x, t.y);
    x.v[1] = make_float2(t.z, t.w);
  } else {
    x.v[0] = __ldg(reinterpret_cast<const float2*>(p));
  }
}

// Narrow tile (V = 1, B = 32): one warp, one group, lane l owns column l; nc < 32
// masks a partial last tile.
template <int R, int B, int V, int U>
__device__ __forceinline__ void group_rows(int64_t g, int64_t n_atoms, const int64_t* __restrict__ gptr,
                                           const float4* __restrict__ gent, const float* __restrict__ diag,
                                           const float* __restrict__ X, int64_t ldx, float* Y, int64_t ldy,
                                           const float* Yin, int64_t ldyin, float* __restrict__ Acc, int64_t ldacc,
                                           int c0, int nc, const Epi& ep, const double* __restrict__ Q,
                                           int64_t ndof, const double* s_coef, int lane) {
  static_assert(B == 32 && V == 1, "narrow tile");
  // acc holds +sum_j w (w . X_j); row_out negates it
  float acc[R][3][1][1];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r][0][0][0] = acc[r][1][0][0] = acc[r][2][0][0] = 0.f;
  const int64_t u1 = gptr[g + 1];
  const float* Xc = X + c0 + lane;
  const bool live = lane < nc;
#pragma unroll U
  for (int64_t u = gptr[g]; u < u1; ++u) {
    float4 s[R];
#pragma unroll
    for (int r = 0; r < R; ++r) s[r] = __ldg(gent + R * u + r);
    const float* xj = Xc + 3 * (int64_t)__float_as_int(s[0].w) * ldx;
    float x0 = 0.f, x1 = 0.f, x2 = 0.f;
    if (live) {
      x0 = __ldg(xj);
      x1 = __ldg(xj + ldx);
      x2 = __ldg(xj + 2 * ldx);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const float dot = __fmaf_rn(s[r].z, x2, __fmaf_rn(s[r].y, x1, s[r].x * x0));
      acc[r][0][0][0] = __fmaf_rn(s[r].x, dot, acc[r][0][0][0]);
      acc[r][1][0][0] = __fmaf_rn(s[r].y, dot, acc[r][1][0][0]);
      acc[r][2][0][0] = __fmaf_rn(s[r].z, dot, acc[r][2][0][0]);
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t i = R * g + r;
    if (i < n_atoms)
      row_out<float, B, V, true>(i, acc[r], nc, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, ep, Q, ndof,
                                 s_coef, lane);
  }
}

// Wide tiles (V = 2 or 4, every column live): the group's unions are walked in
// chunks of U (the store pads each group to whole chunks).  A chunk's U*R weight
// slots are fetched one chunk ahead, one 16-byte slot per lane, then staged in
// this warp's shared slots; the column indices come by shuffle and the weights by
// broadcast shared loads, so the registers in flight hold only the X_j gathers.
template <int R, int B, int V, int U>
__device__ __forceinline__ void group_rows_staged(int64_t g, int64_t n_atoms, const int64_t* __restrict__ gptr,
                                                  const float4* __restrict__ gent, const float* __restrict__ diag,
                                                  const float* __restrict__ X, int64_t ldx, float* Y, int64_t ldy,
                                                  const float* Yin, int64_t ldyin, float* __restrict__ Acc,
                                                  int64_t ldacc, int c0, const Epi& ep, const double* __restrict__ Q,
                                                  int64_t ndof, const double* s_coef, float4* s_w, int lane) {
  static_assert(B == 32 * V && V >= 2, "one warp spans the tile");
  constexpr int NS = U * R;
  static_assert(NS <= 32, "one slot per lane");
  float2 acc[R][3][V / 2];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int p = 0; p < V / 2; ++p) acc[r][0][p] = acc[r][1][p] = acc[r][2][p] = make_float2(0.f, 0.f);
  const int64_t u0 = gptr[g], u1 = gptr[g + 1];
  const float* Xc = X + c0 + lane * V;
  float4 wreg = make_float4(0.f, 0.f, 0.f, 0.f);
  if (u0 < u1 && lane < NS) wreg = __ldg(gent + R * u0 + lane);
#pragma unroll 1
  for (int64_t u = u0; u < u1; u += U) {
    int j[U];
#pragma unroll
    for (int k = 0; k < U; ++k) j[k] = __shfl_sync(0xffffffffu, __float_as_int(wreg.w), k * R);
    __syncwarp();                        // the previous chunk's reads of s_w are done
    if (lane < NS) s_w[lane] = wreg;
    __syncwarp();
    if (u + U < u1 && lane < NS) wreg = __ldg(gent + R * (u + U) + lane);
    F2<V> x[U][3];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const float* xj = Xc + 3 * (int64_t)j[k] * ldx;
      vld2<V>(xj, x[k][0]);
      vld2<V>(xj + ldx, x[k][1]);
      vld2<V>(xj + 2 * ldx, x[k][2]);
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float4 w = s_w[k * R + r];
        const float2 wx = make_float2(w.x, w.x), wy = make_float2(w.y, w.y), wz = make_float2(w.z, w.z);
#pragma unroll
        for (int p = 0; p < V / 2; ++p) {
          float2 dot = __fmul2_rn(wx, x[k][0].v[p]);
          dot = __ffma2_rn(wy, x[k][1].v[p], dot);
          dot = __ffma2_rn(wz, x[k][2].v[p], dot);
          acc[r][0][p] = __ffma2_rn(wx, dot, acc[r][0][p]);
          acc[r][1][p] = __ffma2_rn(wy, dot, acc[r][1][p]);
          acc[r][2][p] = __ffma2_rn(wz, dot, acc[r][2][p]);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t i = R * g + r;
    if (i < n_atoms) {
      float a[3][1][V];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int p = 0; p < V / 2; ++p) {
          a[c][0][2 * p] = acc[r][c][p].x;
          a[c][0][2 * p + 1] = acc[r][c][p].y;
        }
      row_out<float, B, V, true>(i, a, B, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, ep, Q, ndof, s_coef,
                                 lane);
    }
  }
}

template <int R, int B, int V, int U>
__device__ __forceinline__ void group_dispatch(int64_t g, int64_t n_atoms, const int64_t* __restrict__ gptr,
                                               const float4* __restrict__ gent, const float* __restrict__ diag,
                                               const float* __restrict__ X, int64_t ldx, float* Y, int64_t ldy,
                                               const float* Yin, int64_t ldyin, float* __restrict__ Acc,
                                               int64_t ldacc, int c0, int nc, const Epi& ep,
                                               const double* __restrict__ Q, int64_t ndof, const double* s_coef,
                                               float4* s_w, int lane) {
  if constexpr (V >= 2)
    group_rows_staged<R, B, V, (U * R <= 32 ? U : 32 / R)>(g, n_atoms, gptr, gent, diag, X, ldx, Y, ldy, Yin,
                                                          ldyin, Acc, ldacc, c0, ep, Q, ndof, s_coef, s_w, lane);
  else
    group_rows<R, B, V, (U < 4 ? U : 4)>(g, n_atoms, gptr, gent, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0,
                                         nc, ep, Q, ndof, s_coef, lane);
}

// Two resident blocks of 256 threads per SM: 128 registers a thread, which the
// gathers of a 128-column chunk in flight fill.
template <int R, int B, int V, int U, int NT>
__global__ void __launch_bounds__(NT, 2)
k_spmm_group(int64_t n_atoms, const int64_t* __restrict__ gptr, const float4* __restrict__ gent,
             const float* __restrict__ diag, const float* __restrict__ X, int64_t ldx, float* Y, int64_t ldy,
             const float* Yin, int64_t ldyin, float* __restrict__ Acc, int64_t ldacc, int c0, int nc, Epi ep,
             const double* __restrict__ Q, int64_t ndof, const double* __restrict__ coef,
             int* __restrict__ group_counter) {
  __shared__ double s_coef[8 * B];
  __shared__ float4 s_slots[NT / 32][32];
  if (ep.r > 0) {
    for (int t = threadIdx.x; t < ep.r * B; t += NT) s_coef[t] = coef[t];
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  float4* s_w = s_slots[threadIdx.x >> 5];
  const int64_t ng = (n_atoms + R - 1) / R;
  if (group_counter == nullptr) {
    for (int64_t g = (int64_t)blockIdx.x * (NT / 32) + (threadIdx.x >> 5); g < ng;
         g += (int64_t)gridDim.x * (NT / 32))
      group_dispatch<R, B, V, U>(g, n_atoms, gptr, gent, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, nc, ep,
                                 Q, ndof, s_coef, s_w, lane);
    return;
  }
  // each warp takes chunks of kGroupSteps consecutive groups from the counter
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(group_counter, kGroupSteps);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= ng) break;
#pragma unroll 1
    for (int st = 0; st < kGroupSteps; ++st) {
      const int64_t g = (int64_t)base + st;
      if (g < ng)
        group_dispatch<R, B, V, U>(g, n_atoms, gptr, gent, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, nc, ep,
                                   Q, ndof, s_coef, s_w, lane);
    }
  }
}

// Unions in flight per warp of the row-group product (the autotuner's hook): 0
// picks the default of the tile width.
std::atomic<int> g_group_unroll{0};

template <int R, int B, int V>
cudaError_t launch_group_tile(int64_t n_atoms, const int64_t* gptr, const float4* gent, const float* diag,
                              const float* X, int64_t ldx, float* Y, int64_t ldy, const float* Yin, int64_t ldyin,
                              float* Acc, int64_t ldacc, int c0, int nc, Epi ep, const double* Q, double hot_shift,
                              double* partial, double* coef, cudaStream_t stream, int* counter) {
  const int64_t ndof = 3 * n_atoms;
  if (ep.r > 0) {
    dim3 g(kQxBlocks, ep.r);
    k_qx_partial<float, B><<<g, kThreads, 0, stream>>>(Q, ndof, X, ldx, c0, partial, nc);
    k_qx_final<<<(ep.r * B + kThreads / 32 - 1) / (kThreads / 32), kThreads, 0, stream>>>(partial, kQxBlocks,
                                                                                          ep.r, B, hot_shift, coef);
  }
  if (counter != nullptr) {
    const cudaError_t me = cudaMemsetAsync(counter, 0, sizeof(int), stream);
    if (me != cudaSuccess) return me;
  }
  constexpr int NT = 256;
  const int64_t ng = (n_atoms + R - 1) / R;
  const int blocks = grid_for(ng, NT / 32, 148 * g_cols_blocks_per_sm.load());
  const int un = g_group_unroll.load();
#define GROUP_LAUNCH(UU)                                                                                      \
  k_spmm_group<R, B, V, UU, NT><<<blocks, NT, 0, stream>>>(n_atoms, gptr, gent, diag, X, ldx, Y, ldy, Yin,    \
                                                           ldyin, Acc, ldacc, c0, nc, ep, Q, ndof, coef, counter)
  // default: 16 unions in flight on 128-column tiles, 8 on narrower ones (the
  // fastest on the 100k-atom assembly and the 500k-atom shell)
  if (un == 16 || (un == 0 && B == 128)) GROUP_LAUNCH(16);
  else if (un == 4) GROUP_LAUNCH(4);
  else if (un == 2) GROUP_LAUNCH(2);
  else GROUP_LAUNCH(8);
#undef GROUP_LAUNCH
  return cudaGetLastError();
}

template <int R>
cudaError_t run_groups(int64_t n_atoms, const int64_t* gptr, const float4* gent, const float* D, const float* X,
                       int64_t ldx, int b, float* Y, int64_t ldy, const float* Yin, int64_t ldyin, float* Acc,
                       int64_t ldacc, Epi ep, const double* Q, double hot_shift, double* partial, double* coef,
                       cudaStream_t s, int* counter) {
  auto al = [&](int m) {
    const uintptr_t a = (uintptr_t)m * sizeof(float);
    bool ok = (ldx % m == 0) && (ldy % m == 0) && ((uintptr_t)X % a == 0) && ((uintptr_t)Y % a == 0);
    if (ep.has_yin) ok = ok && (ldyin % m == 0) && ((uintptr_t)Yin % a == 0);
    if (ep.accumulate) ok = ok && (ldacc % m == 0) && ((uintptr_t)Acc % a == 0);
    return ok;
  };
  const bool al4 = al(4), al2 = al(2);
  int c0 = 0;
  cudaError_t e = cudaSuccess;
  while (c0 < b && e == cudaSuccess) {
    const int rem = b - c0;
    if (rem >= 128 && al4 && c0 % 4 == 0) {
      e = launch_group_tile<R, 128, 4>(n_atoms, gptr, gent, D, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, 128, ep,
                                       Q, hot_shift, partial, coef, s, counter);
      c0 += 128;
    } else if (rem >= 64 && al2 && c0 % 2 == 0) {
      e = launch_group_tile<R, 64, 2>(n_atoms, gptr, gent, D, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, 64, ep, Q,
                                      hot_shift, partial, coef, s, counter);
      c0 += 64;
    } else {
      const int nc = rem < 32 ? rem : 32;
      e = launch_group_tile<R, 32, 1>(n_atoms, gptr, gent, D, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, nc, ep, Q,
                                      hot_shift, partial, coef, s, counter);
      c0 += nc;
    }
  }
  return e;
}

}  // namespace
}  // namespace inch

using namespace inch;

extern "C" inch_status inch_spmm_tune(int32_t threads_per_block, int32_t blocks_per_sm) {
  // threads_per_block 0 selects the whole-warp-row kernel (batched gathers) where it
  // applies; 256/512/1024 select the lane-group kernel with that block size.
  INCH_REQUIRE(threads_per_block == 0 || threads_per_block == 256 || threads_per_block == 512 ||
                   threads_per_block == 1024,
               INCH_INVALID_ARG, "inch_spmm_tune: threads_per_block must be 0, 256, 512 or 1024");
  g_warp_kernel.store(threads_per_block == 0 ? 1 : 0);
  if (threads_per_block == 0) threads_per_block = 256;
  INCH_REQUIRE(blocks_per_sm >= 1 && blocks_per_sm <= 8, INCH_INVALID_ARG, "inch_spmm_tune: blocks_per_sm in 1..8");
  g_cols_threads.store(threads_per_block);
  g_cols_blocks_per_sm.store(blocks_per_sm);
  return INCH_OK;
}

extern "C" inch_status inch_spmm_traversal(int32_t mode) {
  INCH_REQUIRE(mode >= 0 && mode <= 2, INCH_INVALID_ARG, "inch_spmm_traversal: mode must be 0, 1 or 2");
  g_cols_traversal.store(mode);
  return INCH_OK;
}

extern "C" size_t inch_spmm_workspace_size(int64_t n_atoms, int32_t b, int32_t r) {
  (void)n_atoms;
  (void)b;
  Sizer s;
  s.take<int>(1);                               // row counter of the wide-block kernel
  s.take<double>((size_t)kQxBlocks * 8 * 128);  // partial sums (r <= 8, tile <= 128)
  s.take<double>(8 * 128);                      // coefficients
  (void)r;
  return s.bytes();
}

extern "C" inch_status inch_spmm(int32_t prec, int64_t n_atoms, const int64_t* rowptr, const void* ent,
                                 const void* diag, const void* X, int64_t ldx, int32_t b, void* Y, int64_t ldy,
                                 const void* Yin, int64_t ldyin, void* Acc, int64_t ldacc, const double* q,
                                 const inch_spmm_epilogue* ep_in, void* ws, size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(prec == 32 || prec == 64, INCH_INVALID_ARG, "inch_spmm: prec must be 32 or 64");
  INCH_REQUIRE(rowptr && ent && diag && X && Y && ep_in, INCH_INVALID_ARG, "inch_spmm: NULL argument");
  INCH_REQUIRE(n_atoms >= 1 && n_atoms < (int64_t(1) << 31), INCH_INVALID_ARG, "inch_spmm: n_atoms out of range");
  INCH_REQUIRE(b >= 1 && b <= (prec == 32 ? 128 : 64), INCH_INVALID_ARG, "inch_spmm: b=%d outside 1..%d", b,
               prec == 32 ? 128 : 64);
  INCH_REQUIRE(ldx >= b && ldy >= b, INCH_INVALID_ARG, "inch_spmm: leading dimension below b");
  INCH_REQUIRE(X != Y, INCH_INVALID_ARG, "inch_spmm: X and Y must not alias");
  const inch_spmm_epilogue& e = *ep_in;
  INCH_REQUIRE(e.r >= 0 && e.r <= 8, INCH_INVALID_ARG, "inch_spmm: deflation rank %d outside 0..8", e.r);
  INCH_REQUIRE(e.r == 0 || q != nullptr, INCH_INVALID_ARG, "inch_spmm: deflation basis is NULL");
  INCH_REQUIRE(e.beta == 0.0 || (Yin != nullptr && ldyin >= b), INCH_INVALID_ARG, "inch_spmm: beta != 0 needs Yin");
  INCH_REQUIRE(!e.accumulate || (Acc != nullptr && ldacc >= b), INCH_INVALID_ARG, "inch_spmm: accumulate needs Acc");
  INCH_REQUIRE(((uintptr_t)ent & 15) == 0 && ((uintptr_t)diag & 15) == 0, INCH_INVALID_ARG,
               "inch_spmm: store buffers must be 16-byte aligned");
  // The workspace (when given) holds the wide kernel's row counter and the
  // Hotelling scratch; without one (allowed for r = 0) the wide kernel walks its
  // rows with a fixed grid stride instead of the counter.
  double *partial = nullptr, *coef = nullptr;
  int* counter = nullptr;
  if (ws != nullptr || e.r > 0) {
    Carver c(ws, ws_bytes);
    counter = c.take<int>(1);
    partial = c.take<double>((size_t)kQxBlocks * 8 * 128);
    coef = c.take<double>(8 * 128);
    INCH_REQUIRE(c.ok, INCH_OOM, "inch_spmm: workspace of %zu bytes, need %zu", ws_bytes,
                 inch_spmm_workspace_size(n_atoms, b, e.r));
  }
  Epi ep{e.alpha, e.gamma, e.beta, e.mu, e.r, e.accumulate, (e.beta != 0.0) ? 1 : 0};
  cudaError_t err;
  if (prec == 32)
    err = run<float>(n_atoms, rowptr, ent, diag, X, ldx, b, Y, ldy, Yin, ldyin, Acc, ldacc, ep, q, e.hot_shift,
                     partial, coef, stream, counter);
  else
    err = run<double>(n_atoms, rowptr, ent, diag, X, ldx, b, Y, ldy, Yin, ldyin, Acc, ldacc, ep, q, e.hot_shift,
                      partial, coef, stream, counter);
  INCH_REQUIRE(err == cudaSuccess, INCH_CUDA_ERROR, "inch_spmm: %s", cudaGetErrorString(err));
  return INCH_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of inch_spmm.
//
// Some hosts cannot hand this library a device workspace: a caller that sits on
// top of another runtime's memory manager with no device allocator of its own,
// or a bare FFI binding that only owns its input and output buffers.  For them
// the Hotelling partial sums and coefficients live in the file-scope array
// below.  It is sized for the largest tile the kernels use (64 columns) and the
// largest fused deflation rank (8): kQxBlocks * 8 * 64 + 8 * 64 doubles, about
// 1.2 MB, resident on every GPU that loads the library until the process exits.
// The array's host-side name is not a device address: its address is fetched
// with cudaGetSymbolAddress once per device, with that device current, on the
// first call with deflation vectors (r > 0) made on that device, so make that
// first call before any stream capture; calls with r = 0 never touch the array.
// Nothing in the array has to start at zero: every call writes each
// partial sum and coefficient before reading it.  All calls share the array, so
// calls that overlap on the GPU (different streams, or different host threads on
// the same device) race on it and must be serialised by the caller.
// ---------------------------------------------------------------------------
#include <mutex>

namespace inch {
namespace {
constexpr size_t kNoAllocPartial = (size_t)kQxBlocks * 8 * 64;
constexpr size_t kNoAllocDoubles = kNoAllocPartial + 8 * 64;
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];
std::mutex g_noalloc_mu;
double* g_noalloc_addr[kNoAllocMaxDevices] = {nullptr};
}  // namespace
}  // namespace inch

extern "C" inch_status inch_spmm_noalloc(int32_t prec, int64_t n_atoms, const int64_t* rowptr, const void* ent,
                                         const void* diag, const void* X, int64_t ldx, int32_t b, void* Y,
                                         int64_t ldy, const void* Yin, int64_t ldyin, void* Acc, int64_t ldacc,
                                         const double* q, const inch_spmm_epilogue* ep_in, cudaStream_t stream) {
  INCH_REQUIRE(prec == 32 || prec == 64, INCH_INVALID_ARG, "inch_spmm_noalloc: prec must be 32 or 64");
  INCH_REQUIRE(rowptr && ent && diag && X && Y && ep_in, INCH_INVALID_ARG, "inch_spmm_noalloc: NULL argument");
  INCH_REQUIRE(n_atoms >= 1 && n_atoms < (int64_t(1) << 31), INCH_INVALID_ARG,
               "inch_spmm_noalloc: n_atoms out of range");
  INCH_REQUIRE(b >= 1 && b <= 64, INCH_LIMIT,
               "inch_spmm_noalloc: b=%d exceeds the 64 columns its static scratch holds", b);
  INCH_REQUIRE(ldx >= b && ldy >= b, INCH_INVALID_ARG, "inch_spmm_noalloc: leading dimension below b");
  INCH_REQUIRE(X != Y, INCH_INVALID_ARG, "inch_spmm_noalloc: X and Y must not alias");
  const inch_spmm_epilogue& e = *ep_in;
  INCH_REQUIRE(e.r >= 0 && e.r <= 8, INCH_LIMIT,
               "inch_spmm_noalloc: deflation rank %d exceeds the 8 its static scratch holds", e.r);
  INCH_REQUIRE(e.r == 0 || q != nullptr, INCH_INVALID_ARG, "inch_spmm_noalloc: deflation basis is NULL");
  INCH_REQUIRE(e.beta == 0.0 || (Yin != nullptr && ldyin >= b), INCH_INVALID_ARG,
               "inch_spmm_noalloc: beta != 0 needs Yin");
  INCH_REQUIRE(!e.accumulate || (Acc != nullptr && ldacc >= b), INCH_INVALID_ARG,
               "inch_spmm_noalloc: accumulate needs Acc");
  INCH_REQUIRE(((uintptr_t)ent & 15) == 0 && ((uintptr_t)diag & 15) == 0, INCH_INVALID_ARG,
               "inch_spmm_noalloc: store buffers must be 16-byte aligned");
  double *partial = nullptr, *coef = nullptr;
  if (e.r > 0) {
    // the static scratch holds only the deflation partial sums: look its device
    // address up (once per device) only for calls that use it
    int dev = -1;
    INCH_CUDA(cudaGetDevice(&dev));
    INCH_REQUIRE(dev >= 0 && dev < kNoAllocMaxDevices, INCH_LIMIT, "inch_spmm_noalloc: device %d not supported",
                 dev);
    double* base = nullptr;
    {
      std::lock_guard<std::mutex> lock(g_noalloc_mu);
      if (g_noalloc_addr[dev] == nullptr) {
        void* p = nullptr;
        INCH_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_addr[dev] = static_cast<double*>(p);
      }
      base = g_noalloc_addr[dev];
    }
    partial = base;
    coef = base + kNoAllocPartial;
  }
  Epi ep{e.alpha, e.gamma, e.beta, e.mu, e.r, e.accumulate, (e.beta != 0.0) ? 1 : 0};
  cudaError_t err;
  if (prec == 32)
    err = run<float>(n_atoms, rowptr, ent, diag, X, ldx, b, Y, ldy, Yin, ldyin, Acc, ldacc, ep, q, e.hot_shift,
                     partial, coef, stream);
  else
    err = run<double>(n_atoms, rowptr, ent, diag, X, ldx, b, Y, ldy, Yin, ldyin, Acc, ldacc, ep, q, e.hot_shift,
                      partial, coef, stream);
  INCH_REQUIRE(err == cudaSuccess, INCH_CUDA_ERROR, "inch_spmm_noalloc: %s", cudaGetErrorString(err));
  return INCH_OK;
}

// ---------------------------------------------------------------------------
// Segmented epilogue: block-diagonal stores holding many structures, where each
// structure (segment) needs its own filter coefficients.
// ---------------------------------------------------------------------------
extern "C" inch_status inch_spmm_seg(int32_t prec, int64_t n_atoms, const int64_t* rowptr, const void* ent,
                                     const void* diag, const void* X, int64_t ldx, int32_t b, void* Y, int64_t ldy,
                                     const void* Yin, int64_t ldyin, const int32_t* atom_seg,
                                     const double* seg_coef, cudaStream_t stream) {
  INCH_REQUIRE(prec == 32 || prec == 64, INCH_INVALID_ARG, "inch_spmm_seg: prec must be 32 or 64");
  INCH_REQUIRE(rowptr && ent && diag && X && Y && atom_seg && seg_coef, INCH_INVALID_ARG,
               "inch_spmm_seg: NULL argument");
  INCH_REQUIRE(n_atoms >= 1 && n_atoms < (int64_t(1) << 31), INCH_INVALID_ARG, "inch_spmm_seg: n_atoms out of range");
  INCH_REQUIRE(b >= 1 && b <= 64 && ldx >= b && ldy >= b && X != Y, INCH_INVALID_ARG,
               "inch_spmm_seg: bad b / leading dimension / aliasing");
  INCH_REQUIRE(Yin == nullptr || ldyin >= b, INCH_INVALID_ARG, "inch_spmm_seg: ldyin below b");
  INCH_REQUIRE(((uintptr_t)ent & 15) == 0 && ((uintptr_t)diag & 15) == 0, INCH_INVALID_ARG,
               "inch_spmm_seg: store buffers must be 16-byte aligned");
  Epi ep{0.0, 0.0, 0.0, 0.0, 0, 0, Yin != nullptr ? 1 : 0};
  ep.seg_coef = seg_coef;
  ep.atom_seg = atom_seg;
  cudaError_t err;
  if (prec == 32)
    err = run<float>(n_atoms, rowptr, ent, diag, X, ldx, b, Y, ldy, Yin, ldyin, nullptr, 0, ep, nullptr, 0.0,
                     nullptr, nullptr, stream);
  else
    err = run<double>(n_atoms, rowptr, ent, diag, X, ldx, b, Y, ldy, Yin, ldyin, nullptr, 0, ep, nullptr, 0.0,
                      nullptr, nullptr, stream);
  INCH_REQUIRE(err == cudaSuccess, INCH_CUDA_ERROR, "inch_spmm_seg: %s", cudaGetErrorString(err));
  return INCH_OK;
}

extern "C" inch_status inch_spmm_seg_ws(int32_t prec, int64_t n_atoms, const int64_t* rowptr, const void* ent,
                                        const void* diag, const void* X, int64_t ldx, int32_t b, void* Y,
                                        int64_t ldy, const void* Yin, int64_t ldyin, const int32_t* atom_seg,
                                        const double* seg_coef, void* ws, size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(prec == 32 || prec == 64, INCH_INVALID_ARG, "inch_spmm_seg_ws: prec must be 32 or 64");
  INCH_REQUIRE(rowptr && ent && diag && X && Y && atom_seg && seg_coef && ws, INCH_INVALID_ARG,
               "inch_spmm_seg_ws: NULL argument");
  INCH_REQUIRE(n_atoms >= 1 && n_atoms < (int64_t(1) << 31), INCH_INVALID_ARG,
               "inch_spmm_seg_ws: n_atoms out of range");
  INCH_REQUIRE(b >= 1 && b <= (prec == 32 ? 128 : 64) && ldx >= b && ldy >= b && X != Y, INCH_INVALID_ARG,
               "inch_spmm_seg_ws: bad b / leading dimension / aliasing");
  INCH_REQUIRE(Yin == nullptr || ldyin >= b, INCH_INVALID_ARG, "inch_spmm_seg_ws: ldyin below b");
  INCH_REQUIRE(((uintptr_t)ent & 15) == 0 && ((uintptr_t)diag & 15) == 0, INCH_INVALID_ARG,
               "inch_spmm_seg_ws: store buffers must be 16-byte aligned");
  Carver c(ws, ws_bytes);
  int* counter = c.take<int>(1);
  INCH_REQUIRE(c.ok, INCH_OOM, "inch_spmm_seg_ws: workspace too small");
  Epi ep{0.0, 0.0, 0.0, 0.0, 0, 0, Yin != nullptr ? 1 : 0};
  ep.seg_coef = seg_coef;
  ep.atom_seg = atom_seg;
  cudaError_t err;
  if (prec == 32)
    err = run<float>(n_atoms, rowptr, ent, diag, X, ldx, b, Y, ldy, Yin, ldyin, nullptr, 0, ep, nullptr, 0.0,
                     nullptr, nullptr, stream, counter);
  else
    err = run<double>(n_atoms, rowptr, ent, diag, X, ldx, b, Y, ldy, Yin, ldyin, nullptr, 0, ep, nullptr, 0.0,
                      nullptr, nullptr, stream, counter);
  INCH_REQUIRE(err == cudaSuccess, INCH_CUDA_ERROR, "inch_spmm_seg_ws: %s", cudaGetErrorString(err));
  return INCH_OK;
}

// ---------------------------------------------------------------------------
// Row-group layout: build and product.
// ---------------------------------------------------------------------------
extern "C" size_t inch_group_store_workspace_size(int64_t n_atoms, int32_t rows_per_group) {
  const int R = rows_per_group > 0 ? rows_per_group : 1;
  const int64_t ng = (n_atoms + R - 1) / R;
  size_t cb = 0;
  cub::DeviceScan::InclusiveSum(nullptr, cb, (int64_t*)nullptr, (int64_t*)nullptr, (int)(ng > 0 ? ng : 1));
  Sizer s;
  s.take<int64_t>(ng > 0 ? ng : 1);
  s.take<char>(cb);
  return s.bytes();
}

extern "C" inch_status inch_group_store_count(const int64_t* rowptr, const float* ent32, int64_t n_atoms,
                                              int32_t rows_per_group, int64_t* group_ptr, int64_t* n_union_host,
                                              void* ws, size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(rowptr && ent32 && group_ptr && n_union_host, INCH_INVALID_ARG,
               "inch_group_store_count: NULL argument");
  INCH_REQUIRE(rows_per_group == 2 || rows_per_group == 4, INCH_INVALID_ARG,
               "inch_group_store_count: rows_per_group must be 2 or 4");
  INCH_REQUIRE(n_atoms >= 1 && n_atoms < (int64_t(1) << 31), INCH_INVALID_ARG,
               "inch_group_store_count: n_atoms out of range");
  INCH_REQUIRE(((uintptr_t)ent32 & 15) == 0, INCH_INVALID_ARG,
               "inch_group_store_count: entries must be 16-byte aligned");
  const int R = rows_per_group;
  const int64_t ng = (n_atoms + R - 1) / R;
  Carver c(ws, ws_bytes);
  int64_t* cnt = c.take<int64_t>(ng);
  size_t cb = 0;
  cub::DeviceScan::InclusiveSum(nullptr, cb, (int64_t*)nullptr, (int64_t*)nullptr, (int)ng);
  void* tmp = c.take<char>(cb);
  INCH_REQUIRE(c.ok, INCH_OOM, "inch_group_store_count: workspace of %zu bytes, need %zu", ws_bytes,
               inch_group_store_workspace_size(n_atoms, R));
  const int blocks = grid_for(ng, kGroupBuildThreads, 148 * 16);
  const float4* e4 = reinterpret_cast<const float4*>(ent32);
  if (R == 2)
    k_group_merge<0, 2><<<blocks, kGroupBuildThreads, 0, stream>>>(n_atoms, rowptr, e4, cnt, nullptr, nullptr);
  else
    k_group_merge<0, 4><<<blocks, kGroupBuildThreads, 0, stream>>>(n_atoms, rowptr, e4, cnt, nullptr, nullptr);
  INCH_LAUNCH_CHECK();
  k_set0<<<1, 1, 0, stream>>>(group_ptr);
  INCH_LAUNCH_CHECK();
  INCH_CUDA(cub::DeviceScan::InclusiveSum(tmp, cb, cnt, group_ptr + 1, (int)ng, stream));
  INCH_CUDA(cudaMemcpyAsync(n_union_host, group_ptr + ng, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cudaStreamSynchronize(stream));
  return INCH_OK;
}

extern "C" inch_status inch_group_store_fill(const int64_t* rowptr, const float* ent32, int64_t n_atoms,
                                             int32_t rows_per_group, const int64_t* group_ptr, float* group_ent,
                                             cudaStream_t stream) {
  INCH_REQUIRE(rowptr && ent32 && group_ptr && group_ent, INCH_INVALID_ARG, "inch_group_store_fill: NULL argument");
  INCH_REQUIRE(rows_per_group == 2 || rows_per_group == 4, INCH_INVALID_ARG,
               "inch_group_store_fill: rows_per_group must be 2 or 4");
  INCH_REQUIRE(n_atoms >= 1 && n_atoms < (int64_t(1) << 31), INCH_INVALID_ARG,
               "inch_group_store_fill: n_atoms out of range");
  INCH_REQUIRE(((uintptr_t)ent32 & 15) == 0 && ((uintptr_t)group_ent & 15) == 0, INCH_INVALID_ARG,
               "inch_group_store_fill: entry buffers must be 16-byte aligned");
  const int R = rows_per_group;
  const int64_t ng = (n_atoms + R - 1) / R;
  const int blocks = grid_for(ng, kGroupBuildThreads, 148 * 16);
  const float4* e4 = reinterpret_cast<const float4*>(ent32);
  float4* g4 = reinterpret_cast<float4*>(group_ent);
  if (R == 2)
    k_group_merge<1, 2><<<blocks, kGroupBuildThreads, 0, stream>>>(n_atoms, rowptr, e4, nullptr, group_ptr, g4);
  else
    k_group_merge<1, 4><<<blocks, kGroupBuildThreads, 0, stream>>>(n_atoms, rowptr, e4, nullptr, group_ptr, g4);
  INCH_LAUNCH_CHECK();
  return INCH_OK;
}

extern "C" inch_status inch_spmm_group_tune(int32_t unroll) {
  INCH_REQUIRE(unroll == 0 || unroll == 2 || unroll == 4 || unroll == 8 || unroll == 16, INCH_INVALID_ARG,
               "inch_spmm_group_tune: unroll must be 0, 2, 4, 8 or 16");
  g_group_unroll.store(unroll);
  return INCH_OK;
}

namespace {
inch_status groups_common(const char* who, int64_t n_atoms, int32_t R, const int64_t* gptr, const float* gent,
                          const float* diag, const float* X, int64_t ldx, int32_t b, float* Y, int64_t ldy) {
  INCH_REQUIRE(gptr && gent && diag && X && Y, INCH_INVALID_ARG, "%s: NULL argument", who);
  INCH_REQUIRE(R == 2 || R == 4, INCH_INVALID_ARG, "%s: rows_per_group must be 2 or 4", who);
  INCH_REQUIRE(n_atoms >= 1 && n_atoms < (int64_t(1) << 31), INCH_INVALID_ARG, "%s: n_atoms out of range", who);
  INCH_REQUIRE(b >= 1 && ldx >= b && ldy >= b, INCH_INVALID_ARG, "%s: b=%d or leading dimension below b", who, b);
  INCH_REQUIRE((const void*)X != (const void*)Y, INCH_INVALID_ARG, "%s: X and Y must not alias", who);
  INCH_REQUIRE(((uintptr_t)gent & 15) == 0 && ((uintptr_t)diag & 15) == 0, INCH_INVALID_ARG,
               "%s: store buffers must be 16-byte aligned", who);
  return INCH_OK;
}
}  // namespace

extern "C" inch_status inch_spmm_groups(int64_t n_atoms, int32_t rows_per_group, const int64_t* group_ptr,
                                        const float* group_ent, const float* diag, const float* X, int64_t ldx,
                                        int32_t b, float* Y, int64_t ldy, const float* Yin, int64_t ldyin, float* Acc,
                                        int64_t ldacc, const double* q, const inch_spmm_epilogue* ep_in, void* ws,
                                        size_t ws_bytes, cudaStream_t stream) {
  const inch_status st = groups_common("inch_spmm_groups", n_atoms, rows_per_group, group_ptr, group_ent, diag, X,
                                       ldx, b, Y, ldy);
  if (st != INCH_OK) return st;
  INCH_REQUIRE(ep_in != nullptr, INCH_INVALID_ARG, "inch_spmm_groups: NULL epilogue");
  const inch_spmm_epilogue& e = *ep_in;
  INCH_REQUIRE(e.r >= 0 && e.r <= 8, INCH_INVALID_ARG, "inch_spmm_groups: deflation rank %d outside 0..8", e.r);
  INCH_REQUIRE(e.r == 0 || q != nullptr, INCH_INVALID_ARG, "inch_spmm_groups: deflation basis is NULL");
  INCH_REQUIRE(e.beta == 0.0 || (Yin != nullptr && ldyin >= b), INCH_INVALID_ARG,
               "inch_spmm_groups: beta != 0 needs Yin");
  INCH_REQUIRE(!e.accumulate || (Acc != nullptr && ldacc >= b), INCH_INVALID_ARG,
               "inch_spmm_groups: accumulate needs Acc");
  double *partial = nullptr, *coef = nullptr;
  int* counter = nullptr;
  if (ws != nullptr || e.r > 0) {
    Carver c(ws, ws_bytes);
    counter = c.take<int>(1);
    partial = c.take<double>((size_t)kQxBlocks * 8 * 128);
    coef = c.take<double>(8 * 128);
    INCH_REQUIRE(c.ok, INCH_OOM, "inch_spmm_groups: workspace of %zu bytes, need %zu", ws_bytes,
                 inch_spmm_workspace_size(n_atoms, b, e.r));
  }
  Epi ep{e.alpha, e.gamma, e.beta, e.mu, e.r, e.accumulate, (e.beta != 0.0) ? 1 : 0};
  const float4* g4 = reinterpret_cast<const float4*>(group_ent);
  const cudaError_t err =
      rows_per_group == 2
          ? run_groups<2>(n_atoms, group_ptr, g4, diag, X, ldx, b, Y, ldy, Yin, ldyin, Acc, ldacc, ep, q, e.hot_shift,
                          partial, coef, stream, counter)
          : run_groups<4>(n_atoms, group_ptr, g4, diag, X, ldx, b, Y, ldy, Yin, ldyin, Acc, ldacc, ep, q, e.hot_shift,
                          partial, coef, stream, counter);
  INCH_REQUIRE(err == cudaSuccess, INCH_CUDA_ERROR, "inch_spmm_groups: %s", cudaGetErrorString(err));
  return INCH_OK;
}

extern "C" inch_status inch_spmm_groups_seg(int64_t n_atoms, int32_t rows_per_group, const int64_t* group_ptr,
                                            const float* group_ent, const float* diag, const float* X, int64_t ldx,
                                            int32_t b, float* Y, int64_t ldy, const float* Yin, int64_t ldyin,
                                            const int32_t* atom_seg, const double* seg_coef, void* ws,
                                            size_t ws_bytes, cudaStream_t stream) {
  const inch_status st = groups_common("inch_spmm_groups_seg", n_atoms, rows_per_group, group_ptr, group_ent, diag,
                                       X, ldx, b, Y, ldy);
  if (st != INCH_OK) return st;
  INCH_REQUIRE(atom_seg && seg_coef, INCH_INVALID_ARG, "inch_spmm_groups_seg: NULL segment arrays");
  INCH_REQUIRE(Yin == nullptr || ldyin >= b, INCH_INVALID_ARG, "inch_spmm_groups_seg: ldyin below b");
  int* counter = nullptr;
  if (ws != nullptr) {
    Carver c(ws, ws_bytes);
    counter = c.take<int>(1);
    INCH_REQUIRE(c.ok, INCH_OOM, "inch_spmm_groups_seg: workspace too small");
  }
  Epi ep{0.0, 0.0, 0.0, 0.0, 0, 0, Yin != nullptr ? 1 : 0};
  ep.seg_coef = seg_coef;
  ep.atom_seg = atom_seg;
  const float4* g4 = reinterpret_cast<const float4*>(group_ent);
  const cudaError_t err =
      rows_per_group == 2
          ? run_groups<2>(n_atoms, group_ptr, g4, diag, X, ldx, b, Y, ldy, Yin, ldyin, nullptr, 0, ep, nullptr, 0.0,
                          nullptr, nullptr, stream, counter)
          : run_groups<4>(n_atoms, group_ptr, g4, diag, X, ldx, b, Y, ldy, Yin, ldyin, nullptr, 0, ep, nullptr, 0.0,
                          nullptr, nullptr, stream, counter);
  INCH_REQUIRE(err == cudaSuccess, INCH_CUDA_ERROR, "inch_spmm_groups_seg: %s", cudaGetErrorString(err));
  return INCH_OK;
}

// ---------------------------------------------------------------------------
// Chebyshev filters as single library calls (the SpMM above, looped inside the
// library with its fused epilogue; the caller provides every buffer).
// ---------------------------------------------------------------------------
namespace inch {
namespace {

// Y = s * X over an (n, b) block with leading dimensions.
template <class T>
__global__ void k_scale_copy(const T* __restrict__ X, int64_t ldx, T* __restrict__ Y, int64_t ldy, int64_t n, int b,
                             double s) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * b; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / b;
    const int c = static_cast<int>(t % b);
    Y[i * ldy + c] = static_cast<T>(s * static_cast<double>(X[i * ldx + c]));
  }
}

template <class T>
inch_status cheb_mu(int64_t n_atoms, const int64_t* rowptr, const void* ent, const void* diag, const T* X,
                    int64_t ldx, int b, int degree, const double* mu, double cc, double dd, T* Y, int64_t ldy, T* W1,
                    T* W2, int64_t ldw, cudaStream_t s) {
  const int64_t n = 3 * n_atoms;
  k_scale_copy<T><<<grid_for(n * b, 256, 148 * 16), 256, 0, s>>>(X, ldx, Y, ldy, n, b, mu[0]);
  INCH_LAUNCH_CHECK();
  if (degree == 0) return INCH_OK;
  // X_1 = (H X_0 - cc X_0) / dd;  Y += mu_1 X_1
  Epi ep{1.0 / dd, -cc / dd, 0.0, mu[1], 0, 1, 0};
  cudaError_t e = run<T>(n_atoms, rowptr, ent, diag, X, ldx, b, W1, ldw, nullptr, 0, Y, ldy, ep, nullptr, 0.0,
                         nullptr, nullptr, s);
  INCH_REQUIRE(e == cudaSuccess, INCH_CUDA_ERROR, "inch_cheb_filter: %s", cudaGetErrorString(e));
  // X_{k+1} = 2 (H X_k - cc X_k) / dd - X_{k-1};  Y += mu_{k+1} X_{k+1}.  X_2 goes
  // to W2; from then on X_{k+1} is written over X_{k-1} (never over the input X).
  const T* prev = X;
  int64_t ldprev = ldx;
  T* cur = W1;
  for (int k = 1; k < degree; ++k) {
    T* out = (k == 1) ? W2 : const_cast<T*>(prev);
    Epi ek{2.0 / dd, -2.0 * cc / dd, -1.0, mu[k + 1], 0, 1, 1};
    e = run<T>(n_atoms, rowptr, ent, diag, cur, ldw, b, out, ldw, prev, ldprev, Y, ldy, ek, nullptr, 0.0, nullptr,
               nullptr, s);
    INCH_REQUIRE(e == cudaSuccess, INCH_CUDA_ERROR, "inch_cheb_filter: %s", cudaGetErrorString(e));
    prev = cur;
    ldprev = ldw;
    cur = out;
  }
  return INCH_OK;
}

template <class T>
inch_status cheb_scaled(int64_t n_atoms, const int64_t* rowptr, const void* ent, const void* diag, const T* X,
                        int64_t ldx, int b, int degree, double a, double bup, double a0, T* Y, int64_t ldy, T* W,
                        int64_t ldw, cudaStream_t s) {
  // Zhou & Saad's scaled filter: Y_1 = (sigma_1 / e)(H X - c X), then
  // Y_{t+1} = (2 sigma_{t+1} / e)(H Y_t - c Y_t) - sigma_t sigma_{t+1} Y_{t-1}.
  const double e = (bup - a) / 2.0, c = (bup + a) / 2.0;
  double sigma = e / (a0 - c);
  const double sigma1 = sigma, tau = 2.0 / sigma1;
  Epi ep{sigma1 / e, -sigma1 * c / e, 0.0, 0.0, 0, 0, 0};
  cudaError_t err = run<T>(n_atoms, rowptr, ent, diag, X, ldx, b, Y, ldy, nullptr, 0, nullptr, 0, ep, nullptr, 0.0,
                           nullptr, nullptr, s);
  INCH_REQUIRE(err == cudaSuccess, INCH_CUDA_ERROR, "inch_cheb_filter_scaled: %s", cudaGetErrorString(err));
  // buffers: older -> newer; the newest of the two sits in `cur`
  const T* older = X;
  int64_t ldo = ldx;
  T* cur = Y;
  int64_t ldc = ldy;
  for (int t = 2; t <= degree; ++t) {
    const double s2 = 1.0 / (tau - sigma);
    T* out = (t == 2) ? W : const_cast<T*>(older);       // overwrite the oldest (never X)
    const int64_t ldout = (t == 2) ? ldw : ldo;
    Epi et{2.0 * s2 / e, -2.0 * s2 * c / e, -sigma * s2, 0.0, 0, 0, 1};
    err = run<T>(n_atoms, rowptr, ent, diag, cur, ldc, b, out, ldout, older, ldo, nullptr, 0, et, nullptr, 0.0,
                 nullptr, nullptr, s);
    INCH_REQUIRE(err == cudaSuccess, INCH_CUDA_ERROR, "inch_cheb_filter_scaled: %s", cudaGetErrorString(err));
    older = cur;
    ldo = ldc;
    cur = out;
    ldc = ldout;
    sigma = s2;
  }
  if (cur != Y) {
    INCH_CUDA(cudaMemcpy2DAsync(Y, ldy * sizeof(T), cur, ldc * sizeof(T), b * sizeof(T), 3 * n_atoms,
                                cudaMemcpyDeviceToDevice, s));
  }
  return INCH_OK;
}

}  // namespace
}  // namespace inch

extern "C" inch_status inch_cheb_filter(int32_t prec, int64_t n_atoms, const int64_t* rowptr, const void* ent,
                                        const void* diag, const void* X, int64_t ldx, int32_t b, int32_t degree,
                                        const double* mu_host, double cc, double dd, void* Y, int64_t ldy, void* W1,
                                        void* W2, int64_t ldw, cudaStream_t stream) {
  INCH_REQUIRE(prec == 32 || prec == 64, INCH_INVALID_ARG, "inch_cheb_filter: prec must be 32 or 64");
  INCH_REQUIRE(rowptr && ent && diag && X && Y && mu_host && (degree == 0 || (W1 && W2)), INCH_INVALID_ARG,
               "inch_cheb_filter: NULL argument");
  INCH_REQUIRE(n_atoms >= 1 && b >= 1 && degree >= 0, INCH_INVALID_ARG, "inch_cheb_filter: bad sizes");
  INCH_REQUIRE(dd != 0.0 && std::isfinite(cc) && std::isfinite(dd), INCH_INVALID_ARG,
               "inch_cheb_filter: dd must be finite and non-zero");
  INCH_REQUIRE(ldx >= b && ldy >= b && (degree == 0 || ldw >= b), INCH_INVALID_ARG,
               "inch_cheb_filter: leading dimension below b");
  INCH_REQUIRE(X != Y && X != W1 && X != W2 && Y != W1 && Y != W2 && (degree == 0 || W1 != W2), INCH_INVALID_ARG,
               "inch_cheb_filter: X, Y, W1 and W2 must be distinct");
  if (prec == 32)
    return cheb_mu<float>(n_atoms, rowptr, ent, diag, static_cast<const float*>(X), ldx, b, degree, mu_host, cc, dd,
                          static_cast<float*>(Y), ldy, static_cast<float*>(W1), static_cast<float*>(W2), ldw, stream);
  return cheb_mu<double>(n_atoms, rowptr, ent, diag, static_cast<const double*>(X), ldx, b, degree, mu_host, cc, dd,
                         static_cast<double*>(Y), ldy, static_cast<double*>(W1), static_cast<double*>(W2), ldw, stream);
}

extern "C" inch_status inch_cheb_filter_scaled(int32_t prec, int64_t n_atoms, const int64_t* rowptr,
                                               const void* ent, const void* diag, const void* X, int64_t ldx,
                                               int32_t b, int32_t degree, double a, double b_up, double a0, void* Y,
                                               int64_t ldy, void* W, int64_t ldw, cudaStream_t stream) {
  INCH_REQUIRE(prec == 32 || prec == 64, INCH_INVALID_ARG, "inch_cheb_filter_scaled: prec must be 32 or 64");
  INCH_REQUIRE(rowptr && ent && diag && X && Y && W, INCH_INVALID_ARG, "inch_cheb_filter_scaled: NULL argument");
  INCH_REQUIRE(n_atoms >= 1 && b >= 1 && degree >= 1, INCH_INVALID_ARG, "inch_cheb_filter_scaled: bad sizes");
  INCH_REQUIRE(a0 < a && a < b_up && std::isfinite(a0) && std::isfinite(b_up), INCH_INVALID_ARG,
               "inch_cheb_filter_scaled: need a0 < a < b_up");
  INCH_REQUIRE(ldx >= b && ldy >= b && ldw >= b, INCH_INVALID_ARG, "inch_cheb_filter_scaled: leading dimension below b");
  INCH_REQUIRE(X != Y && X != W && Y != W, INCH_INVALID_ARG, "inch_cheb_filter_scaled: X, Y and W must be distinct");
  if (prec == 32)
    return cheb_scaled<float>(n_atoms, rowptr, ent, diag, static_cast<const float*>(X), ldx, b, degree, a, b_up, a0,
                              static_cast<float*>(Y), ldy, static_cast<float*>(W), ldw, stream);
  return cheb_scaled<double>(n_atoms, rowptr, ent, diag, static_cast<const double*>(X), ldx, b, degree, a, b_up, a0,
                             static_cast<double*>(Y), ldy, static_cast<double*>(W), ldw, stream);
}
