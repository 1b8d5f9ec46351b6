// Row-tile store and the tile SpMM for wide multivectors.
//
// The rank-one store of hessian.cu keeps one entry per (row, neighbour) pair, so a
// row-by-row product gathers X_j once per pair: 12*b bytes from L1/L2 per pair,
// which bounds the wide-block product (b >= 8).  Consecutive rows after
// Cuthill-McKee share most of their neighbours (8 consecutive rows of the
// 100k-atom assembly: 2.5 pairs per distinct column), so here rows are grouped
// into tiles of kTile = 8 consecutive atoms and each tile stores the merged,
// sorted union of its rows' neighbour columns:
//   urec[u]  = (j << 8) | mask       mask bit r: row (tile base + r) has neighbour j
//   pw[p]    = w for every set bit, in (u, r) order  (FP32 {wx,wy,wz,0} 16 B,
//                                                    FP64 {wx,wy,wz,0} 32 B)
//   tile_uptr / tile_pptr: per-tile offsets into urec / pw.
// Self pairs (w = 0) are left out.  The product walks a tile's union once: X_j is
// gathered once per distinct column and applied, through the mask, to every row
// of the tile that needs it (unrolled over the 8 rows, so accumulators stay in
// registers).  Diagonal blocks and the fused epilogue are those of spmm.cu.
#include <cub/cub.cuh>

#include "common.cuh"

namespace inch {
namespace {

constexpr int kTile = 8;
constexpr int kWarpsBuild = 8;

// Lanes 0..kTile-1 each walk one row of the tile; every step the warp takes the
// smallest head column j, the lanes whose head equals j form the mask and advance.
// Pass 0 counts (unions, pairs); pass 1 writes records and w.
template <int PASS>
__global__ void __launch_bounds__(kWarpsBuild * 32)
k_tile_merge(const double* __restrict__ X, int64_t n, double r2, const int64_t* __restrict__ rowptr,
             const int* __restrict__ cols, int64_t* __restrict__ ucount, int64_t* __restrict__ pcount,
             const int64_t* __restrict__ uptr, const int64_t* __restrict__ pptr, uint32_t* __restrict__ urec,
             double* __restrict__ pw64, float* __restrict__ pw32) {
  const int lane = threadIdx.x & 31;
  const int64_t ntiles = (n + kTile - 1) / kTile;
  for (int64_t t = (int64_t)blockIdx.x * kWarpsBuild + (threadIdx.x >> 5); t < ntiles;
       t += (int64_t)gridDim.x * kWarpsBuild) {
    const int64_t row = t * kTile + lane;
    const bool active = lane < kTile && row < n;
    int64_t e = active ? rowptr[row] : 0;
    const int64_t e1 = active ? rowptr[row + 1] : 0;
    double xi = 0, yi = 0, zi = 0;
    if (PASS == 1 && active) {
      xi = X[3 * row];
      yi = X[3 * row + 1];
      zi = X[3 * row + 2];
    }
    int64_t nu = 0, np = 0;
    int64_t u_out = PASS == 1 ? uptr[t] : 0, p_out = PASS == 1 ? pptr[t] : 0;
    for (;;) {
      // skip the self entry
      int head = 0x7fffffff;
      if (active) {
        while (e < e1 && cols[e] == row) ++e;
        if (e < e1) head = cols[e];
      }
      int m = head;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (m == 0x7fffffff) break;
      const bool mine = active && head == m;
      const unsigned mask = __ballot_sync(0xffffffffu, mine) & ((1u << kTile) - 1u);
      if (PASS == 1) {
        if (lane == 0) urec[u_out + nu] = (static_cast<uint32_t>(m) << 8) | mask;
        if (mine) {
          const int64_t p = p_out + np + __popc(mask & ((1u << lane) - 1u));
          const double dx = X[3 * (int64_t)m] - xi, dy = X[3 * (int64_t)m + 1] - yi,
                       dz = X[3 * (int64_t)m + 2] - zi;
          const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
          const bool ok = d2 > 0.0 && d2 <= r2;
          const double inv = ok ? 1.0 / sqrt(d2) : 0.0;
          const double wx = dx * inv, wy = dy * inv, wz = dz * inv;
          if (pw64) {
            pw64[4 * p] = wx;
            pw64[4 * p + 1] = wy;
            pw64[4 * p + 2] = wz;
            pw64[4 * p + 3] = 0.0;
          }
          if (pw32) reinterpret_cast<float4*>(pw32)[p] = make_float4((float)wx, (float)wy, (float)wz, 0.f);
        }
      }
      nu += 1;
      np += __popc(mask);
      if (mine) ++e;
    }
    if (PASS == 0 && lane == 0) {
      ucount[t] = nu;
      pcount[t] = np;
    }
  }
}

__global__ void k_set0_pair(int64_t* a, int64_t* b) {
  a[0] = 0;
  b[0] = 0;
}

template <class T>
struct PW;
template <>
struct PW<float> {
  __device__ __forceinline__ static void load(const void* base, int64_t p, float& wx, float& wy, float& wz) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(base) + p);
    wx = v.x;
    wy = v.y;
    wz = v.z;
  }
};
template <>
struct PW<double> {
  __device__ __forceinline__ static void load(const void* base, int64_t p, double& wx, double& wy, double& wz) {
    const double2* q = reinterpret_cast<const double2*>(base) + 2 * p;
    const double2 a = __ldg(q), b = __ldg(q + 1);
    wx = a.x;
    wy = a.y;
    wz = b.x;
  }
};

template <class T, int V>
__device__ __forceinline__ void vld2(const T* p, T (&x)[V]) {
  if constexpr (V == 1) {
    x[0] = __ldg(p);
  } else if constexpr (sizeof(T) == 4) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
    x[0] = v.x;
    x[1] = v.y;
  } else {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    x[0] = v.x;
    x[1] = v.y;
  }
}

struct EpiT {
  double alpha, gamma, beta, mu;
  int r, accumulate, has_yin;
};

constexpr int kThreads = 256;

// One group of LPR lanes per tile; lane owns V consecutive columns per chunk.
template <class T, int B, int V>
__global__ void __launch_bounds__(kThreads)
k_spmm_tiles(int64_t n_atoms, const int64_t* __restrict__ uptr, const int64_t* __restrict__ pptr,
             const uint32_t* __restrict__ urec, const void* __restrict__ pw, const T* __restrict__ diag,
             const T* __restrict__ X, int64_t ldx, T* Y, int64_t ldy, const T* Yin, int64_t ldyin,
             T* __restrict__ Acc, int64_t ldacc, int c0, EpiT ep, const double* __restrict__ Q, int64_t ndof,
             const double* __restrict__ coef) {
  constexpr int LPR = (B / V) < 32 ? (B / V) : 32;
  constexpr int CPL = B / (LPR * V);
  constexpr int GPW = 32 / LPR;
  constexpr int GPB = (kThreads / 32) * GPW;
  __shared__ double s_coef[8 * B];
  if (ep.r > 0) {
    for (int t = threadIdx.x; t < ep.r * B; t += kThreads) s_coef[t] = coef[t];
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const int cl = lane % LPR;
  const int grp = (threadIdx.x >> 5) * GPW + lane / LPR;
  const int64_t ntiles = (n_atoms + kTile - 1) / kTile;
  const int64_t per = (ntiles + gridDim.x - 1) / gridDim.x;
  const int64_t t_beg = (int64_t)blockIdx.x * per;
  const int64_t t_end = t_beg + per < ntiles ? t_beg + per : ntiles;
  for (int64_t t = t_beg + grp; t < t_end; t += GPB) {
    T acc[kTile][3][CPL][V];
#pragma unroll
    for (int r = 0; r < kTile; ++r)
#pragma unroll
      for (int q = 0; q < CPL; ++q)
#pragma unroll
        for (int v = 0; v < V; ++v) acc[r][0][q][v] = acc[r][1][q][v] = acc[r][2][q][v] = T(0);
    int64_t p = pptr[t];
    const int64_t u1 = uptr[t + 1];
    const T* Xc = X + c0 + cl * V;
    for (int64_t u = uptr[t]; u < u1; ++u) {
      const uint32_t rec = __ldg(urec + u);
      const int64_t j = rec >> 8;
      const unsigned mask = rec & 0xffu;
      const T* xj = Xc + 3 * j * ldx;
      T x0[CPL][V], x1[CPL][V], x2[CPL][V];
#pragma unroll
      for (int q = 0; q < CPL; ++q) {
        vld2<T, V>(xj + q * LPR * V, x0[q]);
        vld2<T, V>(xj + ldx + q * LPR * V, x1[q]);
        vld2<T, V>(xj + 2 * ldx + q * LPR * V, x2[q]);
      }
#pragma unroll
      for (int r = 0; r < kTile; ++r) {
        if (mask & (1u << r)) {
          T wx, wy, wz;
          PW<T>::load(pw, p, wx, wy, wz);
          ++p;
#pragma unroll
          for (int q = 0; q < CPL; ++q)
#pragma unroll
            for (int v = 0; v < V; ++v) {
              const T dot = wx * x0[q][v] + wy * x1[q][v] + wz * x2[q][v];
              acc[r][0][q][v] -= wx * dot;
              acc[r][1][q][v] -= wy * dot;
              acc[r][2][q][v] -= wz * dot;
            }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kTile; ++r) {
      const int64_t i = t * kTile + r;
      if (i >= n_atoms) break;
      const T* d = diag + 8 * i;
      const T dxx = d[0], dyy = d[1], dzz = d[2], dxy = d[3], dxz = d[4], dyz = d[5];
      const int64_t r0 = 3 * i;
#pragma unroll
      for (int q = 0; q < CPL; ++q)
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const int c = (q * LPR + cl) * V + v;
          const T x0 = X[r0 * ldx + c0 + c], x1 = X[(r0 + 1) * ldx + c0 + c], x2 = X[(r0 + 2) * ldx + c0 + c];
          T h[3];
          h[0] = acc[r][0][q][v] + dxx * x0 + dxy * x1 + dxz * x2;
          h[1] = acc[r][1][q][v] + dxy * x0 + dyy * x1 + dyz * x2;
          h[2] = acc[r][2][q][v] + dxz * x0 + dyz * x1 + dzz * x2;
          const T xs[3] = {x0, x1, x2};
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const int64_t row = r0 + a;
            double y = ep.alpha * (double)h[a] + ep.gamma * (double)xs[a];
            if (ep.has_yin) y += ep.beta * (double)Yin[row * ldyin + c0 + c];
            for (int qq = 0; qq < ep.r; ++qq) y += Q[qq * ndof + row] * s_coef[qq * B + c];
            Y[row * ldy + c0 + c] = (T)y;
            if (ep.accumulate) Acc[row * ldacc + c0 + c] += (T)(ep.mu * y);
          }
        }
    }
  }
}

// Hotelling coefficients (same two-stage FP64 reduction as spmm.cu).
template <class T, int B>
__global__ void __launch_bounds__(kThreads)
k_qx_partial_t(const double* __restrict__ Q, int64_t ndof, const T* __restrict__ X, int64_t ldx, int c0,
               double* __restrict__ partial) {
  __shared__ double s[kThreads];
  const int q = blockIdx.y, r = gridDim.y;
  const double* qr = Q + q * ndof;
  const int c = threadIdx.x % B;
  double acc = 0.0;
  const int64_t total = ndof * B;
  for (int64_t p = (int64_t)blockIdx.x * kThreads + threadIdx.x; p < total; p += (int64_t)gridDim.x * kThreads)
    acc += qr[p / B] * (double)X[(p / B) * ldx + c0 + c];
  s[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < B) {
    double t = 0.0;
    for (int u = threadIdx.x; u < kThreads; u += B) t += s[u];
    partial[((int64_t)blockIdx.x * r + q) * B + threadIdx.x] = t;
  }
}

__global__ void k_qx_final_t(const double* __restrict__ partial, int P, int r, int B, double shift,
                             double* __restrict__ coef) {
  for (int t = threadIdx.x; t < r * B; t += blockDim.x) {
    double s = 0.0;
    for (int p = 0; p < P; ++p) s += partial[(int64_t)p * r * B + t];
    coef[t] = shift * s;
  }
}

constexpr int kQxBlocksT = 296;

template <class T, int B>
cudaError_t tile_launch(int64_t n, const int64_t* uptr, const int64_t* pptr, const uint32_t* urec, const void* pw,
                        const T* diag, const T* X, int64_t ldx, T* Y, int64_t ldy, const T* Yin, int64_t ldyin,
                        T* Acc, int64_t ldacc, int c0, EpiT ep, const double* Q, double hot_shift, double* partial,
                        double* coef, cudaStream_t s) {
  const int64_t ndof = 3 * n;
  if (ep.r > 0) {
    k_qx_partial_t<T, B><<<dim3(kQxBlocksT, ep.r), kThreads, 0, s>>>(Q, ndof, X, ldx, c0, partial);
    k_qx_final_t<<<1, 512, 0, s>>>(partial, kQxBlocksT, ep.r, B, hot_shift, coef);
  }
  // float2 gathers only where a whole warp owns one tile (B = 64 in FP32); other
  // widths use scalar gathers with 32 (or B) lanes per tile.
  constexpr int VV = (sizeof(T) == 4 && B >= 64) ? 2 : 1;
  const uintptr_t al = 2 * sizeof(T);
  bool vec = (ldx % 2 == 0) && (ldy % 2 == 0) && (c0 % 2 == 0) && ((uintptr_t)X % al == 0) && ((uintptr_t)Y % al == 0);
  if (ep.has_yin) vec = vec && (ldyin % 2 == 0) && ((uintptr_t)Yin % al == 0);
  if (ep.accumulate) vec = vec && (ldacc % 2 == 0) && ((uintptr_t)Acc % al == 0);
  const int64_t ntiles = (n + kTile - 1) / kTile;
  const int blocks = grid_for(ntiles, 32, 148 * 3);
  if (VV == 2 && vec)
    k_spmm_tiles<T, B, VV><<<blocks, kThreads, 0, s>>>(n, uptr, pptr, urec, pw, diag, X, ldx, Y, ldy, Yin, ldyin,
                                                       Acc, ldacc, c0, ep, Q, ndof, coef);
  else
    k_spmm_tiles<T, B, 1><<<blocks, kThreads, 0, s>>>(n, uptr, pptr, urec, pw, diag, X, ldx, Y, ldy, Yin, ldyin,
                                                      Acc, ldacc, c0, ep, Q, ndof, coef);
  return cudaGetLastError();
}

}  // namespace
}  // namespace inch

using namespace inch;

extern "C" size_t inch_tile_store_workspace_size(int64_t n_atoms) {
  const int64_t nt = (n_atoms + kTile - 1) / kTile;
  size_t cb = 0;
  cub::DeviceScan::InclusiveSum(nullptr, cb, (int64_t*)nullptr, (int64_t*)nullptr, (int)(nt > 0 ? nt : 1));
  Sizer s;
  s.take<int64_t>(nt);
  s.take<int64_t>(nt);
  s.take<char>(cb);
  return s.bytes();
}

extern "C" inch_status inch_tile_store_count(const int64_t* rowptr, const int32_t* cols, int64_t n,
                                             int64_t* tile_uptr, int64_t* tile_pptr, int64_t* n_union_host,
                                             int64_t* n_pairs_host, void* ws, size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(rowptr && cols && tile_uptr && tile_pptr && n_union_host && n_pairs_host, INCH_INVALID_ARG,
               "inch_tile_store_count: NULL argument");
  INCH_REQUIRE(n >= 1 && n < (int64_t(1) << 24), INCH_LIMIT,
               "inch_tile_store_count: n_atoms=%lld outside 1..2^24-1 (column packed in 24 bits)", (long long)n);
  const int64_t nt = (n + kTile - 1) / kTile;
  Carver c(ws, ws_bytes);
  int64_t* uc = c.take<int64_t>(nt);
  int64_t* pc = c.take<int64_t>(nt);
  size_t cb = 0;
  cub::DeviceScan::InclusiveSum(nullptr, cb, (int64_t*)nullptr, (int64_t*)nullptr, (int)nt);
  void* tmp = c.take<char>(cb);
  INCH_REQUIRE(c.ok, INCH_OOM, "inch_tile_store_count: workspace of %zu bytes, need %zu", ws_bytes,
               inch_tile_store_workspace_size(n));
  k_tile_merge<0><<<grid_for(nt, kWarpsBuild, 148 * 16), kWarpsBuild * 32, 0, stream>>>(
      nullptr, n, 0.0, rowptr, cols, uc, pc, nullptr, nullptr, nullptr, nullptr, nullptr);
  INCH_LAUNCH_CHECK();
  k_set0_pair<<<1, 1, 0, stream>>>(tile_uptr, tile_pptr);
  INCH_LAUNCH_CHECK();
  size_t c1 = cb;
  INCH_CUDA(cub::DeviceScan::InclusiveSum(tmp, c1, uc, tile_uptr + 1, (int)nt, stream));
  c1 = cb;
  INCH_CUDA(cub::DeviceScan::InclusiveSum(tmp, c1, pc, tile_pptr + 1, (int)nt, stream));
  INCH_CUDA(cudaMemcpyAsync(n_union_host, tile_uptr + nt, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cudaMemcpyAsync(n_pairs_host, tile_pptr + nt, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cudaStreamSynchronize(stream));
  return INCH_OK;
}

extern "C" inch_status inch_tile_store_fill(const double* X, int64_t n, double rc, const int64_t* rowptr,
                                            const int32_t* cols, const int64_t* tile_uptr, const int64_t* tile_pptr,
                                            uint32_t* urec, double* pw64, float* pw32, cudaStream_t stream) {
  INCH_REQUIRE(X && rowptr && cols && tile_uptr && tile_pptr && urec && (pw64 || pw32), INCH_INVALID_ARG,
               "inch_tile_store_fill: NULL argument");
  INCH_REQUIRE(n >= 1 && n < (int64_t(1) << 24), INCH_LIMIT, "inch_tile_store_fill: n_atoms outside 1..2^24-1");
  INCH_REQUIRE(((uintptr_t)pw64 & 15) == 0 && ((uintptr_t)pw32 & 15) == 0, INCH_INVALID_ARG,
               "inch_tile_store_fill: w buffers must be 16-byte aligned");
  const int64_t nt = (n + kTile - 1) / kTile;
  k_tile_merge<1><<<grid_for(nt, kWarpsBuild, 148 * 16), kWarpsBuild * 32, 0, stream>>>(
      X, n, rc * rc, rowptr, cols, nullptr, nullptr, tile_uptr, tile_pptr, urec, pw64, pw32);
  INCH_LAUNCH_CHECK();
  return INCH_OK;
}

extern "C" size_t inch_spmm_tiles_workspace_size(void) {
  Sizer s;
  s.take<double>((size_t)kQxBlocksT * 8 * 64);
  s.take<double>(8 * 64);
  return s.bytes();
}

extern "C" inch_status inch_spmm_tiles(int32_t prec, int64_t n, const int64_t* tile_uptr, const int64_t* tile_pptr,
                                       const uint32_t* urec, const void* pw, const void* diag, const void* Xv,
                                       int64_t ldx, int32_t b, void* Yv, int64_t ldy, const void* Yinv, int64_t ldyin,
                                       void* Accv, int64_t ldacc, const double* q, const inch_spmm_epilogue* ep_in,
                                       void* ws, size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(prec == 32 || prec == 64, INCH_INVALID_ARG, "inch_spmm_tiles: prec must be 32 or 64");
  INCH_REQUIRE(tile_uptr && tile_pptr && urec && pw && diag && Xv && Yv && ep_in, INCH_INVALID_ARG,
               "inch_spmm_tiles: NULL argument");
  INCH_REQUIRE(n >= 1 && n < (int64_t(1) << 24), INCH_INVALID_ARG, "inch_spmm_tiles: n_atoms out of range");
  INCH_REQUIRE(b >= 1 && b <= 64, INCH_INVALID_ARG, "inch_spmm_tiles: b=%d outside 1..64", b);
  INCH_REQUIRE(ldx >= b && ldy >= b && Xv != Yv, INCH_INVALID_ARG, "inch_spmm_tiles: bad leading dimension or X == Y");
  const inch_spmm_epilogue& e = *ep_in;
  INCH_REQUIRE(e.r >= 0 && e.r <= 8 && (e.r == 0 || q), INCH_INVALID_ARG, "inch_spmm_tiles: bad deflation basis");
  INCH_REQUIRE(e.beta == 0.0 || (Yinv && ldyin >= b), INCH_INVALID_ARG, "inch_spmm_tiles: beta != 0 needs Yin");
  INCH_REQUIRE(!e.accumulate || (Accv && ldacc >= b), INCH_INVALID_ARG, "inch_spmm_tiles: accumulate needs Acc");
  INCH_REQUIRE(((uintptr_t)pw & 15) == 0 && ((uintptr_t)diag & 15) == 0, INCH_INVALID_ARG,
               "inch_spmm_tiles: store buffers must be 16-byte aligned");
  double *partial = nullptr, *coef = nullptr;
  if (e.r > 0) {
    Carver c(ws, ws_bytes);
    partial = c.take<double>((size_t)kQxBlocksT * 8 * 64);
    coef = c.take<double>(8 * 64);
    INCH_REQUIRE(c.ok, INCH_OOM, "inch_spmm_tiles: workspace too small");
  }
  EpiT ep{e.alpha, e.gamma, e.beta, e.mu, e.r, e.accumulate, e.beta != 0.0 ? 1 : 0};
  cudaError_t err = cudaSuccess;
  int c0 = 0;
  while (c0 < b && err == cudaSuccess) {
    const int rem = b - c0;
#define TT(TYPE, BB)                                                                                         \
  err = tile_launch<TYPE, BB>(n, tile_uptr, tile_pptr, urec, pw, static_cast<const TYPE*>(diag),              \
                              static_cast<const TYPE*>(Xv), ldx, static_cast<TYPE*>(Yv), ldy,                  \
                              static_cast<const TYPE*>(Yinv), ldyin, static_cast<TYPE*>(Accv), ldacc, c0, ep, q, \
                              e.hot_shift, partial, coef, stream);                                             \
  c0 += BB;
    if (prec == 32) {
      if (rem >= 64) { TT(float, 64) }
      else if (rem >= 32) { TT(float, 32) }
      else if (rem >= 16) { TT(float, 16) }
      else if (rem >= 8) { TT(float, 8) }
      else if (rem >= 4) { TT(float, 4) }
      else if (rem >= 2) { TT(float, 2) }
      else { TT(float, 1) }
    } else {
      if (rem >= 32) { TT(double, 32) }
      else if (rem >= 16) { TT(double, 16) }
      else if (rem >= 8) { TT(double, 8) }
      else if (rem >= 4) { TT(double, 4) }
      else if (rem >= 2) { TT(double, 2) }
      else { TT(double, 1) }
    }
#undef TT
  }
  INCH_REQUIRE(err == cudaSuccess, INCH_CUDA_ERROR, "inch_spmm_tiles: %s", cudaGetErrorString(err));
  return INCH_OK;
}
