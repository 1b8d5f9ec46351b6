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
#include <atomic>

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

// ---------------------------------------------------------------------------
// Band-tile product (union walk, TMA-staged batches).
//
// One warp owns one 8-row tile and one column panel of P = 32*C columns; lane l
// owns the C consecutive columns [l*C, l*C + C) of the panel.  The tile's union
// columns are processed in batches of kBatch.  A batch is staged in this warp's
// slice of shared memory by the bulk-copy (TMA) engine: lane u (< kBatch) issues
// the three row segments of X_j for union column u of the batch (P values each,
// rows 3j, 3j+1, 3j+2), lane kBatch issues one copy of the batch's w values
// (contiguous in the tile store), and all of them complete on the buffer's
// mbarrier.  Batches are double-buffered: batch b+1 is in flight while batch b
// is multiplied, so a warp keeps up to 2*kBatch gathers outstanding while its
// lanes execute only arithmetic and shared loads.
//
// For each union column, each lane reads its slice of X_j once and applies it to
// every row of the column's mask.  The mask is split in two nibbles; each nibble
// dispatches through a 16-way switch to straight-line code with the accumulator
// rows fixed at compile time, so the accumulators stay in registers.  FP32
// panels with C >= 2 use the packed f32x2 FMAs of sm_100.  The accumulators hold
// S = sum_j w (w . X_j); the epilogue forms (H X)_i = D_i X_i - S.
//
// Every mbarrier wait is bounded; a wait that runs out records kBandTimeout in
// the status word (read by inch_spmm_band_status) and the warp stops after
// draining its outstanding copies.
// ---------------------------------------------------------------------------
constexpr int kBatch = 8;                  // union columns per staged batch
constexpr int kWarpsUT = 4;                // warps per block
constexpr int kMaxPanel = 128;             // widest panel (FP32, C = 4)
constexpr unsigned kWaitSpins = 1u << 24;  // bound of one mbarrier wait
constexpr int kBandTimeout = 1;

__device__ int g_band_status;              // 0, or kBandTimeout after a wait ran out

struct EpiT {
  double alpha, gamma, beta, mu;
  int r, accumulate, has_yin;
  const double* seg_coef;   // optional per-segment (alpha, gamma, beta)
  const int* atom_seg;
};

// w of one pair as stored by the tile store: FP32 {wx,wy,wz,0}, FP64 the same in doubles.
template <class T>
struct WRaw;
template <>
struct WRaw<float> {
  float4 v;
};
template <>
struct WRaw<double> {
  double2 a, b;
};

// One staged batch: this warp's slice of X_j (3 rows x P columns) for kBatch
// union columns and the w of their pairs (at most kTile each).
template <class T, int C>
struct Batch {
  T x[kBatch][3][32 * C];
  WRaw<T> w[kBatch * kTile];
};

template <class T, int C>
struct WarpSmem {
  Batch<T, C> buf[2];
  unsigned long long bar[2];
};

// Register vector type of one lane's columns: NV values of type V.
template <class T, int C>
struct UK;
template <>
struct UK<float, 4> {
  using V = float2;
  static constexpr int NV = 2;
  static constexpr int MINB = 2;
};
template <>
struct UK<float, 2> {
  using V = float2;
  static constexpr int NV = 1;
  static constexpr int MINB = 4;
};
template <>
struct UK<float, 1> {
  using V = float;
  static constexpr int NV = 1;
  static constexpr int MINB = 4;
};
template <>
struct UK<double, 2> {
  using V = double;
  static constexpr int NV = 2;
  static constexpr int MINB = 2;
};
template <>
struct UK<double, 1> {
  using V = double;
  static constexpr int NV = 1;
  static constexpr int MINB = 4;
};

__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float vmul(float a, float b) { return a * b; }
__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double vmul(double a, double b) { return a * b; }
__device__ __forceinline__ double vfma(double a, double b, double c) { return fma(a, b, c); }

__device__ __forceinline__ void get_w(const WRaw<float>& s, float2& wx, float2& wy, float2& wz) {
  const float4 v = s.v;
  wx = make_float2(v.x, v.x);
  wy = make_float2(v.y, v.y);
  wz = make_float2(v.z, v.z);
}
__device__ __forceinline__ void get_w(const WRaw<float>& s, float& wx, float& wy, float& wz) {
  const float4 v = s.v;
  wx = v.x;
  wy = v.y;
  wz = v.z;
}
__device__ __forceinline__ void get_w(const WRaw<double>& s, double& wx, double& wy, double& wz) {
  const double2 a = s.a, b = s.b;
  wx = a.x;
  wy = a.y;
  wz = b.x;
}

// --- mbarrier and bulk-copy helpers (this CTA's shared memory only) ----------
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase with this parity; false if the bound ran out.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  for (unsigned s = 0; s < kWaitSpins; ++s)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// One lane's C columns of row p (p points at the lane's first column).
template <class T, int C, bool GLOBAL>
__device__ __forceinline__ void load_v(const T* p, typename UK<T, C>::V (&v)[UK<T, C>::NV]) {
  if constexpr (sizeof(T) == 4 && C == 4) {
    const float4 q = GLOBAL ? __ldg(reinterpret_cast<const float4*>(p)) : *reinterpret_cast<const float4*>(p);
    v[0] = make_float2(q.x, q.y);
    v[1] = make_float2(q.z, q.w);
  } else if constexpr (sizeof(T) == 4 && C == 2) {
    v[0] = GLOBAL ? __ldg(reinterpret_cast<const float2*>(p)) : *reinterpret_cast<const float2*>(p);
  } else if constexpr (sizeof(T) == 8 && C == 2) {
    const double2 q = GLOBAL ? __ldg(reinterpret_cast<const double2*>(p)) : *reinterpret_cast<const double2*>(p);
    v[0] = q.x;
    v[1] = q.y;
  } else {
    v[0] = GLOBAL ? __ldg(p) : *p;
  }
}

template <class T, int C>
__device__ __forceinline__ void to_scalars(const typename UK<T, C>::V (&v)[UK<T, C>::NV], T (&s)[C]) {
  if constexpr (sizeof(T) == 4 && C >= 2) {
#pragma unroll
    for (int k = 0; k < UK<T, C>::NV; ++k) {
      s[2 * k] = v[k].x;
      s[2 * k + 1] = v[k].y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < C; ++k) s[k] = v[k];
  }
}

template <class T, int C>
__device__ __forceinline__ void load_s(const T* p, T (&s)[C]) {
  typename UK<T, C>::V v[UK<T, C>::NV];
  load_v<T, C, true>(p, v);
  to_scalars<T, C>(v, s);
}

template <class T, int C>
__device__ __forceinline__ void store_s(T* p, const T (&s)[C]) {
  if constexpr (sizeof(T) == 4 && C == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(s[0], s[1], s[2], s[3]);
  } else if constexpr (sizeof(T) == 4 && C == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(s[0], s[1]);
  } else if constexpr (sizeof(T) == 8 && C == 2) {
    *reinterpret_cast<double2*>(p) = make_double2(s[0], s[1]);
  } else {
    p[0] = s[0];
  }
}

// Rows R0 + b for the set bits b of NIB, their w at sw[0], sw[1], ... in bit order.
template <int R0, int NIB, class T, class V, int NV>
__device__ __forceinline__ void nib_rows(V (&acc)[kTile][3][NV], const V (&x)[3][NV], const WRaw<T>* sw) {
  int idx = 0;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    if (NIB & (1 << b)) {
      V wx, wy, wz;
      get_w(sw[idx], wx, wy, wz);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        V d = vmul(wx, x[0][v]);
        d = vfma(wy, x[1][v], d);
        d = vfma(wz, x[2][v], d);
        acc[R0 + b][0][v] = vfma(wx, d, acc[R0 + b][0][v]);
        acc[R0 + b][1][v] = vfma(wy, d, acc[R0 + b][1][v]);
        acc[R0 + b][2][v] = vfma(wz, d, acc[R0 + b][2][v]);
      }
      ++idx;
    }
  }
}

template <int R0, class T, class V, int NV>
__device__ __forceinline__ void nib_dispatch(unsigned nib, V (&acc)[kTile][3][NV], const V (&x)[3][NV],
                                             const WRaw<T>* sw) {
#define INCH_NIB(N)                        \
  case N:                                  \
    nib_rows<R0, N, T, V, NV>(acc, x, sw); \
    break;
  switch (nib) {
    INCH_NIB(1)
    INCH_NIB(2)
    INCH_NIB(3)
    INCH_NIB(4)
    INCH_NIB(5)
    INCH_NIB(6)
    INCH_NIB(7)
    INCH_NIB(8)
    INCH_NIB(9)
    INCH_NIB(10)
    INCH_NIB(11)
    INCH_NIB(12)
    INCH_NIB(13)
    INCH_NIB(14)
    INCH_NIB(15)
    default:
      break;
  }
#undef INCH_NIB
}

template <class T>
__device__ __forceinline__ void zero_val(T& a) {
  a = T(0);
}
__device__ __forceinline__ void zero_val(float2& a) { a = make_float2(0.f, 0.f); }

template <class T, int C>
constexpr size_t band_smem_bytes() {
  return (size_t)kWarpsUT * sizeof(WarpSmem<T, C>);
}

// Exclusive scan of popc(mask) over lanes 0..kBatch-1 (the batch's records);
// the batch's pair count in `tot`.
__device__ __forceinline__ int batch_scan(uint32_t rec, int lane, int& tot) {
  const int pc = __popc(rec & 0xffu);
  int incl = pc;
#pragma unroll
  for (int o = 1; o < kBatch; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  tot = __shfl_sync(0xffffffffu, incl, kBatch - 1);
  return incl - pc;
}

template <class T, int C>
__global__ void __launch_bounds__(kWarpsUT * 32, UK<T, C>::MINB)
k_spmm_band(int n_atoms, const int64_t* __restrict__ uptr, const int64_t* __restrict__ pptr,
            const uint32_t* __restrict__ urec, const void* __restrict__ pw, const T* __restrict__ diag,
            const T* __restrict__ X, int64_t ldx, T* Y, int64_t ldy, const T* Yin, int64_t ldyin,
            T* __restrict__ Acc, int64_t ldacc, int c0, int ncols, EpiT ep, const double* __restrict__ Q,
            int64_t ndof, const double* __restrict__ coef) {
  using V = typename UK<T, C>::V;
  constexpr int NV = UK<T, C>::NV;
  constexpr int P = 32 * C;
  constexpr int WB = (int)sizeof(WRaw<T>);
  constexpr int VEC = 16 / (int)sizeof(T);            // elements per 16 bytes
  extern __shared__ __align__(128) unsigned char band_smem[];
  __shared__ double s_coef[8 * P];
  if (ep.r > 0) {
    for (int t = threadIdx.x; t < ep.r * P; t += kWarpsUT * 32) s_coef[t] = coef[t];
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  WarpSmem<T, C>* sm = reinterpret_cast<WarpSmem<T, C>*>(band_smem) + warp;
  const unsigned bar0 = smem_u32(&sm->bar[0]), bar1 = smem_u32(&sm->bar[1]);
  if (lane == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
  }
  fence_proxy_async();
  __syncwarp();
  unsigned ph0 = 0u, ph1 = 0u;               // parity of the next phase to complete, per buffer
  bool pend0 = false, pend1 = false;         // a staged batch not yet waited for, per buffer
  const bool on = lane * C < ncols;          // lane inside the panel
  // bytes of one staged row segment: the panel's columns rounded up to 16 bytes
  // (the rounding stays inside the row: leading dimensions are multiples of VEC)
  const unsigned row_bytes = (unsigned)(((ncols + VEC - 1) / VEC) * VEC * (int)sizeof(T));
  const T* Xp = X + c0;
  const unsigned char* pwb = static_cast<const unsigned char*>(pw);
  const int ntiles = (n_atoms + kTile - 1) / kTile;
  for (int t = blockIdx.x * kWarpsUT + warp; t < ntiles; t += gridDim.x * kWarpsUT) {
    V acc[kTile][3][NV];
#pragma unroll
    for (int r = 0; r < kTile; ++r)
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int k = 0; k < NV; ++k) zero_val(acc[r][a][k]);
    const int64_t ubase = uptr[t];
    const int nu = (int)(uptr[t + 1] - ubase);
    const int64_t pbase = pptr[t];
    const int nb = (nu + kBatch - 1) / kBatch;
    // records of the batch being multiplied (rc), being staged next (rs) and the
    // one after it (rp), in lanes 0..kBatch-1; ec: their exclusive pair offsets
    auto rec_of = [&](int bb) -> uint32_t {
      const int u = bb * kBatch + lane;
      return (lane < kBatch && u < nu) ? __ldg(urec + ubase + u) : 0u;
    };
    int qstage = 0;                          // tile-relative first pair of the next batch to stage
    // stage batch bb (records r) into buffer bb & 1; returns the exclusive offsets
    auto issue = [&](int bb, uint32_t r) -> int {
      const int s = bb & 1;
      int tot;
      const int ex = batch_scan(r, lane, tot);
      const int cnt = (nu - bb * kBatch) < kBatch ? (nu - bb * kBatch) : kBatch;
      Batch<T, C>* B = &sm->buf[s];
      const unsigned bar = s ? bar1 : bar0;
      if (lane == 0) mbar_expect_tx(bar, (unsigned)cnt * 3u * row_bytes + (unsigned)tot * WB);
      __syncwarp();
      if (lane < cnt) {
        const T* p = Xp + (int64_t)(3 * (int)(r >> 8)) * ldx;
        bulk_g2s(smem_u32(&B->x[lane][0][0]), p, row_bytes, bar);
        bulk_g2s(smem_u32(&B->x[lane][1][0]), p + ldx, row_bytes, bar);
        bulk_g2s(smem_u32(&B->x[lane][2][0]), p + 2 * ldx, row_bytes, bar);
      }
      if (lane == kBatch && tot > 0)
        bulk_g2s(smem_u32(&B->w[0]), pwb + (pbase + qstage) * WB, (unsigned)tot * WB, bar);
      qstage += tot;
      if (s)
        pend1 = true;
      else
        pend0 = true;
      return ex;
    };
    uint32_t rc = rec_of(0), rs = rec_of(1), rp = 0u;
    int ec = 0, es = 0;
    __syncwarp();                            // the previous tile's reads of both buffers are done
    fence_proxy_async();
    if (nb > 0) ec = issue(0, rc);
    bool ok = true;
    for (int bb = 0; bb < nb; ++bb) {
      if (bb + 1 < nb) {
        rp = rec_of(bb + 2);
        __syncwarp();                        // every lane is done reading the buffer issue() refills
        fence_proxy_async();
        es = issue(bb + 1, rs);
      }
      const int s = bb & 1;
      if (!mbar_wait(s ? bar1 : bar0, s ? ph1 : ph0)) {
        ok = false;
        break;
      }
      if (s) {
        ph1 ^= 1u;
        pend1 = false;
      } else {
        ph0 ^= 1u;
        pend0 = false;
      }
      const Batch<T, C>* B = &sm->buf[s];
      const int cnt = (nu - bb * kBatch) < kBatch ? (nu - bb * kBatch) : kBatch;
      for (int k = 0; k < cnt; ++k) {
        const unsigned m = __shfl_sync(0xffffffffu, rc, k) & 0xffu;
        const int qk = __shfl_sync(0xffffffffu, ec, k);
        V x[3][NV];
        load_v<T, C, false>(&B->x[k][0][lane * C], x[0]);
        load_v<T, C, false>(&B->x[k][1][lane * C], x[1]);
        load_v<T, C, false>(&B->x[k][2][lane * C], x[2]);
        const WRaw<T>* sw = B->w + qk;
        nib_dispatch<0, T, V, NV>(m & 15u, acc, x, sw);
        nib_dispatch<4, T, V, NV>(m >> 4, acc, x, sw + __popc(m & 15u));
      }
      rc = rs;
      ec = es;
      rs = rp;
    }
    if (!ok) {
      // a wait ran out: record it, let this warp's outstanding copies land (again
      // bounded), and stop
      if (lane == 0) atomicExch(&g_band_status, kBandTimeout);
      if (pend0) mbar_wait(bar0, ph0);
      if (pend1) mbar_wait(bar1, ph1);
      return;
    }
    // epilogue: (H X)_i = D_i X_i - S_i, then the fused combination per element
    if (!on) continue;
#pragma unroll
    for (int r = 0; r < kTile; ++r) {
      const int i = t * kTile + r;
      if (i >= n_atoms) break;
      const T* d = diag + 8 * (int64_t)i;
      const T dxx = d[0], dyy = d[1], dzz = d[2], dxy = d[3], dxz = d[4], dyz = d[5];
      double al = ep.alpha, ga = ep.gamma, be = ep.beta;
      if (ep.seg_coef != nullptr) {
        const int sg = __ldg(ep.atom_seg + i);
        al = __ldg(ep.seg_coef + 3 * sg);
        ga = __ldg(ep.seg_coef + 3 * sg + 1);
        be = __ldg(ep.seg_coef + 3 * sg + 2);
      }
      const int64_t r0 = 3 * (int64_t)i;
      const T* xr = Xp + r0 * ldx + lane * C;
      T x0[C], x1[C], x2[C];
      load_s<T, C>(xr, x0);
      load_s<T, C>(xr + ldx, x1);
      load_s<T, C>(xr + 2 * ldx, x2);
      T s0[C], s1[C], s2[C];
      to_scalars<T, C>(acc[r][0], s0);
      to_scalars<T, C>(acc[r][1], s1);
      to_scalars<T, C>(acc[r][2], s2);
      const T alf = (T)al, gaf = (T)ga, bef = (T)be;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int64_t row = r0 + a;
        T yv[C], yin[C];
        if (ep.has_yin) load_s<T, C>(Yin + row * ldyin + c0 + lane * C, yin);
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const T h = (a == 0)   ? (dxx * x0[c] + dxy * x1[c] + dxz * x2[c]) - s0[c]
                      : (a == 1) ? (dxy * x0[c] + dyy * x1[c] + dyz * x2[c]) - s1[c]
                                 : (dxz * x0[c] + dyz * x1[c] + dzz * x2[c]) - s2[c];
          const T xa_ = (a == 0) ? x0[c] : (a == 1) ? x1[c] : x2[c];
          T y = alf * h + gaf * xa_;
          if (ep.has_yin) y += bef * yin[c];
          if (ep.r > 0) {
            double yq = (double)y;
            for (int q = 0; q < ep.r; ++q) yq += Q[q * ndof + row] * s_coef[q * P + lane * C + c];
            y = (T)yq;
          }
          yv[c] = y;
        }
        store_s<T, C>(Y + row * ldy + c0 + lane * C, yv);
        if (ep.accumulate) {
          T av[C];
          load_s<T, C>(Acc + row * ldacc + c0 + lane * C, av);
#pragma unroll
          for (int c = 0; c < C; ++c) av[c] = (T)((double)av[c] + ep.mu * (double)yv[c]);
          store_s<T, C>(Acc + row * ldacc + c0 + lane * C, av);
        }
      }
    }
  }
}

constexpr int kThreads = 256;

// Hotelling coefficients coef[q * P + c] = shift * sum_dof Q[q, dof] X[dof, c0 + c]
// for the ncols columns of one panel: per-block partial sums, then one warp per
// (q, c) adds the partials in a fixed order (deterministic, FP64).
template <class T, int P>
__global__ void __launch_bounds__(kThreads)
k_qx_partial_t(const double* __restrict__ Q, int64_t ndof, const T* __restrict__ X, int64_t ldx, int c0, int ncols,
               double* __restrict__ partial) {
  __shared__ double s[kThreads];
  const int q = blockIdx.y, r = gridDim.y;
  const double* qr = Q + q * ndof;
  const int c = threadIdx.x % P;
  constexpr int RPB = kThreads / P;   // dofs per block step
  double acc = 0.0;
  if (c < ncols) {
    for (int64_t dof = (int64_t)blockIdx.x * RPB + threadIdx.x / P; dof < ndof; dof += (int64_t)gridDim.x * RPB)
      acc += qr[dof] * (double)X[dof * ldx + c0 + c];
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  // tree over the threads of one column (P is a power of two dividing kThreads,
  // so t and t + stride always share a column): log2(kThreads / P) steps
#pragma unroll
  for (int stride = kThreads / 2; stride >= P; stride >>= 1) {
    if (threadIdx.x < stride) s[threadIdx.x] += s[threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x < P) partial[((int64_t)blockIdx.x * r + q) * P + threadIdx.x] = s[threadIdx.x];
}

__global__ void __launch_bounds__(kThreads)
k_qx_final_t(const double* __restrict__ partial, int nblk, int r, int P, double shift, double* __restrict__ coef) {
  const int64_t t = (int64_t)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (t >= (int64_t)r * P) return;
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int p = lane; p < nblk; p += 32) s += partial[(int64_t)p * r * P + t];
  s = warp_sum(s);
  if (lane == 0) coef[t] = shift * s;
}

constexpr int kQxBlocksT = 296;

// Process-wide launch choice (autotuner hook): the widest FP32 panel, 128 or 64.
std::atomic<int> g_band_panel32{128};

// Grid of the band kernel: its resident blocks per SM (registers and the ring's
// dynamic shared memory, opted in once per instantiation) times the SM count.
template <class T, int C>
int band_grid(int64_t ntiles) {
  static int per_sm = 0;
  if (per_sm == 0) {
    int nb = 0;
    const size_t sm = band_smem_bytes<T, C>();
    cudaFuncSetAttribute(k_spmm_band<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_spmm_band<T, C>, kWarpsUT * 32, sm) != cudaSuccess ||
        nb < 1)
      nb = 1;
    per_sm = nb;
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return grid_for(ntiles, kWarpsUT, sms * per_sm);
}

template <class T, int C>
cudaError_t band_launch(int64_t n, const int64_t* uptr, const int64_t* pptr, const uint32_t* urec, const void* pw,
                        const T* diag, const T* X, int64_t ldx, T* Y, int64_t ldy, const T* Yin, int64_t ldyin,
                        T* Acc, int64_t ldacc, int c0, int ncols, EpiT ep, const double* Q, double hot_shift,
                        double* partial, double* coef, cudaStream_t s) {
  constexpr int P = 32 * C;
  const int64_t ndof = 3 * n;
  if (ep.r > 0) {
    k_qx_partial_t<T, P><<<dim3(kQxBlocksT, ep.r), kThreads, 0, s>>>(Q, ndof, X, ldx, c0, ncols, partial);
    const int outs = ep.r * P;
    k_qx_final_t<<<(outs + kThreads / 32 - 1) / (kThreads / 32), kThreads, 0, s>>>(partial, kQxBlocksT, ep.r, P,
                                                                                   hot_shift, coef);
  }
  const int64_t ntiles = (n + kTile - 1) / kTile;
k_spmm_band<T, C><<<band_grid<T, C>(ntiles), kWarpsUT * 32, band_smem_bytes<T, C>(), s>>>(
      (int)n, uptr, pptr, urec, pw, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, ncols, ep, Q, ndof, coef);
  return cudaGetLastError();
}



// Whether every vector block starts on 16 bytes with a leading dimension that is a
// multiple of vec elements (the bulk copies and vector stores of the band kernel).
inline bool band_vectors_aligned(int vec, int esize, const void* X, int64_t ldx, const void* Y, int64_t ldy,
                                 const void* Yin, int64_t ldyin, const void* Acc, int64_t ldacc) {
  (void)esize;
  bool ok = (ldx % vec == 0) && (ldy % vec == 0) && ((uintptr_t)X % 16 == 0) && ((uintptr_t)Y % 16 == 0);
  if (Yin) ok = ok && (ldyin % vec == 0) && ((uintptr_t)Yin % 16 == 0);
  if (Acc) ok = ok && (ldacc % vec == 0) && ((uintptr_t)Acc % 16 == 0);
  return ok;
}

template <class T>
cudaError_t band_run(int64_t n, const int64_t* uptr, const int64_t* pptr, const uint32_t* urec, const void* pw,
                     const T* diag, const T* X, int64_t ldx, int b, T* Y, int64_t ldy, const T* Yin, int64_t ldyin,
                     T* Acc, int64_t ldacc, EpiT ep, const double* Q, double hot_shift, double* partial,
                     double* coef, cudaStream_t s) {
  cudaError_t err = cudaSuccess;
  int c0 = 0;
  while (c0 < b && err == cudaSuccess) {
    const int rem = b - c0;
    bool wide = false;
    if constexpr (sizeof(T) == 4) {
      if (g_band_panel32.load() >= 128 && rem >= 128) {
        err = band_launch<T, 4>(n, uptr, pptr, urec, pw, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, 128, ep,
                                Q, hot_shift, partial, coef, s);
        c0 += 128;
        wide = true;
      }
    }
    if (wide) {
    } else if (rem >= 64) {
      err = band_launch<T, 2>(n, uptr, pptr, urec, pw, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, 64, ep, Q,
                              hot_shift, partial, coef, s);
      c0 += 64;
    } else {
      const int nc = rem < 32 ? rem : 32;
      err = band_launch<T, 1>(n, uptr, pptr, urec, pw, diag, X, ldx, Y, ldy, Yin, ldyin, Acc, ldacc, c0, nc, ep, Q,
                              hot_shift, partial, coef, s);
      c0 += nc;
    }
  }
  return err;
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
  s.take<double>((size_t)kQxBlocksT * 8 * kMaxPanel);
  s.take<double>(8 * kMaxPanel);
  return s.bytes();
}

extern "C" inch_status inch_spmm_band_tune(int32_t widest_fp32_panel) {
  INCH_REQUIRE(widest_fp32_panel == 64 || widest_fp32_panel == 128, INCH_INVALID_ARG,
               "inch_spmm_band_tune: widest FP32 panel must be 64 or 128");
  g_band_panel32.store(widest_fp32_panel);
  return INCH_OK;
}

extern "C" inch_status inch_spmm_band_status(int32_t* status_host) {
  INCH_REQUIRE(status_host != nullptr, INCH_INVALID_ARG, "inch_spmm_band_status: NULL argument");
  int v = 0, zero = 0;
  INCH_CUDA(cudaMemcpyFromSymbol(&v, g_band_status, sizeof(int)));
  INCH_CUDA(cudaMemcpyToSymbol(g_band_status, &zero, sizeof(int)));
  *status_host = v;
  return INCH_OK;
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
  INCH_REQUIRE(b >= 1, INCH_INVALID_ARG, "inch_spmm_tiles: b=%d below 1", b);
  INCH_REQUIRE(ldx >= b && ldy >= b && Xv != Yv, INCH_INVALID_ARG, "inch_spmm_tiles: bad leading dimension or X == Y");
  const inch_spmm_epilogue& e = *ep_in;
  INCH_REQUIRE(e.r >= 0 && e.r <= 8 && (e.r == 0 || q), INCH_INVALID_ARG, "inch_spmm_tiles: bad deflation basis");
  INCH_REQUIRE(e.beta == 0.0 || (Yinv && ldyin >= b), INCH_INVALID_ARG, "inch_spmm_tiles: beta != 0 needs Yin");
  INCH_REQUIRE(!e.accumulate || (Accv && ldacc >= b), INCH_INVALID_ARG, "inch_spmm_tiles: accumulate needs Acc");
  INCH_REQUIRE(((uintptr_t)pw & 15) == 0 && ((uintptr_t)diag & 15) == 0, INCH_INVALID_ARG,
               "inch_spmm_tiles: store buffers must be 16-byte aligned");
  const int vec = prec == 32 ? 4 : 2;
  INCH_REQUIRE(band_vectors_aligned(vec, prec == 32 ? 4 : 8, Xv, ldx, Yv, ldy, e.beta != 0.0 ? Yinv : nullptr, ldyin,
                                    e.accumulate ? Accv : nullptr, ldacc),
               INCH_INVALID_ARG,
               "inch_spmm_tiles: vector blocks must start on 16 bytes with leading dimensions multiples of %d", vec);
  double *partial = nullptr, *coef = nullptr;
  if (e.r > 0) {
    Carver c(ws, ws_bytes);
    partial = c.take<double>((size_t)kQxBlocksT * 8 * kMaxPanel);
    coef = c.take<double>(8 * kMaxPanel);
    INCH_REQUIRE(c.ok, INCH_OOM, "inch_spmm_tiles: workspace of %zu bytes, need %zu", ws_bytes,
                 inch_spmm_tiles_workspace_size());
  }
  EpiT ep{e.alpha, e.gamma, e.beta, e.mu, e.r, e.accumulate, e.beta != 0.0 ? 1 : 0, nullptr, nullptr};
  cudaError_t err;
  if (prec == 32)
    err = band_run<float>(n, tile_uptr, tile_pptr, urec, pw, static_cast<const float*>(diag),
                          static_cast<const float*>(Xv), ldx, b, static_cast<float*>(Yv), ldy,
                          static_cast<const float*>(Yinv), ldyin, static_cast<float*>(Accv), ldacc, ep, q,
                          e.hot_shift, partial, coef, stream);
  else
    err = band_run<double>(n, tile_uptr, tile_pptr, urec, pw, static_cast<const double*>(diag),
                           static_cast<const double*>(Xv), ldx, b, static_cast<double*>(Yv), ldy,
                           static_cast<const double*>(Yinv), ldyin, static_cast<double*>(Accv), ldacc, ep, q,
                           e.hot_shift, partial, coef, stream);
  INCH_REQUIRE(err == cudaSuccess, INCH_CUDA_ERROR, "inch_spmm_tiles: %s", cudaGetErrorString(err));
  return INCH_OK;
}

extern "C" inch_status inch_spmm_tiles_seg(int32_t prec, int64_t n, const int64_t* tile_uptr,
                                           const int64_t* tile_pptr, const uint32_t* urec, const void* pw,
                                           const void* diag, const void* Xv, int64_t ldx, int32_t b, void* Yv,
                                           int64_t ldy, const void* Yinv, int64_t ldyin, const int32_t* atom_seg,
                                           const double* seg_coef, cudaStream_t stream) {
  INCH_REQUIRE(prec == 32 || prec == 64, INCH_INVALID_ARG, "inch_spmm_tiles_seg: prec must be 32 or 64");
  INCH_REQUIRE(tile_uptr && tile_pptr && urec && pw && diag && Xv && Yv && atom_seg && seg_coef, INCH_INVALID_ARG,
               "inch_spmm_tiles_seg: NULL argument");
  INCH_REQUIRE(n >= 1 && n < (int64_t(1) << 24), INCH_INVALID_ARG, "inch_spmm_tiles_seg: n_atoms out of range");
  INCH_REQUIRE(b >= 1 && ldx >= b && ldy >= b && Xv != Yv, INCH_INVALID_ARG,
               "inch_spmm_tiles_seg: bad b / leading dimension / aliasing");
  INCH_REQUIRE(Yinv == nullptr || ldyin >= b, INCH_INVALID_ARG, "inch_spmm_tiles_seg: ldyin below b");
  INCH_REQUIRE(((uintptr_t)pw & 15) == 0 && ((uintptr_t)diag & 15) == 0, INCH_INVALID_ARG,
               "inch_spmm_tiles_seg: store buffers must be 16-byte aligned");
  const int vec = prec == 32 ? 4 : 2;
  INCH_REQUIRE(band_vectors_aligned(vec, prec == 32 ? 4 : 8, Xv, ldx, Yv, ldy, Yinv, ldyin, nullptr, 0),
               INCH_INVALID_ARG,
               "inch_spmm_tiles_seg: vector blocks must start on 16 bytes with leading dimensions multiples of %d",
               vec);
  EpiT ep{0.0, 0.0, 0.0, 0.0, 0, 0, Yinv != nullptr ? 1 : 0, seg_coef, atom_seg};
  cudaError_t err;
  if (prec == 32)
    err = band_run<float>(n, tile_uptr, tile_pptr, urec, pw, static_cast<const float*>(diag),
                          static_cast<const float*>(Xv), ldx, b, static_cast<float*>(Yv), ldy,
                          static_cast<const float*>(Yinv), ldyin, nullptr, 0, ep, nullptr, 0.0, nullptr, nullptr,
                          stream);
  else
    err = band_run<double>(n, tile_uptr, tile_pptr, urec, pw, static_cast<const double*>(diag),
                           static_cast<const double*>(Xv), ldx, b, static_cast<double*>(Yv), ldy,
                           static_cast<const double*>(Yinv), ldyin, nullptr, 0, ep, nullptr, 0.0, nullptr, nullptr,
                           stream);
  INCH_REQUIRE(err == cudaSuccess, INCH_CUDA_ERROR, "inch_spmm_tiles_seg: %s", cudaGetErrorString(err));
  return INCH_OK;
}
