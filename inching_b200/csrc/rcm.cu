// Level-synchronous Cuthill-McKee that reproduces the sequential BFS of the
// reference (InchingLiteInteger/Fuel/Coordinate/T1.py:254-323) bit for bit.
//
// Sequential rule: frontier atoms are processed in order; each appends its
// still-unvisited neighbours (descending index) and then stably sorts that run by
// degree.  Hence, within one level,
//   * child j belongs to the EARLIEST frontier position q adjacent to it
//     (atomicMin over positions), and
//   * the children of q are ordered by (degree ascending, index descending),
//   * runs are concatenated in parent order (exclusive scan of run lengths).
// Each level costs four kernels (claim, count, scan, write) plus a one-thread
// advance kernel that also seeds the next connected component from the
// caller's argsort(degree) order.  The host reads the level bounds back once per
// level.
#include <cub/cub.cuh>

#include "common.cuh"

namespace inch {
namespace {

constexpr int kWarps = 8;
constexpr int kCap = INCH_MAX_DEGREE;

struct State {
  int64_t ls, le, n, seedptr;
};

__global__ void k_init(int* __restrict__ pos, int* __restrict__ claim, int64_t n, State* st) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    pos[i] = -1;
    claim[i] = 0x7fffffff;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->ls = 0;
    st->le = 0;
    st->n = 0;
    st->seedptr = 0;
  }
}

// Frontier atom at position q claims every neighbour unvisited at level start.
__global__ void k_claim(const int64_t* __restrict__ rowptr, const int* __restrict__ cols,
                        const int* __restrict__ order, const int* __restrict__ pos, int* __restrict__ claim,
                        const State* __restrict__ st) {
  const int64_t ls = st->ls, le = st->le;
  const int lane = threadIdx.x & 31;
  for (int64_t q = ls + (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5); q < le;
       q += (int64_t)gridDim.x * kWarps) {
    int i = order[q];
    for (int64_t e = rowptr[i] + lane; e < rowptr[i + 1]; e += 32) {
      int j = cols[e];
      if (pos[j] < 0) atomicMin(&claim[j], static_cast<int>(q));
    }
  }
}

__global__ void k_count(const int64_t* __restrict__ rowptr, const int* __restrict__ cols,
                        const int* __restrict__ order, const int* __restrict__ claim, int* __restrict__ cnt,
                        const State* __restrict__ st) {
  const int64_t ls = st->ls, le = st->le;
  const int lane = threadIdx.x & 31;
  for (int64_t q = ls + (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5); q < le;
       q += (int64_t)gridDim.x * kWarps) {
    int i = order[q];
    int c = 0;
    for (int64_t e = rowptr[i] + lane; e < rowptr[i + 1]; e += 32) c += claim[cols[e]] == static_cast<int>(q);
    c = warp_sum(c);
    if (lane == 0) cnt[q - ls] = c;
  }
}

// Writes the children of q, ordered by (degree asc, index desc), after the level.
__global__ void __launch_bounds__(kWarps * 32)
k_write(const int64_t* __restrict__ rowptr, const int* __restrict__ cols, const int* __restrict__ degree,
        int* __restrict__ order, int* __restrict__ pos, const int* __restrict__ claim,
        const int* __restrict__ off, const State* __restrict__ st, int64_t n_atoms, int* __restrict__ flag) {
  __shared__ int buf[kWarps][kCap];
  const int64_t ls = st->ls, le = st->le;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int* s = buf[w];
  for (int64_t q = ls + (int64_t)blockIdx.x * kWarps + w; q < le; q += (int64_t)gridDim.x * kWarps) {
    int i = order[q];
    int m = 0;
    for (int64_t e0 = rowptr[i]; e0 < rowptr[i + 1]; e0 += 32) {
      int64_t e = e0 + lane;
      bool ok = false;
      int j = 0;
      if (e < rowptr[i + 1]) {
        j = cols[e];
        ok = claim[j] == static_cast<int>(q);
      }
      unsigned b = __ballot_sync(0xffffffffu, ok);
      if (ok) s[m + __popc(b & ((1u << lane) - 1u))] = j;   // m + rank < degree(i) <= kCap
      m += __popc(b);
    }
    __syncwarp();
    const int64_t base = le + off[q - ls];
    for (int t = lane; t < m; t += 32) {
      int jt = s[t];
      int dt = degree[jt];
      int rank = 0;
      for (int u = 0; u < m; ++u) {
        int ju = s[u];
        int du = degree[ju];
        rank += (du < dt) || (du == dt && ju > jt);
      }
      if (base + rank < n_atoms) {
        order[base + rank] = jt;
        pos[jt] = static_cast<int>(base + rank);
      } else {
        atomicExch(flag, 4);
      }
    }
    __syncwarp();
  }
}

// Closes the level and, when the frontier is empty, seeds the next component.
__global__ void k_advance(int* __restrict__ order, int* __restrict__ pos, const int* __restrict__ off,
                          const int64_t* __restrict__ seed_order, int64_t n_atoms, State* st) {
  int64_t L = st->le - st->ls;
  int64_t added = L > 0 ? off[L] : 0;
  int64_t n = st->n + added;
  st->ls = st->le;
  st->le = n;
  st->n = n;
  if (st->ls == st->le && n < n_atoms) {
    int64_t p = st->seedptr;
    while (p < n_atoms && pos[seed_order[p]] >= 0) ++p;
    if (p < n_atoms) {
      int s = static_cast<int>(seed_order[p]);
      order[n] = s;
      pos[s] = static_cast<int>(n);
      st->ls = n;
      st->le = n + 1;
      st->n = n + 1;
      st->seedptr = p + 1;
    }
  }
}

__global__ void k_finish(const int* __restrict__ order, int64_t n, int64_t* __restrict__ rcm,
                         int64_t* __restrict__ undo) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t a = order[n - 1 - i];
    rcm[i] = a;
    undo[a] = i;
  }
}

__global__ void k_check_seeds(const int64_t* __restrict__ seed_order, int64_t n, int* __restrict__ seen,
                              int* __restrict__ bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t s = seed_order[i];
    if (s < 0 || s >= n || atomicAdd(&seen[s], 1) != 0) atomicExch(bad, 1);
  }
}

__global__ void k_check_degree(const int64_t* __restrict__ rowptr, const int* __restrict__ cols,
                               const int* __restrict__ degree, int64_t n, int* __restrict__ bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t d = rowptr[i + 1] - rowptr[i];
    if (d < 0 || d > kCap) atomicExch(bad, 2);
    for (int64_t e = rowptr[i]; e < rowptr[i + 1] && d >= 0 && d <= kCap; ++e)
      if (cols[e] < 0 || cols[e] >= n) atomicExch(bad, 3);
  }
}

struct RcmWs {
  int *pos, *claim, *order, *cnt, *off, *flag;
  State* st;
  void* cub_tmp;
  size_t cub_bytes;
};

template <class C>
void carve_rcm(C& c, int64_t n, RcmWs* w) {
  size_t cb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cb, (int*)nullptr, (int*)nullptr, (int)(n + 1));
  if constexpr (std::is_same<C, Carver>::value) {
    w->pos = c.template take<int>(n);
    w->claim = c.template take<int>(n);
    w->order = c.template take<int>(n);
    w->cnt = c.template take<int>(n + 1);
    w->off = c.template take<int>(n + 1);
    w->flag = c.template take<int>(4);
    w->st = c.template take<State>(1);
    w->cub_tmp = c.template take<char>(cb);
    w->cub_bytes = cb;
  } else {
    for (int k = 0; k < 3; ++k) c.template take<int>(n);
    c.template take<int>(n + 1);
    c.template take<int>(n + 1);
    c.template take<int>(4);
    c.template take<State>(1);
    c.template take<char>(cb);
  }
}

}  // namespace
}  // namespace inch

using namespace inch;

extern "C" size_t inch_rcm_workspace_size(int64_t n) {
  if (n < 1) return 0;
  Sizer s;
  RcmWs w;
  carve_rcm(s, n, &w);
  return s.bytes();
}

extern "C" inch_status inch_rcm(const int64_t* rowptr, const int32_t* cols, const int32_t* degree,
                                const int64_t* seed_order, int64_t n, int64_t* rcm_order, int64_t* undo,
                                int32_t* n_levels_host, void* ws, size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(rowptr && cols && degree && seed_order && rcm_order && undo, INCH_INVALID_ARG,
               "inch_rcm: NULL argument");
  INCH_REQUIRE(n >= 1 && n < (int64_t(1) << 31), INCH_INVALID_ARG, "inch_rcm: n_atoms out of range");
  Carver c(ws, ws_bytes);
  RcmWs w;
  carve_rcm(c, n, &w);
  INCH_REQUIRE(c.ok, INCH_OOM, "inch_rcm: workspace of %zu bytes, need %zu", ws_bytes, inch_rcm_workspace_size(n));
  const int bl = grid_for(n, 256, 148 * 16);
  // Validate the inputs that index memory: seed_order must be a permutation,
  // rows at most kCap long with in-range columns.
  INCH_CUDA(cudaMemsetAsync(w.flag, 0, sizeof(int) * 4, stream));
  INCH_CUDA(cudaMemsetAsync(w.pos, 0, sizeof(int) * n, stream));
  k_check_seeds<<<bl, 256, 0, stream>>>(seed_order, n, w.pos, w.flag);
  INCH_LAUNCH_CHECK();
  k_check_degree<<<bl, 256, 0, stream>>>(rowptr, cols, degree, n, w.flag);
  INCH_LAUNCH_CHECK();
  int bad = 0;
  INCH_CUDA(cudaMemcpyAsync(&bad, w.flag, sizeof(int), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cudaStreamSynchronize(stream));
  INCH_REQUIRE(bad != 1, INCH_INVALID_ARG, "inch_rcm: seed_order is not a permutation of 0..n-1");
  INCH_REQUIRE(bad != 2, INCH_LIMIT, "inch_rcm: a row has more than %d neighbours", kCap);
  INCH_REQUIRE(bad == 0, INCH_INVALID_ARG, "inch_rcm: column index out of range");

  k_init<<<bl, 256, 0, stream>>>(w.pos, w.claim, n, w.st);
  INCH_LAUNCH_CHECK();
  k_advance<<<1, 1, 0, stream>>>(w.order, w.pos, w.off, seed_order, n, w.st);
  INCH_LAUNCH_CHECK();
  State h{};
  INCH_CUDA(cudaMemcpyAsync(&h, w.st, sizeof(State), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cudaStreamSynchronize(stream));
  int levels = 0;
  while (h.ls < h.le) {
    const int64_t L = h.le - h.ls;
    const int gw = grid_for(L, kWarps, 148 * 8);
    k_claim<<<gw, kWarps * 32, 0, stream>>>(rowptr, cols, w.order, w.pos, w.claim, w.st);
    INCH_LAUNCH_CHECK();
    k_count<<<gw, kWarps * 32, 0, stream>>>(rowptr, cols, w.order, w.claim, w.cnt, w.st);
    INCH_LAUNCH_CHECK();
    INCH_CUDA(cudaMemsetAsync(w.cnt + L, 0, sizeof(int), stream));
    size_t cb = w.cub_bytes;
    INCH_CUDA(cub::DeviceScan::ExclusiveSum(w.cub_tmp, cb, w.cnt, w.off, (int)(L + 1), stream));
    k_write<<<gw, kWarps * 32, 0, stream>>>(rowptr, cols, degree, w.order, w.pos, w.claim, w.off, w.st, n,
                                           w.flag);
    INCH_LAUNCH_CHECK();
    k_advance<<<1, 1, 0, stream>>>(w.order, w.pos, w.off, seed_order, n, w.st);
    INCH_LAUNCH_CHECK();
    INCH_CUDA(cudaMemcpyAsync(&h, w.st, sizeof(State), cudaMemcpyDeviceToHost, stream));
    INCH_CUDA(cudaStreamSynchronize(stream));
    ++levels;
    INCH_CUDA(cudaMemcpyAsync(&bad, w.flag, sizeof(int), cudaMemcpyDeviceToHost, stream));
    INCH_CUDA(cudaStreamSynchronize(stream));
    INCH_REQUIRE(bad == 0, INCH_INVALID_ARG, "inch_rcm: adjacency lists contain duplicates");
    INCH_REQUIRE(h.n <= n && levels <= n + 1, INCH_INVALID_ARG, "inch_rcm: inconsistent adjacency (not symmetric?)");
  }
  INCH_REQUIRE(h.n == n, INCH_INVALID_ARG, "inch_rcm: visited %lld of %lld atoms", (long long)h.n, (long long)n);
  k_finish<<<bl, 256, 0, stream>>>(w.order, n, rcm_order, undo);
  INCH_LAUNCH_CHECK();
  if (n_levels_host) *n_levels_host = levels;
  return INCH_OK;
}
