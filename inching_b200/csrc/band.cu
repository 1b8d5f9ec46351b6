// Ungapped band slices per row batch.
//
// Reference: X_KdUngappedMinMaxNeighbor (InchingLiteInteger/Fuel/Coordinate/T1.py:
// 371-481) takes, for every row batch, the sorted set of distinct neighbour columns
// and splits it wherever two consecutive distinct columns are more than GapSize
// apart, except for the first five gaps, the gap at position len(unique)-5 and gaps
// that touch the diagonal band.
//
// Here: one segmented sort of each batch's adjacency entries (CUB), then one block
// per batch that ranks the distinct columns with a block scan, collects the
// candidate gaps (position, left, right) and lets one thread apply the reference's
// sequential acceptance rules (they depend on the previously accepted gap).
#include <cub/cub.cuh>

#include "common.cuh"

namespace inch {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxCand = 2048;

__global__ void k_offsets(const int64_t* __restrict__ rowptr, const int64_t* __restrict__ head, int64_t nb,
                          int64_t n_atoms, int64_t* __restrict__ beg, int64_t* __restrict__ end,
                          int* __restrict__ bad) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nb; b += (int64_t)gridDim.x * blockDim.x) {
    const int64_t h0 = head[b], h1 = head[b + 1];
    if (h0 < 0 || h1 > n_atoms || h1 <= h0) {
      atomicExch(bad, 1);
      beg[b] = end[b] = 0;
      continue;
    }
    beg[b] = rowptr[h0];
    end[b] = rowptr[h1];
    if (end[b] <= beg[b]) atomicExch(bad, 1);
  }
}

__global__ void __launch_bounds__(kThreads)
k_slices(const int* __restrict__ s, const int64_t* __restrict__ beg_a, const int64_t* __restrict__ end_a,
         const int64_t* __restrict__ head, int64_t gap, int max_slices, int64_t* __restrict__ starts,
         int64_t* __restrict__ ends, int* __restrict__ counts, int* __restrict__ err) {
  using Scan = cub::BlockScan<int, kThreads>;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ int c_iii[kMaxCand];
  __shared__ int c_l[kMaxCand], c_r[kMaxCand];
  __shared__ int n_cand;
  __shared__ int overflow;
  const int64_t b = blockIdx.x;
  const int64_t beg = beg_a[b], end = end_a[b];
  if (threadIdx.x == 0) {
    n_cand = 0;
    overflow = 0;
  }
  __syncthreads();
  int U = 0;  // distinct columns seen so far
  for (int64_t k0 = beg; k0 < end; k0 += kThreads) {
    const int64_t k = k0 + threadIdx.x;
    int flag = 0;
    if (k < end) flag = (k == beg) || (s[k] != s[k - 1]);
    int rank, total;
    Scan(tmp).ExclusiveSum(flag, rank, total);
    if (flag && k > beg && (int64_t)s[k] - (int64_t)s[k - 1] > gap) {
      int slot = atomicAdd(&n_cand, 1);
      if (slot < kMaxCand) {
        c_iii[slot] = U + rank - 1;
        c_l[slot] = s[k - 1];
        c_r[slot] = s[k];
      } else {
        overflow = 1;
      }
    }
    U += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int nc = n_cand < kMaxCand ? n_cand : kMaxCand;
    // candidates arrive out of order: insertion sort by position
    for (int a = 1; a < nc; ++a) {
      int ki = c_iii[a], kl = c_l[a], kr = c_r[a];
      int p = a;
      while (p > 0 && c_iii[p - 1] > ki) {
        c_iii[p] = c_iii[p - 1];
        c_l[p] = c_l[p - 1];
        c_r[p] = c_r[p - 1];
        --p;
      }
      c_iii[p] = ki;
      c_l[p] = kl;
      c_r[p] = kr;
    }
    const int64_t start = head[b], height = head[b + 1] - head[b];
    int64_t last = s[beg];  // bounds[-1]
    int ns = 0;
    int64_t* st = starts + b * (int64_t)max_slices;
    int64_t* en = ends + b * (int64_t)max_slices;
    int64_t cur = s[beg];
    bool ok = !overflow;
    for (int a = 0; a < nc && ok; ++a) {
      const int iii = c_iii[a];
      if (iii == U - 5) continue;
      if (iii < 5) continue;
      if ((last + 5 >= start) && ((int64_t)c_l[a] + 1 <= start + height + 5)) continue;
      if (ns + 1 >= max_slices) {
        ok = false;
        break;
      }
      st[ns] = cur;
      en[ns] = (int64_t)c_l[a] + 1;
      ++ns;
      cur = c_r[a];
      last = c_r[a];
    }
    if (ok) {
      st[ns] = cur;
      en[ns] = (int64_t)s[end - 1] + 1;
      ++ns;
      counts[b] = ns;
    } else {
      counts[b] = -1;
      atomicExch(err, 1);
    }
  }
}

struct BandWs {
  int* sorted;
  int64_t *beg, *end;
  int* err;
  void* cub_tmp;
  size_t cub_bytes;
};

}  // namespace
}  // namespace inch

using namespace inch;

extern "C" size_t inch_band_slices_workspace_size(int64_t n_batches, int64_t nnz) {
  size_t cb = 0;
  cub::DeviceSegmentedSort::SortKeys(nullptr, cb, (const int*)nullptr, (int*)nullptr, (int)nnz, (int)n_batches,
                                     (const int64_t*)nullptr, (const int64_t*)nullptr);
  Sizer s;
  s.take<int>(nnz);
  s.take<int64_t>(n_batches);
  s.take<int64_t>(n_batches);
  s.take<int>(4);
  s.take<char>(cb);
  return s.bytes();
}

extern "C" inch_status inch_band_slices(const int64_t* rowptr, const int32_t* cols, int64_t n_atoms,
                                        const int64_t* head, int64_t nb, int64_t gap, int32_t max_slices,
                                        int64_t* starts, int64_t* ends, int32_t* counts, int64_t* total_host,
                                        void* ws, size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(rowptr && cols && head && starts && ends && counts && total_host, INCH_INVALID_ARG,
               "inch_band_slices: NULL argument");
  INCH_REQUIRE(nb >= 1 && nb < (int64_t(1) << 31) && max_slices >= 1 && n_atoms >= 1, INCH_INVALID_ARG,
               "inch_band_slices: bad batch count, atom count or max_slices");
  int64_t nnz = 0;
  INCH_CUDA(cudaMemcpyAsync(&nnz, rowptr + n_atoms, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cudaStreamSynchronize(stream));
  INCH_REQUIRE(nnz >= n_atoms && nnz < (int64_t(1) << 31), INCH_LIMIT,
               "inch_band_slices: adjacency size %lld outside [n_atoms, 2^31)", (long long)nnz);
  const size_t need = inch_band_slices_workspace_size(nb, nnz);
  Carver c(ws, ws_bytes);
  BandWs w;
  w.sorted = c.take<int>(nnz);
  w.beg = c.take<int64_t>(nb);
  w.end = c.take<int64_t>(nb);
  w.err = c.take<int>(4);
  size_t cb = 0;
  cub::DeviceSegmentedSort::SortKeys(nullptr, cb, (const int*)nullptr, (int*)nullptr, (int)nnz, (int)nb,
                                     (const int64_t*)nullptr, (const int64_t*)nullptr);
  w.cub_tmp = c.take<char>(cb);
  INCH_REQUIRE(c.ok, INCH_OOM, "inch_band_slices: workspace of %zu bytes, need %zu", ws_bytes, need);
  INCH_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int) * 4, stream));
  k_offsets<<<grid_for(nb, 256), 256, 0, stream>>>(rowptr, head, nb, n_atoms, w.beg, w.end, w.err);
  INCH_LAUNCH_CHECK();
  int herr[2] = {0, 0};
  int64_t span[2] = {0, 0};
  INCH_CUDA(cudaMemcpyAsync(herr, w.err, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cudaStreamSynchronize(stream));
  INCH_REQUIRE(herr[0] == 0, INCH_INVALID_ARG, "inch_band_slices: batch heads must increase within [0, n_atoms]");
  INCH_CUDA(cudaMemcpyAsync(&span[0], w.beg, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cudaMemcpyAsync(&span[1], w.end + nb - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cub::DeviceSegmentedSort::SortKeys(w.cub_tmp, cb, cols, w.sorted, (int)nnz, (int)nb, w.beg, w.end,
                                               stream));
  k_slices<<<(unsigned)nb, kThreads, 0, stream>>>(w.sorted, w.beg, w.end, head, gap, max_slices, starts, ends,
                                                   counts, w.err + 1);
  INCH_LAUNCH_CHECK();
  INCH_CUDA(cudaMemcpyAsync(herr, w.err, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cudaStreamSynchronize(stream));
  INCH_REQUIRE(herr[1] == 0, INCH_LIMIT, "inch_band_slices: a batch has more than %d slices or %d gap candidates",
               max_slices, kMaxCand);
  *total_host = span[1] - span[0];
  return INCH_OK;
}
