// Cell-list cutoff neighbour search.
//
// Replaces the k-d-tree queries of the reference (scipy cKDTree.query_ball_point
// in InchingLiteInteger/Fuel/Coordinate/T1.py:218-245 and :276) with a uniform
// grid: cells of edge rc*(1+1e-6) so that every neighbour of an atom lies in the
// 3x3x3 block of cells around it, atoms counting-sorted by cell, and one pass
// that tests every candidate with the exact distance rule of cKDTree
// (((dx*dx) + dy*dy) + dz*dz <= rc*rc, every operation rounded, no FMA).
//
// Pass 1 (count): one thread per cell-sorted atom, writes degree[] (self included).
// Pass 2 (fill):  one warp per atom, ballot-compacts the accepted candidates into
//                 shared memory, bitonic-sorts them, writes the row of cols[].
#include <cub/cub.cuh>
#include <cstdarg>
#include <cmath>

#include "common.cuh"

namespace inch {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}

const char* last_error() { return g_err.c_str(); }

namespace {

constexpr int kFillWarps = 8;            // warps per block in the fill kernel
constexpr int kCap = INCH_MAX_DEGREE;    // per-warp candidate buffer

struct GridDev {
  double ox, oy, oz, inv_cell;
  int dx, dy, dz;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Cell of a point, clamped to the grid (in double, before the integer cast, so
// periodic-image queries far outside the grid stay defined).  A clamped cell's
// 3x3x3 neighbourhood still contains every atom within rc of the point.
__device__ __forceinline__ int cell_axis(double v, double o, double inv, int d) {
  const double f = fmin(fmax(floor((v - o) * inv), 0.0), static_cast<double>(d - 1));
  return clampi(static_cast<int>(f), 0, d - 1);
}

__device__ __forceinline__ void cell_of(const GridDev& g, double x, double y, double z, int& cx, int& cy,
                                        int& cz) {
  cx = cell_axis(x, g.ox, g.inv_cell, g.dx);
  cy = cell_axis(y, g.oy, g.inv_cell, g.dy);
  cz = cell_axis(z, g.oz, g.inv_cell, g.dz);
}

// Periodic images in x and y, in the reference's instruction order
// (Fuel/Coordinate/T1.py:98-107): centre, +x, -x, +y, -y, +x+y, +x-y, -x+y, -x-y.
__device__ __forceinline__ void image_shift(int k, double bx, double by, double& sx, double& sy) {
  const int ix = (k == 1 || k == 5 || k == 6) ? 1 : ((k == 2 || k == 7 || k == 8) ? -1 : 0);
  const int iy = (k == 3 || k == 5 || k == 7) ? 1 : ((k == 4 || k == 6 || k == 8) ? -1 : 0);
  sx = ix == 0 ? 0.0 : (ix > 0 ? bx : -bx);
  sy = iy == 0 ? 0.0 : (iy > 0 ? by : -by);
}

constexpr int kImageShift = 27;                       // sort key = image << 27 | column (PBC rows)
constexpr int kColMask = (1 << kImageShift) - 1;

// Squared distance in cKDTree's operation order, no contraction.
__device__ __forceinline__ double sqdist(double ax, double ay, double az, double bx, double by, double bz) {
  double dx = __dsub_rn(bx, ax), dy = __dsub_rn(by, ay), dz = __dsub_rn(bz, az);
  double s = __dmul_rn(dx, dx);
  s = __dadd_rn(s, __dmul_rn(dy, dy));
  s = __dadd_rn(s, __dmul_rn(dz, dz));
  return s;
}

__global__ void k_bbox(const double* __restrict__ X, int64_t n, double* __restrict__ out) {
  __shared__ double smin[3][256], smax[3][256];
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  int nonfinite = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    for (int a = 0; a < 3; ++a) {
      double v = X[3 * i + a];
      if (!isfinite(v)) nonfinite = 1;
      mn[a] = fmin(mn[a], v);
      mx[a] = fmax(mx[a], v);
    }
  }
  nonfinite = __syncthreads_or(nonfinite);
  for (int a = 0; a < 3; ++a) {
    smin[a][threadIdx.x] = mn[a];
    smax[a][threadIdx.x] = mx[a];
  }
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int a = 0; a < 3; ++a) {
        smin[a][threadIdx.x] = fmin(smin[a][threadIdx.x], smin[a][threadIdx.x + s]);
        smax[a][threadIdx.x] = fmax(smax[a][threadIdx.x], smax[a][threadIdx.x + s]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int a = 0; a < 3; ++a) {
      out[a] = smin[a][0];
      out[3 + a] = smax[a][0];
    }
    out[6] = nonfinite ? 1.0 : 0.0;
  }
}

__global__ void k_assign(const double* __restrict__ X, int64_t n, GridDev g, int* __restrict__ cell_cnt,
                         int* __restrict__ cell_id, int* __restrict__ slot) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int cx, cy, cz;
    cell_of(g, X[3 * i], X[3 * i + 1], X[3 * i + 2], cx, cy, cz);
    int c = (cx * g.dy + cy) * g.dz + cz;
    cell_id[i] = c;
    slot[i] = atomicAdd(&cell_cnt[c], 1);
  }
}

__global__ void k_scatter(const double* __restrict__ X, int64_t n, const int* __restrict__ cell_start,
                          const int* __restrict__ cell_id, const int* __restrict__ slot,
                          double4* __restrict__ sorted) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int p = cell_start[cell_id[i]] + slot[i];
    sorted[p] = make_double4(X[3 * i], X[3 * i + 1], X[3 * i + 2], static_cast<double>(i));
  }
}

// Candidate z-runs: for fixed (ax, ay) the cells cz-1..cz+1 are contiguous in
// the cell order, hence contiguous in the sorted atom array.
__device__ __forceinline__ bool zrun(const GridDev& g, const int* __restrict__ cell_start, int cx, int cy,
                                     int cz, int r, int& beg, int& end) {
  int ax = cx + (r / 3) - 1, ay = cy + (r % 3) - 1;
  if (ax < 0 || ax >= g.dx || ay < 0 || ay >= g.dy) return false;
  int z0 = cz > 0 ? cz - 1 : 0;
  int z1 = cz < g.dz - 1 ? cz + 1 : g.dz - 1;
  int base = (ax * g.dy + ay) * g.dz;
  beg = cell_start[base + z0];
  end = cell_start[base + z1 + 1];
  return true;
}

// NIMG = 1: plain cutoff graph; NIMG = 9: the query point is also shifted by
// each periodic xy image (x_i + s, rounded once, as numpy's xx + box * instr).
template <int NIMG>
__global__ void k_count(const double4* __restrict__ sorted, int64_t n, GridDev g,
                        const int* __restrict__ cell_start, double r2, double bx, double by,
                        int* __restrict__ degree, int64_t* __restrict__ deg64) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    double4 a = sorted[t];
    int cnt = 0;
    for (int k = 0; k < NIMG; ++k) {
      double sx = 0.0, sy = 0.0;
      if (NIMG > 1) image_shift(k, bx, by, sx, sy);
      const double qx = NIMG > 1 ? __dadd_rn(a.x, sx) : a.x, qy = NIMG > 1 ? __dadd_rn(a.y, sy) : a.y;
      int cx, cy, cz;
      cell_of(g, qx, qy, a.z, cx, cy, cz);
      for (int r = 0; r < 9; ++r) {
        int beg, end;
        if (!zrun(g, cell_start, cx, cy, cz, r, beg, end)) continue;
        for (int p = beg; p < end; ++p) {
          double4 b = sorted[p];
          cnt += sqdist(qx, qy, a.z, b.x, b.y, b.z) <= r2;
        }
      }
    }
    int64_t i = static_cast<int64_t>(a.w);
    degree[i] = cnt;
    deg64[i] = cnt;
  }
}

template <int NIMG>
__global__ void __launch_bounds__(kFillWarps * 32)
k_fill(const double4* __restrict__ sorted, int64_t n, GridDev g, const int* __restrict__ cell_start,
       double r2, double bx, double by, const int64_t* __restrict__ rowptr, int* __restrict__ cols,
       int8_t* __restrict__ image, int* __restrict__ err) {
  __shared__ int buf[kFillWarps][kCap];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* s = buf[w];
  for (int64_t t = (int64_t)blockIdx.x * kFillWarps + w; t < n; t += (int64_t)gridDim.x * kFillWarps) {
    double4 a = sorted[t];
    int cnt = 0;
    bool over = false;
    for (int k = 0; k < NIMG; ++k) {
      double sx = 0.0, sy = 0.0;
      if (NIMG > 1) image_shift(k, bx, by, sx, sy);
      const double qx = NIMG > 1 ? __dadd_rn(a.x, sx) : a.x, qy = NIMG > 1 ? __dadd_rn(a.y, sy) : a.y;
      int cx, cy, cz;
      cell_of(g, qx, qy, a.z, cx, cy, cz);
      for (int r = 0; r < 9; ++r) {
        int beg, end;
        if (!zrun(g, cell_start, cx, cy, cz, r, beg, end)) continue;
        for (int p0 = beg; p0 < end; p0 += 32) {
          int p = p0 + lane;
          bool ok = false;
          int j = 0;
          if (p < end) {
            double4 b = sorted[p];
            ok = sqdist(qx, qy, a.z, b.x, b.y, b.z) <= r2;
            j = static_cast<int>(b.w);
            if (NIMG > 1) j |= k << kImageShift;   // rows list image 0 first, then 1, ... (each sorted)
          }
          unsigned m = __ballot_sync(0xffffffffu, ok);
          int pos = cnt + __popc(m & ((1u << lane) - 1u));
          if (ok) {
            if (pos < kCap) s[pos] = j;
            else over = true;
          }
          cnt += __popc(m);
        }
      }
    }
    over = __any_sync(0xffffffffu, over);
    int64_t i = static_cast<int64_t>(a.w);
    int64_t row = rowptr[i];
    int expect = static_cast<int>(rowptr[i + 1] - row);
    if (over || cnt != expect) {
      if (lane == 0) atomicExch(err, over ? 1 : 2);
      continue;
    }
    int P = 1;
    while (P < cnt) P <<= 1;
    for (int q = cnt + lane; q < P; q += 32) s[q] = 0x7fffffff;
    __syncwarp();
    for (int k = 2; k <= P; k <<= 1) {
      for (int jj = k >> 1; jj > 0; jj >>= 1) {
        for (int q = lane; q < P; q += 32) {
          int o = q ^ jj;
          if (o > q) {
            int x = s[q], y = s[o];
            bool up = (q & k) == 0;
            if ((x > y) == up) {
              s[q] = y;
              s[o] = x;
            }
          }
        }
        __syncwarp();
      }
    }
    for (int q = lane; q < cnt; q += 32) {
      if (NIMG > 1) {
        cols[row + q] = s[q] & kColMask;
        image[row + q] = static_cast<int8_t>(s[q] >> kImageShift);
      } else {
        cols[row + q] = s[q];
      }
    }
    __syncwarp();
  }
}

__global__ void k_set0(int64_t* p) { p[0] = 0; }

struct NbrWs {
  int* cell_cnt;     // ncells + 1
  int* cell_start;   // ncells + 1
  int* cell_id;      // n
  int* slot;         // n
  double4* sorted;   // n
  int64_t* deg64;    // n
  int* err;          // 1
  void* cub_tmp;
  size_t cub_bytes;
};

size_t cub_bytes_for(int64_t ncells, int64_t n) {
  size_t a = 0, b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, a, (int*)nullptr, (int*)nullptr, (int)(ncells + 1));
  cub::DeviceScan::InclusiveSum(nullptr, b, (int64_t*)nullptr, (int64_t*)nullptr, (int)n);
  return a > b ? a : b;
}

template <class C>
void carve_nbr(C& c, const inch_cell_grid& g, NbrWs* w) {
  int64_t n = g.n_atoms, nc = g.ncells;
  size_t cb = cub_bytes_for(nc, n > 0 ? n : 1);
  if constexpr (std::is_same<C, Carver>::value) {
    w->cell_cnt = c.template take<int>(nc + 1);
    w->cell_start = c.template take<int>(nc + 1);
    w->cell_id = c.template take<int>(n);
    w->slot = c.template take<int>(n);
    w->sorted = c.template take<double4>(n);
    w->deg64 = c.template take<int64_t>(n);
    w->err = c.template take<int>(4);
    w->cub_tmp = c.template take<char>(cb);
    w->cub_bytes = cb;
  } else {
    c.template take<int>(nc + 1);
    c.template take<int>(nc + 1);
    c.template take<int>(n);
    c.template take<int>(n);
    c.template take<double4>(n);
    c.template take<int64_t>(n);
    c.template take<int>(4);
    c.template take<char>(cb);
  }
}

GridDev to_dev(const inch_cell_grid& g) {
  GridDev d;
  d.ox = g.origin[0];
  d.oy = g.origin[1];
  d.oz = g.origin[2];
  d.inv_cell = 1.0 / g.cell;
  d.dx = g.dims[0];
  d.dy = g.dims[1];
  d.dz = g.dims[2];
  return d;
}

}  // namespace
}  // namespace inch

using namespace inch;

extern "C" const char* inch_last_error_string(void) { return inch::last_error(); }
extern "C" int inch_abi_version(void) { return 1; }

extern "C" inch_status inch_cell_grid_plan(const double* X, int64_t n, double rc, inch_cell_grid* grid,
                                           void* ws, size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(grid != nullptr, INCH_INVALID_ARG, "inch_cell_grid_plan: grid is NULL");
  INCH_REQUIRE(n >= 1 && n < (int64_t(1) << 31), INCH_INVALID_ARG, "inch_cell_grid_plan: n_atoms=%lld out of range",
               (long long)n);
  INCH_REQUIRE(X != nullptr, INCH_INVALID_ARG, "inch_cell_grid_plan: X is NULL");
  INCH_REQUIRE(rc > 0 && std::isfinite(rc), INCH_INVALID_ARG, "inch_cell_grid_plan: rc must be > 0");
  INCH_REQUIRE(ws != nullptr && ws_bytes >= 64, INCH_OOM, "inch_cell_grid_plan: needs 64 bytes of workspace");
  double* d = static_cast<double*>(ws);
  k_bbox<<<1, 256, 0, stream>>>(X, n, d);
  INCH_LAUNCH_CHECK();
  double h[8];
  INCH_CUDA(cudaMemcpyAsync(h, d, 7 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cudaStreamSynchronize(stream));
  INCH_REQUIRE(h[6] == 0.0, INCH_INVALID_ARG, "ABORTED. coordinates contain NaN or Inf");
  // Cell edge slightly above rc so that floor() rounding can never separate two
  // atoms within rc by more than one cell.  Grow it if the grid gets too large.
  double cell = rc * (1.0 + 1e-6);
  for (;;) {
    int64_t nc = 1;
    for (int a = 0; a < 3; ++a) {
      int64_t da = static_cast<int64_t>(std::floor((h[3 + a] - h[a]) / cell)) + 1;
      grid->dims[a] = static_cast<int32_t>(da < 1 ? 1 : da);
      nc *= grid->dims[a];
    }
    if (nc <= (int64_t(1) << 26) || nc <= 4 * n) {
      grid->ncells = nc;
      break;
    }
    cell *= 1.25;
  }
  for (int a = 0; a < 3; ++a) grid->origin[a] = h[a];
  grid->cell = cell;
  grid->n_atoms = n;
  return INCH_OK;
}

extern "C" size_t inch_neighbors_workspace_size(const inch_cell_grid* g) {
  if (g == nullptr) return 0;
  Sizer s;
  NbrWs w;
  carve_nbr(s, *g, &w);
  return s.bytes();
}

namespace {
template <int NIMG>
inch_status neighbors_count_impl(const char* who, const double* X, const inch_cell_grid* grid, double rc, double bx,
                                 double by, int32_t* degree, int64_t* rowptr, int64_t* nnz_host, void* ws,
                                 size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(X && grid && degree && rowptr && nnz_host, INCH_INVALID_ARG, "%s: NULL argument", who);
  INCH_REQUIRE(rc > 0 && grid->cell >= rc, INCH_INVALID_ARG, "%s: cell edge below rc", who);
  const int64_t n = grid->n_atoms;
  Carver c(ws, ws_bytes);
  NbrWs w;
  carve_nbr(c, *grid, &w);
  INCH_REQUIRE(c.ok, INCH_OOM, "%s: workspace of %zu bytes, need %zu", who, ws_bytes,
               inch_neighbors_workspace_size(grid));
  GridDev g = to_dev(*grid);
  INCH_CUDA(cudaMemsetAsync(w.cell_cnt, 0, sizeof(int) * (grid->ncells + 1), stream));
  INCH_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int) * 4, stream));
  int blocks = grid_for(n, 256, 148 * 16);
  k_assign<<<blocks, 256, 0, stream>>>(X, n, g, w.cell_cnt, w.cell_id, w.slot);
  INCH_LAUNCH_CHECK();
  size_t cb = w.cub_bytes;
  INCH_CUDA(cub::DeviceScan::ExclusiveSum(w.cub_tmp, cb, w.cell_cnt, w.cell_start, (int)(grid->ncells + 1), stream));
  k_scatter<<<blocks, 256, 0, stream>>>(X, n, w.cell_start, w.cell_id, w.slot, w.sorted);
  INCH_LAUNCH_CHECK();
  k_count<NIMG><<<blocks, 256, 0, stream>>>(w.sorted, n, g, w.cell_start, rc * rc, bx, by, degree, w.deg64);
  INCH_LAUNCH_CHECK();
  k_set0<<<1, 1, 0, stream>>>(rowptr);
  INCH_LAUNCH_CHECK();
  cb = w.cub_bytes;
  INCH_CUDA(cub::DeviceScan::InclusiveSum(w.cub_tmp, cb, w.deg64, rowptr + 1, (int)n, stream));
  INCH_CUDA(cudaMemcpyAsync(nnz_host, rowptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cudaStreamSynchronize(stream));
  return INCH_OK;
}

template <int NIMG>
inch_status neighbors_fill_impl(const char* who, const double* X, const inch_cell_grid* grid, double rc, double bx,
                                double by, const int64_t* rowptr, int32_t* cols, int8_t* image, void* ws,
                                size_t ws_bytes, cudaStream_t stream) {
  INCH_REQUIRE(X && grid && rowptr && cols && (NIMG == 1 || image), INCH_INVALID_ARG, "%s: NULL argument", who);
  const int64_t n = grid->n_atoms;
  Carver c(ws, ws_bytes);
  NbrWs w;
  carve_nbr(c, *grid, &w);
  INCH_REQUIRE(c.ok, INCH_OOM, "%s: workspace too small", who);
  GridDev g = to_dev(*grid);
  INCH_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int) * 4, stream));
  int blocks = grid_for(n, kFillWarps, 148 * 8);
  k_fill<NIMG><<<blocks, kFillWarps * 32, 0, stream>>>(w.sorted, n, g, w.cell_start, rc * rc, bx, by, rowptr, cols,
                                                       image, w.err);
  INCH_LAUNCH_CHECK();
  int herr = 0;
  INCH_CUDA(cudaMemcpyAsync(&herr, w.err, sizeof(int), cudaMemcpyDeviceToHost, stream));
  INCH_CUDA(cudaStreamSynchronize(stream));
  INCH_REQUIRE(herr != 1, INCH_LIMIT, "%s: an atom has more than %d neighbours within the cutoff", who, kCap);
  INCH_REQUIRE(herr == 0, INCH_INVALID_ARG, "%s: neighbour counts differ from the count pass (different X or rc?)",
               who);
  return INCH_OK;
}

inch_status check_box(const char* who, const inch_cell_grid* grid, double rc, double bx, double by) {
  INCH_REQUIRE(grid != nullptr, INCH_INVALID_ARG, "%s: grid is NULL", who);
  INCH_REQUIRE(std::isfinite(bx) && std::isfinite(by), INCH_INVALID_ARG, "%s: box sizes must be finite", who);
  INCH_REQUIRE(bx > rc, INCH_INVALID_ARG, "ABORTED. The PBC box size X is smaller than rc gamma.");
  INCH_REQUIRE(by > rc, INCH_INVALID_ARG, "ABORTED. The PBC box size Y is smaller than rc gamma.");
  INCH_REQUIRE(grid->n_atoms < (int64_t(1) << kImageShift), INCH_INVALID_ARG,
               "%s: periodic neighbour lists take at most 2^27 atoms", who);
  return INCH_OK;
}
}  // namespace

extern "C" inch_status inch_neighbors_count(const double* X, const inch_cell_grid* grid, double rc,
                                            int32_t* degree, int64_t* rowptr, int64_t* nnz_host, void* ws,
                                            size_t ws_bytes, cudaStream_t stream) {
  return neighbors_count_impl<1>("inch_neighbors_count", X, grid, rc, 0.0, 0.0, degree, rowptr, nnz_host, ws,
                                 ws_bytes, stream);
}

extern "C" inch_status inch_neighbors_count_pbc_xy(const double* X, const inch_cell_grid* grid, double rc,
                                                   double box_x, double box_y, int32_t* degree, int64_t* rowptr,
                                                   int64_t* nnz_host, void* ws, size_t ws_bytes,
                                                   cudaStream_t stream) {
  inch_status st = check_box("inch_neighbors_count_pbc_xy", grid, rc, box_x, box_y);
  if (st != INCH_OK) return st;
  return neighbors_count_impl<9>("inch_neighbors_count_pbc_xy", X, grid, rc, box_x, box_y, degree, rowptr,
                                 nnz_host, ws, ws_bytes, stream);
}

extern "C" inch_status inch_neighbors_fill(const double* X, const inch_cell_grid* grid, double rc,
                                           const int64_t* rowptr, int32_t* cols, void* ws, size_t ws_bytes,
                                           cudaStream_t stream) {
  return neighbors_fill_impl<1>("inch_neighbors_fill", X, grid, rc, 0.0, 0.0, rowptr, cols, nullptr, ws, ws_bytes,
                                stream);
}

extern "C" inch_status inch_neighbors_fill_pbc_xy(const double* X, const inch_cell_grid* grid, double rc,
                                                  double box_x, double box_y, const int64_t* rowptr, int32_t* cols,
                                                  int8_t* image, void* ws, size_t ws_bytes, cudaStream_t stream) {
  inch_status st = check_box("inch_neighbors_fill_pbc_xy", grid, rc, box_x, box_y);
  if (st != INCH_OK) return st;
  return neighbors_fill_impl<9>("inch_neighbors_fill_pbc_xy", X, grid, rc, box_x, box_y, rowptr, cols, image, ws,
                                ws_bytes, stream);
}
