/*
 * C restatement of oracle/graph.py's neighbour search and Cuthill-McKee order,
 * for inputs of millions of atoms.  TEST INFRASTRUCTURE ONLY: only the tests load
 * it (through oracle.graph), as a checker.  It is pinned to the Python oracle and
 * through it to the reference-generated goldens (tests/test_cpu_oracle_c.py).
 *
 * Neighbours: the distance rule of scipy's cKDTree.query_ball_point as the
 * reference calls it (InchingLiteInteger/Fuel/Coordinate/T1.py:239,276): the
 * squared distance accumulated in axis order ((dx*dx) + dy*dy) + dz*dz, each step
 * rounded to double, compared with rc*rc; self included; rows sorted ascending.
 *
 * Cuthill-McKee: InchingLiteInteger/Fuel/Coordinate/T1.py:254-323 over an
 * adjacency list: seeds in the given order (the reference's np.argsort(degree)),
 * each frontier atom appends its unvisited neighbours in descending index order,
 * the appended run is stably sorted by degree, and the order is reversed.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  double lo[3], cell;
  int64_t dims[3];
  int64_t *start; /* (ncells + 1) offsets into idx */
  int64_t *idx;   /* atoms sorted by cell */
} grid_t;

static int64_t cell_of(const grid_t *g, const double *x, int64_t c[3]) {
  for (int a = 0; a < 3; ++a) {
    int64_t v = (int64_t)floor((x[a] - g->lo[a]) / g->cell);
    if (v < 0) v = 0;
    if (v >= g->dims[a]) v = g->dims[a] - 1;
    c[a] = v;
  }
  return (c[0] * g->dims[1] + c[1]) * g->dims[2] + c[2];
}

static int grid_build(grid_t *g, const double *X, int64_t n, double rc) {
  double hi[3];
  for (int a = 0; a < 3; ++a) g->lo[a] = hi[a] = X[a];
  for (int64_t i = 1; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      if (X[3 * i + a] < g->lo[a]) g->lo[a] = X[3 * i + a];
      if (X[3 * i + a] > hi[a]) hi[a] = X[3 * i + a];
    }
  /* cells a little wider than rc, so that a pair within rc is never two cells apart */
  g->cell = rc * (1.0 + 1e-6);
  int64_t nc = 1;
  for (int a = 0; a < 3; ++a) {
    g->dims[a] = (int64_t)floor((hi[a] - g->lo[a]) / g->cell) + 1;
    nc *= g->dims[a];
  }
  if (nc > (int64_t)1 << 31) return -1;
  g->start = (int64_t *)calloc((size_t)nc + 1, sizeof(int64_t));
  g->idx = (int64_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
  int64_t *key = (int64_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
  if (!g->start || !g->idx || !key) return -2;
  int64_t c[3];
  for (int64_t i = 0; i < n; ++i) {
    key[i] = cell_of(g, X + 3 * i, c);
    g->start[key[i] + 1]++;
  }
  for (int64_t k = 0; k < nc; ++k) g->start[k + 1] += g->start[k];
  int64_t *fill = (int64_t *)malloc((size_t)nc * sizeof(int64_t));
  if (!fill) return -2;
  memcpy(fill, g->start, (size_t)nc * sizeof(int64_t));
  for (int64_t i = 0; i < n; ++i) g->idx[fill[key[i]]++] = i;
  free(fill);
  free(key);
  return 0;
}

static void grid_free(grid_t *g) {
  free(g->start);
  free(g->idx);
}

static int cmp_i32(const void *a, const void *b) {
  const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

/* Visits the neighbours of atom i; writes them to out (if not NULL), returns the count. */
static int64_t row(const grid_t *g, const double *X, int64_t i, double r2, int32_t *out) {
  int64_t c[3], cnt = 0;
  cell_of(g, X + 3 * i, c);
  const double xi = X[3 * i], yi = X[3 * i + 1], zi = X[3 * i + 2];
  for (int64_t a = c[0] - 1; a <= c[0] + 1; ++a) {
    if (a < 0 || a >= g->dims[0]) continue;
    for (int64_t b = c[1] - 1; b <= c[1] + 1; ++b) {
      if (b < 0 || b >= g->dims[1]) continue;
      for (int64_t d = c[2] - 1; d <= c[2] + 1; ++d) {
        if (d < 0 || d >= g->dims[2]) continue;
        const int64_t k = (a * g->dims[1] + b) * g->dims[2] + d;
        for (int64_t p = g->start[k]; p < g->start[k + 1]; ++p) {
          const int64_t j = g->idx[p];
          const double dx = X[3 * j] - xi, dy = X[3 * j + 1] - yi, dz = X[3 * j + 2] - zi;
          double s = dx * dx;
          s = s + dy * dy;
          s = s + dz * dz;
          if (s <= r2) {
            if (out) out[cnt] = (int32_t)j;
            ++cnt;
          }
        }
      }
    }
  }
  if (out) qsort(out, (size_t)cnt, sizeof(int32_t), cmp_i32);
  return cnt;
}

/* degree (n,), rowptr (n+1,) filled; returns nnz, or < 0 on failure. */
int64_t oracle_neighbor_count(const double *X, int64_t n, double rc, int32_t *degree, int64_t *rowptr) {
  grid_t g;
  if (grid_build(&g, X, n, rc) != 0) return -1;
  const double r2 = rc * rc;
  rowptr[0] = 0;
  for (int64_t i = 0; i < n; ++i) {
    degree[i] = (int32_t)row(&g, X, i, r2, NULL);
    rowptr[i + 1] = rowptr[i] + degree[i];
  }
  grid_free(&g);
  return rowptr[n];
}

int oracle_neighbor_fill(const double *X, int64_t n, double rc, const int64_t *rowptr, int32_t *cols) {
  grid_t g;
  if (grid_build(&g, X, n, rc) != 0) return -1;
  const double r2 = rc * rc;
  for (int64_t i = 0; i < n; ++i) row(&g, X, i, r2, cols + rowptr[i]);
  grid_free(&g);
  return 0;
}

/* stable insertion sort of seg[0..m) by degree (strict '<', as the reference) */
static void sort_by_degree(int64_t *seg, int64_t m, const int32_t *degree) {
  for (int64_t a = 1; a < m; ++a) {
    const int64_t v = seg[a];
    const int32_t dv = degree[v];
    int64_t b = a - 1;
    while (b >= 0 && dv < degree[seg[b]]) {
      seg[b + 1] = seg[b];
      --b;
    }
    seg[b + 1] = v;
  }
}

/* order_out (n,): reversed Cuthill-McKee order; returns 0, or < 0 on failure. */
int oracle_cuthill_mckee(int64_t n, const int64_t *rowptr, const int32_t *cols, const int32_t *degree,
                         const int64_t *seed_order, int64_t *order_out) {
  unsigned char *visited = (unsigned char *)calloc((size_t)(n > 0 ? n : 1), 1);
  if (!visited) return -1;
  int64_t N = 0;
  for (int64_t zz = 0; zz < n && N < n; ++zz) {
    const int64_t seed = seed_order[zz];
    if (seed < 0 || seed >= n) {
      free(visited);
      return -2;
    }
    if (visited[seed]) continue;
    order_out[N++] = seed;
    visited[seed] = 1;
    int64_t ls = N - 1, le = N;
    while (ls < le) {
      for (int64_t ii = ls; ii < le; ++ii) {
        const int64_t i = order_out[ii];
        const int64_t n_old = N;
        for (int64_t e = rowptr[i + 1] - 1; e >= rowptr[i]; --e) {
          const int64_t j = cols[e];
          if (!visited[j]) {
            visited[j] = 1;
            order_out[N++] = j;
          }
        }
        sort_by_degree(order_out + n_old, N - n_old, degree);
      }
      ls = le;
      le = N;
    }
  }
  free(visited);
  if (N != n) return -3;
  for (int64_t a = 0, b = n - 1; a < b; ++a, --b) {
    const int64_t t = order_out[a];
    order_out[a] = order_out[b];
    order_out[b] = t;
  }
  return 0;
}
