/*
 * inching_b200 C ABI: B200-native kernels for the Inching normal-mode hot path
 * (ANM Hessian build, Cuthill-McKee banding, Hessian x multivector products).
 *
 * Conventions
 *   - Every pointer argument named *_dev is device memory (cudaMalloc'd or a torch
 *     tensor's data_ptr); *_host is host memory.
 *   - Every entry point takes the cudaStream_t it enqueues on.  Entry points that
 *     must read a size back to the host say "synchronises" and do so on that stream.
 *   - The library never frees caller memory.  Kernel scratch comes from a
 *     caller-provided workspace whose size is queried first.  The one device
 *     allocation the library makes itself is cuBLAS's: the solver building blocks
 *     (inch_block_orth, inch_rr_project, inch_rr_rotate) create one cuBLAS handle
 *     per device on first use, which allocates cuBLAS's own internal state.
 *   - Return value: INCH_OK or an error code; inch_last_error_string() gives a
 *     message for the calling thread's last error.
 *   - Coordinates are float64 nanometres, atoms in caller order; degrees of
 *     freedom are dof = 3*atom + axis.
 *
 * Reference interfaces replaced (paths inside jhmlam/Inching):
 *   inch_neighbors_*  -> cKDTree.query_ball_point in X_KdCuthillMckeeOrder /
 *                        X_KdUngappedMinMaxNeighbor (InchingLiteInteger/Fuel/Coordinate/T1.py:218-245,397)
 *   inch_rcm          -> the BFS of X_KdCuthillMckeeOrder (Fuel/Coordinate/T1.py:254-323)
 *   inch_band_slices  -> the gap scan of X_KdUngappedMinMaxNeighbor (Fuel/Coordinate/T1.py:371-481)
 *   inch_hessian_assemble -> Xnumpy_SparseCupyMatrixUngappped.ReturnCupyHLowerTriangleInt32/64
 *                        (InchingLiteInteger/Fuel/T1.py:228-660, 666-1048)
 *   inch_spmm         -> OOC2_HalfMemS_v_KrylovAv_VOID / OOC2_FullMemS_v_KrylovAv_VOID
 *                        (InchingLiteInteger/Burn/Krylov/T3.py:54-239), with the Hotelling update
 *                        of Burn/Orthogonalization/T3.py:62-164 and one step of the Chebyshev
 *                        recurrence of Burn/PolynomialFilters/T2.py:59-80 fused in its epilogue
 */
#ifndef INCHING_B200_H
#define INCHING_B200_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  INCH_OK = 0,
  INCH_INVALID_ARG = 1,
  INCH_OOM = 2,            /* workspace too small */
  INCH_NOT_CONVERGED = 3,
  INCH_TIMEOUT = 4,
  INCH_CUDA_ERROR = 5,
  INCH_LIMIT = 6           /* an input exceeds a documented kernel limit */
} inch_status;

/* Message for the calling thread's most recent error ("" if none). */
const char* inch_last_error_string(void);
/* ABI version of this library (bumped on any signature change). */
int inch_abi_version(void);

/* ---------------------------------------------------------------------------
 * Cell-list neighbour search.  j is a neighbour of i iff
 *   ((dx*dx) + dy*dy) + dz*dz <= rc*rc   (each step rounded to double, no FMA),
 * the distance rule of scipy cKDTree.query_ball_point(p=2, eps=0) used by the
 * reference.  Lists include i itself and are sorted ascending.
 * ------------------------------------------------------------------------- */
typedef struct {
  double origin[3];      /* lower corner of the cell grid (nm) */
  double cell;           /* cell edge (nm), >= rc */
  int32_t dims[3];       /* cells per axis */
  int64_t ncells;
  int64_t n_atoms;
} inch_cell_grid;

/* Bounding box of X_dev (N,3) -> grid with cell edge rc.  Needs 64 bytes of
 * workspace.  Synchronises the stream.  Replaces the cKDTree construction of
 * Fuel/Coordinate/T1.py:218-226. */
inch_status inch_cell_grid_plan(const double* X_dev, int64_t n_atoms, double rc,
                                inch_cell_grid* grid_host, void* ws_dev, size_t ws_bytes,
                                cudaStream_t stream);

/* Workspace bytes for inch_neighbors_count / inch_neighbors_fill on this grid. */
size_t inch_neighbors_workspace_size(const inch_cell_grid* grid_host);

/* Builds the cell list in the workspace, writes degree_dev[N] (neighbours incl.
 * self) and rowptr_dev[N+1] (exclusive prefix sum, int64), and copies the total
 * neighbour count to *nnz_host.  Synchronises the stream.
 * Replaces the degree pass of Fuel/Coordinate/T1.py:236-245. */
inch_status inch_neighbors_count(const double* X_dev, const inch_cell_grid* grid_host, double rc,
                                 int32_t* degree_dev, int64_t* rowptr_dev, int64_t* nnz_host,
                                 void* ws_dev, size_t ws_bytes, cudaStream_t stream);

/* Fills cols_dev[nnz] with the sorted neighbour lists.  Must follow
 * inch_neighbors_count with the same workspace (the cell list is reused).
 * At most INCH_MAX_DEGREE neighbours per atom (else INCH_LIMIT).  Synchronises.
 * Replaces query_ball_point(..., return_sorted=True) (Fuel/Coordinate/T1.py:276,397). */
#define INCH_MAX_DEGREE 1024
inch_status inch_neighbors_fill(const double* X_dev, const inch_cell_grid* grid_host, double rc,
                                const int64_t* rowptr_dev, int32_t* cols_dev,
                                void* ws_dev, size_t ws_bytes, cudaStream_t stream);

/* Periodic images in x and y (membrane systems): atom j is a neighbour of i
 * through image s when |x_j - (x_i + s)| <= rc, s in the nine shifts
 * {0, +-box_x, +-box_y, +-box_x +-box_y} in the order centre, +x, -x, +y, -y,
 * +x+y, +x-y, -x+y, -x-y.  degree counts every (j, image) pair; each row lists
 * image 0's neighbours (ascending j), then image 1's, ..., with image_dev[e] the
 * image code 0..8 of entry e.  Requires box_x, box_y > rc (the reference's
 * "ABORTED. The PBC box size X/Y is smaller than rc gamma.") and N < 2^27.
 * Same grid and workspace as the non-periodic pair of calls.
 * Replaces X_cKDTreePbcXy.query_ball_point (Fuel/Coordinate/T1.py:67-161) as used
 * by X_KdCuthillMckeeOrder / X_KdUngappedMinMaxNeighbor with User_DictCharmmGuiPbc. */
inch_status inch_neighbors_count_pbc_xy(const double* X_dev, const inch_cell_grid* grid_host, double rc,
                                        double box_x, double box_y, int32_t* degree_dev, int64_t* rowptr_dev,
                                        int64_t* nnz_host, void* ws_dev, size_t ws_bytes, cudaStream_t stream);
inch_status inch_neighbors_fill_pbc_xy(const double* X_dev, const inch_cell_grid* grid_host, double rc,
                                       double box_x, double box_y, const int64_t* rowptr_dev, int32_t* cols_dev,
                                       int8_t* image_dev, void* ws_dev, size_t ws_bytes, cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * Cuthill-McKee ordering (level-synchronous, bit-exact with the sequential BFS
 * of Fuel/Coordinate/T1.py:254-323).  seed_order_dev is np.argsort(degree) as
 * computed by the reference (its tie order is the caller's numpy's); the next
 * unvisited atom in that order seeds each connected component.
 * Outputs the REVERSED order (rcm_order_dev, int64 N) and its inverse
 * (undo_dev, int64 N), as X_KdCuthillMckeeOrder(..., Reverse=True) returns.
 * Synchronises once per BFS level.
 * ------------------------------------------------------------------------- */
size_t inch_rcm_workspace_size(int64_t n_atoms);
inch_status inch_rcm(const int64_t* rowptr_dev, const int32_t* cols_dev, const int32_t* degree_dev,
                     const int64_t* seed_order_dev, int64_t n_atoms,
                     int64_t* rcm_order_dev, int64_t* undo_dev, int32_t* n_levels_host,
                     void* ws_dev, size_t ws_bytes, cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * Ungapped band slices of X_KdUngappedMinMaxNeighbor (Fuel/Coordinate/T1.py:371-481)
 * from the adjacency of the (reordered) structure.  batch_head_dev holds
 * n_batches+1 row heads.  For batch b, slices are written to
 * starts/ends[b*max_slices ...] and their number to counts_dev[b].  *total_nbrs_host
 * receives the sum of all degrees (for HalfNnz).  A batch with more than
 * max_slices slices, or more than 2048 gaps wider than `gap`, returns INCH_LIMIT.
 * nnz = rowptr[n_atoms] < 2^31.  Synchronises.
 * ------------------------------------------------------------------------- */
size_t inch_band_slices_workspace_size(int64_t n_batches, int64_t nnz);
inch_status inch_band_slices(const int64_t* rowptr_dev, const int32_t* cols_dev, int64_t n_atoms,
                             const int64_t* batch_head_dev, int64_t n_batches, int64_t gap,
                             int32_t max_slices, int64_t* starts_dev, int64_t* ends_dev,
                             int32_t* counts_dev, int64_t* total_nbrs_host,
                             void* ws_dev, size_t ws_bytes, cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * ANM Hessian store.  Off-diagonal block (i,j) = -(x x^T)/d^2 for 0 < d^2 <= rc^2,
 * x = X_j - X_i, is rank one: it is stored as w = x/d, so block = -w w^T.
 * Diagonal block (i,i) = sum_j w w^T + plus_i * I, stored as 6 unique values
 * (xx, yy, zz, xy, xz, yz) padded to 8.
 *   entries: one per adjacency entry (self included, w = 0 there), same order
 *            as cols: f64 layout {wx, wy, wz, (double)col} (32 B),
 *            f32 layout {wx, wy, wz, col bits} (16 B).
 *   diag:    f64 (N,8) and f32 (N,8).
 * Pass NULL for a precision that is not wanted.
 * Replaces Fuel/T1.py:276-455 (pair blocks, diagonal row sum, +PlusI).
 * ------------------------------------------------------------------------- */
inch_status inch_hessian_assemble(const double* X_dev, int64_t n_atoms, double rc, double plus_i,
                                  const int64_t* rowptr_dev, const int32_t* cols_dev,
                                  double* ent64_dev, double* diag64_dev,
                                  float* ent32_dev, float* diag32_dev, cudaStream_t stream);

/* As inch_hessian_assemble with a spring constant per adjacency entry
 * (pair_weight_dev[e] >= 0, the same value for both directions of a pair): block
 * (i,j) = -gamma_e u u^T, stored as w = sqrt(gamma_e) u.  Used by the learned
 * bead model of the warm start; no reference counterpart (the reference's
 * gamma is 1). */
inch_status inch_hessian_assemble_weighted(const double* X_dev, int64_t n_atoms, double rc, double plus_i,
                                           const int64_t* rowptr_dev, const int32_t* cols_dev,
                                           const double* pair_weight_dev, double* ent64_dev, double* diag64_dev,
                                           float* ent32_dev, float* diag32_dev, cudaStream_t stream);

/* Hessian of a structure with periodic xy images, from the lists of
 * inch_neighbors_*_pbc_xy: entry e (found with the query x_i + s) gets the block
 * of d = (x_j - s) - x_i, the reference's (x_j + box * instr) - x_i with
 * instr = -s (a pair seen through two images contributes two blocks); the
 * diagonal sums them all.
 * Replaces the image loop of Xnumpy_SparseCupyMatrixUngappped (Fuel/T1.py:317-396). */
inch_status inch_hessian_assemble_pbc_xy(const double* X_dev, int64_t n_atoms, double rc, double plus_i,
                                         const int64_t* rowptr_dev, const int32_t* cols_dev,
                                         const int8_t* image_dev, double box_x, double box_y, double* ent64_dev,
                                         double* diag64_dev, float* ent32_dev, float* diag32_dev,
                                         cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * Message-passing network kernels of the learned warm start (no reference
 * counterpart).  Directed bead-graph edges in CSR by destination: rowptr (N+1),
 * src[e] / dst[e] per edge.  Dense layers are GEMMs done by the caller.
 *   edge_concat      Z[e] = [H[src[e]], EF[e]]           (+ bwd: scatter-add)
 *   segment_sum      M[i] = mean of A over the edges of row i (+ bwd: gather / deg)
 *   bias_relu        Y = relu(Y + b);  relu_bwd  dY *= (Y > 0)
 *   edge_pair        R[e] = [H[dst] + H[src], EF[e]]     (+ bwd)
 *   softplus         gamma = softplus(s) + floor, or ds = sigmoid(s) * dgamma
 *   hf_grad          out[e] = 1/2 sum_t c[t] (u_e . (V_t[a] - V_t[b]))^2
 *                    (Hellmann-Feynman eigenvalue gradient of the bead Hessian)
 *   adam             one bias-corrected Adam step
 *   gemm             the dense layers (forward, weight and input gradients)
 * ------------------------------------------------------------------------- */
inch_status inch_mp_edge_concat(const float* H, const float* EF, const int32_t* src, int64_t E, int32_t F,
                                int32_t G, float* Z, cudaStream_t stream);
inch_status inch_mp_edge_concat_bwd(const float* dZ, const int32_t* src, int64_t E, int32_t F, int32_t G,
                                    float* dH, cudaStream_t stream);
inch_status inch_mp_segment_sum(const float* A, const int64_t* rowptr, int64_t N, int32_t F, float* M,
                                cudaStream_t stream);
inch_status inch_mp_segment_sum_bwd(const float* dM, const int64_t* rowptr, const int32_t* dst, int64_t E,
                                    int32_t F, float* dA, cudaStream_t stream);
inch_status inch_mp_bias_relu(float* Y, const float* b, int64_t R, int32_t F, cudaStream_t stream);
inch_status inch_mp_relu_bwd(float* dY, const float* Y, int64_t n, cudaStream_t stream);
inch_status inch_mp_edge_pair(const float* H, const float* EF, const int32_t* src, const int32_t* dst, int64_t E,
                              int32_t F, int32_t G, float* R, cudaStream_t stream);
inch_status inch_mp_edge_pair_bwd(const float* dR, const int32_t* src, const int32_t* dst, int64_t E, int32_t F,
                                  int32_t G, float* dH, cudaStream_t stream);
inch_status inch_mp_softplus(const float* s, int64_t E, float floor_v, double* gamma, const double* dgamma,
                             float* ds, cudaStream_t stream);
inch_status inch_mp_hf_grad(const double* P, const int64_t* rowptr, const int32_t* src, const int32_t* dst,
                            const double* V, int32_t m, const double* c, int64_t E, double* out,
                            cudaStream_t stream);
inch_status inch_mp_adam(float* w, const float* g, float* m1, float* m2, int64_t n, float lr, float b1, float b2,
                         float eps, int32_t step, cudaStream_t stream);
/* The network's dense layers: C = A B + beta C in FP32, with element (i, k) of A at
 * A[i*sai + k*sak] and (k, j) of B at B[k*sbk + j*sbn] (so transposed operands are
 * strides), C row-major with leading dimension ldc.  A product with a small output
 * and a long K splits K into partial tiles added in a fixed order (deterministic);
 * ws: inch_mp_gemm_workspace_size(M, N, K) bytes.  No reference counterpart. */
size_t inch_mp_gemm_workspace_size(int32_t M, int32_t N, int32_t K);
inch_status inch_mp_gemm(int32_t M, int32_t N, int32_t K, const float* A, int64_t sai, int64_t sak,
                         const float* B, int64_t sbk, int64_t sbn, float* C, int64_t ldc, float beta,
                         void* ws_dev, size_t ws_bytes, cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * Hessian x multivector with fused epilogue.  X and Y are (3N, b) row-major with
 * leading dimension ld (>= b), element (dof, c) at dof*ld + c.
 *   Y = alpha*(H X) + gamma*X + beta*Yin + hot_shift * Q^T (Q X)   [Acc += mu*Y]
 * where Q is the (r, 3N) row-major FP64 deflation basis (r <= 8; explicit
 * Hotelling deflation); its coefficients Q X are reduced inside the call.
 * Yin may alias Y.  prec: 64 -> f64 store and f64 vectors; 32 -> f32 store and
 * f32 vectors.  Supported b: 1..128 in FP32 (128-column tiles with float4 gathers
 * when every vector block is 16-byte aligned with leading dimensions and column
 * offset multiples of 4, else 64-column tiles), 1..64 in FP64 (two 32-column
 * tiles).  With a workspace the wide-block kernel hands out its rows from a
 * counter in it (inch_spmm_traversal); calls that share a workspace must not
 * overlap on the GPU.
 * ------------------------------------------------------------------------- */
typedef struct {
  double alpha, gamma, beta, mu, hot_shift;
  int32_t r;              /* deflation rank (0 = none) */
  int32_t accumulate;     /* 1 -> Acc += mu*Y */
} inch_spmm_epilogue;

size_t inch_spmm_workspace_size(int64_t n_atoms, int32_t b, int32_t r);
/* Row traversal of inch_spmm's wide-block kernel (b >= 8) for this process (the
 * autotuner's hook; no reference counterpart): 0 a fixed block-interleaved grid
 * stride; 1 (default) chunks of consecutive rows that each warp takes from a
 * counter in the workspace; 2 chunks that each block takes from it.  Modes 1 and
 * 2 keep every SM on one compact frontier of rows, so the gathered X rows stay
 * in L2 on large structures; they need the workspace (calls without one use 0),
 * and calls that share one workspace must not overlap on the GPU. */
inch_status inch_spmm_traversal(int32_t mode);
/* inch_spmm with per-segment coefficients (no reference counterpart): for a
 * block-diagonal store holding many structures, atom i uses (alpha, gamma, beta) =
 * seg_coef[3*atom_seg[i] .. +2] in Y = alpha*(H X) + gamma*X + beta*Yin, so each
 * structure gets its own Chebyshev filter step in the same launch.  Yin may be
 * NULL (then beta is ignored) and may alias Y.  No deflation or accumulation. */
inch_status inch_spmm_seg(int32_t prec, int64_t n_atoms, const int64_t* rowptr_dev,
                          const void* ent_dev, const void* diag_dev,
                          const void* X_dev, int64_t ldx, int32_t b,
                          void* Y_dev, int64_t ldy, const void* Yin_dev, int64_t ldyin,
                          const int32_t* atom_seg_dev, const double* seg_coef_dev, cudaStream_t stream);
/* inch_spmm_seg with a workspace (inch_spmm_workspace_size bytes): the wide-block
 * kernel then hands out its rows from the counter in it (inch_spmm_traversal) and
 * FP32 takes up to 128 columns per call, as in inch_spmm.  Used by the CUDA-graph
 * Chebyshev filter.  Calls sharing a workspace must not overlap on the GPU. */
inch_status inch_spmm_seg_ws(int32_t prec, int64_t n_atoms, const int64_t* rowptr_dev, const void* ent_dev,
                             const void* diag_dev, const void* X_dev, int64_t ldx, int32_t b, void* Y_dev,
                             int64_t ldy, const void* Yin_dev, int64_t ldyin, const int32_t* atom_seg_dev,
                             const double* seg_coef_dev, void* ws_dev, size_t ws_bytes, cudaStream_t stream);

/* Launch shape of the wide-block (b >= 8) SpMM kernel for this process: threads
 * per block (256, 512 or 1024) and resident blocks per SM (1..8); each block walks
 * one contiguous slab of rows.  threads_per_block = 0 selects instead, for tiles of
 * >= 32 columns per lane-row, the whole-warp-row kernel that loads 32 entries at
 * once and batches 4 entries' gathers.  Hook of the autotuner (inching_b200.autotune);
 * default 256 x 5.  No reference counterpart. */
inch_status inch_spmm_tune(int32_t threads_per_block, int32_t blocks_per_sm);
inch_status inch_spmm(int32_t prec, int64_t n_atoms, const int64_t* rowptr_dev,
                      const void* ent_dev, const void* diag_dev,
                      const void* X_dev, int64_t ldx, int32_t b,
                      void* Y_dev, int64_t ldy, const void* Yin_dev, int64_t ldyin,
                      void* Acc_dev, int64_t ldacc,
                      const double* q_dev /* (r, 3N) row-major, FP64 */,
                      const inch_spmm_epilogue* ep,
                      void* ws_dev, size_t ws_bytes, cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * Solver building blocks as single calls (for hosts that drive an iteration
 * through this ABI).  Tall blocks are row-major (n rows, b columns, leading
 * dimension ld >= b); n = 3 * n_atoms for the Hessian.  Every buffer, including
 * scratch, is the caller's.
 * ------------------------------------------------------------------------- */

/* Y = sum_{k=0..degree} mu[k] T_k((H - cc)/dd) X on the store (prec 32 or 64),
 * the three-term recurrence fused with its accumulation in each SpMM; W1, W2:
 * work blocks of the same shape (leading dimension ldw).  X is not modified.
 * Any b (column panels of 64 inside).  mu_host: degree + 1 host doubles.
 * Replaces OOC2_A_Adiag_ChebyshevAv.ChebyshevAv (Burn/PolynomialFilters/T2.py:28-92). */
inch_status inch_cheb_filter(int32_t prec, int64_t n_atoms, const int64_t* rowptr_dev, const void* ent_dev,
                             const void* diag_dev, const void* X_dev, int64_t ldx, int32_t b, int32_t degree,
                             const double* mu_host, double cc, double dd, void* Y_dev, int64_t ldy,
                             void* W1_dev, void* W2_dev, int64_t ldw, cudaStream_t stream);

/* Scaled Chebyshev filter of degree m damping [a, b_up], normalised at a0 < a
 * (Zhou & Saad, J. Comput. Phys. 219 (2006)): Y = p_m(H) X; W: one work block.
 * No reference counterpart (the block solver's filter; the reference filters one
 * vector at a time through ChebyshevAv). */
inch_status inch_cheb_filter_scaled(int32_t prec, int64_t n_atoms, const int64_t* rowptr_dev, const void* ent_dev,
                                    const void* diag_dev, const void* X_dev, int64_t ldx, int32_t b, int32_t degree,
                                    double a, double b_up, double a0, void* Y_dev, int64_t ldy, void* W_dev,
                                    int64_t ldw, cudaStream_t stream);

/* FP64 block orthonormalisation: Y <- Y - B^T (B Y) twice for each of the two
 * optional row bases B1 (r1 x n, leading dimension ldb1) and B2 (locked modes,
 * rigid-body basis), then `passes` Cholesky-QR passes (G = Y^T Y = L L^T,
 * Y <- Y L^{-T}; a Gram matrix that is not numerically positive is retried once
 * with a 1e-12 * max-diagonal shift; still not positive -> INCH_INVALID_ARG,
 * "rank deficient").  cuBLAS runs the GEMMs and the triangular solve; its handle
 * is created on a device's first call (cuBLAS's own small allocation), its GEMM
 * workspace comes from ws.  Synchronises the stream once per pass.
 * Replaces the Gram-Schmidt of Burn/Orthogonalization/T1.py:56-64 and
 * T2.py:64-137 (one vector against the basis there, a whole block here). */
size_t inch_block_orth_workspace_size(int32_t b, int64_t r_max);
inch_status inch_block_orth(int64_t n, int32_t b, double* Y_dev, int64_t ldy, const double* B1_dev, int64_t r1,
                            int64_t ldb1, const double* B2_dev, int64_t r2, int64_t ldb2, int32_t passes,
                            void* ws_dev, size_t ws_bytes, cudaStream_t stream);

/* Rayleigh-Ritz: G (b x b, symmetric, column-major) = sym(Y^T HY) for an
 * orthonormal Y and HY = H Y (both FP64 blocks); and Z (n x m) = Y W for the m
 * leading columns of the (column-major, b x b) eigenvector matrix W of G.  The
 * small eigenproblem itself stays with the caller (LAPACK / cuSOLVER).
 * Replaces the projected matrix of JacobiDavidsonHotellingDeflation/T1.py:440-451
 * and the restart rotations of T1.py:662-666 / ThickRestartLanczos.../T1.py. */
size_t inch_rr_workspace_size(void);
inch_status inch_rr_project(int64_t n, int32_t b, const double* Y_dev, int64_t ldy, const double* HY_dev,
                            int64_t ldh, double* G_dev, void* ws_dev, size_t ws_bytes, cudaStream_t stream);
inch_status inch_rr_rotate(int64_t n, int32_t b, int32_t m, const double* Y_dev, int64_t ldy, const double* W_dev,
                           double* Z_dev, int64_t ldz, void* ws_dev, size_t ws_bytes, cudaStream_t stream);

/* res_dev[c] = || HY[:, c] - theta_dev[c] * Y[:, c] ||_2 in FP64 (deterministic
 * two-stage reduction, no (n x b) temporary).
 * Replaces the Ritz residual of JacobiDavidsonHotellingDeflation/T1.py:543-560. */
size_t inch_residual_workspace_size(int32_t b);
inch_status inch_residual_fp64(int64_t n, int32_t b, const double* HY_dev, int64_t ldh, const double* Y_dev,
                               int64_t ldy, const double* theta_dev, double* res_dev, void* ws_dev,
                               size_t ws_bytes, cudaStream_t stream);

/* Eigenpairs of n_mat symmetric p x p FP64 matrices (row-major, one after the
 * other; p <= 64): W (n_mat, p) ascending, V (n_mat, p, p) with eigenvector k in
 * column k.  One CTA per matrix, cyclic Jacobi in shared memory, sweeps until the
 * off-diagonal norm is below tol times the matrix's or max_sweeps (<= 100; the
 * count used per matrix goes to sweeps_used if not NULL).  No reference
 * counterpart: the small projected eigenproblems of the batched solve (one per
 * structure), which the reference would solve one at a time with numpy. */
inch_status inch_eigh_batched_small(const double* A_dev, int64_t n_mat, int32_t p, double* W_dev, double* V_dev,
                                    int32_t max_sweeps, double tol, int32_t* sweeps_used_dev, cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * Row-tile store for wide multivectors (no reference counterpart; an alternative
 * layout of the same matrix).  Atoms are grouped in tiles of 8 consecutive rows;
 * per tile, the merged sorted union of the rows' neighbour columns is stored as
 * urec = (j << 8) | row-mask, followed in pw by w = x/|x| for every set mask bit
 * (FP64 {wx,wy,wz,0} 32 B, FP32 {wx,wy,wz,0} 16 B); self pairs are omitted.
 * tile_uptr / tile_pptr: (n_tiles + 1) offsets.  n_atoms < 2^24.
 * count (synchronises, returns the totals) then fill; inch_spmm_tiles is
 * inch_spmm on this layout (same epilogue, diagonal from inch_hessian_assemble).
 * ------------------------------------------------------------------------- */
size_t inch_tile_store_workspace_size(int64_t n_atoms);
inch_status inch_tile_store_count(const int64_t* rowptr_dev, const int32_t* cols_dev, int64_t n_atoms,
                                  int64_t* tile_uptr_dev, int64_t* tile_pptr_dev, int64_t* n_union_host,
                                  int64_t* n_pairs_host, void* ws_dev, size_t ws_bytes, cudaStream_t stream);
inch_status inch_tile_store_fill(const double* X_dev, int64_t n_atoms, double rc, const int64_t* rowptr_dev,
                                 const int32_t* cols_dev, const int64_t* tile_uptr_dev,
                                 const int64_t* tile_pptr_dev, uint32_t* urec_dev, double* pw64_dev,
                                 float* pw32_dev, cudaStream_t stream);
size_t inch_spmm_tiles_workspace_size(void);
/* The band-tile product: one warp per 8-row tile and column panel (FP32 panels of
 * 128 columns with the packed f32x2 FMAs of sm_100, or 64 / 32; FP64 panels of
 * 64 / 32), each union column's X_j staged once by the bulk-copy (TMA) engine
 * and applied to all rows of its mask.  Any b >= 1 (the library walks the
 * panels; the last one may be partial).  Replaces the same two cuSPARSE SpMVs as
 * inch_spmm (Burn/Krylov/T3.py:138-156), with the same fused epilogue.  Every
 * vector block (X, Y, Yin, Acc) must start on 16 bytes and have a leading
 * dimension that is a multiple of 4 (FP32) or 2 (FP64) elements, else
 * INCH_INVALID_ARG; rows of X are read up to the next 16-byte boundary past the
 * last column, which the leading dimension keeps inside the row.  ws: inch_spmm_tiles_workspace_size() bytes, used only when
 * ep->r > 0. */
inch_status inch_spmm_tiles(int32_t prec, int64_t n_atoms, const int64_t* tile_uptr_dev,
                            const int64_t* tile_pptr_dev, const uint32_t* urec_dev, const void* pw_dev,
                            const void* diag_dev, const void* X_dev, int64_t ldx, int32_t b,
                            void* Y_dev, int64_t ldy, const void* Yin_dev, int64_t ldyin,
                            void* Acc_dev, int64_t ldacc, const double* q_dev,
                            const inch_spmm_epilogue* ep, void* ws_dev, size_t ws_bytes, cudaStream_t stream);
/* inch_spmm_seg on the band tiles (per-segment alpha, gamma, beta; any b >= 1).
 * Used by the CUDA-graph Chebyshev filter, whose coefficients live in a device
 * table (PolynomialFilters/T2.py:59-80 as one graph replay). */
inch_status inch_spmm_tiles_seg(int32_t prec, int64_t n_atoms, const int64_t* tile_uptr_dev,
                                const int64_t* tile_pptr_dev, const uint32_t* urec_dev, const void* pw_dev,
                                const void* diag_dev, const void* X_dev, int64_t ldx, int32_t b,
                                void* Y_dev, int64_t ldy, const void* Yin_dev, int64_t ldyin,
                                const int32_t* atom_seg_dev, const double* seg_coef_dev, cudaStream_t stream);
/* Widest FP32 panel of the band-tile product for this process (128 or 64
 * columns): the autotuner's hook (no reference counterpart). */
inch_status inch_spmm_band_tune(int32_t widest_fp32_panel);
/* Status word of the band-tile kernels (synchronises): 0, or 1 if a bounded
 * wait for a staged batch ran out in some launch since the last call (the
 * affected launch stopped early; its output is incomplete).  Reading clears it.
 * No reference counterpart. */
inch_status inch_spmm_band_status(int32_t* status_host);

/* ---------------------------------------------------------------------------
 * Row-group store, FP32 (no reference counterpart; an alternative layout of the
 * same matrix, built from the FP32 pair entries of inch_hessian_assemble).
 * R = rows_per_group (2 or 4) consecutive atoms form a group; the group's
 * neighbour lists are merged into one sorted union, and union u stores R float4
 * slots group_ent[R*u + r] = {wx, wy, wz, .} of row R*g + r's entry for that
 * column (zeros where the row has none), slot 0's last field holding the column
 * index as int bits.  Each group's union count is padded with zero-weight unions
 * to a multiple of 16.  group_ptr: (ceil(n_atoms / R) + 1) offsets in unions.
 * A row's entries keep their order, so the product gives the bits of inch_spmm
 * on the pair store.  count (synchronises, returns the union total) then fill
 * (group_ent: n_union * R float4, 16-byte aligned). */
size_t inch_group_store_workspace_size(int64_t n_atoms, int32_t rows_per_group);
inch_status inch_group_store_count(const int64_t* rowptr_dev, const float* ent32_dev, int64_t n_atoms,
                                   int32_t rows_per_group, int64_t* group_ptr_dev, int64_t* n_union_host,
                                   void* ws_dev, size_t ws_bytes, cudaStream_t stream);
inch_status inch_group_store_fill(const int64_t* rowptr_dev, const float* ent32_dev, int64_t n_atoms,
                                  int32_t rows_per_group, const int64_t* group_ptr_dev, float* group_ent_dev,
                                  cudaStream_t stream);
/* The row-group product: inch_spmm (prec 32) on the row-group store, any b >= 1
 * (tiles of 128 / 64 columns where the vector blocks allow float4 / float2
 * access, else 32-column tiles, the last one partial).  One warp per group and
 * tile; each X_j gather serves every row of the group.  Replaces the same two
 * cuSPARSE SpMVs as inch_spmm (Burn/Krylov/T3.py:138-156), with the same fused
 * epilogue.  ws: inch_spmm_workspace_size() bytes (row counter and deflation
 * scratch), or NULL when ep->r == 0. */
inch_status inch_spmm_groups(int64_t n_atoms, int32_t rows_per_group, const int64_t* group_ptr_dev,
                             const float* group_ent_dev, const float* diag_dev, const float* X_dev, int64_t ldx,
                             int32_t b, float* Y_dev, int64_t ldy, const float* Yin_dev, int64_t ldyin,
                             float* Acc_dev, int64_t ldacc, const double* q_dev, const inch_spmm_epilogue* ep,
                             void* ws_dev, size_t ws_bytes, cudaStream_t stream);
/* inch_spmm_seg on the row-group store (per-segment alpha, gamma, beta; any b). */
inch_status inch_spmm_groups_seg(int64_t n_atoms, int32_t rows_per_group, const int64_t* group_ptr_dev,
                                 const float* group_ent_dev, const float* diag_dev, const float* X_dev, int64_t ldx,
                                 int32_t b, float* Y_dev, int64_t ldy, const float* Yin_dev, int64_t ldyin,
                                 const int32_t* atom_seg_dev, const double* seg_coef_dev, void* ws_dev,
                                 size_t ws_bytes, cudaStream_t stream);
/* Unions a warp of the row-group product keeps in flight (2, 4, 8 or 16; 0 = the
 * default: 16 on 128-column tiles, 8 on narrower ones): the autotuner's hook (no
 * reference counterpart). */
inch_status inch_spmm_group_tune(int32_t unroll);

/* Allocation-free form of inch_spmm (no counterpart in the reference).  For
 * callers that cannot provide device scratch -- hosts running on another
 * runtime's memory manager without a device allocator of their own, or thin FFI
 * bindings that own only their input and output buffers -- the deflation partial
 * sums live in a static device array of about 1.2 MB held by every GPU that
 * loads the library until exit.  Limits: b <= 64 columns and r <= 8 deflation
 * vectors (else INCH_LIMIT).  The array is used only when ep->r > 0: the first
 * such call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and keeps it for the process; make that first call
 * before any stream capture.  The kept address is not refreshed after a
 * cudaDeviceReset, so a caller that resets a device must not call this entry
 * point on it afterwards.  All calls share the array: calls with r > 0 that
 * overlap on the GPU race and must be serialised by the caller.  Allocates
 * nothing. */
inch_status inch_spmm_noalloc(int32_t prec, int64_t n_atoms, const int64_t* rowptr_dev,
                              const void* ent_dev, const void* diag_dev,
                              const void* X_dev, int64_t ldx, int32_t b,
                              void* Y_dev, int64_t ldy, const void* Yin_dev, int64_t ldyin,
                              void* Acc_dev, int64_t ldacc, const double* q_dev,
                              const inch_spmm_epilogue* ep, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* INCHING_B200_H */
