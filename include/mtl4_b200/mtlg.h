/*
 * mtl4_b200 C ABI: the drop-in boundary for MTL4's sparse-solve hot path on
 * one B200 GPU (sm_100a).  Plain pointers and sizes only; every function
 * returns an int status (MTLG_OK == 0).
 *
 * Reference surface each group replaces (paths inside simunova/mtl4):
 *   mtlg_csr_*     mtl::compressed2D<T> raw-array constructor
 *                  (boost/numeric/mtl/matrix/compressed2D.hpp:355-364)
 *   mtlg_vec_*     mtl::dense_vector<T>(n, address)
 *                  (boost/numeric/mtl/vector/dense_vector.hpp:122)
 *   mtlg_spmv      w = A*v, w += A*v, w -= A*v
 *                  (boost/numeric/mtl/vector/crtp_base_vector.hpp:94-101,
 *                   boost/numeric/mtl/operation/mat_vec_mult.hpp:614-683)
 *   mtlg_dot / mtlg_two_norm
 *                  mtl::dot, mtl::two_norm
 *                  (boost/numeric/mtl/operation/dot.hpp:228,
 *                   boost/numeric/mtl/operation/two_norm.hpp:54)
 *   mtlg_pc_*      itl::pc::identity / diagonal / ilu_0 / ic_0 and
 *                  solve(P, x) / adjoint_solve(P, x)
 *                  (boost/numeric/itl/pc/identity.hpp:25, diagonal.hpp:29-64,
 *                   ilu_0.hpp:34-92, ilu.hpp:74-115, ic_0.hpp:40-107)
 *   mtlg_solve     itl::cg(A,x,b,P,iter) (boost/numeric/itl/krylov/cg.hpp:76),
 *                  itl::bicgstab (bicgstab.hpp:29),
 *                  itl::gmres(A,x,b,L,R,iter,restart) (gmres.hpp:124) with
 *                  itl::basic_iteration<double>
 *                  (boost/numeric/itl/iteration/basic_iteration.hpp:24-93)
 *   mtlg_refine_solve, mtlg_batch_*, mtlg_server_*
 *                  no reference counterpart: FP64 iterative refinement around
 *                  an FP32 inner solve, batched and served solves.
 */
#ifndef MTL4_B200_MTLG_H
#define MTL4_B200_MTLG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (mapped to the reference's exception types by the C++
 * front end: utility/exception.hpp:116-204, itl/utility/exception.hpp:22-31) */
enum {
    MTLG_OK = 0,
    MTLG_ERR_INVALID_ARG = 1,       /* null handle, bad enum, negative size     */
    MTLG_ERR_NOT_SQUARE = 2,        /* mtl::matrix_not_square                   */
    MTLG_ERR_MISSING_DIAGONAL = 3,  /* mtl::missing_diagonal                    */
    MTLG_ERR_ZERO_PIVOT = 4,        /* factorization produced a non-finite pivot */
    MTLG_ERR_BREAKDOWN = 5,         /* itl::unexpected_orthogonality            */
    MTLG_ERR_OOM = 6,               /* device allocation failed / over budget   */
    MTLG_ERR_TIMEOUT = 7,           /* a bounded device-side wait expired       */
    MTLG_ERR_CUDA = 8,              /* CUDA runtime error                       */
    MTLG_ERR_INCOMPATIBLE_SIZE = 9, /* mtl::incompatible_size                   */
    MTLG_ERR_UNSORTED = 10,         /* CSR rows must be sorted, in range        */
    MTLG_ERR_TOO_LARGE = 11,        /* nnz or n beyond int32 device indexing    */
    MTLG_ERR_NOT_SUPPORTED = 12,
    MTLG_ERR_ADMISSION = 13,        /* serving: request does not fit the budget */
    MTLG_ERR_NOT_FOUND = 14,        /* serving: unknown request id              */
    MTLG_PENDING = 15,              /* serving: request not finished yet        */
    MTLG_ERR_FILE_NOT_FOUND = 16,   /* mtl::io::file_not_found                  */
    MTLG_ERR_FORMAT = 17            /* malformed input file (mtl::runtime_error) */
};

typedef enum { MTLG_F64 = 0, MTLG_F32 = 1 } mtlg_dtype;
typedef enum { MTLG_ASSIGN = 0, MTLG_PLUS = 1, MTLG_MINUS = 2 } mtlg_assign;
typedef enum { MTLG_PC_IDENTITY = 0, MTLG_PC_DIAGONAL = 1, MTLG_PC_ILU0 = 2, MTLG_PC_IC0 = 3 } mtlg_pc_kind;
typedef enum {
    MTLG_CG = 0, MTLG_BICGSTAB = 1, MTLG_GMRES = 2,
    /* host-driven bodies on device vectors (itl/krylov/*.hpp) */
    MTLG_BICG = 3,          /* itl::bicg (bicg.hpp:28)        adjoint(A), adjoint_solve(L)  */
    MTLG_CGS = 4,           /* itl::cgs (cgs.hpp:28)                                         */
    MTLG_TFQMR = 5,         /* itl::tfqmr (tfqmr.hpp:30)      left L, right R                */
    MTLG_QMR = 6,           /* itl::qmr (qmr.hpp:31)          left L, right R, trans(A)      */
    MTLG_BICGSTAB_2 = 7,    /* itl::bicgstab_2 (bicgstab_2.hpp:29)                          */
    MTLG_BICGSTAB_ELL = 8,  /* itl::bicgstab_ell (bicgstab_ell.hpp:29)  ell = params->restart */
    MTLG_IDR_S = 9          /* itl::idr_s (idr_s.hpp:31)      s = params->restart           */
} mtlg_solver;

/* Termination state of one solve; mirrors itl::basic_iteration. */
enum {
    MTLG_ST_RUNNING = 0,
    MTLG_ST_CONVERGED = 1,   /* resid <= rtol*norm_r0 or resid <= atol   error_code 0 */
    MTLG_ST_MAXIT = 2,       /* "Too many iterations."                    error_code 1 */
    MTLG_ST_BREAKDOWN = 3,   /* zero rho/gamma/omega (BiCGSTAB) or NaN    */
    MTLG_ST_NO_DIRECTION = 4, /* GMRES found no direction                 error_code 2 */
    MTLG_ST_STALLED = 5       /* refinement: an FP64 outer step failed to halve the
                                 residual (operator too ill-conditioned for the FP32
                                 inner solve); no counterpart in the reference */
};

typedef struct mtlg_ctx mtlg_ctx;
typedef struct mtlg_csr mtlg_csr;
typedef struct mtlg_vec mtlg_vec;
typedef struct mtlg_pc mtlg_pc;
typedef struct mtlg_batch mtlg_batch;
typedef struct mtlg_ell mtlg_ell;
typedef struct mtlg_banded mtlg_banded;
typedef struct mtlg_server mtlg_server;

/* basic_iteration<double>(r0 or norm, max_iter, rtol, atol).  norm_r0 < 0
 * means "take ||b||" as the reference's constructor from b does
 * (basic_iteration.hpp:32-34). */
typedef struct {
    int max_iter;
    int restart;        /* GMRES restart length (gmres.hpp:124-137) */
    double rtol;
    double atol;
    double norm_r0;
} mtlg_iter_params;

typedef struct {
    int iterations;     /* iter.iterations(); total inner iterations for refinement */
    int error_code;     /* iter.error_code(): 0 converged, 1 too many iterations, 2 GMRES */
    int status;         /* MTLG_ST_* */
    int outer_iterations;
    double resid;       /* iter.resid() */
    double relresid;    /* iter.relresid() = resid / norm_r0 */
    double norm_r0;
    double seconds;     /* device time of the solve (CUDA events) */
    int fp64_fallback;  /* refinement: 1 when the system was finished by a plain
                           FP64 solve after the FP32-inner refinement stalled or
                           broke down (iterations then include that solve's) */
    int reserved;
} mtlg_iter_result;

/* FP64 iterative refinement around an FP32 inner Krylov solve. */
typedef struct {
    int max_outer;      /* refinement steps */
    int max_inner;      /* inner iterations per step */
    int restart;
    int pad;
    double rtol;        /* outer: ||b - A x||_FP64 <= rtol * ||b|| */
    double inner_rtol;  /* inner: relative to the step's right-hand side */
} mtlg_refine_params;

/* ---- context -------------------------------------------------------------- */
int mtlg_ctx_create(int device, size_t hbm_budget, mtlg_ctx** out);
int mtlg_ctx_destroy(mtlg_ctx* ctx);
int mtlg_ctx_synchronize(mtlg_ctx* ctx);
/* Use an external cudaStream_t (e.g. torch's current stream); NULL restores
 * the context's own stream. */
int mtlg_ctx_set_stream(mtlg_ctx* ctx, void* cuda_stream);
void* mtlg_ctx_stream(mtlg_ctx* ctx);
/* Kernels this library enqueued on the context since creation (graph replays
 * count every kernel node they run). */
int64_t mtlg_ctx_kernel_launches(mtlg_ctx* ctx);
/* Launch-shape tuning (used by the autotuner): "sweep_blocks_per_sm"
 * (default 1), "sweep_blocks" (absolute grid of the triangular sweeps,
 * overrides the former when > 0), "sweep_sleep_ns" (poll back-off, default
 * 0), "loop_mode" (0: the Krylov loop runs as chunks of 8 iterations in
 * plain CUDA graphs, two in flight; 1: one graph with a WHILE conditional
 * node per solve; 2: the loop bodies launched directly, no graph -- for
 * profilers that do not see kernels inside graphs), "spmv_kernel" (standalone SpMV: 0 chooses by row
 * lengths, 1 shared-memory stream tiles, 2 row-aligned warp tasks, 3 one
 * thread per row from global memory), "sweep_kernel" (0: chunked sweeps,
 * one CTA per chunk of rows, default; 1: flat level-order sweeps),
 * "grid_sweep" (1, default: factors whose pattern is a 5- or 7-point grid
 * stencil in natural order get, at set-up, a layout of x-lines per lane and
 * are swept by the grid kernel when sweep_kernel is 0; 0: chunked or flat
 * only), "grid_warps" (compute warps per grid-sweep CTA: 4 or 8; 0,
 * default: 8 where the shared memory fits, else 4),
 * "chunk_rows" (rows per chunk of preconditioners created afterwards; 0:
 * 16384 for FP32 factors, 8192 for FP64), "sweep_cluster" (CTAs per
 * thread-block cluster of the chunked sweeps, whose neighbouring chunks
 * hand results over through shared memory: 1, 2, 4, 8 or 16; 0, default:
 * chosen per plan), "vec_ctas_per_sm" (CTAs per SM of the fused vector
 * passes, 1-16, default 2), "pc_apply_sync" (1, default:
 * mtlg_pc_apply waits for its sweeps and reports an expired device wait;
 * 0: it only enqueues them, and an expired wait is reported by the next
 * synchronous apply of the same preconditioner), "reduction_order" (FP64
 * dots and norms of mtlg_dot, mtlg_two_norm, mtlg_spmv_dot and the CG /
 * BiCGSTAB solves: 0, default, tile-parallel sums; 1, the reference build's
 * summation order -- four strided partial sums per reduction, combined as
 * mtl::dot, two_norm and the fused lazy dots do -- so that FP64 results and
 * iteration counts equal the reference's bitwise, at about a microsecond
 * per thousand entries per reduction), "admission_free_bytes" (servers
 * without a byte budget admit by the device's free memory; > 0 stands in for
 * cudaMemGetInfo's figure, 0 queries it) and "admission_reserve_bytes"
 * (memory kept out of admission; -1, default: max(1 GiB, 2% of the
 * device)), "spin_limit" (polls before a device-side dependency wait of the
 * triangular sweeps or factorizations gives up and the call returns
 * MTLG_ERR_TIMEOUT; 0, default: 2^20, about half a second; applies to
 * mtlg_pc_apply at once and to solves of preconditioners created
 * afterwards).
 * Read-only keys for get: "sweep_max_blocks_per_sm", "sm_count". */
int mtlg_ctx_set_tuning(mtlg_ctx* ctx, const char* key, int64_t value);
int mtlg_ctx_get_tuning(mtlg_ctx* ctx, const char* key, int64_t* value);
/* Residual log of CG and BiCGSTAB solves made through mtlg_solve: with a
 * capacity > 0 every termination test of the next solves (basic_iteration::
 * finished, basic_iteration.hpp:50-65; BiCGSTAB tests r at the loop top and s
 * mid-iteration) is recorded on the device as (iteration, residual) and read
 * back for the last solve with mtlg_ctx_residual_log: pairs[2k], pairs[2k+1]
 * for k < min(count, capacity); count may exceed the capacity (truncated).
 * Replaying the pairs through finished() gives a cyclic_iteration /
 * noisy_iteration (itl/iteration/cyclic_iteration.hpp:29-95) its per-cycle
 * output.  0 turns the log off (default).  GMRES records no log. */
int mtlg_ctx_set_residual_log(mtlg_ctx* ctx, int capacity);
int mtlg_ctx_residual_log(mtlg_ctx* ctx, double* pairs, int capacity, int* count);
/* Bytes of device memory the context's objects hold. */
size_t mtlg_ctx_bytes_in_use(mtlg_ctx* ctx);
const char* mtlg_status_string(int status);
const char* mtlg_last_error_message(void);

/* ---- tracing (the reference's vampir_trace<N> hooks,
 * boost/numeric/mtl/interface/vpt.hpp:37-78, ids from interface/vpt.cpp) ---
 * Every traced entry point pushes an NVTX range "<id> <name>" (e.g.
 * "7004 bicgstab", "5038 ilu_0::factorize", "3049 crs_cvec_mult"; 9xxx for
 * steps without a reference id: set-up phases, refinement, batch, server).
 * While enabled (this call, or MTLG_TRACE=1 in the environment) each scope
 * also adds its host wall time to a per-event tally; the report is one line
 * per event, "id name calls total_ms".  needed (may be NULL) receives the
 * report's length + 1. */
int mtlg_trace_enable(int on);
int mtlg_trace_reset(void);
int mtlg_trace_report(char* buf, size_t cap, size_t* needed);

/* ---- CSR matrix (compressed2D) --------------------------------------------- */
/* Host arrays are copied.  Columns must be sorted and in range in every row
 * (the reference's trisolves require sorted rows, lower_trisolve.hpp:105). */
int mtlg_csr_create(mtlg_ctx* ctx, int64_t n_rows, int64_t n_cols, int64_t nnz, const int64_t* row_ptr,
                    const int32_t* col, const void* val, mtlg_dtype val_dtype, mtlg_csr** out);
int mtlg_csr_destroy(mtlg_csr* A);
int mtlg_csr_info(const mtlg_csr* A, int64_t* n_rows, int64_t* n_cols, int64_t* nnz);
/* Matrix Market input (the reference's mtl::io::matrix_market_istream >>
 * compressed2D, boost/numeric/mtl/io/matrix_market.hpp:44-214): coordinate
 * or array files with real, integer or pattern values (pattern entries are
 * stored as 0.0, as the reference does) and general, symmetric,
 * skew-symmetric or Hermitian symmetry (off-diagonal entries mirrored as v,
 * -v, v); a later entry at the same position replaces an earlier one; rows
 * sorted by column.  Complex files are refused (MTLG_ERR_FORMAT), as the
 * reference refuses them for a real matrix.  mtlg_mm_read puts the matrix
 * on the device as FP64 CSR; mtlg_mm_read_host fills host arrays (call with
 * null arrays to get the sizes). */
int mtlg_mm_read(mtlg_ctx* ctx, const char* path, mtlg_csr** out);
int mtlg_mm_read_host(const char* path, int64_t* n_rows, int64_t* n_cols, int64_t* nnz, int64_t* row_ptr,
                      int32_t* col, double* val);
/* Replace the values (same pattern), e.g. a new operator with the old graph. */
int mtlg_csr_update_values(mtlg_csr* A, const void* val, mtlg_dtype val_dtype);
/* SpMV tiling statistics: tiles by kind (0 stream, 1 long row, 2 unused). */
int mtlg_csr_plan_info(const mtlg_csr* A, int64_t* tiles_by_kind3, int* max_row_len);

/* ---- ELL and sparse_banded matrices ------------------------------------------ */
/* mtl::mat::ell_matrix (boost/numeric/mtl/matrix/ell_matrix.hpp:31-170) in its
 * own layout: entry j of row r at k = r + j * stride (stride >= n_rows; the
 * reference rounds n_rows up to 32), `slots` entries per row, short rows
 * padded with value 0 (the reference repeats the row's last column there).
 * minor[slots * stride], data likewise (val_dtype).  y (=|+=|-=) E x sums each
 * row's slots in order with rounded products, as the reference build does
 * (operation/mat_vec_mult.hpp:686-700): FP64 bitwise the reference's. */
int mtlg_ell_create(mtlg_ctx* ctx, int64_t n_rows, int64_t n_cols, int64_t slots, int64_t stride,
                    const int64_t* minor, const void* data, mtlg_dtype val_dtype, mtlg_ell** out);
int mtlg_ell_destroy(mtlg_ell* E);
int mtlg_ell_spmv(mtlg_ctx* ctx, mtlg_ell* E, const mtlg_vec* x, mtlg_vec* y, int assign);
/* mtl::mat::sparse_banded (matrix/sparse_banded.hpp:38-160): nbands strictly
 * increasing diagonal offsets (column - row) and the values row by row, one
 * per band (data[r * nbands + b]; entries outside the matrix are ignored).
 * y (=|+=|-=) S x sums each row's bands inside the matrix in increasing order
 * with the reference build's roundings (operation/mat_vec_mult.hpp:704-803:
 * rows in 4-row blocks add rounded products in pairs and fuse an odd last
 * band, other rows with >= 4 bands in fours with the rest fused, shorter ones
 * round every product): FP64 bitwise the reference's.  Rows with no band
 * inside the matrix get 0 for '=' and are left alone by '+=' / '-='. */
int mtlg_banded_create(mtlg_ctx* ctx, int64_t n_rows, int64_t n_cols, int64_t nbands, const int64_t* bands,
                       const void* data, mtlg_dtype val_dtype, mtlg_banded** out);
int mtlg_banded_destroy(mtlg_banded* S);
int mtlg_banded_spmv(mtlg_ctx* ctx, mtlg_banded* S, const mtlg_vec* x, mtlg_vec* y, int assign);

/* ---- dense vectors (dense_vector) ----------------------------------------- */
int mtlg_vec_create(mtlg_ctx* ctx, int64_t n, mtlg_dtype dtype, mtlg_vec** out);   /* zero-filled */
/* Borrow caller-owned device memory (not freed by mtlg_vec_destroy). */
int mtlg_vec_wrap(mtlg_ctx* ctx, int64_t n, mtlg_dtype dtype, void* device_ptr, mtlg_vec** out);
int mtlg_vec_destroy(mtlg_vec* v);
int mtlg_vec_upload(mtlg_vec* v, const void* host, int64_t n);     /* host dtype == vector dtype */
int mtlg_vec_download(const mtlg_vec* v, void* host, int64_t n);
int mtlg_vec_fill(mtlg_vec* v, double value);
void* mtlg_vec_device_ptr(const mtlg_vec* v);
int64_t mtlg_vec_size(const mtlg_vec* v);

/* ---- level-1 / SpMV --------------------------------------------------------- */
/* y (=|+=|-=) A x.  FP64 vectors use the FP64 values, FP32 vectors the FP32
 * copy of the values (made once, on first use).  Rows of up to 32 entries are
 * summed sequentially in storage order, as the reference does. */
int mtlg_spmv(mtlg_ctx* ctx, mtlg_csr* A, const mtlg_vec* x, mtlg_vec* y, int assign);
/* Fused q = A p and the dot p.q (cg.hpp:103 lazy pair) in one pass. */
int mtlg_spmv_dot(mtlg_ctx* ctx, mtlg_csr* A, const mtlg_vec* p, mtlg_vec* q, double* pq);
/* Allocation-free q = A p with p.q, for callers that cannot allocate device
 * memory (a fully reserved budget, a foreign memory pool, a real-time loop
 * where cudaMalloc may block).  No counterpart in the reference.  All
 * pointers are caller-owned device memory (CSR with int32 row_ptr/col, FP64
 * values; *dot written on the device); stream is a cudaStream_t (NULL: the
 * legacy default stream).  Scratch is a file-scope device array of 4096 CTA
 * partial sums (~32 KiB per GPU, held until exit), so n_rows <= 1,048,576
 * (MTLG_ERR_TOO_LARGE beyond); square matrices only.  Calls share that
 * array: calls that can overlap on the GPU race and must be serialized.  The
 * first call on a device looks up the array's address; make it before any
 * stream capture. */
int mtlg_spmv_dot_noalloc(int64_t n_rows, int64_t n_cols, const int32_t* row_ptr, const int32_t* col,
                          const double* val, const double* p, double* q, double* dot, void* stream);
/* Roofline probe (no reference counterpart): one pass that streams A's FP64
 * values and columns and gathers x[col] for every entry, without the row
 * structure -- the memory-system floor of any y = A x on A, to time beside
 * mtlg_spmv.  Partial sums land in a device scratch array of A. */
int mtlg_spmv_gather_floor(mtlg_ctx* ctx, mtlg_csr* A, const mtlg_vec* x);
int mtlg_dot(mtlg_ctx* ctx, const mtlg_vec* x, const mtlg_vec* y, double* out);
int mtlg_two_norm(mtlg_ctx* ctx, const mtlg_vec* x, double* out);
/* y += a x */
int mtlg_axpy(mtlg_ctx* ctx, double a, const mtlg_vec* x, mtlg_vec* y);

/* ---- preconditioners -------------------------------------------------------- */
/* storage = value type of the stored factors / inverse diagonal (the `Value`
 * template argument).  ILU(0)/IC(0) always factorize in FP64 on the GPU. */
int mtlg_pc_create(mtlg_ctx* ctx, mtlg_csr* A, int kind, mtlg_dtype storage, mtlg_pc** out);
int mtlg_pc_destroy(mtlg_pc* P);
/* y = solve(P, x); y = adjoint_solve(P, x).  x and y have the same dtype. */
int mtlg_pc_apply(mtlg_ctx* ctx, mtlg_pc* P, const mtlg_vec* x, mtlg_vec* y);
int mtlg_pc_adjoint_apply(mtlg_ctx* ctx, mtlg_pc* P, const mtlg_vec* x, mtlg_vec* y);
/* Stored factors as CSR on the host (which: 0 = L, 1 = U).  ILU(0): L strict
 * lower with implied unit diagonal, U upper with inverted diagonal first in
 * each row.  IC(0): U with diagonal 1/sqrt(pivot) first, L = trans(U) with
 * the diagonal last.  Call with null arrays to query nnz. */
int mtlg_pc_factor(const mtlg_pc* P, int which, int64_t* nnz, int64_t* row_ptr, int32_t* col, double* val);
/* Number of dependency levels of the L and U sweeps. */
int mtlg_pc_levels(const mtlg_pc* P, int* levels_L, int* levels_U);
/* Launch plan of the sweeps for vectors of `dtype` under the context's
 * current tuning, as 8 integers.  Chunked sweeps: rows per chunk, chunks of
 * L, CTAs resident at once, shared memory per CTA (bytes), compute threads
 * per CTA, entries per row (register bucket), rows and entries per staged
 * segment.  Grid sweeps (grid-stencil factors): 0, 0, CTAs resident at
 * once, shared memory per CTA, compute threads per CTA (two receiver warps
 * more), entries per row, tiles of L, steps per warp unit.  All zero when
 * the flat level-order sweeps run instead.  Not part of the reference's
 * interface (introspection for tuning). */
int mtlg_pc_sweep_plan(mtlg_ctx* ctx, mtlg_pc* P, int dtype, int32_t* out8);
/* Grid structure of a sparse pattern as the triangular sweeps see it: the
 * strictly lower (lower != 0) or strictly upper entries of the n x n CSR
 * pattern (row_ptr, col) are tested for a 5- or 7-point grid stencil in
 * natural order (the preconditioners whose factors pass get the grid sweep
 * and grid factorization).  out8: nx, ny, nz, entries per row, entry order
 * (1 farthest neighbour first, 2 nearest first, 0 none), 1 when rows depend
 * on their neighbours, 0, 0; all zero when the pattern is not a grid
 * stencil (a pattern without entries reports a grid of independent rows).
 * Host-only, no device work.  Not part of the reference's interface
 * (introspection). */
int mtlg_grid_structure(int64_t n, const int64_t* row_ptr, const int32_t* col, int lower, int32_t* out8);

/* ---- solvers ---------------------------------------------------------------- */
/* x is in/out (initial guess on entry).  pc_right may be NULL (identity); CG
 * and BiCGSTAB ignore it as the reference does.  Returns MTLG_OK when the
 * solve ran (convergence is reported in `result`), MTLG_ERR_BREAKDOWN when
 * BiCGSTAB hit a zero rho/gamma/omega (the reference throws). */
int mtlg_solve(mtlg_ctx* ctx, int solver, mtlg_csr* A, mtlg_pc* pc_left, mtlg_pc* pc_right, mtlg_vec* x,
               const mtlg_vec* b, const mtlg_iter_params* params, mtlg_iter_result* result);
/* x, b FP64; the inner solve runs on the FP32 values and FP32 vectors with
 * `pc` (storage FP32, factorized in FP64). */
int mtlg_refine_solve(mtlg_ctx* ctx, int solver, mtlg_csr* A, mtlg_pc* pc, mtlg_vec* x, const mtlg_vec* b,
                      const mtlg_refine_params* params, mtlg_iter_result* result);

/* ---- matrix-free 2D Poisson operator ------------------------------------------ */
/* mtl::mat::poisson2D_dirichlet(m, n) (matrix/poisson2D_dirichlet.hpp:24-80):
 * the 5-point Laplacian on an m x n grid (unknown k = i n + j, Dirichlet
 * boundary) applied without a matrix; results bitwise the reference's.
 * mtlg_poisson2d_solve runs any mtlg_solver except GMRES on it, host-driven,
 * without preconditioning (the reference's tutorial use), FP64 vectors. */
int mtlg_poisson2d_spmv(mtlg_ctx* ctx, int m, int n, const mtlg_vec* x, mtlg_vec* y, int assign);
int mtlg_poisson2d_solve(mtlg_ctx* ctx, int solver, int m, int n, mtlg_vec* x, const mtlg_vec* b,
                         const mtlg_iter_params* params, mtlg_iter_result* result);

/* ---- batched solves ------------------------------------------------------- */
/* Many independent systems of uneven size solved together: every kernel of an
 * iteration covers all unfinished systems.  Each system keeps its own
 * iteration state, so its result does not depend on the others. */
int mtlg_batch_create(mtlg_ctx* ctx, mtlg_batch** out);
int mtlg_batch_destroy(mtlg_batch* B);
/* Adds a system (host arrays copied); returns its index in *index. */
int mtlg_batch_add(mtlg_batch* B, int64_t n, int64_t nnz, const int64_t* row_ptr, const int32_t* col,
                   const double* val, const double* b, int solver, int pc_kind, const mtlg_iter_params* params,
                   int* index);
/* precision MTLG_F64: plain FP64 solves; MTLG_F32: FP32 inner with FP64
 * refinement (refine may be NULL for defaults). */
int mtlg_batch_solve(mtlg_batch* B, int precision, const mtlg_refine_params* refine);
int mtlg_batch_result(const mtlg_batch* B, int index, double* x_host, mtlg_iter_result* result);
int mtlg_batch_size(const mtlg_batch* B);

/* ---- several GPUs (one process per GPU) ------------------------------------- */
/* Independent systems shard by whole systems, with no collective on the data
 * path: every rank computes the same assignment, solves its share on its own
 * GPU, and the results are gathered on the host.  Size-balanced greedy
 * (longest processing time first): by decreasing cost (e.g. nnz + n), each
 * system goes to the part with the least cost so far.  part_of[n_systems]
 * receives the part of each system, part_cost[n_parts] (may be NULL) each
 * part's total.  Host only, needs no GPU.  No reference counterpart (MTL4
 * has no multi-process code). */
int mtlg_partition_systems(int64_t n_systems, const int64_t* cost, int n_parts, int32_t* part_of,
                           int64_t* part_cost);

/* ---- served solves (continuous batching) ----------------------------------- */
typedef struct {
    size_t hbm_budget;        /* bytes the server may hold on the device; 0: admit by
                                 the device's free memory (mtlg_server_admission) */
    int max_active;           /* systems advanced together */
    int iters_per_step;       /* inner iterations per engine step */
    int precision;            /* MTLG_F64 or MTLG_F32 (FP32 inner + FP64 refinement) */
    int pad;
    double rtol;
    double inner_rtol;
} mtlg_server_opts;

typedef struct {
    int64_t submitted, admitted, completed, rejected, cancelled;
    int64_t active, queued;
    int64_t steps;
    size_t bytes_in_use;
} mtlg_server_stats;

int mtlg_server_create(mtlg_ctx* ctx, const mtlg_server_opts* opts, mtlg_server** out);
int mtlg_server_destroy(mtlg_server* S);
/* Queue a request (host arrays copied to pinned staging).  Fails with
 * MTLG_ERR_ADMISSION only if the request could never fit the budget. */
int mtlg_server_submit(mtlg_server* S, int64_t n, int64_t nnz, const int64_t* row_ptr, const int32_t* col,
                       const double* val, const double* b, int solver, int pc_kind, int max_iter,
                       int64_t* request_id);
/* One engine step: admit queued requests that fit, advance every active
 * system by up to iters_per_step iterations, retire finished ones. */
int mtlg_server_step(mtlg_server* S);
/* MTLG_OK with the solution once finished, MTLG_PENDING before. */
int mtlg_server_poll(mtlg_server* S, int64_t request_id, double* x_host, mtlg_iter_result* result);
int mtlg_server_cancel(mtlg_server* S, int64_t request_id);
int mtlg_server_stats_get(const mtlg_server* S, mtlg_server_stats* stats);
/* The server's admission rule (host only, needs no GPU).  With a budget
 * (> 0): admit while held + request <= budget; never when request > budget.
 * Without: free_bytes (cudaMemGetInfo, or the context tuning key
 * "admission_free_bytes") less reserve_bytes (tuning key
 * "admission_reserve_bytes"; default max(1 GiB, 2% of the device)) must hold
 * the request now; otherwise it waits while the server's held bytes would
 * make room once active requests retire, and never fits beyond that.
 * Returns 1 admit, 0 wait, -1 never fits (submit then fails with
 * MTLG_ERR_ADMISSION).  No reference counterpart. */
int mtlg_server_admission(size_t request_bytes, size_t held_bytes, size_t budget, size_t free_bytes,
                          size_t reserve_bytes);

#ifdef __cplusplus
}
#endif
#endif /* MTL4_B200_MTLG_H */
