/*
 * honei_b200 -- C ABI of the B200 (sm_100a) backend for HONEI's sparse Poisson
 * solver path.
 *
 * This is the drop-in boundary.  It replaces the old CUDA backend's launcher
 * table (honei/backends/cuda/operations.hh:29-128) and the tag glue in
 * honei/la/ *-cuda.cc and honei/math/ *-cuda.cc.  A new HONEI tag, tags::B200,
 * specialises Product, Defect, ScaledSum, DotProduct, Norm,
 * Sum, Scale, Difference, ElementProduct, copy/fill/convert, Prolongation,
 * Restriction and the CG / MG / IR solvers with thin shims over these calls.
 *
 * Conventions
 *   - Plain C: pointers, sizes, enums.  No exceptions cross this boundary.
 *   - Every function returns an int status: HB2_OK (0) or a negative code;
 *     hb2_last_error() gives the message of the last failure on this thread.
 *     Size mismatches that the reference reports as VectorSizeDoesNotMatch /
 *     MatrixRowsDoNotMatch (e.g. la/product.hh:155-162) return
 *     HB2_ERR_SIZE before anything is launched.
 *   - Vector arguments are device pointers of the matrix's element type;
 *     `stream` orders the work (0 = legacy default stream).  Operators are
 *     asynchronous; functions returning host scalars synchronise `stream`.
 *   - Reductions are deterministic: the same inputs and sizes give the same
 *     bits on every run, alone or interleaved with other work.
 *   - Matrices live on the device in a B200 layout (hb2_ell / hb2_q1 handles),
 *     built once from the reference's arrays or assembled on the device.
 */
#ifndef HONEI_B200_H
#define HONEI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define HB2_API __attribute__((visibility("default")))
#else
#define HB2_API
#endif

#ifndef __CUDA_RUNTIME_H__
typedef struct CUstream_st *cudaStream_t;
#endif

typedef enum
{
    HB2_F64 = 0, /* double */
    HB2_F32 = 1  /* float  */
} hb2_dtype;

enum
{
    HB2_OK = 0,
    HB2_ERR_ARG = -1,       /* invalid argument / null pointer */
    HB2_ERR_SIZE = -2,      /* VectorSizeDoesNotMatch / MatrixRowsDoNotMatch */
    HB2_ERR_CUDA = -3,      /* CUDA runtime error */
    HB2_ERR_NOMEM = -4,     /* device allocation failed or over budget */
    HB2_ERR_TIMEOUT = -5,   /* a bounded device-side wait expired */
    HB2_ERR_UNSUPPORTED = -6,
    HB2_ERR_NOT_FINITE = -7 /* a solver produced a NaN/Inf norm */
};

typedef struct hb2_ell_s *hb2_ell; /* SparseMatrixELL<DT> resident on the device */
typedef struct hb2_q1_s *hb2_q1;   /* BandedMatrixQx<Q1Type, DT> resident on the device */
typedef struct hb2_mg_s *hb2_mg;   /* MGData + V-cycle OperatorList resident on the device */
typedef struct hb2_batch_s *hb2_batch; /* many Q1 systems solved together (batched PCG) */
typedef struct hb2_csr_s *hb2_csr; /* SparseMatrixCSR<DT> resident on the device */
typedef struct hb2_krylov_s *hb2_krylov; /* a Krylov solver with its vectors and CUDA graph */
typedef struct hb2_lmg_s *hb2_lmg; /* the legacy banded multigrid solver (MGInfo + its CUDA graph) */

/* ---------------------------------------------------------------- runtime */
HB2_API const char *hb2_last_error(void);
HB2_API const char *hb2_version(void);
/* number of kernels this library launched on this host thread since load */
HB2_API uint64_t hb2_launch_count(void);
/* number of per-(device, stream) reduction workspaces this library has
 * allocated since load (each is created on the first fused reduction on a
 * stream and kept until exit) */
HB2_API uint64_t hb2_workspace_count(void);

/* ---------------------------------------------------------------- matrices */
/* Upload a SparseMatrixELL in the reference layout (la/sparse_matrix_ell-impl.hh:42-72:
 * Aj/Ax of num_cols_per_row*stride slots, slot k of row r at (k%T)+r*T+(k/T)*stride,
 * Arl[r] used slot groups).  Replaces the MemoryArbiter upload of Aj/Ax/Arl that
 * Product<tags::GPU::CUDA>(DV, SMELL, DV) performs (la/product-cuda.cc:197-231).
 * host_ptrs != 0: Aj/Ax/Arl are host pointers; else device pointers. */
HB2_API int hb2_ell_create(hb2_ell *out, hb2_dtype dtype, uint64_t rows, uint64_t cols, uint64_t stride,
                   uint64_t num_cols_per_row, uint64_t threads, const uint64_t *Aj, const void *Ax,
                   const uint64_t *Arl, int host_ptrs, cudaStream_t stream);
/* Assemble on the device the level-L Q1 Poisson operator that
 * FillMatrix<Tag, POISSON, DIRICHLET_0> (math/fill_matrix.hh:37-79) followed by
 * SparseMatrixELL(SparseMatrix(BandedMatrixQx)) (la/sparse_matrix_ell-impl.hh:75-122)
 * produces; aniso != 1 scales the x-coupling (DL/DU) and the diagonal. */
HB2_API int hb2_ell_create_q1(hb2_ell *out, hb2_dtype dtype, unsigned level, double aniso, cudaStream_t stream);
/* Assemble on the device P = ProlongationMatrix (level-1 -> level) with identity
 * index maps (math/prolongation_matrix.hh:44-100) and its transpose R
 * (math/transposition.hh:36-50), both as ELL.  Their single-vector products
 * (hb2_product_ell, hb2_product_add_ell, the MG hierarchy's transfers) run on
 * kernels that derive each row's columns and weights from the grid instead of
 * reading the matrix, with the same bits; HB2_Q1_TRANSFER=0 reads the matrices. */
HB2_API int hb2_ell_create_transfer(hb2_ell *prol, hb2_ell *res, hb2_dtype dtype, unsigned fine_level,
                            cudaStream_t stream);
/* Same matrix in another element type (values rounded like DT(double)). */
HB2_API int hb2_ell_convert(hb2_ell *out, hb2_ell src, hb2_dtype dtype, cudaStream_t stream);
HB2_API int hb2_ell_destroy(hb2_ell A);
/* rows, cols, reference stride / num_cols_per_row / threads, device bytes */
HB2_API int hb2_ell_info(hb2_ell A, uint64_t *rows, uint64_t *cols, uint64_t *stride, uint64_t *num_cols_per_row,
                 uint64_t *threads, uint64_t *device_bytes);
/* Device layout the matrix-vector kernels (no fused reduction) run on, chosen by
 * timing at creation among the lossless layouts the matrix admits:
 *   *layout = 0  plain: values + int32 columns (*table_size = 0);
 *             1  compressed: 1-byte value codes into a table of *table_size
 *                distinct values + 16-bit column offsets from the row;
 *             2  row patterns (square matrices): a 1-byte pattern id per row into
 *                a table of *table_size patterns of (value, column - row) slots;
 *             3  BF16 values + 16-bit offsets or int32 columns (hb2_ell_create_bf16).
 * *row_bytes = matrix bytes read per row.  Every layout gives the same bits.
 * No counterpart in the reference (its device copy is the raw arrays). */
HB2_API int hb2_ell_layout(hb2_ell A, int *layout, uint32_t *table_size, uint32_t *row_bytes);
/* The kernel behind that choice, per kernel class (cls 0: products, sweeps and
 * transfers; 1: defects with a fused norm): its layout (as above), rows per thread,
 * and *windowed = the kernel kind on the row-pattern layout (0 general, 1 x staged
 * in shared-memory windows, 2 / 3 / 4 / 5 the Q1 stencil kernel's bulk-copy, gather,
 * pair and strip forms).  No counterpart in the reference. */
HB2_API int hb2_ell_layout_variant(hb2_ell A, int cls, int *layout, int *rows_per_thread, int *windowed);
/* Launch shape of that kernel: threads per block (128, 256 or 512; timed by the
 * autotuner for the plain, compressed and Q1 gather kernels, 256 for the others;
 * at most 256 for the plain kernel with one thread per row) and threads per row
 * (1, or 2 on the plain layout).  HB2_ELL_BLOCK and
 * HB2_ELL_TPR override the tuned values for matrices created while they are set.
 * The reference's counterparts are its block-size settings
 * (honei/honeirc:50-51) and the T threads per row of the ELL kernel
 * (backends/cuda/product.cu:148-200); every shape gives the same bits. */
HB2_API int hb2_ell_launch_shape(hb2_ell A, int cls, int *block_threads, int *threads_per_row);
/* Download the matrix in the reference layout (host arrays of K*stride, K*stride
 * and rows elements); Arl as the reference computes it. */
HB2_API int hb2_ell_export(hb2_ell A, uint64_t *Aj, void *Ax, uint64_t *Arl);
/* MatrixIO<io_formats::ELL>::read_matrix / write_matrix (math/matrix_io.hh:433-560):
 * the reference's binary ELL file (five uint64: size, rows, columns, stride,
 * num_cols_per_row; then size uint64 column indices and size doubles), read
 * into the device layout (values rounded to dtype) or written from an F64
 * matrix with one thread per row. */
HB2_API int hb2_ell_read(hb2_ell *out, const char *path, hb2_dtype dtype, cudaStream_t stream);
HB2_API int hb2_ell_write(hb2_ell A, const char *path);
/* Transposition<Tag>::value (math/transposition.hh:36-50): A^T assembled like the
 * reference (each row's entries in ascending column order); MGUtil::load_data
 * builds every restriction matrix this way from its prolongation. */
HB2_API int hb2_ell_transpose(hb2_ell *out, hb2_ell A, cudaStream_t stream);
/* A BF16-stored copy of A for the FP32 inner solve of mixed-precision iterative
 * refinement: every entry stored as q = bf16(s * a) (one rounding from the double
 * s * a, to nearest, ties to even), s the first of 1, 3, ..., 15 with the smallest
 * largest relative rounding error of the stored entries (3 for the Q1 operator:
 * 8, -1 and 3 exactly), column offsets in 16 bits where they fit.  compensate = 1
 * (square matrices): the diagonal in FP32, each row's diagonal absorbing the
 * rounding errors of its off-diagonal entries, d = s a_ii + sum (s a_ij - q_ij),
 * so the row sums of s * A are kept.  Products accumulate in FP32 (fmaf, slot
 * order) and divide by s once per row; the vectors are F32 and *out is an F32
 * matrix (hb2_ell_layout reports layout 3) usable wherever an F32 ELL matrix is,
 * its plain arrays holding q / s.  *scale and *max_rel_error (nullable): s and
 * that largest error.  No counterpart in the reference. */
HB2_API int hb2_ell_create_bf16(hb2_ell *out, hb2_ell A, int compensate, double *scale, double *max_rel_error,
                                cudaStream_t stream);

/* SparseMatrixCSR<DT>(blocksize, rows, columns, Aj, Ax, Ar, used) (la/sparse_matrix_csr-impl.hh:40-71,
 * 140-145): Ar[rows + 1] block offsets, Aj[Ar[rows]] first column of each block,
 * Ax[Ar[rows] * blocksize] values (dtype).  Replaces the upload that
 * Product<tags::GPU::CUDA>(DV, SMCSR, DV) performs (la/product-cuda.cc:317-400).
 * host_ptrs != 0: host arrays; else device arrays. */
HB2_API int hb2_csr_create(hb2_csr *out, hb2_dtype dtype, uint64_t rows, uint64_t cols, uint64_t blocksize,
                   const uint64_t *Ar, const uint64_t *Aj, const void *Ax, int host_ptrs, cudaStream_t stream);
/* SparseMatrixCSR(SparseMatrixELL) (la/sparse_matrix_csr-impl.hh:85-135) with csr::blocksize = blocksize */
HB2_API int hb2_csr_from_ell(hb2_csr *out, hb2_ell A, uint64_t blocksize, cudaStream_t stream);
HB2_API int hb2_csr_destroy(hb2_csr A);
/* rows, cols, blocksize, blocks (Ar[rows]), device bytes */
HB2_API int hb2_csr_info(hb2_csr A, uint64_t *rows, uint64_t *cols, uint64_t *blocksize, uint64_t *nblocks,
                 uint64_t *device_bytes);
/* Ar (rows + 1), Aj (blocks), Ax (blocks * blocksize) into host arrays */
HB2_API int hb2_csr_export(hb2_csr A, uint64_t *Ar, uint64_t *Aj, void *Ax);
/* Device layout the products run on: rows of at most 128 entries in 32-row
 * slices stored slot-major (SELL-C-sigma; *slots = slots incl. padding), longer
 * rows as 128-entry chunks (*long_rows, *long_entries); *unroll = slots per lane
 * and round (8 or 16, timed at creation). */
HB2_API int hb2_csr_layout(hb2_csr A, uint64_t *slots, uint64_t *long_rows, uint64_t *long_entries, uint32_t *unroll);

/* BandedMatrixQx<Q1Type, DT> (la/banded_matrix_qx-impl.hh:45-466): 9 bands of n,
 * band-major LL LD LU DL DD DU UL UD UU; n must be (2^L+1)^2. */
HB2_API int hb2_q1_create(hb2_q1 *out, hb2_dtype dtype, uint64_t n, const void *bands, int host_ptrs,
                  cudaStream_t stream);
HB2_API int hb2_q1_create_poisson(hb2_q1 *out, hb2_dtype dtype, unsigned level, double aniso, cudaStream_t stream);
HB2_API int hb2_q1_destroy(hb2_q1 A);

/* ---------------------------------------------------------------- operators */
/* Product<Tag>::value(y, A, x) on ELL (la/product.hh:148-206; old CUDA launcher
 * cuda_product_smell_dv_{float,double}, backends/cuda/operations.hh:93-99). */
HB2_API int hb2_product_ell(hb2_ell A, const void *x, void *y, cudaStream_t stream);
/* Product<Tag>::value(y, A, x) on CSR (la/product.hh:208-244; old launcher
 * cuda_product_csr_dv_{float,double}, backends/cuda/operations.hh:95-99): each row
 * one fma chain over its blocks in order, a block value past x skipped. */
HB2_API int hb2_product_csr(hb2_csr A, const void *x, void *y, cudaStream_t stream);
/* Defect<Tag>::value(r, rhs, A, x) on CSR (math/defect.hh:385-420; old launcher
 * cuda_defect_csr_dv_*, operations.hh:49-53): r = rhs - (the product's row sum). */
HB2_API int hb2_defect_csr(hb2_csr A, const void *rhs, const void *x, void *r, cudaStream_t stream);
/* Defect<Tag>::value(r, rhs, A, x) = rhs - A x (math/defect.hh:357-383; old launcher
 * cuda_defect_smell_dv_*, operations.hh:40-46).  norm2_dev (nullable, device double):
 * receives ||r||_2^2 computed in the same pass (Norm<vnt_l_two,false>, la/norm.hh:290-305). */
HB2_API int hb2_defect_ell(hb2_ell A, const void *rhs, const void *x, void *r, double *norm2_dev,
                   cudaStream_t stream);
/* Defect with the fused ||r||_2^2 like hb2_defect_ell, but allocating nothing:
 * no counterpart in the reference.  For callers that must not allocate device
 * memory (a hard device-memory budget with every byte reserved up front, or a
 * latency-critical loop where a cudaMalloc would stall the device):
 * hb2_defect_ell's reduction workspace is cudaMalloc'd on first use of a stream,
 * this variant keeps the reduction scratch in a fixed file-scope device array
 * (about 134 KiB per GPU that loads the library, held until exit).  norm2_dev
 * is required.  Limit: at most 8,388,608 rows in F64 and 16,777,216 in F32;
 * larger matrices return HB2_ERR_UNSUPPORTED before any launch.  The answer
 * depends on the row count and element type only (a tuned layout whose row
 * blocks would not fit the scratch runs with more rows per thread: the same
 * defect bits; the norm within rounding of hb2_defect_ell's).  All calls on a
 * device share the array, so calls that overlap on the GPU race; calls ordered on
 * one stream are safe.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and caches it: make it before any stream capture. */
HB2_API int hb2_defect_ell_noalloc(hb2_ell A, const void *rhs, const void *x, void *r, double *norm2_dev,
                                   cudaStream_t stream);
/* y = A x and dot_dev = <y, x> in one pass (the CG step Product + DotProduct, math/cg.hh:97-98) */
HB2_API int hb2_product_dot_ell(hb2_ell A, const void *x, void *y, double *dot_dev, cudaStream_t stream);
/* y += A x (Prolongation<PROLMAT> followed by Sum, math/mg.hh:627-629) */
HB2_API int hb2_product_add_ell(hb2_ell A, const void *x, void *y, cudaStream_t stream);
/* Product<Tag>(y, BandedMatrixQx<Q1>, x) (la/product.hh:370-403; old launcher
 * cuda_product_bmdv_q1_*, operations.hh:82-90) and Defect on Q1 (math/defect.hh:194-198;
 * cuda_defect_q1_*, operations.hh:30-38). */
HB2_API int hb2_product_q1(hb2_q1 A, const void *x, void *y, cudaStream_t stream);
HB2_API int hb2_defect_q1(hb2_q1 A, const void *rhs, const void *x, void *r, cudaStream_t stream);

/* BLAS-1 on DenseVector<DT> (n elements, device pointers):
 *   ScaledSum x += b*y        la/scaled_sum.hh:73-88   (cuda_scaled_sum_*, operations.hh:117-120)
 *   ScaledSum r = b*y + x     la/scaled_sum.hh:91-110
 *   Sum x += y                la/sum.hh                (cuda_sum_two_*, operations.hh:125-126)
 *   Difference x -= y; r = x - y   la/difference.hh    (cuda_difference_*, operations.hh:54-57)
 *   Scale x *= a              la/scale.hh              (cuda_scale_one_*, operations.hh:122-123)
 *   ElementProduct r = a (.) b la/element_product.hh / la/product.hh:1198-1204
 *   fill, copy, convert       la/algorithm.hh:50-86, 370-440, 163-245 (transfer.cu:28-46)
 * DotProduct / Norm write a device double (nullable) and, when host_out is
 * non-null, synchronise and store it on the host (la/dot_product.hh:72-89,
 * la/norm.hh:290-381; the old launchers finished the sum on the host,
 * backends/cuda/dot_product.cu:101-105). */
HB2_API int hb2_scaled_sum(hb2_dtype dt, void *x, const void *y, double b, uint64_t n, cudaStream_t stream);
HB2_API int hb2_scaled_sum3(hb2_dtype dt, void *r, const void *x, const void *y, double b, uint64_t n,
                    cudaStream_t stream);
HB2_API int hb2_sum(hb2_dtype dt, void *x, const void *y, uint64_t n, cudaStream_t stream);
HB2_API int hb2_difference(hb2_dtype dt, void *x, const void *y, uint64_t n, cudaStream_t stream);
HB2_API int hb2_difference3(hb2_dtype dt, void *r, const void *x, const void *y, uint64_t n, cudaStream_t stream);
HB2_API int hb2_scale(hb2_dtype dt, void *x, double a, uint64_t n, cudaStream_t stream);
HB2_API int hb2_element_product(hb2_dtype dt, void *r, const void *a, const void *b, uint64_t n,
                        cudaStream_t stream);
HB2_API int hb2_fill(hb2_dtype dt, void *x, double value, uint64_t n, cudaStream_t stream);
HB2_API int hb2_copy(hb2_dtype dt, void *dst, const void *src, uint64_t n, cudaStream_t stream);
HB2_API int hb2_convert(hb2_dtype dst_dt, void *dst, hb2_dtype src_dt, const void *src, uint64_t n,
                cudaStream_t stream);
HB2_API int hb2_dot(hb2_dtype dt, const void *x, const void *y, uint64_t n, double *dev_out, double *host_out,
            cudaStream_t stream);
HB2_API int hb2_norm_l2(hb2_dtype dt, const void *x, uint64_t n, int root, double *dev_out, double *host_out,
                cudaStream_t stream);
/* DotProduct<tags::CPU> / Norm<vnt_l_two, root, tags::CPU> in the reference's own
 * summation order (la/dot_product.hh:72-89: one sequential fma chain in the element
 * type; la/norm.hh:363-381: sqrt in the element type): its bits, at the speed of one
 * thread.  For bit-for-bit comparisons with the reference; hb2_dot / hb2_norm_l2 are
 * the fast (tree-ordered) reductions.  Same outputs as hb2_dot. */
HB2_API int hb2_dot_ordered(hb2_dtype dt, const void *x, const void *y, uint64_t n, int root, double *dev_out,
                            double *host_out, cudaStream_t stream);

/* ---------------------------------------------------------------- grid transfer */
/* Matrix-free Prolongation<Tag, NONE> (math/prolongation.hh:42-139) and
 * Restriction<Tag, NONE> (math/restriction.hh:41-173), each followed by
 * ApplyDirichletBoundaries with the 8-entry mask (host array; 2 = Dirichlet,
 * math/apply_dirichlet_boundaries.hh:29-84).  Old launchers:
 * cuda_prolongation_* / cuda_restriction_* (operations.hh:101-111).
 * Bit-identical to the reference (same summation order per node). */
HB2_API int hb2_prolongation(hb2_dtype dt, void *fine, uint64_t n_fine, const void *coarse, uint64_t n_coarse,
                     const uint64_t *mask, cudaStream_t stream);
HB2_API int hb2_restriction(hb2_dtype dt, void *coarse, uint64_t n_coarse, const void *fine, uint64_t n_fine,
                    const uint64_t *mask, cudaStream_t stream);

/* ---------------------------------------------------------------- solvers */
/* RISmoother<Tag>::value(A, P, b, x, temps, iters) (math/ri.hh:110-133): `sweeps`
 * damped-Jacobi sweeps x += P (.) (b - A x), fused into one pass per sweep.
 * tmp: device vector of A.rows (ping-pong buffer). */
HB2_API int hb2_jacobi_ell(hb2_ell A, const void *P, const void *b, void *x, void *tmp, uint64_t sweeps,
                   cudaStream_t stream);
/* One sweep of RISmoother (math/ri.hh:125-129) into a separate output:
 * x_out = x_in + P (.) (b - A x_in), one fused pass (no copy). */
HB2_API int hb2_jacobi_sweep_ell(hb2_ell A, const void *P, const void *b, const void *x_in, void *x_out,
                                 cudaStream_t stream);
/* P = omega / diag(A): PreconFill "jac" (math/mg.hh:266-273) */
HB2_API int hb2_jacobi_precon(hb2_ell A, double omega, void *P, cudaStream_t stream);

/* CGSolver<Tag, methods::NONE>::value(A, P, b, x, max_iters, used_iters, eps)
 * (math/cg.hh:64-135): unpreconditioned CG with the reference's relative-or-
 * absolute stop sqrt(r.r) < eps*||r0|| or < eps.  One cooperative launch per
 * solve; all scalars stay on the device.  final_defect: sqrt(r.r) at exit.
 * Synchronises `stream`. */
HB2_API int hb2_cg_solve(hb2_ell A, const void *b, void *x, uint64_t max_iters, double eps, uint64_t *used_iters,
                 double *final_defect, cudaStream_t stream);

/* Krylov solvers with a variable preconditioner, FP64:
 *   HB2_CG_VAR        CGSolver<Tag, methods::VAR> (math/cg.hh:142-210)
 *   HB2_BICGSTAB_VAR  BiCGStabSolver<Tag, methods::VAR> (math/bicgstab.hh:60-210)
 *   HB2_CG_SMOOTHER   CGSmoother (math/cg.hh:217-290): exactly max_iters steps
 * P is either the ELL matrix P or the vector pdiag (n doubles, host or device,
 * copied: the element-wise product P (.) r); the other is NULL.  The handle
 * keeps a reference to A and P (they must outlive it) and owns its vectors and
 * the CUDA graph of the solve (prefix, a conditional WHILE node over the
 * iterations, IF nodes for BiCGStab's early exits). */
enum { HB2_CG_VAR = 0, HB2_BICGSTAB_VAR = 1, HB2_CG_SMOOTHER = 2 };
HB2_API int hb2_krylov_create(hb2_krylov *out, int method, hb2_ell A, hb2_ell P, const double *pdiag,
                      uint64_t max_iters, double eps_relative, cudaStream_t stream);
HB2_API int hb2_krylov_destroy(hb2_krylov K);
/* b, x: device vectors (x: initial guess in, result out).  used_iters: the
 * reference's used_iters (CG VAR: the iteration that met a stop test, 0 if none
 * ran; BiCGStab: iterations + 1; smoother: max_iters); final_defect: ||r||
 * (CG VAR), the squared defect norm (BiCGStab, as the reference's
 * Norm<vnt_l_two, false>), 0 (smoother).  Synchronises `stream`. */
HB2_API int hb2_krylov_solve(hb2_krylov K, const void *b, void *x, uint64_t *used_iters, double *final_defect,
                     cudaStream_t stream);

/* The legacy multigrid solver Multigrid<Tag, OuterTag, methods::NONE, methods::JAC,
 * methods::CYCLE::V, methods::FIXED> on BandedMatrixQx (math/multigrid.hh:151-466,
 * 781-825): its MGInfo configuration (math/multigrid.hh:65-149); the levels'
 * diags_inverted are built as the reference's tests build them, omega * (1 / DD). */
typedef struct
{
    uint64_t n_max_iter;               /* 16: cycles at most */
    int initial_zero;                  /* 1: d = b (the initial guess is not applied to the defect) */
    int convergence_check;             /* 0: skip the solve when ||d0|| <= tolerance */
    int is_smoother;                   /* 0: 1 = no norms, exactly n_max_iter cycles */
    double tolerance;                  /* 1e-8: stop when ||d|| <= ||d0|| * tolerance */
    uint64_t n_pre_smooth;             /* 2: Jacobi sweeps before and after the coarse correction */
    double adapt_correction_factor;    /* 1.0: x += factor * P x(coarser) */
    double omega;                      /* 0.7 */
    uint64_t macro_border_mask[8];     /* 2 = Dirichlet, 1 = Neumann (edges and corners) */
    int adaptive;                      /* 0; 1 = the MIXED class's kernel: a correction factor of 0
                                          means alpha = <d, c> / <A c, c> (math/multigrid.hh:1712-1721) */
} hb2_lmg_params;
/* A: max_level - min_level + 1 banded matrices, levels min_level (>= 1) .. max_level,
 * one element type; the handle keeps references to them. */
HB2_API int hb2_lmg_create(hb2_lmg *out, unsigned min_level, unsigned max_level, const hb2_q1 *A,
                   const hb2_lmg_params *params, cudaStream_t stream);
HB2_API int hb2_lmg_destroy(hb2_lmg mg);
/* Multigrid::value(system, b, x, ...): b, x device vectors of the finest level (x:
 * initial guess in -- its first row, last row and first column replaced by b's values
 * -- result out).  cycles: cycles run; defect: the last ||d|| of the finest level.
 * Synchronises `stream`. */
HB2_API int hb2_lmg_solve(hb2_lmg mg, const void *b, void *x, uint64_t *cycles, double *defect, cudaStream_t stream);
/* Multigrid<Tag, OuterTag, NONE, JAC, CYCLE::V, MIXED>::value (math/multigrid.hh:2252-2394):
 * `mg` an F32 hierarchy (its MGInfo), A the F64 finest matrix, b and x F64 device vectors.
 * The FP64 defect of the initial guess (b's Dirichlet values applied) is scaled into the
 * inner right-hand side, the inner kernel runs on its persistent iterate, result (from 0)
 * += scale x_inner, until ||b - A result|| < tolerance (the MGInfo's, through float)
 * times the initial norm; at most max_outer outer steps (the reference has no cap:
 * HB2_ERR_NOT_FINITE when it is reached).  Synchronises `stream`. */
HB2_API int hb2_lmg_solve_mixed(hb2_lmg mg, hb2_q1 A, const void *b, void *x, uint64_t max_outer,
                        uint64_t *outer_steps, uint64_t *inner_cycles, double *final_defect, cudaStream_t stream);

/* MG hierarchy: MGData (math/mg.hh:57-240) + MGCycleCreation<V::STATIC,
 * CGSolver<NONE>, RISmoother, Restriction<PROLMAT>, Prolongation<PROLMAT>>
 * (math/mg.hh:567-656), captured once as a CUDA graph.  Levels are given
 * coarsest first: A[0..nlev-1]; prol[i], res[i] connect level i and i+1
 * (i = 0..nlev-2).  Jacobi P = omega/diag(A) per level.  The handle keeps
 * references to the matrices (they must outlive it) and owns its vectors. */
typedef struct
{
    uint64_t n_pre_smooth, n_post_smooth;   /* 4, 4 */
    uint64_t max_iters;                     /* MG cycles */
    uint64_t max_iters_coarse;              /* coarse CG iterations */
    double eps_relative;                    /* MG stop: ||r|| < eps * ||r0|| */
    double coarse_eps;                      /* coarse CG eps (reference: = eps_relative) */
    double omega;                           /* Jacobi damping, 0.7 */
    int coarse_exact;                       /* 1: coarse CG dots in the reference's sequential fma order */
    int no_fused_levels;                    /* 1: one kernel per operator on every level (0: levels below
                                               ~20k rows run as two thread-block-cluster kernels per cycle) */
    int coarse_fp64;                        /* F32 hierarchies: 1 runs the coarsest CG in FP64 on an FP64 copy
                                               of the coarse operator (<= 128 rows, 1-9 slots); 0: FP32 as the reference */
    int cycle;                              /* 0: V-cycle (MGCycleCreation<V::STATIC>, math/mg.hh:567-656);
                                               1: W-cycle (MGCycleCreation<W::STATIC>, math/mg.hh:658-740) */
} hb2_mg_params;

HB2_API int hb2_mg_create(hb2_mg *out, uint32_t num_levels, const hb2_ell *A, const hb2_ell *prol, const hb2_ell *res,
                  const hb2_mg_params *params, cudaStream_t stream);
/* Q1 Poisson hierarchy min_level..max_level assembled on the device */
HB2_API int hb2_mg_create_q1(hb2_mg *out, hb2_dtype dtype, unsigned min_level, unsigned max_level, double aniso,
                     const hb2_mg_params *params, cudaStream_t stream);
HB2_API int hb2_mg_destroy(hb2_mg mg);
/* MGSolver<Tag, Norm<vnt_l_two, true>>::value(data, cycle) (math/mg.hh:1094-1127):
 * b, x: finest-level device vectors (x = initial guess in, solution out).
 * stats (nullable, host, 4 doubles): used_iters, ||r0||, ||r_final||, coarse iters
 * of the last cycle.  Synchronises `stream`. */
HB2_API int hb2_mg_solve(hb2_mg mg, const void *b, void *x, double *stats, cudaStream_t stream);
/* one V-cycle on the finest level (OperatorList::value, math/operator_list.hh:69-76) */
HB2_API int hb2_mg_cycle(hb2_mg mg, const void *b, void *x, cudaStream_t stream);

/* IRSolver<OuterTag, InnerTag, Norm> (math/ir.hh:31-80): FP64 outer defect, norm
 * and update around an inner MG solve on `inner` (an F32 or F64 hierarchy whose
 * finest level matches A).  reset_inner = 0 keeps the reference's behaviour
 * (inner initial guess carried over); 1 restarts it from zero each outer step.
 * stats (nullable, host, 4 doubles): outer iters, ||r0||, ||r_final||, total
 * inner cycles.  Synchronises `stream`. */
HB2_API int hb2_ir_solve(hb2_ell A, hb2_mg inner, const void *b, void *x, double eps, uint64_t max_iters,
                 int reset_inner, double *stats, cudaStream_t stream);

/* Batched solves: num_systems Q1 Poisson systems (level levels[s], nrhs[s]
 * right-hand sides each, nrhs NULL = 1) solved together by
 * CGSolver<Tag, methods::VAR> (math/cg.hh:142-210) with an MG V-cycle as the
 * variable preconditioner.  Outer recurrence, dots, norms and stop test FP64 on
 * the FP64 operator; the preconditioner is one V-cycle (Jacobi omega,
 * n_pre/n_post sweeps, bilinear transfers) in FP32 with the coarsest-level CG
 * (level coarse_level, 1..3) in FP64 arithmetic.  Each PCG step of the whole
 * batch is one CUDA graph whose launch count depends on the deepest hierarchy,
 * not on the number of systems: every stage is one launch over the (row block,
 * right-hand side) pairs of all systems at that level.  A right-hand side's
 * iterates do not depend on which other systems share the batch. */
typedef struct
{
    uint64_t max_iters;                     /* PCG iterations per right-hand side (100) */
    double eps_relative;                    /* default stop ||r|| < eps ||r0|| or ||r|| < eps (1e-8) */
    uint64_t n_pre_smooth, n_post_smooth;   /* 4, 4 */
    uint64_t max_iters_coarse;              /* coarse CG iterations (100) */
    double coarse_eps;                      /* coarse CG relative tolerance (1e-10) */
    double omega;                           /* Jacobi damping (0.7) */
} hb2_batch_params;

HB2_API int hb2_batch_create_q1(hb2_batch *out, uint32_t num_systems, const uint32_t *levels, const uint32_t *nrhs,
                        unsigned coarse_level, const hb2_batch_params *params, cudaStream_t stream);
HB2_API int hb2_batch_destroy(hb2_batch B);
/* right-hand sides in total, device bytes held, kernel launches per PCG step */
HB2_API int hb2_batch_info(hb2_batch B, uint32_t *num_vectors, uint64_t *device_bytes, uint64_t *launches_per_step);
/* which = 0: set b, 1: set x (initial guess), 2: read x.  buf (host or device)
 * holds the system's nrhs vectors of (2^level+1)^2 doubles one after another. */
HB2_API int hb2_batch_copy(hb2_batch B, uint32_t system, int which, void *buf, cudaStream_t stream);
/* queue a system for solving at the next step (eps_relative <= 0: the default);
 * zero_guess = 1 starts from x = 0, else from the x it holds */
HB2_API int hb2_batch_start(hb2_batch B, uint32_t system, double eps_relative, int zero_guess, cudaStream_t stream);
/* run `steps` PCG steps of every queued or running system; done (nullable, host,
 * num_systems bytes) receives 1 for each system with nothing left to do.
 * Synchronises `stream`. */
HB2_API int hb2_batch_step(hb2_batch B, uint32_t steps, uint8_t *done, cudaStream_t stream);
/* start every system and step until all are done, in one graph launch (the loop
 * runs on the device); steps (nullable) receives the number of steps.
 * Synchronises `stream`. */
HB2_API int hb2_batch_solve(hb2_batch B, int zero_guess, uint64_t *steps, cudaStream_t stream);
/* iterations and final ||r||/||r0|| of one right-hand side, as of the last
 * hb2_batch_step / hb2_batch_solve */
HB2_API int hb2_batch_result(hb2_batch B, uint32_t system, uint32_t rhs, uint64_t *iters, double *rel_defect);

#ifdef __cplusplus
}
#endif
#endif
