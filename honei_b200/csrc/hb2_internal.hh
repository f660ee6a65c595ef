// Internal host-side structures shared by the backend's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#include "hb2_common.cuh"

namespace hb2
{
    // Launch shape of the ELL family: blocks of 256 threads, each thread owns
    // kRowsPerThread consecutive rows (one 128-bit load of values per slot for
    // FP64, two rows; four rows for FP32).
    constexpr int kEllThreads = 256;
    // The plain, compressed and Q1 gather kernels also run as blocks of 128 or 512
    // threads, and the plain one with two threads per row: the autotuner times
    // those shapes (their launch bounds are sized for the largest block; the
    // plain kernel with one thread per row takes at most 256).
    constexpr int kEllMaxThreads = 512;
    constexpr uint32_t kMaxReduceBlocks = 1u << 16;

    // Launch with programmatic dependent launch (pdl_entry in the kernel) when
    // HB2_PDL=1: the kernel's blocks may start while the stream's previous
    // kernel finishes (a chain of small kernels, a V-cycle's small levels).
    bool pdl_enabled();
    template <typename... KArgs, typename... Args>
    inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                  Args &&... args)
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = block;
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = pdl_enabled() ? 1 : 0;
        return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
    }

    void count_launches(uint64_t n);
    void set_launch_count(uint64_t n);   // undo the counting of captured (not launched) kernels
    int stream_workspace(cudaStream_t stream, Workspace ** out);

    template <typename T> struct RowsPerThread;
    template <> struct RowsPerThread<double> { static constexpr int value = 2; };
    template <> struct RowsPerThread<float> { static constexpr int value = 4; };

    // Device view of an ELL matrix in the B200 layout: slot-major like the
    // reference (coalesced across rows), int32 column indices, -1 marking the
    // slots past a row's length, leading dimension padded to 64 rows so each
    // slot column starts 256-byte aligned and every vector load is in bounds.
    template <typename T>
    struct EllView
    {
        const T * val;
        const int32_t * col;
        uint64_t rows;
        uint64_t ld;
        uint32_t K;
    };
}

struct hb2_ell_s
{
    int dtype;
    int device;
    uint64_t rows, cols;
    uint32_t K;        // device slots per row (reference num_cols_per_row * threads)
    uint64_t ld;       // device leading dimension
    void * val;        // K * ld values
    int32_t * col;     // K * ld column indices (-1 = empty)
    uint64_t ref_stride, ref_K, ref_T;
    uint64_t bytes;
    // optional compressed layout (ell_compact.cu): 1-byte value codes into
    // `table`, 16-bit column offsets from the row's base column
    uint8_t * code = nullptr;
    int16_t * delta = nullptr;
    void * table = nullptr;
    uint32_t ntable = 0;
    uint64_t compact_bytes = 0;
    int compact_rpt = 2;       // rows per thread of the compressed kernel (autotuned)
    int compact_rpt_red = 2;   // the same for the modes with a fused reduction
    // optional row-pattern layout (ell_pattern.cu, square matrices): 1-byte
    // pattern id per row, npat * K (value, column offset) table entries
    uint8_t * pat = nullptr;
    void * ptab = nullptr;
    uint32_t npat = 0;
    uint64_t pattern_bytes = 0;
    // m when every pattern offset lies in the three bands around -m, 0, +m of a
    // square matrix of m^2 rows (the Q1 operators): the windowed pattern kernel
    // applies (rpt | kPatWin); 0 otherwise
    int64_t pat_win_m = 0;
    // the pattern holding the full nine-point stencil (columns i-m-1 .. i+m+1 in
    // ascending slot order) and its values, or -1: the Q1 stencil kernel applies
    // (rpt | kPatQ1, ell_q1.cu)
    int q1_full = -1;
    double q1_val[9] = {};
    // optional BF16 layout (ell_bf16.cu, F32 matrices made by hb2_ell_create_bf16):
    // bform 0: per slot one 32-bit word (BF16 bits of s * a, 16-bit column offset)
    // in chunks of 32 rows, the chunk's slots one after another; bform 1: BF16
    // values and int32 columns (bidx) slot-major.  With the row-sum compensated
    // form, bdiag holds each row's diagonal remainder (FP32, the BF16 part sits in
    // the diagonal's slot).  val / col hold the same operator in FP32 (a = q / s)
    // for the paths that read them.
    void * bval = nullptr;
    void * bidx = nullptr;
    float * bdiag = nullptr;
    float bscale = 1.f;
    int bform = 0;
    uint64_t bf16_bytes = 0;
    // row patterns of a small square matrix for the fused small-level kernels
    // (subcycle.cu), built on the host when the matrix joins a hierarchy
    uint8_t * spat = nullptr;
    void * sptab = nullptr;     // snpat * K hb2::PatEnt<T>
    uint32_t snpat = 0;
    // layout each kernel class runs on (index 0: no fused reduction, 1: fused
    // reduction): hb2::kLayoutPlain / kLayoutCompact / kLayoutPattern, and
    // its rows per thread
    int layout[2] = {0, 0};
    int rpt[2] = {2, 2};
    // threads per block (128, 256 or 512) and, on the plain layout, threads per
    // row (1 or 2) of each kernel class: autotuned where the kernel takes them
    // (hb2::ell_block), else 256 and 1
    int bs[2] = {hb2::kEllThreads, hb2::kEllThreads};
    int tpr[2] = {1, 1};
    // the Q1 transfer matrices of hb2_ell_create_transfer: +L for the prolongation
    // into fine level L, -L for its transposition, the restriction; 0 otherwise.
    // Their products run on kernels that know the rows' columns and weights
    // (launch_q1_transfer) instead of reading the matrix.
    int q1_transfer = 0;

    template <typename T> hb2::EllView<T> view() const
    {
        hb2::EllView<T> v;
        v.val = (const T *)val;
        v.col = col;
        v.rows = rows;
        v.ld = ld;
        v.K = K;
        return v;
    }
};

struct hb2_q1_s
{
    int dtype;
    uint64_t n, m;
    void * bands;      // 9 * n, band-major LL LD LU DL DD DU UL UD UU
};

namespace hb2
{
    // ELL kernel family (ell.cu).  Modes of the fused epilogue:
    enum EllMode
    {
        kPlain = 0,     // y = A x
        kDefect = 1,    // y = aux - A x             (+ optional ||y||^2)
        kDot = 2,       // y = A x, red = <y, x>
        kAdd = 3,       // y = y + A x
        kJacobi = 4,    // y = x + P (.) (aux - A x) (ping-pong sweep)
        kRestrict = 5,  // y = A x, zero[0..rows) = 0
        kDefectIR = 6,  // FP64 r = aux - A x: (float) r and its ||r|| (the IR outer defect, Q1 kernels only)
        kJacobiNorm = 7 // kJacobi with ||aux - A x||^2 into red: the kernels' template mode when a Jacobi
                        // launch asks for the norm, so that the plain sweep carries no reduction code
    };

    __host__ __device__ constexpr bool is_jacobi(int mode) { return mode == kJacobi || mode == kJacobiNorm; }

    // Pass flags of the ELL family: kReverse walks the row blocks from the end
    // (consecutive passes over one matrix in alternating directions start where
    // the previous pass left its lines in L2); kKeepL2 caches the matrix stream
    // in L2 (ld.cg) instead of marking it evict-first (ld.cs).
    // kSplitSum (set by launch_ell): the fused reduction only stores one partial per
    // block, partials[blockIdx.y * gridDim.x + blockIdx.x], and a second launch
    // (launch_sum_partials) adds them; for launches of many blocks, where the fence
    // and ticket every block of grid_sum_finish waits for before it exits cost more
    // than that launch.
    enum EllFlags
    {
        kReverse = 1,
        kKeepL2 = 2,
        kSplitSum = 4
    };
    constexpr uint64_t kSplitSumMinBlocks = 4096;

    // end of a fused reduction in an ELL kernel: the block's sum, then its partial
    // (kSplitSum) or the two-level finish of grid_sum_finish
    __device__ __forceinline__ void ell_block_reduce(double part, ReduceSlot rs, double * red, int want_sqrt, int flags,
                                                     double * scratch)
    {
        const double s = block_sum(part, scratch);
        if (flags & kSplitSum)
        {
            if (threadIdx.x == 0) rs.partials[(uint64_t)blockIdx.y * gridDim.x + blockIdx.x] = s;
        }
        else grid_sum_finish(s, rs, red, want_sqrt, scratch);
    }

    // out[j] (sqrt when asked) = the sum of partials[j * G .. j * G + G) in a fixed
    // order, j < nvec; one block of 1,024 threads per vector (ell.cu)
    void launch_sum_partials(const double * partials, unsigned G, unsigned nvec, double * out, int want_sqrt,
                             cudaStream_t stream);

    // Batch dimension of the ELL family: nvec vectors stored one after another
    // (vector j of y / aux at element offset j * vstride, of x at j * xstride
    // -- xstride 0 means vstride; a rectangular transfer matrix reads and
    // writes vectors of two levels --, of zero at j * zstride, of red at j);
    // the matrix and aux2 (the Jacobi vector) are shared; a vector whose
    // active[j] is 0 is skipped entirely.  With a work list (list, count on the
    // device) the vectors are list[0 .. *count - 1] instead, walked by a
    // persistent grid, so idle vectors cost no blocks (no fused reduction).
    struct Batch
    {
        uint32_t nvec = 1;
        uint64_t vstride = 0;
        uint64_t xstride = 0;
        uint64_t zstride = 0;          // element offset between the `zero` vectors
        const uint8_t * active = nullptr;
        const uint32_t * list = nullptr;
        const uint32_t * count = nullptr;
        uint32_t gx = 0;               // row blocks per vector (set by launch_ell)
        uint64_t cap = 0;              // blocks of a work-list launch (0: list_grid_cap())
    };

    // Launch one ELL kernel on `stream`.  aux: rhs / b; aux2: Jacobi P; zero:
    // vector cleared by kRestrict; red: device double receiving the fused
    // reduction (nullable, kDefect / kDot); ws: workspace for the reduction
    // (max_blocks must cover the grid times nvec).
    int launch_ell(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux, const void * aux2,
                   void * zero, double * red, int want_sqrt, const Workspace * ws, cudaStream_t stream,
                   int flags = 0, const Batch * batch = nullptr);

    uint64_t list_grid_cap();

    // one slot of a row pattern: value and column - row (kPatEmpty past the row)
    // aligned to its size so that one entry is one 128-bit (FP64) / 64-bit (FP32)
    // shared-memory load
    template <typename T>
    struct alignas(2 * sizeof(T)) PatEnt
    {
        T val;
        int32_t off;
    };
    constexpr int32_t kPatEmpty = (-2147483647 - 1);
    constexpr int kPatWin = 0x10;    // rpt flag: the windowed row-pattern kernel
    constexpr int kPatQ1 = 0x20;     // rpt flag: the Q1 stencil kernel (ell_q1.cu)
    constexpr int kPatQ1G = 0x40;    // rpt flag: the Q1 stencil kernel's gather form (ell_q1.cu)
    constexpr int kPatQ1P = 0x80;    // rpt flag: the Q1 stencil kernel's pair form (ell_q1.cu)
    constexpr int kPatQ1S = 0x100;   // rpt flag: the Q1 stencil kernel's strip form (ell_q1.cu)
    constexpr int kPatFlags = kPatWin | kPatQ1 | kPatQ1G | kPatQ1P | kPatQ1S;
    constexpr int kSubPatMax = 8;    // patterns of a small-level operator in the fused kernels
    int ell_small_patterns(hb2_ell_s * A);

    enum LayoutKind
    {
        kLayoutPlain = 0,
        kLayoutCompact = 1,
        kLayoutPattern = 2,
        kLayoutBF16 = 3
    };
    constexpr int kPatMax = 32;     // patterns per matrix
    constexpr int kPatMaxK = 16;    // slots per row of the pattern layout

    // row blocks of one launch on A for the kernel class (reducing or not), its
    // block size and rows per block, for the kernel of the class's layout (the
    // Q1 gather form where the layout names it)
    unsigned ell_grid(const hb2_ell_s * A, bool reducing);
    unsigned ell_block(const hb2_ell_s * A, bool reducing);
    bool ell_shape_tunable(const hb2_ell_s * A, int cls);   // the class's kernel takes a tuned block size
    uint64_t ell_rows_per_block(const hb2_ell_s * A, bool reducing);

    // row-pattern layout (ell_pattern.cu)
    int ell_build_pattern(hb2_ell_s * A, cudaStream_t stream);
    void ell_free_pattern(hb2_ell_s * A);
    // bs: threads per block of the Q1 gather form (the other pattern kernels run 256)
    void launch_ell_pattern(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux,
                            const void * aux2, void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid,
                            cudaStream_t stream, int flags, Batch b, int R, unsigned bs);

    // Q1 stencil kernel for row-pattern matrices with the full nine-point stencil (ell_q1.cu)
    void ell_find_q1_stencil(hb2_ell_s * A);
    bool ell_q1_stencil_applies(const hb2_ell_s * A, int mode, const void * x, int rpt, const Batch & b);
    unsigned q1_strip_grid(const hb2_ell_s * A, int S, unsigned bs);   // blocks of a strip-form launch
    void launch_ell_q1_stencil(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux,
                               const void * aux2, double * red, int want_sqrt, ReduceSlot rs, dim3 grid,
                               cudaStream_t stream, int flags, int R, unsigned bs);

    // compressed ELL layout (ell_compact.cu)
    int ell_build_compact(hb2_ell_s * A, cudaStream_t stream);
    void ell_free_compact(hb2_ell_s * A);
    void launch_ell_compact(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux,
                            const void * aux2, void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid,
                            cudaStream_t stream, int flags, Batch b, unsigned bs);

    // BF16 layout (ell_bf16.cu)
    void ell_free_bf16(hb2_ell_s * A);
    void launch_ell_bf16(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux,
                         const void * aux2, void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid,
                         cudaStream_t stream, int flags, Batch b, unsigned bs);
    // time the layouts and launch shapes the matrix admits, keep the fastest (ell_compact.cu)
    int ell_autotune(hb2_ell_s * A, cudaStream_t stream);

    // BLAS-1 helpers (blas1.cu) usable from other translation units.
    int launch_fill(int dt, void * x, double value, uint64_t n, cudaStream_t stream);
    int launch_copy(int dt, void * dst, const void * src, uint64_t n, cudaStream_t stream);

    // banded Q1 kernels (q1.cu): mode 0 y = A x, 1 y = rhs - A x, 2 the Jacobi sweep
    // y = x + (rhs - A x) (.) dinv (y != x); err: device flag of the bounded copy wait
    // y = P x, y += P x (kAdd) or y = R x with zero[] cleared (kRestrict) for a matrix
    // with q1_transfer set: the products and slot-ordered sums of its rows, bit-identical
    // to the ELL kernels, without the matrix reads (transfer.cu)
    int launch_q1_transfer(const hb2_ell_s * A, int mode, const void * x, void * y, void * zero,
                           cudaStream_t stream);
    int launch_q1(const hb2_q1_s * A, int mode, const void * x, void * y, const void * rhs, const void * dinv,
                  int * err, cudaStream_t stream);
    int launch_norm(int dt, const void * x, uint64_t n, int root, double * dev_out, const Workspace * ws,
                    cudaStream_t stream);
    int launch_convert(int dst_dt, void * dst, int src_dt, const void * src, uint64_t n, cudaStream_t stream);
    // x64 += (double) c  (IR update, math/ir.hh:73-75)
    int launch_add_converted(void * x64, int c_dt, const void * c, uint64_t n, cudaStream_t stream);
    // IR outer defect of an F64 matrix: r = b - A x, b32 = (float) r, x32 = 0 (x32
    // nullable), red = ||r|| -- one pass on the Q1 stencil kernel, else a defect
    // into r64, a conversion and a fill
    int launch_ir_defect(const hb2_ell_s * A, const double * x, const double * b, float * b32, float * x32,
                         double * r64, double * red, const Workspace * ws, cudaStream_t stream);

    // small levels of a V-cycle as cluster kernels (subcycle.cu)
    struct SubLevelDesc
    {
        const hb2_ell_s * A;
        const hb2_ell_s * R;   // restriction to the next coarser level (levels > 0)
        const hb2_ell_s * P;   // prolongation from the next coarser level (levels > 0)
        void * x;
        void * b;
        void * store;
        void * tmp;
        const void * jac;
    };
    constexpr uint64_t kSubMaxRows = 20000;
    int launch_subcycle(int dtype, const SubLevelDesc * lev, int top, int t1, int n_pre, int n_post, bool down,
                        cudaStream_t stream);
    int subcycle_prepare();
    // the whole bottom of the cycle (levels 0..top, coarsest CG included) in one
    // launch; levels 1..t1 run in one CTA (subcycle.cu)
    constexpr uint64_t kSubLocalRows = 1100;
    bool subvcycle_supported(const hb2_ell_s * coarse, const hb2_ell_s * coarse64);
    int launch_subvcycle(int dtype, const SubLevelDesc * lev, int top, int t1, int n_pre, int n_post,
                         const hb2_ell_s * coarse, const hb2_ell_s * coarse64, uint64_t max_iters, double eps, int exact,
                         uint64_t * used, double * defect, cudaStream_t stream);

    // small-system CG in one thread block (cg.cu); returns HB2_ERR_UNSUPPORTED
    // when the system does not fit in shared memory.
    int launch_cg_small(const hb2_ell_s * A, const void * b, void * x, uint64_t max_iters, double eps, int exact,
                        uint64_t * used_dev, double * defect_dev, cudaStream_t stream);
    bool cg_small_fits(const hb2_ell_s * A);
    bool cg_mixed_supported(const hb2_ell_s * A64);
    int launch_cg_small_f32io(const hb2_ell_s * A64, const void * b32, void * x32, uint64_t max_iters, double eps,
                              int exact, uint64_t * used_dev, double * defect_dev, cudaStream_t stream);
    int launch_cg_warp_batched(const hb2_ell_s * A, int vec_dtype, const void * b, void * x, uint32_t nvec,
                               uint64_t vstride, const uint8_t * active, uint64_t max_iters, double eps,
                               cudaStream_t stream, const uint32_t * list = nullptr, const uint32_t * count = nullptr,
                               uint64_t cap = 0);
}
