// SparseMatrixELL on the B200: device layout, device-side assembly of the Q1
// Poisson operator and the grid-transfer matrices, and the fused ELL kernel
// family (SpMV, defect, defect+norm, SpMV+dot, SpMV-add, Jacobi sweep,
// restriction+clear).
//
// Layout.  The reference stores num_cols_per_row x stride slots, slot k of row r
// at (k%T) + r*T + (k/T)*stride with uint64 column indices
// (la/sparse_matrix_ell-impl.hh:75-122).  The product loop visits the
// Arl[r]*T entries of a row in that order (la/product.hh:148-206).  On the
// device every row's entries are flattened into K = num_cols_per_row*T slots in
// the same visiting order, slot-major with leading dimension ld (rows rounded
// up to 64), int32 columns and -1 past the row's length.  Each slot column is a
// contiguous run over rows, so a warp's loads of one slot are fully coalesced
// 128-bit vector loads, and the index stream is half the reference's bytes.
//
// Arithmetic.  Products and sums are rounded separately (no fma), in slot
// order, exactly like the reference's compiled tags::CPU loop, so SpMV, defect
// and the Jacobi sweep are bit-identical to it.
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <algorithm>
#include <cstdlib>
#include <vector>

namespace hb2
{
    template <typename T> struct Vec;
    template <> struct Vec<double> { typedef double2 V; typedef int2 I; };
    template <> struct Vec<float> { typedef float4 V; typedef int4 I; };

    template <typename T, int R>
    union VLoad { typename Vec<T>::V v; T a[R]; };
    template <int R>
    union ILoad { typename Vec<double>::I v2; int4 v4; int a[R]; };

    template <typename T, int R>
    __device__ __forceinline__ void load_slot(const T * val, const int32_t * col, T (&v)[R], int (&c)[R], bool keep)
    {
        VLoad<T, R> lv;
        lv.v = keep ? __ldcg((const typename Vec<T>::V *)val) : __ldcs((const typename Vec<T>::V *)val);
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = lv.a[i];
        if (R == 2)
        {
            int2 t = keep ? __ldcg((const int2 *)col) : __ldcs((const int2 *)col);
            c[0] = t.x;
            c[1] = t.y;
        }
        else
        {
            int4 t = keep ? __ldcg((const int4 *)col) : __ldcs((const int4 *)col);
            c[0] = t.x;
            if (R > 1) c[1] = t.y;
            if (R > 2) c[2] = t.z;
            if (R > 3) c[3] = t.w;
        }
    }

    // One thread (TPR = 1) or a pair of adjacent lanes (TPR = 2): R consecutive
    // rows; KT = compile-time slot count (0: runtime).  With two lanes per row
    // the lanes load alternate slots (the even lane 0, 2, 4, ..., the odd one
    // 1, 3, 5, ...) and form their products; the odd lane's products move to the
    // even lane by shuffle, which adds all of them in slot order, so the sums are
    // the one-lane kernel's bit for bit.  The even lane runs the epilogue.
    // One thread per row takes blocks of up to 256 threads, two up to 512: bounded
    // at 512 the one-thread FP64 kernel got 44 registers instead of 32 (defect: 64
    // instead of 40) and the level-11 SpMV ran 20 % slower.
    template <typename T, int KT, int MODE, int TPR>
    __global__ void __launch_bounds__(TPR == 1 ? kEllThreads : kEllMaxThreads)
    ell_kernel(EllView<T> A, const T * __restrict__ x_, T * __restrict__ y_, const T * __restrict__ aux_,
               const T * __restrict__ aux2, T * __restrict__ zero_, ReduceSlot rs, double * red_, int want_sqrt,
               int flags, Batch bt)
    {
        constexpr int R = RowsPerThread<T>::value;
        typedef Arith<T> M;
        pdl_entry();
        // work items: (vector j, row block) -- the launch grid (blockIdx.x, blockIdx.y),
        // or, with a device work list, items 0 .. count * gx - 1 walked by a
        // persistent grid (vector list[item / gx], row block item % gx)
        const bool listed = bt.list != nullptr;
        const uint32_t total = listed ? *bt.count * bt.gx : 1;
        for (uint32_t item = listed ? blockIdx.x : 0; item < total; item += listed ? gridDim.x : 1)
        {
        const uint32_t j = listed ? bt.list[item / bt.gx] : blockIdx.y;
        if (! listed && bt.active && ! bt.active[j]) return;
        const uint64_t vo = (uint64_t)j * bt.vstride;
        const T * __restrict__ x = x_ + (uint64_t)j * (bt.xstride ? bt.xstride : bt.vstride);
        T * __restrict__ y = y_ + vo;
        const T * __restrict__ aux = aux_ ? aux_ + vo : aux_;
        T * __restrict__ zero = zero_ ? zero_ + (uint64_t)j * bt.zstride : zero_;
        double * red = red_ ? red_ + j : red_;   // the block reduction offsets its partials / counters itself
        const uint64_t bx = listed ? item % bt.gx : blockIdx.x;
        const uint64_t blk = (flags & kReverse) ? (gridDim.x - 1 - bx) : bx;
        const bool keep = (flags & kKeepL2) != 0;
        const uint64_t r0 = (blk * (blockDim.x / TPR) + threadIdx.x / TPR) * R;
        const int K = KT > 0 ? KT : (int)A.K;
        const int lane2 = TPR == 2 ? (int)(threadIdx.x & 1) : 0;
        T acc[R];
#pragma unroll
        for (int i = 0; i < R; ++i) acc[i] = T(0);
        if constexpr (TPR == 1)
        {
        if (r0 < A.rows)
        {
            const T * vp = A.val + r0;
            const int32_t * cp = A.col + r0;
            if constexpr (KT > 0)
            {
                // issue every slot load of the thread before the first gather:
                // K * 24 (FP64) / K * 32 (FP32) bytes in flight per thread
                T v[KT][R];
                int c[KT][R];
#pragma unroll
                for (int k = 0; k < KT; ++k)
                    load_slot<T, R>(vp + (uint64_t)k * A.ld, cp + (uint64_t)k * A.ld, v[k], c[k], keep);
#pragma unroll
                for (int k = 0; k < KT; ++k)
#pragma unroll
                    for (int i = 0; i < R; ++i)
                        if (c[k][i] >= 0) acc[i] = M::add(acc[i], M::mul(v[k][i], __ldg(x + c[k][i])));
            }
            else
            {
                for (int k = 0; k < K; ++k)
                {
                    T v[R];
                    int c[R];
                    load_slot<T, R>(vp + (uint64_t)k * A.ld, cp + (uint64_t)k * A.ld, v, c, keep);
#pragma unroll
                    for (int i = 0; i < R; ++i)
                        if (c[i] >= 0) acc[i] = M::add(acc[i], M::mul(v[i], __ldg(x + c[i])));
                }
            }
        }
        }
        else
        {
            // both lanes of a pair run every shuffle (the whole warp does: r0 and K
            // are the same for the pair, the loads are guarded instead)
            const bool live = r0 < A.rows;
            const T * vp = A.val + (live ? r0 : 0);
            const int32_t * cp = A.col + (live ? r0 : 0);
            constexpr int KH = KT > 0 ? (KT + 1) / 2 : 1;
            const int kh = (K + 1) / 2;
#pragma unroll (KT > 0 ? KH : 1)
            for (int h = 0; h < kh; ++h)
            {
                const int k = 2 * h + lane2;
                T v[R], pr[R];
                int c[R];
                if (live && k < K) load_slot<T, R>(vp + (uint64_t)k * A.ld, cp + (uint64_t)k * A.ld, v, c, keep);
                else
                {
#pragma unroll
                    for (int i = 0; i < R; ++i) { v[i] = T(0); c[i] = -1; }
                }
                unsigned ok = 0;
#pragma unroll
                for (int i = 0; i < R; ++i)
                {
                    pr[i] = c[i] >= 0 ? M::mul(v[i], __ldg(x + c[i])) : T(0);
                    ok |= c[i] >= 0 ? 1u << i : 0u;
                }
                const unsigned ok_odd = __shfl_down_sync(0xffffffffu, ok, 1);
#pragma unroll
                for (int i = 0; i < R; ++i)
                {
                    const T odd = __shfl_down_sync(0xffffffffu, pr[i], 1);
                    if (ok & (1u << i)) acc[i] = M::add(acc[i], pr[i]);             // slot 2h
                    if (ok_odd & (1u << i)) acc[i] = M::add(acc[i], odd);           // slot 2h + 1
                }
            }
        }
        double part = 0.0;
#pragma unroll
        for (int i = 0; i < R; ++i)
        {
            const uint64_t r = r0 + i;
            if (r >= A.rows || lane2) break;
            if (MODE == kPlain) y[r] = acc[i];
            else if (MODE == kDefect)
            {
                T d = M::sub(aux[r], acc[i]);
                y[r] = d;
                part = fma((double)d, (double)d, part);
            }
            else if (MODE == kDot)
            {
                y[r] = acc[i];
                part = fma((double)acc[i], (double)x[r], part);
            }
            else if (MODE == kAdd) y[r] = M::add(y[r], acc[i]);
            else if (is_jacobi(MODE))
            {
                // the sweep's defect b - A x, and its square for a fused norm
                const T d = M::sub(aux[r], acc[i]);
                y[r] = M::add(x[r], M::mul(aux2[r], d));
                part = fma((double)d, (double)d, part);
            }
            else if (MODE == kRestrict) { y[r] = acc[i]; zero[r] = T(0); }
        }
        if ((MODE == kDefect || MODE == kDot || MODE == kJacobiNorm) && red != 0)
        {
            __shared__ double scratch[32];
            ell_block_reduce(part, rs, red, want_sqrt, flags, scratch);
        }
        }
    }

    template <typename T, int MODE, int TPR>
    static void launch_shape(const hb2_ell_s * A, const void * x, void * y, const void * aux, const void * aux2,
                             void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid, cudaStream_t s,
                             int flags, Batch b, unsigned bs)
    {
        EllView<T> v = A->view<T>();
        const T * xp = (const T *)x;
        T * yp = (T *)y;
        if (A->K == 9)
            launch_pdl(ell_kernel<T, 9, MODE, TPR>, grid, dim3(bs), 0, s, v, xp, yp, (const T *)aux, (const T *)aux2,
                       (T *)zero, rs, red, want_sqrt, flags, b);
        else if (A->K == 4)
            launch_pdl(ell_kernel<T, 4, MODE, TPR>, grid, dim3(bs), 0, s, v, xp, yp, (const T *)aux, (const T *)aux2,
                       (T *)zero, rs, red, want_sqrt, flags, b);
        else
            launch_pdl(ell_kernel<T, 0, MODE, TPR>, grid, dim3(bs), 0, s, v, xp, yp, (const T *)aux, (const T *)aux2,
                       (T *)zero, rs, red, want_sqrt, flags, b);
    }

    template <typename T, int MODE>
    static void launch_mode(const hb2_ell_s * A, const void * x, void * y, const void * aux, const void * aux2,
                            void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid, cudaStream_t s,
                            int flags, Batch b, unsigned bs, int tpr)
    {
        if (tpr == 2) launch_shape<T, MODE, 2>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, flags, b, bs);
        else launch_shape<T, MODE, 1>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, flags, b, bs);
    }

    template <typename T>
    static void launch_typed(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux,
                             const void * aux2, void * zero, double * red, int want_sqrt, ReduceSlot rs,
                             dim3 grid, cudaStream_t s, int f, Batch b, unsigned bs, int tpr)
    {
        switch (mode)
        {
            case kPlain: launch_mode<T, kPlain>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, tpr); break;
            case kDefect: launch_mode<T, kDefect>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, tpr); break;
            case kDot: launch_mode<T, kDot>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, tpr); break;
            case kAdd: launch_mode<T, kAdd>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, tpr); break;
            case kJacobi:
                if (red) launch_mode<T, kJacobiNorm>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, tpr);
                else launch_mode<T, kJacobi>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, tpr);
                break;
            case kRestrict: launch_mode<T, kRestrict>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, tpr); break;
        }
    }

    // blocks of a work-list launch: at most 32 per SM, or HB2_LIST_GRID (0: one
    // block per possible work item).  Measured on the 512-system batch: 8 per
    // SM (one resident wave, each block looping over its items) is 15 % slower
    // than one block per item, 16 per SM within 2 %; the cap keeps a mostly idle
    // batch from paying for hundreds of thousands of empty blocks.
    uint64_t list_grid_cap()
    {
        static const uint64_t cap = [] {
            const char * v = getenv("HB2_LIST_GRID");
            const uint64_t c = v && *v ? strtoull(v, 0, 10) : (uint64_t)num_sms() * 32;
            return c ? c : ~0ull;
        }();
        return cap;
    }

    // rows per block of a launch of bs threads on the class's layout
    static uint64_t rows_per_block(const hb2_ell_s * A, int cls, uint64_t bs)
    {
        if (A->layout[cls] == kLayoutPattern) return bs * (A->rpt[cls] & ~kPatFlags);
        if (A->layout[cls] == kLayoutCompact) return bs * (cls ? A->compact_rpt_red : A->compact_rpt);
        if (A->layout[cls] == kLayoutBF16) return bs * A->rpt[cls];
        return bs / A->tpr[cls] * (A->dtype == HB2_F64 ? RowsPerThread<double>::value : RowsPerThread<float>::value);
    }

    // the tuned block size where the class's kernel takes one (plain, compressed,
    // the Q1 gather form), else 256
    bool ell_shape_tunable(const hb2_ell_s * A, int cls)
    {
        return A->layout[cls] != kLayoutPattern || (A->rpt[cls] & (kPatQ1G | kPatQ1S));
    }

    unsigned ell_block(const hb2_ell_s * A, bool reducing)
    {
        const int cls = reducing ? 1 : 0;
        if (! ell_shape_tunable(A, cls)) return kEllThreads;
        // the plain kernel with one thread per row is bounded at 256 threads
        if (A->layout[cls] == kLayoutPlain && A->tpr[cls] == 1) return std::min(A->bs[cls], kEllThreads);
        return (unsigned)A->bs[cls];
    }

    uint64_t ell_rows_per_block(const hb2_ell_s * A, bool reducing)
    {
        return rows_per_block(A, reducing ? 1 : 0, ell_block(A, reducing));
    }

    // blocks of a launch of bs threads with the class's kernel (q1: the Q1 stencil
    // kernel runs it, where the layout names one)
    static unsigned grid_blocks(const hb2_ell_s * A, int cls, unsigned bs, bool q1)
    {
        if (q1 && A->layout[cls] == kLayoutPattern && (A->rpt[cls] & kPatQ1S))
            return q1_strip_grid(A, A->rpt[cls] & ~kPatFlags, bs);
        return ceil_div(A->rows, rows_per_block(A, cls, bs));
    }

    unsigned ell_grid(const hb2_ell_s * A, bool reducing)
    {
        return grid_blocks(A, reducing ? 1 : 0, ell_block(A, reducing), true);
    }

    // HB2_Q1_TRANSFER=0 runs the Q1 transfer matrices on their stored layout instead
    // (read at every launch, so a process can compare both)
    static bool q1_transfer_kernels_enabled()
    {
        const char * v = getenv("HB2_Q1_TRANSFER");
        return ! (v && strcmp(v, "0") == 0);
    }

    int launch_ell(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux, const void * aux2,
                   void * zero, double * red, int want_sqrt, const Workspace * ws, cudaStream_t stream, int flags,
                   const Batch * batch)
    {
        Batch b = batch ? *batch : Batch();
        if (A->rows == 0)
        {
            // empty matrix: defined results without a launch
            if (red) HB2_CUDA(cudaMemsetAsync(red, 0, sizeof(double), stream));
            return HB2_OK;
        }
        // the launch shape: the class's tuned one, except where a Q1 gather layout
        // hands this launch to the general row-pattern kernel (256 threads)
        const int cls = red != 0;
        unsigned bs = ell_block(A, red != 0);
        const bool q1 = A->layout[cls] == kLayoutPattern && ell_q1_stencil_applies(A, mode, x, A->rpt[cls], b);
        if (A->layout[cls] == kLayoutPattern && ! q1) bs = kEllThreads;
        const unsigned gx = grid_blocks(A, cls, bs, q1);
        if (b.nvec == 0 || b.nvec > 65535) return fail(HB2_ERR_ARG, "ELL batch: 1..65535 vectors");
        dim3 grid(gx, b.nvec);
        if (b.list)
        {
            // persistent grid over the work list: at most 8 blocks per SM
            if (red || ! b.count) return fail(HB2_ERR_ARG, "ELL work list: no fused reduction, count required");
            b.gx = gx;
            grid = dim3((unsigned)std::min<uint64_t>((uint64_t)gx * b.nvec, b.cap ? b.cap : list_grid_cap()), 1);
        }
        ReduceSlot rs;
        rs.partials = 0;
        rs.gpart = 0;
        rs.ticket = 0;
        rs.max_blocks = 0;
        if (red)
        {
            if (! ws) return fail(HB2_ERR_ARG, "fused reduction without a workspace");
            const uint64_t ngroups = (gx + kReduceGroup - 1) / kReduceGroup;
            if ((uint64_t)gx * b.nvec > ws->max_blocks || (ngroups + 1) * b.nvec > ws->max_tickets ||
                ngroups * b.nvec > ws->max_blocks / kReduceGroup + 4096)
                return fail(HB2_ERR_UNSUPPORTED, "matrix / batch too large for the reduction workspace");
            rs = ws->slot();
        }
        if (A->q1_transfer && ! red && b.nvec == 1 && ! b.list && ! b.active &&
            (mode == kPlain || mode == kAdd || mode == kRestrict) && q1_transfer_kernels_enabled())
            return launch_q1_transfer(A, mode, x, y, zero, stream);
        // the fused reduction split into per-block partials and a second launch: always
        // on the Q1 stencil kernels, elsewhere from kSplitSumMinBlocks blocks
        const bool split = red && (q1 || (uint64_t)gx * b.nvec >= kSplitSumMinBlocks);
        if (split) flags |= kSplitSum;
        if (A->layout[cls] == kLayoutPattern)
            launch_ell_pattern(A, mode, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, stream, flags, b, A->rpt[cls], bs);
        else if (A->layout[cls] == kLayoutCompact)
            launch_ell_compact(A, mode, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, stream, flags, b, bs);
        else if (A->layout[cls] == kLayoutBF16)
            launch_ell_bf16(A, mode, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, stream, flags, b, bs);
        else if (A->dtype == HB2_F64)
            launch_typed<double>(A, mode, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, stream, flags, b, bs, A->tpr[cls]);
        else launch_typed<float>(A, mode, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, stream, flags, b, bs, A->tpr[cls]);
        count_launches(1);
        if (split) launch_sum_partials(rs.partials, gx, b.nvec, red, want_sqrt, stream);
        HB2_LAUNCH_CHECK("ell kernel launch");
        return HB2_OK;
    }

    // ------------------------------------------------------------------
    // construction

    static uint64_t pad_ld(uint64_t rows) { return std::max<uint64_t>(64, (rows + 63) / 64 * 64); }

    static int alloc_ell(hb2_ell_s ** out, int dtype, uint64_t rows, uint64_t cols, uint32_t K)
    {
        if (cols > 0x7fffffffULL) return fail(HB2_ERR_UNSUPPORTED, "more than 2^31-1 columns");
        hb2_ell_s * A = new hb2_ell_s();
        A->dtype = dtype;
        cudaGetDevice(&A->device);
        A->rows = rows;
        A->cols = cols;
        A->K = K;
        A->ld = pad_ld(rows);
        size_t nslots = (size_t)K * A->ld;
        size_t vbytes = nslots * dtype_size(dtype), cbytes = nslots * sizeof(int32_t);
        cudaError_t e = cudaMalloc(&A->val, std::max<size_t>(vbytes, 16));
        if (e != cudaSuccess) { delete A; return cuda_status(e, "ELL values cudaMalloc"); }
        e = cudaMalloc(&A->col, std::max<size_t>(cbytes, 16));
        if (e != cudaSuccess) { cudaFree(A->val); delete A; return cuda_status(e, "ELL indices cudaMalloc"); }
        A->bytes = vbytes + cbytes;
        *out = A;
        return HB2_OK;
    }

    // reference arrays -> device layout
    template <typename T>
    __global__ void ell_from_ref_kernel(const uint64_t * __restrict__ Aj, const T * __restrict__ Ax,
                                        const uint64_t * __restrict__ Arl, uint64_t rows, uint64_t cols,
                                        uint64_t stride, uint64_t T_, uint32_t K, uint64_t ld, T * val,
                                        int32_t * col, int * bad)
    {
        uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (r >= ld) return;
        uint64_t used = r < rows ? Arl[r] * T_ : 0;
        if (used > K) { atomicExch(bad, 1); used = K; }
        for (uint32_t t = 0; t < K; ++t)
        {
            T v = T(0);
            int32_t c = -1;
            if (t < used)
            {
                uint64_t src = (t % T_) + r * T_ + (t / T_) * stride;
                uint64_t j = Aj[src];
                if (j >= cols) { atomicExch(bad, 2); j = 0; }
                c = (int32_t)j;
                v = Ax[src];
            }
            val[(uint64_t)t * ld + r] = v;
            col[(uint64_t)t * ld + r] = c;
        }
    }

    // Q1 Poisson operator (math/fill_matrix.hh:37-79 -> SparseMatrix -> ELL):
    // 1-based row i is a Dirichlet unit row when i <= M, i > N-M, i%M == 1 or
    // i%M == 0; interior rows hold the 9 stencil entries in ascending column order.
    template <typename T>
    __global__ void ell_q1_kernel(uint64_t M, double aniso, uint64_t ld, T * val, int32_t * col)
    {
        uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (r >= ld) return;
        const uint64_t N = M * M;
        if (r >= N)
        {
            for (int k = 0; k < 9; ++k) { val[k * ld + r] = T(0); col[k * ld + r] = -1; }
            return;
        }
        const uint64_t i = r + 1;
        const bool dir = (i <= M || i > N - M || (i % M) == 1 || (i % M) == 0);
        if (dir)
        {
            val[r] = T(1.0);
            col[r] = (int32_t)r;
            for (int k = 1; k < 9; ++k) { val[k * ld + r] = T(0); col[k * ld + r] = -1; }
            return;
        }
        const int64_t m = (int64_t)M;
        const int64_t off[9] = {-m - 1, -m, -m + 1, -1, 0, 1, m - 1, m, m + 1};
        const T nb = T(-1.0 / 3.0);
        for (int k = 0; k < 9; ++k)
        {
            T v = nb;
            if (k == 4) v = aniso == 1.0 ? T(8.0 / 3.0) : T((6.0 + 2.0 * aniso) / 3.0);
            else if ((k == 3 || k == 5) && aniso != 1.0) v = T(-aniso / 3.0);
            val[k * ld + r] = v;
            col[k * ld + r] = (int32_t)((int64_t)r + off[k]);
        }
    }

    // ProlongationMatrix (math/prolongation_matrix.hh:44-100) with identity maps:
    // fine node (i, j) takes coarse (i/2, j/2) with weight 1, the two coarse
    // neighbours with 1/2 on a coarse row or column, the four with 1/4 otherwise;
    // columns ascending (SparseVector order).
    template <typename T>
    __global__ void ell_prol_kernel(uint64_t mf, uint64_t ld, T * val, int32_t * col)
    {
        uint64_t f = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (f >= ld) return;
        int32_t c[4] = {-1, -1, -1, -1};
        T v[4] = {T(0), T(0), T(0), T(0)};
        if (f < mf * mf)
        {
            const uint64_t mc = (mf + 1) / 2, i = f / mf, j = f % mf;
            if (i % 2 == 0 && j % 2 == 0) { c[0] = (int32_t)((i / 2) * mc + j / 2); v[0] = T(1); }
            else if (i % 2 == 0)
            {
                c[0] = (int32_t)((i / 2) * mc + (j - 1) / 2); v[0] = T(0.5);
                c[1] = (int32_t)((i / 2) * mc + (j + 1) / 2); v[1] = T(0.5);
            }
            else if (j % 2 == 0)
            {
                c[0] = (int32_t)(((i - 1) / 2) * mc + j / 2); v[0] = T(0.5);
                c[1] = (int32_t)(((i + 1) / 2) * mc + j / 2); v[1] = T(0.5);
            }
            else
            {
                c[0] = (int32_t)(((i - 1) / 2) * mc + (j - 1) / 2);
                c[1] = (int32_t)(((i - 1) / 2) * mc + (j + 1) / 2);
                c[2] = (int32_t)(((i + 1) / 2) * mc + (j - 1) / 2);
                c[3] = (int32_t)(((i + 1) / 2) * mc + (j + 1) / 2);
                v[0] = v[1] = v[2] = v[3] = T(0.25);
            }
        }
        for (int k = 0; k < 4; ++k) { val[k * ld + f] = v[k]; col[k * ld + f] = c[k]; }
    }

    // R = P^T (math/transposition.hh:36-50): coarse node (I, J) collects the fine
    // nodes (2I+di, 2J+dj), di, dj in {-1, 0, 1}, inside the grid, ascending,
    // with weight 1 / 2^(|di|+|dj|).
    template <typename T>
    __global__ void ell_res_kernel(uint64_t mf, uint64_t ld, T * val, int32_t * col)
    {
        uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (r >= ld) return;
        const uint64_t mc = (mf + 1) / 2;
        int k = 0;
        if (r < mc * mc)
        {
            const int64_t I = (int64_t)(r / mc), J = (int64_t)(r % mc);
            for (int di = -1; di <= 1; ++di)
                for (int dj = -1; dj <= 1; ++dj)
                {
                    int64_t fi = 2 * I + di, fj = 2 * J + dj;
                    if (fi < 0 || fj < 0 || fi >= (int64_t)mf || fj >= (int64_t)mf) continue;
                    int w = (di != 0) + (dj != 0);
                    val[k * ld + r] = w == 0 ? T(1) : (w == 1 ? T(0.5) : T(0.25));
                    col[k * ld + r] = (int32_t)(fi * (int64_t)mf + fj);
                    ++k;
                }
        }
        for (; k < 9; ++k) { val[k * ld + r] = T(0); col[k * ld + r] = -1; }
    }

    // device layout -> reference arrays
    template <typename T>
    __global__ void ell_to_ref_kernel(const T * __restrict__ val, const int32_t * __restrict__ col, uint64_t rows,
                                      uint64_t ld, uint32_t K, uint64_t stride, uint64_t T_, uint64_t * Aj, T * Ax,
                                      uint64_t * Arl)
    {
        uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (r >= rows) return;
        uint32_t used = 0;
        for (uint32_t t = 0; t < K; ++t)
        {
            int32_t c = col[(uint64_t)t * ld + r];
            uint64_t dst = (t % T_) + r * T_ + (t / T_) * stride;
            if (c >= 0) { Aj[dst] = (uint64_t)c; Ax[dst] = val[(uint64_t)t * ld + r]; used = t + 1; }
        }
        Arl[r] = (used + T_ - 1) / T_;
    }

    template <typename S, typename D>
    __global__ void ell_convert_kernel(const S * __restrict__ src, D * __restrict__ dst, uint64_t n)
    {
        uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (i < n) dst[i] = D(src[i]);
    }

    // P = omega / A(j, j) with the reference's element access
    // (la/sparse_matrix_ell-impl.hh:325-337: scan slot groups while the group's
    // first column <= j).
    template <typename T>
    __global__ void jacobi_precon_kernel(EllView<T> A, uint64_t T_, double omega, T * P)
    {
        uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (r >= A.rows) return;
        T d = T(0);
        for (uint32_t g = 0; g * T_ < A.K; ++g)
        {
            int32_t first = A.col[(uint64_t)(g * T_) * A.ld + r];
            if (first < 0 || (uint64_t)first > r) break;
            bool found = false;
            for (uint64_t t = 0; t < T_ && g * T_ + t < A.K; ++t)
            {
                uint64_t s = (uint64_t)(g * T_ + t) * A.ld + r;
                if (A.col[s] == (int32_t)r) { d = A.val[s]; found = true; break; }
            }
            if (found) break;
        }
        P[r] = Arith<T>::div(T(omega), d);
    }
}

using namespace hb2;

extern "C" int hb2_ell_create(hb2_ell * out, hb2_dtype dtype, uint64_t rows, uint64_t cols, uint64_t stride,
                              uint64_t num_cols_per_row, uint64_t threads, const uint64_t * Aj, const void * Ax,
                              const uint64_t * Arl, int host_ptrs, cudaStream_t stream)
{
    if (! out || (dtype != HB2_F64 && dtype != HB2_F32)) return fail(HB2_ERR_ARG, "hb2_ell_create: bad argument");
    if (threads == 0 || num_cols_per_row == 0) return fail(HB2_ERR_ARG, "hb2_ell_create: zero threads/slots");
    if (rows > 0 && (! Aj || ! Ax || ! Arl)) return fail(HB2_ERR_ARG, "hb2_ell_create: null array");
    if (stride < rows * threads) return fail(HB2_ERR_SIZE, "hb2_ell_create: stride < rows * threads");
    uint64_t K = num_cols_per_row * threads;
    if (K > 4096) return fail(HB2_ERR_UNSUPPORTED, "hb2_ell_create: more than 4096 slots per row");
    hb2_ell_s * A = 0;
    int st = alloc_ell(&A, dtype, rows, cols, (uint32_t)K);
    if (st) return st;
    A->ref_stride = stride;
    A->ref_K = num_cols_per_row;
    A->ref_T = threads;
    size_t es = dtype_size(dtype), nslots = num_cols_per_row * stride;
    const uint64_t * dAj = Aj;
    const void * dAx = Ax;
    const uint64_t * dArl = Arl;
    void * tmp = 0;
    int * bad = 0;
    cudaError_t e = cudaSuccess;
    if (host_ptrs && rows > 0)
    {
        // Aj | Ax | Arl, each part 256-byte aligned (an F32 Ax of an odd slot count
        // would leave the uint64 Arl 4-byte aligned)
        const size_t ax_off = nslots * 8, arl_off = (ax_off + nslots * es + 255) / 256 * 256;
        size_t bytes = arl_off + rows * 8;
        e = cudaMalloc(&tmp, bytes);
        if (e == cudaSuccess)
        {
            char * p = (char *)tmp;
            cudaMemcpyAsync(p, Aj, nslots * 8, cudaMemcpyHostToDevice, stream);
            cudaMemcpyAsync(p + ax_off, Ax, nslots * es, cudaMemcpyHostToDevice, stream);
            e = cudaMemcpyAsync(p + arl_off, Arl, rows * 8, cudaMemcpyHostToDevice, stream);
            dAj = (const uint64_t *)p;
            dAx = p + ax_off;
            dArl = (const uint64_t *)(p + arl_off);
        }
    }
    if (e == cudaSuccess) e = cudaMalloc(&bad, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int), stream);
    if (e == cudaSuccess)
    {
        unsigned grid = ceil_div(A->ld, 256);
        if (dtype == HB2_F64)
            ell_from_ref_kernel<double><<<grid, 256, 0, stream>>>(dAj, (const double *)dAx, dArl, rows, cols, stride,
                                                                  threads, A->K, A->ld, (double *)A->val, A->col, bad);
        else
            ell_from_ref_kernel<float><<<grid, 256, 0, stream>>>(dAj, (const float *)dAx, dArl, rows, cols, stride,
                                                                 threads, A->K, A->ld, (float *)A->val, A->col, bad);
        count_launches(1);
        e = cudaGetLastError();
    }
    int hbad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (tmp) cudaFree(tmp);
    if (bad) cudaFree(bad);
    if (e != cudaSuccess) { hb2_ell_destroy(A); return cuda_status(e, "hb2_ell_create"); }
    if (hbad)
    {
        hb2_ell_destroy(A);
        return fail(HB2_ERR_ARG, hbad == 1 ? "hb2_ell_create: Arl exceeds num_cols_per_row"
                                           : "hb2_ell_create: column index >= columns");
    }
    int cst = ell_build_compact(A, stream);
    if (cst) { hb2_ell_destroy(A); return cst; }
    *out = A;
    return HB2_OK;
}

extern "C" int hb2_ell_create_q1(hb2_ell * out, hb2_dtype dtype, unsigned level, double aniso, cudaStream_t stream)
{
    if (! out || level < 1 || level > 14 || ! (aniso > 0.0)) return fail(HB2_ERR_ARG, "hb2_ell_create_q1: bad argument");
    uint64_t M = (1ULL << level) + 1, n = M * M;
    hb2_ell_s * A = 0;
    int st = alloc_ell(&A, dtype, n, n, 9);
    if (st) return st;
    A->ref_stride = 32 * ((n + 31) / 32);
    A->ref_K = 9;
    A->ref_T = 1;
    unsigned grid = ceil_div(A->ld, 256);
    if (dtype == HB2_F64) ell_q1_kernel<double><<<grid, 256, 0, stream>>>(M, aniso, A->ld, (double *)A->val, A->col);
    else ell_q1_kernel<float><<<grid, 256, 0, stream>>>(M, aniso, A->ld, (float *)A->val, A->col);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { hb2_ell_destroy(A); return cuda_status(e, "hb2_ell_create_q1"); }
    int cst = ell_build_compact(A, stream);
    if (cst) { hb2_ell_destroy(A); return cst; }
    *out = A;
    return HB2_OK;
}

extern "C" int hb2_ell_create_transfer(hb2_ell * prol, hb2_ell * res, hb2_dtype dtype, unsigned fine_level,
                                       cudaStream_t stream)
{
    if (! prol || ! res || fine_level < 2 || fine_level > 14) return fail(HB2_ERR_ARG, "hb2_ell_create_transfer: bad argument");
    uint64_t mf = (1ULL << fine_level) + 1, mc = (mf + 1) / 2, nf = mf * mf, nc = mc * mc;
    hb2_ell_s * P = 0, * R = 0;
    int st = alloc_ell(&P, dtype, nf, nc, 4);
    if (st) return st;
    st = alloc_ell(&R, dtype, nc, nf, 9);
    if (st) { hb2_ell_destroy(P); return st; }
    P->ref_stride = 32 * ((nf + 31) / 32);
    P->ref_K = 4;
    P->ref_T = 1;
    R->ref_stride = 32 * ((nc + 31) / 32);
    R->ref_K = 9;
    R->ref_T = 1;
    if (dtype == HB2_F64)
    {
        ell_prol_kernel<double><<<ceil_div(P->ld, 256), 256, 0, stream>>>(mf, P->ld, (double *)P->val, P->col);
        ell_res_kernel<double><<<ceil_div(R->ld, 256), 256, 0, stream>>>(mf, R->ld, (double *)R->val, R->col);
    }
    else
    {
        ell_prol_kernel<float><<<ceil_div(P->ld, 256), 256, 0, stream>>>(mf, P->ld, (float *)P->val, P->col);
        ell_res_kernel<float><<<ceil_div(R->ld, 256), 256, 0, stream>>>(mf, R->ld, (float *)R->val, R->col);
    }
    count_launches(2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { hb2_ell_destroy(P); hb2_ell_destroy(R); return cuda_status(e, "hb2_ell_create_transfer"); }
    int cst = ell_build_compact(P, stream);
    if (! cst) cst = ell_build_compact(R, stream);
    if (cst) { hb2_ell_destroy(P); hb2_ell_destroy(R); return cst; }
    P->q1_transfer = (int)fine_level;
    R->q1_transfer = -(int)fine_level;
    *prol = P;
    *res = R;
    return HB2_OK;
}

extern "C" int hb2_ell_convert(hb2_ell * out, hb2_ell src, hb2_dtype dtype, cudaStream_t stream)
{
    if (! out || ! src) return fail(HB2_ERR_ARG, "hb2_ell_convert: null argument");
    hb2_ell_s * A = 0;
    int st = alloc_ell(&A, dtype, src->rows, src->cols, src->K);
    if (st) return st;
    A->ref_stride = src->ref_stride;
    A->ref_K = src->ref_K;
    A->ref_T = src->ref_T;
    uint64_t n = (uint64_t)src->K * src->ld;
    unsigned grid = ceil_div(n, 256);
    if (src->dtype == HB2_F64 && dtype == HB2_F32)
        ell_convert_kernel<double, float><<<grid, 256, 0, stream>>>((const double *)src->val, (float *)A->val, n);
    else if (src->dtype == HB2_F32 && dtype == HB2_F64)
        ell_convert_kernel<float, double><<<grid, 256, 0, stream>>>((const float *)src->val, (double *)A->val, n);
    else
        cudaMemcpyAsync(A->val, src->val, n * dtype_size(dtype), cudaMemcpyDeviceToDevice, stream);
    count_launches(1);
    cudaError_t e = cudaMemcpyAsync(A->col, src->col, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) { hb2_ell_destroy(A); return cuda_status(e, "hb2_ell_convert"); }
    int cst = ell_build_compact(A, stream);
    if (cst) { hb2_ell_destroy(A); return cst; }
    *out = A;
    return HB2_OK;
}

extern "C" int hb2_ell_destroy(hb2_ell A)
{
    if (! A) return HB2_OK;
    cudaFree(A->val);
    cudaFree(A->col);
    ell_free_compact(A);
    ell_free_pattern(A);
    ell_free_bf16(A);
    cudaFree(A->spat);
    cudaFree(A->sptab);
    delete A;
    return HB2_OK;
}

extern "C" int hb2_ell_info(hb2_ell A, uint64_t * rows, uint64_t * cols, uint64_t * stride, uint64_t * K,
                            uint64_t * threads, uint64_t * device_bytes)
{
    if (! A) return fail(HB2_ERR_ARG, "hb2_ell_info: null matrix");
    if (rows) *rows = A->rows;
    if (cols) *cols = A->cols;
    if (stride) *stride = A->ref_stride;
    if (K) *K = A->ref_K;
    if (threads) *threads = A->ref_T;
    if (device_bytes) *device_bytes = A->bytes + A->compact_bytes + A->pattern_bytes + A->bf16_bytes;
    return HB2_OK;
}

extern "C" int hb2_ell_layout(hb2_ell A, int * layout, uint32_t * table_size, uint32_t * row_bytes)
{
    if (! A) return fail(HB2_ERR_ARG, "hb2_ell_layout: null matrix");
    const int l = A->layout[0];
    if (layout) *layout = l;
    if (table_size) *table_size = l == kLayoutPattern ? A->npat : (l == kLayoutCompact ? A->ntable : 0u);
    if (row_bytes)
        *row_bytes = l == kLayoutPattern   ? 1u
                     : l == kLayoutBF16    ? A->K * (A->bform == 0 ? 4u : 6u) + (A->bdiag ? 4u : 0u)
                     : l == kLayoutCompact ? A->K * 3u
                                           : A->K * (uint32_t)(dtype_size(A->dtype) + 4);
    return HB2_OK;
}

extern "C" int hb2_ell_layout_variant(hb2_ell A, int cls, int * layout, int * rows_per_thread, int * windowed)
{
    if (! A) return fail(HB2_ERR_ARG, "hb2_ell_layout_variant: null matrix");
    if (cls != 0 && cls != 1) return fail(HB2_ERR_ARG, "hb2_ell_layout_variant: class must be 0 or 1");
    const int l = A->layout[cls];
    if (layout) *layout = l;
    if (rows_per_thread) *rows_per_thread = (int)(ell_rows_per_block(A, cls == 1) * A->tpr[cls] / ell_block(A, cls == 1));
    if (windowed)
        *windowed = l != kLayoutPattern ? 0 : (A->rpt[cls] & kPatWin) ? 1 : (A->rpt[cls] & kPatQ1) ? 2
                                                                      : (A->rpt[cls] & kPatQ1G) ? 3
                                                                      : (A->rpt[cls] & kPatQ1P) ? 4
                                                                      : (A->rpt[cls] & kPatQ1S) ? 5 : 0;
    return HB2_OK;
}

extern "C" int hb2_ell_launch_shape(hb2_ell A, int cls, int * block_threads, int * threads_per_row)
{
    if (! A) return fail(HB2_ERR_ARG, "hb2_ell_launch_shape: null matrix");
    if (cls != 0 && cls != 1) return fail(HB2_ERR_ARG, "hb2_ell_launch_shape: class must be 0 or 1");
    if (block_threads) *block_threads = (int)ell_block(A, cls == 1);
    if (threads_per_row) *threads_per_row = A->layout[cls] == kLayoutPlain ? A->tpr[cls] : 1;
    return HB2_OK;
}

extern "C" int hb2_ell_export(hb2_ell A, uint64_t * Aj, void * Ax, uint64_t * Arl)
{
    if (! A || ! Aj || ! Ax || ! Arl) return fail(HB2_ERR_ARG, "hb2_ell_export: null argument");
    size_t nslots = A->ref_K * A->ref_stride, es = dtype_size(A->dtype);
    // Aj | Ax | Arl in one buffer, Arl 256-byte aligned
    const size_t arl_off = (nslots * 8 + nslots * es + 255) / 256 * 256;
    void * d = 0;
    HB2_CUDA(cudaMalloc(&d, arl_off + A->rows * 8 + 16));
    char * p = (char *)d;
    cudaError_t e = cudaMemset(p, 0, nslots * 8 + nslots * es);
    if (e == cudaSuccess && A->rows > 0)
    {
        unsigned grid = ceil_div(A->rows, 256);
        if (A->dtype == HB2_F64)
            ell_to_ref_kernel<double><<<grid, 256>>>((const double *)A->val, A->col, A->rows, A->ld, A->K, A->ref_stride,
                                                     A->ref_T, (uint64_t *)p, (double *)(p + nslots * 8),
                                                     (uint64_t *)(p + arl_off));
        else
            ell_to_ref_kernel<float><<<grid, 256>>>((const float *)A->val, A->col, A->rows, A->ld, A->K, A->ref_stride,
                                                    A->ref_T, (uint64_t *)p, (float *)(p + nslots * 8),
                                                    (uint64_t *)(p + arl_off));
        count_launches(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(Aj, p, nslots * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(Ax, p + nslots * 8, nslots * es, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && A->rows > 0) e = cudaMemcpy(Arl, p + arl_off, A->rows * 8, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_status(e, "hb2_ell_export");
    return HB2_OK;
}

// ---------------------------------------------------------------------- operators

static int check_vec(const void * p, uint64_t n, const char * what)
{
    if (n > 0 && ! p) return fail(HB2_ERR_ARG, std::string("null vector: ") + what);
    return HB2_OK;
}

extern "C" int hb2_product_ell(hb2_ell A, const void * x, void * y, cudaStream_t stream)
{
    if (! A) return fail(HB2_ERR_ARG, "hb2_product_ell: null matrix");
    if (check_vec(x, A->cols, "x") || check_vec(y, A->rows, "y")) return HB2_ERR_ARG;
    return launch_ell(A, kPlain, x, y, 0, 0, 0, 0, 0, 0, stream);
}

extern "C" int hb2_defect_ell(hb2_ell A, const void * rhs, const void * x, void * r, double * norm2_dev,
                              cudaStream_t stream)
{
    if (! A) return fail(HB2_ERR_ARG, "hb2_defect_ell: null matrix");
    if (A->rows != A->cols) return fail(HB2_ERR_SIZE, "hb2_defect_ell: VectorSizeDoesNotMatch (rhs vs columns)");
    if (check_vec(rhs, A->rows, "rhs") || check_vec(x, A->cols, "x") || check_vec(r, A->rows, "r")) return HB2_ERR_ARG;
    Workspace * ws = 0;
    if (norm2_dev)
    {
        int st = stream_workspace(stream, &ws);
        if (st) return st;
    }
    return launch_ell(A, kDefect, x, r, rhs, 0, 0, norm2_dev, 0, ws, stream);
}

extern "C" int hb2_product_dot_ell(hb2_ell A, const void * x, void * y, double * dot_dev, cudaStream_t stream)
{
    if (! A || ! dot_dev) return fail(HB2_ERR_ARG, "hb2_product_dot_ell: null argument");
    if (A->rows != A->cols) return fail(HB2_ERR_SIZE, "hb2_product_dot_ell: needs a square matrix");
    Workspace * ws = 0;
    int st = stream_workspace(stream, &ws);
    if (st) return st;
    return launch_ell(A, kDot, x, y, 0, 0, 0, dot_dev, 0, ws, stream);
}

extern "C" int hb2_product_add_ell(hb2_ell A, const void * x, void * y, cudaStream_t stream)
{
    if (! A) return fail(HB2_ERR_ARG, "hb2_product_add_ell: null matrix");
    return launch_ell(A, kAdd, x, y, 0, 0, 0, 0, 0, 0, stream);
}

extern "C" int hb2_jacobi_precon(hb2_ell A, double omega, void * P, cudaStream_t stream)
{
    if (! A || ! P) return fail(HB2_ERR_ARG, "hb2_jacobi_precon: null argument");
    if (A->rows == 0) return HB2_OK;
    unsigned grid = ceil_div(A->rows, 256);
    if (A->dtype == HB2_F64) jacobi_precon_kernel<double><<<grid, 256, 0, stream>>>(A->view<double>(), A->ref_T, omega, (double *)P);
    else jacobi_precon_kernel<float><<<grid, 256, 0, stream>>>(A->view<float>(), A->ref_T, omega, (float *)P);
    count_launches(1);
    HB2_LAUNCH_CHECK("hb2_jacobi_precon");
    return HB2_OK;
}

extern "C" int hb2_jacobi_sweep_ell(hb2_ell A, const void * P, const void * b, const void * x_in, void * x_out,
                                    cudaStream_t stream)
{
    if (! A || ! P || ! b || ! x_in || ! x_out) return fail(HB2_ERR_ARG, "hb2_jacobi_sweep_ell: null argument");
    if (A->rows != A->cols) return fail(HB2_ERR_SIZE, "hb2_jacobi_sweep_ell: needs a square matrix");
    if (x_in == x_out) return fail(HB2_ERR_ARG, "hb2_jacobi_sweep_ell: x_in and x_out must differ (Jacobi, not Gauss-Seidel)");
    return launch_ell(A, kJacobi, x_in, x_out, b, P, 0, 0, 0, 0, stream);
}

extern "C" int hb2_jacobi_ell(hb2_ell A, const void * P, const void * b, void * x, void * tmp, uint64_t sweeps,
                              cudaStream_t stream)
{
    if (! A || ! P || ! b || ! x || (sweeps > 0 && ! tmp)) return fail(HB2_ERR_ARG, "hb2_jacobi_ell: null argument");
    if (A->rows != A->cols) return fail(HB2_ERR_SIZE, "hb2_jacobi_ell: needs a square matrix");
    // ping-pong: sweep s reads cur, writes nxt (true Jacobi, as the reference's
    // separate defect / element product / sum passes)
    void * cur = x, * nxt = tmp;
    for (uint64_t s = 0; s < sweeps; ++s)
    {
        int st = launch_ell(A, kJacobi, cur, nxt, b, P, 0, 0, 0, 0, stream);
        if (st) return st;
        std::swap(cur, nxt);
    }
    if (cur != x) return launch_copy(A->dtype, x, cur, A->rows, stream);
    return HB2_OK;
}
