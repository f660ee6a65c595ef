// Q1 stencil kernel for square row-pattern ELL matrices whose rows are the
// nine-point stencil of an m x m node grid (the Q1 operators of
// math/fill_matrix.hh:37-79 at every level, and any matrix with the same
// structure).
//
// The general row-pattern kernels (ell_pattern.cu) look up each row's pattern
// in a table and gather x through per-slot offsets: about 200-230 instructions
// per row, most of them address arithmetic, so they issue-bind well below the
// HBM roofline.  Here the pattern that holds the full stencil -- nine slots,
// columns i-m-1, i-m, i-m+1, i-1, i, i+1, i+m-1, i+m, i+m+1 in that slot order --
// is known when the layout is built, and its nine values travel as kernel
// parameters (constant-bank operands of the multiplies).  A block owns
// B = 256 R consecutive rows, interleaved over its threads; thread 0 stages the
// three windows of x the stencil touches ([r0-m-1, r0+B-m+1), [r0-1, r0+B+1),
// [r0+m-1, r0+B+m+1)) with bulk copies (cp.async.bulk, no multicast, completion
// on an mbarrier with a bounded wait) while every thread streams its rows'
// pattern ids, rhs and Jacobi vector.  A full-stencil row then reads its nine x
// values at fixed shared-memory offsets from its own position: no table, no
// per-slot integer work.  Rows of any other pattern (Dirichlet identity rows,
// the grid's boundary) take the general slot loop over the pattern table.
// Both paths form the products and slot-ordered sums of the plain layout
// (la/product.hh:148-206: sum = 0, then sum += a_k x_k slot by slot, each
// product and sum rounded), so results are bit-identical to it and to the
// reference.  If the copies do not complete within the bounded wait, the block
// computes from global memory instead (same bits) and records the event.
#include "hb2_common.cuh"
#include "hb2_internal.hh"
#include "tma.cuh"

#include <cstdlib>
#include <vector>

namespace hb2
{
    template <typename T>
    struct Q1Stencil
    {
        T v[9];                  // the full stencil row's values, in slot order
        const uint8_t * pat;     // pattern id per row
        const PatEnt<T> * tab;   // npat * 9 (value, column - row) entries
        int64_t n, m;
        uint32_t full;           // pattern id of the full stencil row
        int64_t pf = 0;          // gather form: L2 prefetch distance in rows (0: none)
    };


    // diagnostic: set when a block's window copies did not complete in time
    __device__ int g_q1_stencil_timeout = 0;

    // x window w of the block starting at row r0: its first element's global index
    // (16-byte aligned: the bulk copy's start), the valid range and the ragged tail
    template <int B, int E>
    __device__ __forceinline__ void q1_window(int64_t start, int64_t n, int64_t & lo, int64_t & hi, int64_t & alo,
                                              int64_t & ahi)
    {
        lo = start < 0 ? 0 : start;
        hi = start + B + 2 > n ? n : start + B + 2;
        if (hi < lo) hi = lo;
        alo = lo - (lo % E);
        ahi = hi - (hi % E);
    }

    // one row of any pattern: slots in table order, x from the windows (or from
    // global memory when the copies did not complete)
    template <typename T, int W>
    __device__ __noinline__ T q1_any_row(const PatEnt<T> * __restrict__ te, const T * __restrict__ x, int64_t i,
                                         const T * win, int64_t alo0, int64_t alo1, int64_t alo2, bool fast)
    {
        typedef Arith<T> M;
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < 9; ++j)
        {
            const PatEnt<T> e = te[j];
            if (e.off == kPatEmpty) continue;
            const int64_t g = i + e.off;
            T xv;
            if (! fast) xv = __ldg(x + g);
            else if (e.off <= -2) xv = win[g - alo0];
            else if (e.off <= 1) xv = win[W + (g - alo1)];
            else xv = win[2 * W + (g - alo2)];
            acc = M::add(acc, M::mul(e.val, xv));
        }
        return acc;
    }

    template <typename T, int MODE, int R>
    __global__ void __launch_bounds__(kEllThreads)
    q1_stencil_kernel(const __grid_constant__ Q1Stencil<T> s, const T * __restrict__ x, T * __restrict__ y,
                      const T * __restrict__ aux, const T * __restrict__ aux2, ReduceSlot rs, double * red,
                      int want_sqrt, int flags)
    {
        typedef Arith<T> M;
        constexpr int B = kEllThreads * R;
        constexpr int E = 16 / sizeof(T);
        constexpr int W = (B + 2 + 2 * E + E - 1) / E * E;
        extern __shared__ __align__(128) unsigned char q1_smem[];
        T * win = reinterpret_cast<T *>(q1_smem);
        __shared__ alignas(8) uint64_t bar;
        const int64_t n = s.n, m = s.m;
        const int t = (int)threadIdx.x;
        const int64_t blk = (flags & kReverse) ? (int64_t)(gridDim.x - 1 - blockIdx.x) : (int64_t)blockIdx.x;
        const int64_t r0 = blk * B;
        const int64_t i0 = r0 + t;
        // pattern ids are constant: fetched before waiting on the previous kernel
        uint32_t p[R];
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int64_t i = i0 + k * kEllThreads;
            p[k] = i < n ? (uint32_t)((flags & kKeepL2) ? __ldcg(s.pat + i) : __ldcs(s.pat + i)) : s.full;
        }
        pdl_entry();   // x, rhs and P may come from the previous kernel
        T ea[R], ep[R];
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int64_t i = i0 + k * kEllThreads;
            const bool ok = i < n;
            ea[k] = (ok && (MODE == kDefect || is_jacobi(MODE))) ? aux[i] : T(0);
            ep[k] = (ok && is_jacobi(MODE)) ? aux2[i] : T(0);
        }
        int64_t lo[3], hi[3], alo[3], ahi[3];
#pragma unroll
        for (int w = 0; w < 3; ++w) q1_window<B, E>(r0 + (w - 1) * m - 1, n, lo[w], hi[w], alo[w], ahi[w]);
        if (t == 0)
        {
            mbar_init(&bar, 1);
            unsigned total = 0;
#pragma unroll
            for (int w = 0; w < 3; ++w) total += (unsigned)((ahi[w] - alo[w]) * sizeof(T));
            mbar_expect_tx(&bar, total);
#pragma unroll
            for (int w = 0; w < 3; ++w)
                if (ahi[w] > alo[w])
                    bulk_g2s(win + w * W, x + alo[w], (unsigned)((ahi[w] - alo[w]) * sizeof(T)), &bar);
        }
        else if (t <= 3 * (E - 1))
        {
            // the windows' ragged tails (at most E - 1 elements each) by plain loads
            const int w = (t - 1) / (E - 1), e = (t - 1) % (E - 1);
            const int64_t from = w == 0 ? (ahi[0] > lo[0] ? ahi[0] : lo[0])
                                        : (w == 1 ? (ahi[1] > lo[1] ? ahi[1] : lo[1]) : (ahi[2] > lo[2] ? ahi[2] : lo[2]));
            const int64_t j = from + e;
            const int64_t h = w == 0 ? hi[0] : (w == 1 ? hi[1] : hi[2]);
            const int64_t a = w == 0 ? alo[0] : (w == 1 ? alo[1] : alo[2]);
            if (j < h) win[w * W + (j - a)] = x[j];
        }
        __syncthreads();
        const bool fast = mbar_wait_bounded(&bar, 0, 1000000000ull);
        if (! fast && t == 0) atomicExch(&g_q1_stencil_timeout, 1);
        // x[i - m - 1 + j], x[i - 1 + j], x[i + m - 1 + j] of row i = i0 + k * 256 at
        // c0[k * 256 + j], c1[...], c2[...]: compile-time offsets from three
        // per-thread positions (negative only for rows the full stencil does not reach)
        const int o0 = (int)(i0 - m - 1 - alo[0]);
        const int o1 = W + (int)(i0 - 1 - alo[1]);
        const int o2 = 2 * W + (int)(i0 + m - 1 - alo[2]);
        double part = 0.0;
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int64_t i = i0 + k * kEllThreads;
            if (i >= n) break;
            const int l = k * kEllThreads;
            T acc, xc;
            if (fast && p[k] == s.full)
            {
                const T * c0 = win + (o0 + l);
                const T * c1 = win + (o1 + l);
                const T * c2 = win + (o2 + l);
                acc = M::add(T(0), M::mul(s.v[0], c0[0]));
                acc = M::add(acc, M::mul(s.v[1], c0[1]));
                acc = M::add(acc, M::mul(s.v[2], c0[2]));
                acc = M::add(acc, M::mul(s.v[3], c1[0]));
                xc = c1[1];
                acc = M::add(acc, M::mul(s.v[4], xc));
                acc = M::add(acc, M::mul(s.v[5], c1[2]));
                acc = M::add(acc, M::mul(s.v[6], c2[0]));
                acc = M::add(acc, M::mul(s.v[7], c2[1]));
                acc = M::add(acc, M::mul(s.v[8], c2[2]));
            }
            else
            {
                acc = q1_any_row<T, W>(s.tab + p[k] * 9u, x, i, win, alo[0], alo[1], alo[2], fast);
                xc = (is_jacobi(MODE) || MODE == kDot) ? (fast ? win[o1 + l + 1] : x[i]) : T(0);
            }
            if (MODE == kPlain) y[i] = acc;
            else if (MODE == kDefect)
            {
                const T d = M::sub(ea[k], acc);
                y[i] = d;
                part = fma((double)d, (double)d, part);
            }
            else if (MODE == kDot)
            {
                y[i] = acc;
                part = fma((double)acc, (double)xc, part);
            }
            else if (is_jacobi(MODE))
            {
                const T d = M::sub(ea[k], acc);
                y[i] = M::add(xc, M::mul(ep[k], d));
                part = fma((double)d, (double)d, part);
            }
        }
        if ((MODE == kDefect || MODE == kDot || MODE == kJacobiNorm) && red != 0)
        {
            __shared__ double scratch[32];
            ell_block_reduce(part, rs, red, want_sqrt, flags, scratch);
        }
        // copies still in flight must land before the block's shared memory is reused
        if (! fast) mbar_wait_bounded(&bar, 0, 1000000000ull);
    }

    // ------------------------------------------------------------------
    // Gather form: no shared memory, no block barrier, no bulk copies.  Each thread
    // owns R rows interleaved over the block (coalesced) and issues every load of
    // all of them before the first use: the pattern ids, rhs and Jacobi vector,
    // and the nine x values of each row as three runs of three (x[i-m-1..i-m+1],
    // x[i-1..i+1], x[i+m-1..i+m+1]: one base pointer per run, immediate offsets),
    // which the L1 serves after the first lane of a warp brought the line in.
    // Measured on B200: small bulk copies complete one after another within a CTA
    // (about 0.57 us per copy of 4 or 8 KiB, whatever the number issued ahead), so
    // a block that stages three x windows pays three serialised latencies; plain
    // loads of all rows of all resident blocks are in flight together.
    template <typename T, int MODE>
    __device__ __forceinline__ void q1_epilogue(T * __restrict__ y, int64_t i, T acc, T xc, T ea, T ep, double & part,
                                                float * __restrict__ y32 = nullptr, float * __restrict__ z32 = nullptr)
    {
        typedef Arith<T> M;
        if (MODE == kDefectIR)
        {
            // the outer defect in FP64, handed to the FP32 inner solve as its
            // right-hand side (round to nearest, as convert<> does), the inner
            // guess cleared
            const T d = M::sub(ea, acc);
            y32[i] = (float)d;
            if (z32) z32[i] = 0.f;
            part = fma((double)d, (double)d, part);
        }
        else if (MODE == kPlain) y[i] = acc;
        else if (MODE == kDefect)
        {
            const T d = M::sub(ea, acc);
            y[i] = d;
            part = fma((double)d, (double)d, part);
        }
        else if (MODE == kDot)
        {
            y[i] = acc;
            part = fma((double)acc, (double)xc, part);
        }
        else if (is_jacobi(MODE))
        {
            const T d = M::sub(ea, acc);
            y[i] = M::add(xc, M::mul(ep, d));
            part = fma((double)d, (double)d, part);
        }
    }

    // blocks of 128, 256 or 512 threads (autotuned); one row per thread keeps 2,048
    // threads resident per SM (32 registers)
    template <typename T, int MODE, int R>
    __global__ void __launch_bounds__(kEllMaxThreads, R == 1 ? 2048 / kEllMaxThreads : 1)
    q1_gather_kernel(const __grid_constant__ Q1Stencil<T> s, const T * __restrict__ x, T * __restrict__ y,
                     const T * __restrict__ aux, const T * __restrict__ aux2, ReduceSlot rs, double * red,
                     int want_sqrt, int flags, float * __restrict__ y32, float * __restrict__ z32)
    {
        typedef Arith<T> M;
        const int64_t n = s.n, m = s.m;
        const int t = (int)threadIdx.x;
        const int64_t blk = (flags & kReverse) ? (int64_t)(gridDim.x - 1 - blockIdx.x) : (int64_t)blockIdx.x;
        const int64_t nt = (int64_t)blockDim.x;
        const int64_t i0 = blk * (nt * R) + t;
        uint32_t p[R];
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int64_t i = i0 + k * nt;
            p[k] = i < n ? (uint32_t)((flags & kKeepL2) ? __ldcg(s.pat + i) : __ldcs(s.pat + i)) : s.full;
        }
        pdl_entry();   // x, rhs and P may come from the previous kernel
        if (s.pf)
        {
            // the rows a later wave of blocks will take (in the pass's direction): their
            // pattern ids, x, rhs and P into L2 while this wave's loads are in flight
            const int64_t j = (flags & kReverse) ? i0 - s.pf : i0 + s.pf;
            if (j >= 0 && j < n)
            {
                if ((t & 31) == 0) prefetch_l2(s.pat + j);
                prefetch_l2(x + j);
                if (MODE == kDefect || is_jacobi(MODE) || MODE == kDefectIR) prefetch_l2(aux + j);
                if (is_jacobi(MODE)) prefetch_l2(aux2 + j);
            }
        }
        T xv[R][9], ea[R], ep[R];
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int64_t i = i0 + k * nt;
            // every neighbour of a row inside [m + 1, n - m - 1) exists; the full
            // stencil's rows all lie there, the others read through the table below
            if (i >= m + 1 && i + m + 1 < n)
            {
                const T * a = x + (i - m - 1), * b = x + (i - 1), * c = x + (i + m - 1);
#pragma unroll
                for (int q = 0; q < 3; ++q)
                {
                    xv[k][q] = a[q];
                    xv[k][3 + q] = b[q];
                    xv[k][6 + q] = c[q];
                }
            }
            else
            {
#pragma unroll
                for (int q = 0; q < 9; ++q) xv[k][q] = T(0);
            }
            const bool ok = i < n;
            ea[k] = (ok && (MODE == kDefect || is_jacobi(MODE) || MODE == kDefectIR)) ? aux[i] : T(0);
            ep[k] = (ok && is_jacobi(MODE)) ? aux2[i] : T(0);
        }
        double part = 0.0;
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int64_t i = i0 + k * nt;
            if (i >= n) break;
            T acc, xc;
            if (p[k] == s.full && i >= m + 1 && i + m + 1 < n)
            {
                acc = M::add(T(0), M::mul(s.v[0], xv[k][0]));
#pragma unroll
                for (int q = 1; q < 9; ++q) acc = M::add(acc, M::mul(s.v[q], xv[k][q]));
                xc = xv[k][4];
            }
            else
            {
                acc = q1_any_row<T, 1>(s.tab + p[k] * 9u, x, i, nullptr, 0, 0, 0, false);
                xc = (is_jacobi(MODE) || MODE == kDot) ? x[i] : T(0);
            }
            q1_epilogue<T, MODE>(y, i, acc, xc, ea[k], ep[k], part, y32, z32);
        }
        if ((MODE == kDefect || MODE == kDot || MODE == kDefectIR || MODE == kJacobiNorm) && red != 0)
        {
            // one partial per block; sum_partials_kernel adds them in block order after
            // this launch (no fence or ticket on the block's way out)
            __shared__ double scratch[32];
            const double sum = block_sum(part, scratch);
            if (t == 0) rs.partials[blockIdx.x] = sum;
        }
    }

    // the fused reduction's second step: for vector j = blockIdx.x, partials[j G ..
    // j G + G) summed in a fixed order (thread t adds t, t + 1024, t + 2048, ... in
    // that order, eight independent loads in flight at a time; then the block
    // tree), so the result depends on the data and the launch shape only
    constexpr int kSumThreads = 1024;
    __global__ void __launch_bounds__(kSumThreads) sum_partials_kernel(const double * __restrict__ partials,
                                                                       unsigned G, double * out, int want_sqrt)
    {
        __shared__ double scratch[32];
        partials += (uint64_t)blockIdx.x * G;
        out += blockIdx.x;
        pdl_entry();
        double s = 0.0;
        for (unsigned b0 = threadIdx.x; b0 < G; b0 += 8 * kSumThreads)
        {
            double v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q)
            {
                const unsigned b = b0 + q * kSumThreads;
                v[q] = b < G ? partials[b] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) s += v[q];
        }
        s = block_sum(s, scratch);
        if (threadIdx.x == 0) out[0] = want_sqrt ? sqrt(s) : s;
    }

    void launch_sum_partials(const double * partials, unsigned G, unsigned nvec, double * out, int want_sqrt,
                             cudaStream_t stream)
    {
        launch_pdl(sum_partials_kernel, dim3(nvec), dim3(kSumThreads), 0, stream, partials, G, out, want_sqrt);
        count_launches(1);
    }

    // ------------------------------------------------------------------
    // Pair form: each thread owns two adjacent rows i0 = 2g, i0 + 1 (a warp 64
    // consecutive rows).  The two rows share their x values: per grid row of the
    // stencil four consecutive elements, fetched as two aligned pairs (16 bytes in
    // FP64, 8 in FP32: i0 - m - 1 and i0 + m - 1 are even because m is odd) or, for
    // the centre row, an element, a pair and an element; rhs, P, the pattern ids and
    // the output move as pairs too.  About ten loads per two rows instead of
    // twenty-two, and one index computation: the kernel issues a third of the
    // instructions of the one-row form.  Needs x, rhs, P and y aligned to the pair
    // size (else the interleaved form with two rows per thread runs instead).
    template <typename T> struct Pair;
    template <> struct Pair<double> { typedef double2 type; };
    template <> struct Pair<float> { typedef float2 type; };

    template <typename T, int MODE>
    __device__ __forceinline__ T q1_pair_out(T acc, T xc, T ea, T ep, double & part)
    {
        typedef Arith<T> M;
        if (MODE == kPlain) return acc;
        if (MODE == kDefect || MODE == kDefectIR)
        {
            const T d = M::sub(ea, acc);
            part = fma((double)d, (double)d, part);
            return d;
        }
        if (MODE == kDot)
        {
            part = fma((double)acc, (double)xc, part);
            return acc;
        }
        const T d = M::sub(ea, acc);                       // kJacobi
        part = fma((double)d, (double)d, part);
        return M::add(xc, M::mul(ep, d));
    }

    template <typename T>
    __device__ __forceinline__ T q1_row9(const Q1Stencil<T> & s, const T * a, const T * c, const T * d)
    {
        typedef Arith<T> M;
        T acc = M::add(T(0), M::mul(s.v[0], a[0]));
        acc = M::add(acc, M::mul(s.v[1], a[1]));
        acc = M::add(acc, M::mul(s.v[2], a[2]));
        acc = M::add(acc, M::mul(s.v[3], c[0]));
        acc = M::add(acc, M::mul(s.v[4], c[1]));
        acc = M::add(acc, M::mul(s.v[5], c[2]));
        acc = M::add(acc, M::mul(s.v[6], d[0]));
        acc = M::add(acc, M::mul(s.v[7], d[1]));
        return M::add(acc, M::mul(s.v[8], d[2]));
    }

    template <typename T, int MODE>
    __global__ void __launch_bounds__(kEllThreads)
    q1_pair_kernel(const __grid_constant__ Q1Stencil<T> s, const T * __restrict__ x, T * __restrict__ y,
                   const T * __restrict__ aux, const T * __restrict__ aux2, ReduceSlot rs, double * red, int flags,
                   float * __restrict__ y32, float * __restrict__ z32)
    {
        typedef typename Pair<T>::type V;
        const int n = (int)s.n, m = (int)s.m;
        const int t = (int)threadIdx.x;
        const int blk = (flags & kReverse) ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
        const int i0 = 2 * (blk * kEllThreads + t);
        const bool any = i0 < n, two = i0 + 1 < n;
        uint32_t p0 = s.full, p1 = s.full;
        if (two)
        {
            const uint32_t pp = (uint32_t)((flags & kKeepL2) ? __ldcg((const unsigned short *)(s.pat + i0))
                                                            : __ldcs((const unsigned short *)(s.pat + i0)));
            p0 = pp & 0xffu;
            p1 = pp >> 8;
        }
        else if (any) p0 = s.pat[i0];
        pdl_entry();   // x, rhs and P may come from the previous kernel
        // both rows' neighbours exist: x[i0 - m - 1 .. i0 + m + 2]
        const bool inner = two && i0 >= m + 1 && i0 + m + 2 < n;
        T a[4], c[4], d[4];
        if (inner)
        {
            const V a01 = *(const V *)(x + (i0 - m - 1)), a23 = *(const V *)(x + (i0 - m + 1));
            const V c12 = *(const V *)(x + i0);
            const V d01 = *(const V *)(x + (i0 + m - 1)), d23 = *(const V *)(x + (i0 + m + 1));
            c[0] = x[i0 - 1];
            c[3] = x[i0 + 2];
            a[0] = a01.x; a[1] = a01.y; a[2] = a23.x; a[3] = a23.y;
            c[1] = c12.x; c[2] = c12.y;
            d[0] = d01.x; d[1] = d01.y; d[2] = d23.x; d[3] = d23.y;
        }
        T ea0 = T(0), ea1 = T(0), ep0 = T(0), ep1 = T(0);
        if (MODE == kDefect || is_jacobi(MODE) || MODE == kDefectIR)
        {
            if (two) { const V v = *(const V *)(aux + i0); ea0 = v.x; ea1 = v.y; }
            else if (any) ea0 = aux[i0];
        }
        if (is_jacobi(MODE))
        {
            if (two) { const V v = *(const V *)(aux2 + i0); ep0 = v.x; ep1 = v.y; }
            else if (any) ep0 = aux2[i0];
        }
        double part = 0.0;
        T o0 = T(0), o1 = T(0);
        if (any)
        {
            T acc, xc;
            if (inner && p0 == s.full) { acc = q1_row9(s, a, c, d); xc = c[1]; }
            else
            {
                acc = q1_any_row<T, 1>(s.tab + p0 * 9u, x, i0, nullptr, 0, 0, 0, false);
                xc = (is_jacobi(MODE) || MODE == kDot) ? x[i0] : T(0);
            }
            o0 = q1_pair_out<T, MODE>(acc, xc, ea0, ep0, part);
        }
        if (two)
        {
            T acc, xc;
            if (inner && p1 == s.full) { acc = q1_row9(s, a + 1, c + 1, d + 1); xc = c[2]; }
            else
            {
                acc = q1_any_row<T, 1>(s.tab + p1 * 9u, x, i0 + 1, nullptr, 0, 0, 0, false);
                xc = (is_jacobi(MODE) || MODE == kDot) ? x[i0 + 1] : T(0);
            }
            o1 = q1_pair_out<T, MODE>(acc, xc, ea1, ep1, part);
        }
        if (MODE == kDefectIR)
        {
            // the FP64 defect handed to the FP32 inner solve (round to nearest, as
            // convert<> does), the inner guess cleared
            if (two)
            {
                *(float2 *)(y32 + i0) = make_float2((float)o0, (float)o1);
                if (z32) *(float2 *)(z32 + i0) = make_float2(0.f, 0.f);
            }
            else if (any)
            {
                y32[i0] = (float)o0;
                if (z32) z32[i0] = 0.f;
            }
        }
        else if (two)
        {
            V v;
            v.x = o0;
            v.y = o1;
            *(V *)(y + i0) = v;
        }
        else if (any) y[i0] = o0;
        if ((MODE == kDefect || MODE == kDot || MODE == kDefectIR || MODE == kJacobiNorm) && red != 0)
        {
            __shared__ double scratch[32];
            const double sum = block_sum(part, scratch);
            if (t == 0) rs.partials[blockIdx.x] = sum;
        }
    }

    template <typename T, int R>
    static constexpr size_t q1_stencil_smem()
    {
        return (size_t)3 * ((kEllThreads * R + 2 + 2 * (16 / sizeof(T)) + 16 / sizeof(T) - 1) / (16 / sizeof(T)) *
                            (16 / sizeof(T))) * sizeof(T);
    }

    template <typename T, int MODE, int R>
    static void q1_stencil_launch(const Q1Stencil<T> & s, dim3 grid, cudaStream_t st, const void * x, void * y,
                                  const void * aux, const void * aux2, ReduceSlot rs, double * red, int want_sqrt,
                                  int flags)
    {
        constexpr size_t smem = q1_stencil_smem<T, R>();
        if (smem > 48 * 1024)
        {
            // dynamic shared memory above 48 KiB needs the kernel's opt-in, once per device
            static bool done[64] = {};
            int dev = 0;
            cudaGetDevice(&dev);
            if (dev >= 0 && dev < 64 && ! done[dev])
            {
                cudaFuncSetAttribute(q1_stencil_kernel<T, MODE, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem);
                done[dev] = true;
            }
        }
        launch_pdl(q1_stencil_kernel<T, MODE, R>, grid, dim3(kEllThreads), smem, st, s, (const T *)x, (T *)y,
                   (const T *)aux, (const T *)aux2, rs, red, want_sqrt, flags);
    }

    // ------------------------------------------------------------------
    // Strip form (a pin, HB2_ELL_COMPACT=q1stripS; measured slower than the gather
    // form on B200 at every level, precision, strip length and block size, so the
    // autotuner does not time it): thread g (of m * ceil(m / S)) owns grid column j = g % m and the
    // S grid rows r = S (g / m) .. S (g / m) + S - 1 of that column, node i = r m + j.
    // The three x values a node takes from each stencil row (flattened indices
    // r' m + j - 1, r' m + j, r' m + j + 1 for r' = r - 1, r, r + 1) stay in registers
    // as the strip moves down: each node loads the three of the row below it, not
    // nine.  A warp's 32 threads are 32 consecutive columns (contiguous loads).  The
    // registers hold exactly the values the gather form reads at i - m - 1 ..
    // i + m + 1 (loads outside [0, n) give 0 and are used by no full-stencil row), so
    // the sums are the gather form's bit for bit; rows of other patterns take the
    // general slot loop.  The per-block partial of a fused reduction goes to
    // rs.partials as in the gather form.
    template <typename T>
    __device__ __forceinline__ void q1_strip_row(const T * __restrict__ x, int64_t b, int64_t n, bool keep,
                                                 T (&v)[3])
    {
        // x[b - 1], x[b], x[b + 1], 0 outside [0, n)
#pragma unroll
        for (int q = 0; q < 3; ++q)
        {
            const int64_t g = b - 1 + q;
            v[q] = (g >= 0 && g < n) ? (keep ? __ldcg(x + g) : __ldg(x + g)) : T(0);
        }
    }

    template <typename T, int MODE, int S>
    __global__ void __launch_bounds__(kEllMaxThreads)
    q1_strip_kernel(const __grid_constant__ Q1Stencil<T> s, const T * __restrict__ x, T * __restrict__ y,
                    const T * __restrict__ aux, const T * __restrict__ aux2, ReduceSlot rs, double * red, int flags,
                    float * __restrict__ y32, float * __restrict__ z32)
    {
        const int64_t n = s.n, m = s.m;
        const int64_t strips = (m + S - 1) / S;
        const int64_t blk = (flags & kReverse) ? (int64_t)(gridDim.x - 1 - blockIdx.x) : (int64_t)blockIdx.x;
        const int64_t g = blk * blockDim.x + threadIdx.x;
        const bool keep = (flags & kKeepL2) != 0;
        pdl_entry();   // x, rhs and P may come from the previous kernel
        double part = 0.0;
        if (g < m * strips)
        {
            const int64_t j = g % m, r0 = (g / m) * S;
            T up[3], mid[3];
            q1_strip_row<T>(x, (r0 - 1) * m + j, n, keep, up);
            q1_strip_row<T>(x, r0 * m + j, n, keep, mid);
#pragma unroll
            for (int t = 0; t < S; ++t)
            {
                const int64_t r = r0 + t;
                if (r >= m) break;
                const int64_t i = r * m + j;
                T lo[3];
                q1_strip_row<T>(x, i + m, n, keep, lo);
                const uint32_t p = keep ? __ldcg(s.pat + i) : __ldcs(s.pat + i);
                const T ea = (MODE == kDefect || is_jacobi(MODE) || MODE == kDefectIR) ? aux[i] : T(0);
                const T ep = is_jacobi(MODE) ? aux2[i] : T(0);
                T acc;
                if (p == s.full && i >= m + 1 && i + m + 1 < n) acc = q1_row9<T>(s, up, mid, lo);
                else acc = q1_any_row<T, 1>(s.tab + p * 9u, x, i, nullptr, 0, 0, 0, false);
                q1_epilogue<T, MODE>(y, i, acc, mid[1], ea, ep, part, y32, z32);
#pragma unroll
                for (int q = 0; q < 3; ++q)
                {
                    up[q] = mid[q];
                    mid[q] = lo[q];
                }
            }
        }
        if ((MODE == kDefect || MODE == kDot || MODE == kDefectIR || MODE == kJacobiNorm) && red != 0)
        {
            __shared__ double scratch[32];
            const double sum = block_sum(part, scratch);
            if (threadIdx.x == 0) rs.partials[blockIdx.x] = sum;
        }
    }

    // blocks of a strip-form launch
    unsigned q1_strip_grid(const hb2_ell_s * A, int S, unsigned bs)
    {
        const uint64_t m = (uint64_t)A->pat_win_m, strips = (m + S - 1) / S;
        return ceil_div(m * strips, bs);
    }

    template <typename T, int MODE>
    static void q1_stencil_mode(const hb2_ell_s * A, int R, dim3 grid, cudaStream_t st, const void * x, void * y,
                                const void * aux, const void * aux2, ReduceSlot rs, double * red, int want_sqrt,
                                int flags, unsigned bs)
    {
        Q1Stencil<T> s;
        for (int k = 0; k < 9; ++k) s.v[k] = (T)A->q1_val[k];
        s.pat = A->pat;
        s.tab = (const PatEnt<T> *)A->ptab;
        s.n = (int64_t)A->rows;
        s.m = A->pat_win_m;
        s.full = (uint32_t)A->q1_full;
        s.pf = (R & kPatQ1G) ? l2_prefetch_rows(sizeof(T)) : 0;
        if (R & kPatQ1P)
        {
            // two adjacent rows per thread; the interleaved form where the vectors are
            // not aligned to pairs (same rows per block)
            // (the pairs of the x rows at -m and +m are aligned because m is odd)
            const uintptr_t al = 2 * sizeof(T) - 1;
            if ((((uintptr_t)x | (uintptr_t)y | (uintptr_t)aux | (uintptr_t)aux2) & al) == 0 && (A->pat_win_m & 1) &&
                A->rows < (1ull << 31) - 4096)
            {
                launch_pdl(q1_pair_kernel<T, MODE>, grid, dim3(kEllThreads), 0, st, s, (const T *)x, (T *)y,
                           (const T *)aux, (const T *)aux2, rs, red, flags, (float *)nullptr, (float *)nullptr);
                return;
            }
            R = kPatQ1G | 2;
        }
        if (R & kPatQ1S)
        {
            R &= ~kPatQ1S;
#define HB2_Q1S_(S_) launch_pdl(q1_strip_kernel<T, MODE, S_>, grid, dim3(bs), 0, st, s, (const T *)x, (T *)y,      \
                                (const T *)aux, (const T *)aux2, rs, red, flags, (float *)nullptr, (float *)nullptr)
            if (R == 2) HB2_Q1S_(2);
            else if (R == 4) HB2_Q1S_(4);
            else HB2_Q1S_(8);
#undef HB2_Q1S_
            return;
        }
        if (R & kPatQ1G)
        {
            R &= ~kPatQ1G;
#define HB2_Q1G(R_) launch_pdl(q1_gather_kernel<T, MODE, R_>, grid, dim3(bs), 0, st, s, (const T *)x, (T *)y, \
                               (const T *)aux, (const T *)aux2, rs, red, want_sqrt, flags, (float *)nullptr,      \
                               (float *)nullptr)
            if (R == 1) HB2_Q1G(1);
            else if (R == 2) HB2_Q1G(2);
            else HB2_Q1G(4);
#undef HB2_Q1G
            return;
        }
        if (R == 2) q1_stencil_launch<T, MODE, 2>(s, grid, st, x, y, aux, aux2, rs, red, want_sqrt, flags);
        else if (R == 4) q1_stencil_launch<T, MODE, 4>(s, grid, st, x, y, aux, aux2, rs, red, want_sqrt, flags);
        else q1_stencil_launch<T, MODE, 8>(s, grid, st, x, y, aux, aux2, rs, red, want_sqrt, flags);
    }

    bool ell_q1_stencil_applies(const hb2_ell_s * A, int mode, const void * x, int rpt, const Batch & b)
    {
        // the windows' bulk copies need a 16-byte aligned x (the gather form needs nothing)
        const bool aligned = (rpt & (kPatQ1G | kPatQ1P | kPatQ1S)) || ((uintptr_t)x & 15) == 0;
        return A->q1_full >= 0 && A->pat_win_m && A->K == 9 && ! b.list && b.nvec == 1 && ! b.active &&
               (mode == kPlain || mode == kDefect || mode == kDot || mode == kJacobi) && aligned;
    }

    void launch_ell_q1_stencil(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux,
                               const void * aux2, double * red, int want_sqrt, ReduceSlot rs, dim3 grid,
                               cudaStream_t stream, int flags, int R, unsigned bs)
    {
        // R: rows per thread, with kPatQ1G for the gather form, kPatQ1P for the pair form
#define HB2_Q1S(T_, M_) q1_stencil_mode<T_, M_>(A, R, grid, stream, x, y, aux, aux2, rs, red, want_sqrt, flags, bs)
        if (A->dtype == HB2_F64)
        {
            if (mode == kPlain) HB2_Q1S(double, kPlain);
            else if (mode == kDefect) HB2_Q1S(double, kDefect);
            else if (mode == kDot) HB2_Q1S(double, kDot);
            else if (red) HB2_Q1S(double, kJacobiNorm);
            else HB2_Q1S(double, kJacobi);
        }
        else
        {
            if (mode == kPlain) HB2_Q1S(float, kPlain);
            else if (mode == kDefect) HB2_Q1S(float, kDefect);
            else if (mode == kDot) HB2_Q1S(float, kDot);
            else if (red) HB2_Q1S(float, kJacobiNorm);
            else HB2_Q1S(float, kJacobi);
        }
#undef HB2_Q1S
    }

    int launch_ir_defect(const hb2_ell_s * A, const double * x, const double * b, float * b32, float * x32,
                         double * r64, double * red, const Workspace * ws, cudaStream_t stream)
    {
        const uint64_t n = A->rows;
        const unsigned grid = ceil_div(n, kEllThreads);
        if (A->dtype == HB2_F64 && A->q1_full >= 0 && A->pat && A->pat_win_m && A->K == 9 && n > 0 &&
            grid <= ws->max_blocks)
        {
            Q1Stencil<double> s;
            for (int k = 0; k < 9; ++k) s.v[k] = A->q1_val[k];
            s.pat = A->pat;
            s.tab = (const PatEnt<double> *)A->ptab;
            s.n = (int64_t)n;
            s.m = A->pat_win_m;
            s.full = (uint32_t)A->q1_full;
            const ReduceSlot rs = ws->slot();
            const unsigned pgrid = ceil_div(n, 2 * kEllThreads);
            if (((((uintptr_t)x | (uintptr_t)b) & 15) | (((uintptr_t)b32 | (uintptr_t)x32) & 7)) == 0 &&
                (A->pat_win_m & 1) && n < (1ull << 31) - 4096)
            {
                launch_pdl(q1_pair_kernel<double, kDefectIR>, dim3(pgrid), dim3(kEllThreads), 0, stream, s, x,
                           (double *)nullptr, b, (const double *)nullptr, rs, red, 0, b32, x32);
                launch_pdl(sum_partials_kernel, dim3(1), dim3(kSumThreads), 0, stream, (const double *)rs.partials,
                           pgrid, red, 1);
                count_launches(2);
                HB2_LAUNCH_CHECK("IR defect launch");
                return HB2_OK;
            }
            launch_pdl(q1_gather_kernel<double, kDefectIR, 1>, dim3(grid), dim3(kEllThreads), 0, stream, s, x,
                       (double *)nullptr, b, (const double *)nullptr, rs, red, 1, 0, b32, x32);
            launch_pdl(sum_partials_kernel, dim3(1), dim3(kSumThreads), 0, stream, (const double *)rs.partials, grid,
                       red, 1);
            count_launches(2);
            HB2_LAUNCH_CHECK("IR defect launch");
            return HB2_OK;
        }
        int st = launch_ell(A, kDefect, x, r64, b, 0, 0, red, 1, ws, stream);
        if (! st) st = launch_convert(HB2_F32, b32, HB2_F64, r64, n, stream);
        if (! st && x32) st = launch_fill(HB2_F32, x32, 0.0, n, stream);
        return st;
    }

    // After the row-pattern layout is built: the pattern, if any, that holds the
    // full nine-point stencil of an m x m grid in ascending column order (at most
    // one is used; rows of other full patterns take the general slot loop).
    template <typename T>
    static void find_q1_stencil_typed(hb2_ell_s * A)
    {
        const int64_t m = A->pat_win_m;
        std::vector<PatEnt<T>> tab((size_t)A->npat * 9);
        if (cudaMemcpy(tab.data(), A->ptab, tab.size() * sizeof(PatEnt<T>), cudaMemcpyDeviceToHost) != cudaSuccess)
        {
            cudaGetLastError();
            return;
        }
        const int64_t want[9] = {-m - 1, -m, -m + 1, -1, 0, 1, m - 1, m, m + 1};
        for (uint32_t q = 0; q < A->npat; ++q)
        {
            bool full = true;
            for (int k = 0; k < 9 && full; ++k) full = tab[(size_t)q * 9 + k].off == want[k];
            if (! full) continue;
            A->q1_full = (int)q;
            for (int k = 0; k < 9; ++k) A->q1_val[k] = (double)tab[(size_t)q * 9 + k].val;
            return;
        }
    }

    void ell_find_q1_stencil(hb2_ell_s * A)
    {
        A->q1_full = -1;
        if (! A->pat || ! A->ptab || ! A->pat_win_m || A->K != 9 || A->pat_win_m > (1 << 20)) return;
        if (A->dtype == HB2_F64) find_q1_stencil_typed<double>(A);
        else find_q1_stencil_typed<float>(A);
    }
}
