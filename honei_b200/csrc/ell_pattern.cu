// Row-pattern device layout for square SparseMatrixELL matrices.
//
// Stencil and FEM operators on structured grids repeat a handful of rows: every
// interior row of the Q1 Poisson matrix has the same nine (value, column - row)
// pairs, every Dirichlet row the same single one.  When a square matrix has at
// most kPatMax distinct rows in that sense (its compressed layout -- value codes
// and 16-bit column offsets, ell_compact.cu -- exists and repeats), each row is
// stored as a one-byte pattern id and the pattern table (K (value, offset)
// entries per pattern) lives in shared memory: 1 byte per row instead of 3 per
// slot.  A warp computes 32 consecutive rows per step (one per lane, R steps per
// thread), so every pattern, vector and gather load is coalesced, and the
// kernel forms exactly the products and slot-ordered sums of the plain layout:
// results are bit-identical.  Creation: each row's (code, offset) signature is
// hashed, distinct hashes are collected in a small device hash set, every row
// is verified against its pattern's representative row (a hash collision
// abandons the layout), and the autotuner (ell_compact.cu) then decides per
// kernel class whether this layout is the fastest.
#include "hb2_common.cuh"
#include "hb2_internal.hh"
#include "tma.cuh"

#include <climits>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace hb2
{
    constexpr uint32_t kPatSlots = 1024;                  // hash set
    constexpr unsigned long long kPatEmptyKey = ~0ull;

    template <typename T>
    struct EllPatternView
    {
        const uint8_t * pat;
        const PatEnt<T> * tab;   // npat * K entries
        uint64_t rows;
        uint32_t K, npat;
    };

    __device__ __forceinline__ unsigned long long row_signature(const uint8_t * code, const int16_t * delta, uint64_t ld,
                                                                uint32_t K, uint64_t r)
    {
        unsigned long long h = 0xcbf29ce484222325ull;
        for (uint32_t k = 0; k < K; ++k)
        {
            const uint32_t w = (uint32_t)code[(uint64_t)k * ld + r] | ((uint32_t)(uint16_t)delta[(uint64_t)k * ld + r] << 8);
            h = (h ^ w) * 0x100000001b3ull;
            h ^= h >> 29;
        }
        return h == kPatEmptyKey ? h - 1 : h;
    }

    __device__ __forceinline__ uint32_t pat_hash(unsigned long long k)
    {
        k ^= k >> 31;
        k *= 0x9e3779b97f4a7c15ull;
        return (uint32_t)(k >> 40) & (kPatSlots - 1);
    }

    // signatures into the hash set; one insert per distinct signature of a warp
    __global__ void pat_insert_kernel(const uint8_t * code, const int16_t * delta, uint64_t ld, uint32_t K,
                                      uint64_t rows, unsigned long long * sig, unsigned long long * keys,
                                      unsigned * nkeys, int * flag)
    {
        const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
        for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < rows; base += stride)
        {
            const uint64_t r = base + threadIdx.x;
            const bool ok = r < rows;
            const unsigned long long h = ok ? row_signature(code, delta, ld, K, r) : kPatEmptyKey;
            if (ok) sig[r] = h;
            const unsigned peers = __match_any_sync(0xffffffffu, h);
            if (! ok || (threadIdx.x & 31) != (unsigned)(__ffs(peers) - 1)) continue;
            uint32_t s = pat_hash(h);
            bool placed = false;
            for (uint32_t p = 0; p < kPatSlots; ++p)
            {
                const unsigned long long prev = atomicCAS(keys + s, kPatEmptyKey, h);
                if (prev == kPatEmptyKey) { atomicAdd(nkeys, 1u); placed = true; break; }
                if (prev == h) { placed = true; break; }
                s = (s + 1) & (kPatSlots - 1);
            }
            if (! placed) atomicExch(flag, 1);
        }
    }

    // pattern id per row, and the smallest row of each pattern (its representative)
    __global__ void pat_encode_kernel(const unsigned long long * sig, uint64_t rows, const unsigned long long * keys,
                                      const uint8_t * id_of_slot, uint8_t * pat, unsigned * rep, int * flag)
    {
        const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
        for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < rows; base += stride)
        {
            const uint64_t r = base + threadIdx.x;
            int id = -1;
            if (r < rows)
            {
                const unsigned long long h = sig[r];
                uint32_t s = pat_hash(h), p = 0;
                while (keys[s] != h && p < kPatSlots) { s = (s + 1) & (kPatSlots - 1); ++p; }
                if (p == kPatSlots) atomicExch(flag, 2);
                else
                {
                    id = id_of_slot[s];
                    pat[r] = (uint8_t)id;
                }
            }
            // the lowest lane of each id in the warp holds the warp's smallest row of it
            const unsigned peers = __match_any_sync(0xffffffffu, id);
            if (id >= 0 && (threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) atomicMin(rep + id, (unsigned)r);
        }
    }

    // every row equals its pattern's representative row, slot by slot
    __global__ void pat_verify_kernel(const uint8_t * code, const int16_t * delta, uint64_t ld, uint32_t K, uint64_t rows,
                                      const uint8_t * pat, const unsigned * rep, int * flag)
    {
        const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
        for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += stride)
        {
            const uint64_t q = rep[pat[r]];
            for (uint32_t k = 0; k < K; ++k)
                if (code[(uint64_t)k * ld + r] != code[(uint64_t)k * ld + q] || delta[(uint64_t)k * ld + r] != delta[(uint64_t)k * ld + q])
                {
                    atomicExch(flag, 3);
                    break;
                }
        }
    }

    // ------------------------------------------------------------------ kernel
    // One warp: 32 consecutive rows per step, R steps (rows w*32R + i*32 + lane).
    template <typename T, int KT, int MODE, int R>
    __global__ void __launch_bounds__(kEllThreads)
    ell_pattern_kernel(EllPatternView<T> A, const T * __restrict__ x_, T * __restrict__ y_, const T * __restrict__ aux_,
                       const T * __restrict__ aux2, T * __restrict__ zero_, ReduceSlot rs, double * red_, int want_sqrt,
                       int flags, Batch bt)
    {
        typedef Arith<T> M;
        __shared__ PatEnt<T> tab[kPatMax * kPatMaxK];
        const int K = KT > 0 ? KT : (int)A.K;
        for (uint32_t i = threadIdx.x; i < A.npat * (uint32_t)K; i += blockDim.x) tab[i] = A.tab[i];
        __syncthreads();
        pdl_entry();   // the pattern table is constant: loaded before the wait
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
            double * red = red_ ? red_ + j : red_;
            const uint64_t bx = listed ? item % bt.gx : blockIdx.x;
            const uint64_t blk = (flags & kReverse) ? (gridDim.x - 1 - bx) : bx;
            const uint64_t r0 = blk * (uint64_t)kEllThreads * R + (uint64_t)(threadIdx.x >> 5) * 32 * R + (threadIdx.x & 31);
            // every load that does not depend on the pattern is issued first
            uint32_t p[R];
            T acc[R], ea[R], ep[R], ex[R];
#pragma unroll
            for (int i = 0; i < R; ++i)
            {
                const uint64_t r = r0 + 32 * i;
                const bool ok = r < A.rows;
                p[i] = ok ? (uint32_t)__ldcs(A.pat + r) : 0u;
                acc[i] = T(0);
                if (MODE == kDefect || is_jacobi(MODE)) ea[i] = ok ? aux[r] : T(0);
                if (is_jacobi(MODE)) { ep[i] = ok ? aux2[r] : T(0); ex[i] = ok ? x[r] : T(0); }
                if (MODE == kDot) ex[i] = ok ? x[r] : T(0);
                if (MODE == kAdd) ex[i] = ok ? y[r] : T(0);
            }
            // per row, once: the bound test, the row's x pointer (a gather is then one
            // sign-extended offset) and its pattern's table entries
            bool rok[R];
            const T * xr[R];
            const PatEnt<T> * te[R];
#pragma unroll
            for (int i = 0; i < R; ++i)
            {
                const uint64_t r = r0 + 32 * i;
                rok[i] = r < A.rows;
                xr[i] = x + (rok[i] ? r : 0);
                te[i] = tab + p[i] * (uint32_t)K;
            }
#pragma unroll
            for (int k = 0; k < (KT > 0 ? KT : kPatMaxK); ++k)
            {
                if (KT == 0 && k >= K) break;
#pragma unroll
                for (int i = 0; i < R; ++i)
                {
                    const PatEnt<T> e = te[i][k];
                    if (rok[i] && e.off != kPatEmpty) acc[i] = M::add(acc[i], M::mul(e.val, __ldg(xr[i] + e.off)));
                }
            }
            double part = 0.0;
#pragma unroll
            for (int i = 0; i < R; ++i)
            {
                const uint64_t r = r0 + 32 * i;
                if (r >= A.rows) continue;
                if (MODE == kPlain) y[r] = acc[i];
                else if (MODE == kDefect)
                {
                    const T d = M::sub(ea[i], acc[i]);
                    y[r] = d;
                    part = fma((double)d, (double)d, part);
                }
                else if (MODE == kDot)
                {
                    y[r] = acc[i];
                    part = fma((double)acc[i], (double)ex[i], part);
                }
                else if (MODE == kAdd) y[r] = M::add(ex[i], acc[i]);
                else if (is_jacobi(MODE))
                {
                    const T d = M::sub(ea[i], acc[i]);
                    y[r] = M::add(ex[i], M::mul(ep[i], d));
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

    // diagnostic: set when a windowed block's copies did not complete in time (the
    // block then computed from global memory)
    __device__ int g_pat_win_timeout = 0;

    // Extent of one x window of the windowed kernel: rows [lo, hi) of x (the
    // window's B + 2 rows clipped to the vector), of which the bulk copy moves
    // [alo, ahi) (ends rounded down to 16 bytes); plain loads fetch the ragged
    // tail [max(ahi, lo), hi), at most E - 1 elements.
    struct WinGeom
    {
        int64_t lo, hi, alo, ahi;
    };

    template <int B, int E>
    __device__ __forceinline__ WinGeom win_geom(int64_t start, int64_t n)
    {
        WinGeom g;
        g.lo = start < 0 ? 0 : start;
        g.hi = start + B + 2 > n ? n : start + B + 2;
        if (g.hi < g.lo) g.hi = g.lo;
        g.alo = g.lo - (g.lo % E);
        g.ahi = g.hi - (g.hi % E);
        return g;
    }

    // The row-pattern kernel for a square matrix whose pattern offsets all lie in the
    // three bands around -m, 0, +m (the Q1 operators, m^2 rows).  A block owns
    // B = 256 R rows, interleaved over its threads; thread 0 stages the three windows
    // of x that the bands touch with bulk copies (as the banded kernel does) and
    // threads 1 .. 3 (E - 1) fetch the windows' ragged tails, while every thread loads
    // its rows' pattern ids and vectors and its share of the pattern table; the
    // block meets once, and the gathers then read shared memory.  Each table entry
    // carries its window-relative offset for this block (every thread computes the
    // window geometry itself).  If the copies have not completed within the bounded
    // wait, the block computes from global memory (same bits) and waits for them
    // once more before it exits.
    template <typename T, int MODE, int R>
    __global__ void __launch_bounds__(kEllThreads)
    ell_pattern_win_kernel(EllPatternView<T> A, int64_t m, const T * __restrict__ x, T * __restrict__ y,
                           const T * __restrict__ aux, const T * __restrict__ aux2, T * __restrict__ zero,
                           ReduceSlot rs, double * red, int want_sqrt, int flags)
    {
        typedef Arith<T> M;
        constexpr int K = 9;
        constexpr int B = kEllThreads * R;
        constexpr int E = 16 / sizeof(T);
        constexpr int W = (B + 2 + 2 * E + E - 1) / E * E;
        constexpr int TE = (kPatMax * K + kEllThreads - 1) / kEllThreads;   // table entries per thread
        struct alignas(16) WEnt
        {
            T val;
            int32_t off;    // column - row (kPatEmpty past the row)
            int32_t rel;    // index in `win` minus the row
        };
        __shared__ WEnt tab[kPatMax * K];
        __shared__ alignas(128) T win[3 * W];
        __shared__ alignas(8) uint64_t bar;
        const int64_t n = (int64_t)A.rows;
        const int64_t r0 = (int64_t)blockIdx.x * B;
        const unsigned t = threadIdx.x;
        const int64_t starts[3] = {r0 - m - 1, r0 - 1, r0 + m - 1};
        uint32_t p[R];
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int64_t i = r0 + (int64_t)k * kEllThreads + t;
            p[k] = i < n ? (uint32_t)__ldcs(A.pat + i) : 0u;
        }
        // the pattern table is constant: fetched before the wait on the previous kernel
        const uint32_t nent = A.npat * (uint32_t)K;
        PatEnt<T> mine[TE];
#pragma unroll
        for (int q = 0; q < TE; ++q)
        {
            const uint32_t j = t + q * kEllThreads;
            if (j < nent) mine[q] = A.tab[j];
        }
        pdl_entry();   // the vectors below may come from the previous kernel
        T ea[R], ep[R], ey[R];
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int64_t i = r0 + (int64_t)k * kEllThreads + t;
            const bool ok = i < n;
            ea[k] = (ok && (MODE == kDefect || is_jacobi(MODE))) ? aux[i] : T(0);
            ep[k] = (ok && is_jacobi(MODE)) ? aux2[i] : T(0);
            ey[k] = (ok && MODE == kAdd) ? y[i] : T(0);
        }
        if (t == 0)
        {
            mbar_init(&bar, 1);
            WinGeom g[3];
            unsigned total = 0;
#pragma unroll
            for (int w = 0; w < 3; ++w)
            {
                g[w] = win_geom<B, E>(starts[w], n);
                total += (unsigned)((g[w].ahi - g[w].alo) * sizeof(T));
            }
            mbar_expect_tx(&bar, total);
#pragma unroll
            for (int w = 0; w < 3; ++w)
                if (g[w].ahi > g[w].alo)
                    bulk_g2s(&win[w * W], x + g[w].alo, (unsigned)((g[w].ahi - g[w].alo) * sizeof(T)), &bar);
        }
        else if (t <= 3 * (E - 1))
        {
            const int w = (int)(t - 1) / (E - 1), e = (int)(t - 1) % (E - 1);
            const WinGeom g = win_geom<B, E>(w == 0 ? starts[0] : (w == 1 ? starts[1] : starts[2]), n);
            const int64_t j = (g.ahi > g.lo ? g.ahi : g.lo) + e;
            if (j < g.hi) win[w * W + (j - g.alo)] = x[j];
        }
        int64_t wbase[3];
#pragma unroll
        for (int w = 0; w < 3; ++w) wbase[w] = win_geom<B, E>(starts[w], n).alo;
#pragma unroll
        for (int q = 0; q < TE; ++q)
        {
            const uint32_t j = t + q * kEllThreads;
            if (j < nent)
            {
                const PatEnt<T> e = mine[q];
                WEnt qe;
                qe.val = e.val;
                qe.off = e.off;
                qe.rel = 0;
                if (e.off != kPatEmpty)
                {
                    const int w = e.off <= -2 ? 0 : (e.off <= 1 ? 1 : 2);
                    const int64_t wb = w == 0 ? wbase[0] : (w == 1 ? wbase[1] : wbase[2]);
                    qe.rel = (int32_t)((int64_t)e.off - wb + (int64_t)w * W);
                }
                tab[j] = qe;
            }
        }
        __syncthreads();
        const bool fast = mbar_wait_bounded(&bar, 0, 1000000000ull);
        if (! fast && t == 0) atomicExch(&g_pat_win_timeout, 1);
        double part = 0.0;
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int64_t i = r0 + (int64_t)k * kEllThreads + t;
            if (i >= n) continue;
            const WEnt * te = tab + p[k] * K;
            T acc = T(0);
#pragma unroll
            for (int j = 0; j < K; ++j)
            {
                const WEnt e = te[j];
                if (e.off != kPatEmpty)
                {
                    const T xv = fast ? win[i + e.rel] : __ldg(x + (i + e.off));
                    acc = M::add(acc, M::mul(e.val, xv));
                }
            }
            const T xc = (is_jacobi(MODE) || MODE == kDot) ? (fast ? win[(i - wbase[1]) + W] : x[i]) : T(0);
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
            else if (MODE == kAdd) y[i] = M::add(ey[k], acc);
            else if (is_jacobi(MODE))
            {
                const T d = M::sub(ea[k], acc);
                y[i] = M::add(xc, M::mul(ep[k], d));
                part = fma((double)d, (double)d, part);
            }
            else if (MODE == kRestrict) { y[i] = acc; zero[i] = T(0); }
        }
        if ((MODE == kDefect || MODE == kDot || MODE == kJacobiNorm) && red != 0)
        {
            __shared__ double scratch[32];
            ell_block_reduce(part, rs, red, want_sqrt, flags, scratch);
        }
        // copies still in flight must land before the block's shared memory is reused
        if (! fast) mbar_wait_bounded(&bar, 0, 1000000000ull);
    }

    template <typename T, int MODE>
    static void pattern_mode(const hb2_ell_s * A, const void * x, void * y, const void * aux, const void * aux2,
                             void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid, cudaStream_t s,
                             int flags, Batch b, int R, unsigned bs)
    {
        EllPatternView<T> v;
        v.pat = A->pat;
        v.tab = (const PatEnt<T> *)A->ptab;
        v.rows = A->rows;
        v.K = A->K;
        v.npat = A->npat;
        if ((R & (kPatQ1 | kPatQ1G | kPatQ1S)) && ell_q1_stencil_applies(A, MODE, x, R, b))
        {
            launch_ell_q1_stencil(A, MODE, x, y, aux, aux2, red, want_sqrt, rs, grid, s, flags,
                                  (R & ~kPatFlags) | (R & (kPatQ1G | kPatQ1S)), bs);
            return;
        }
        // the window copies need a 16-byte aligned x
        if ((R & kPatWin) && A->pat_win_m && A->K == 9 && ! b.list && b.nvec == 1 && ! b.active &&
            ((uintptr_t)x & 15) == 0)
        {
            const int Rw = R & ~kPatWin;
            if (Rw == 1)
                launch_pdl(ell_pattern_win_kernel<T, MODE, 1>, grid, dim3(kEllThreads), 0, s, v, A->pat_win_m,
                           (const T *)x, (T *)y, (const T *)aux, (const T *)aux2, (T *)zero, rs, red, want_sqrt, flags);
            else
                launch_pdl(ell_pattern_win_kernel<T, MODE, 2>, grid, dim3(kEllThreads), 0, s, v, A->pat_win_m,
                           (const T *)x, (T *)y, (const T *)aux, (const T *)aux2, (T *)zero, rs, red, want_sqrt, flags);
            return;
        }
        R &= ~kPatFlags;
#define HB2_PAT_LAUNCH(KT_, R_)                                                                              \
        launch_pdl(ell_pattern_kernel<T, KT_, MODE, R_>, grid, dim3(kEllThreads), 0, s, v, (const T *)x, (T *)y, \
                   (const T *)aux, (const T *)aux2, (T *)zero, rs, red, want_sqrt, flags, b)
        // (8 rows per thread only as the fallback of the Q1 stencil kernel's widest shape)
        if (A->K == 9)
        {
            if (R == 1) HB2_PAT_LAUNCH(9, 1);
            else if (R == 2) HB2_PAT_LAUNCH(9, 2);
            else if (R == 4) HB2_PAT_LAUNCH(9, 4);
            else HB2_PAT_LAUNCH(9, 8);
        }
        else { if (R == 1) HB2_PAT_LAUNCH(0, 1); else if (R == 2) HB2_PAT_LAUNCH(0, 2); else HB2_PAT_LAUNCH(0, 4); }
#undef HB2_PAT_LAUNCH
    }

    template <typename T>
    static void pattern_typed(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux,
                              const void * aux2, void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid,
                              cudaStream_t s, int f, Batch b, int R, unsigned bs)
    {
        switch (mode)
        {
            case kPlain: pattern_mode<T, kPlain>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, R, bs); break;
            case kDefect: pattern_mode<T, kDefect>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, R, bs); break;
            case kDot: pattern_mode<T, kDot>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, R, bs); break;
            case kAdd: pattern_mode<T, kAdd>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, R, bs); break;
            case kJacobi:
                if (red) pattern_mode<T, kJacobiNorm>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, R, bs);
                else pattern_mode<T, kJacobi>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, R, bs);
                break;
            case kRestrict: pattern_mode<T, kRestrict>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, R, bs); break;
        }
    }

    void launch_ell_pattern(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux,
                            const void * aux2, void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid,
                            cudaStream_t stream, int flags, Batch b, int R, unsigned bs)
    {
        if (A->dtype == HB2_F64) pattern_typed<double>(A, mode, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, stream, flags, b, R, bs);
        else pattern_typed<float>(A, mode, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, stream, flags, b, R, bs);
    }

    // ------------------------------------------------------------------ build
    template <typename T>
    static int build_pattern_typed(hb2_ell_s * A, cudaStream_t s)
    {
        const uint64_t rows = A->rows;
        unsigned long long * sig = 0, * keys = 0;
        unsigned * nkeys = 0, * rep = 0;
        int * flag = 0;
        uint8_t * ids = 0, * pcode = 0;
        int16_t * pdelta = 0;
        void * tmp = 0;
        // one temporary block: signatures | hash set | counters | representatives | id map
        const size_t bytes = rows * 8 + kPatSlots * 8 + 64 + kPatMax * 4 + kPatSlots + 256;
        HB2_CUDA(cudaMalloc(&tmp, bytes));
        char * p = (char *)tmp;
        sig = (unsigned long long *)p; p += rows * 8;
        keys = (unsigned long long *)p; p += kPatSlots * 8;
        nkeys = (unsigned *)p; flag = (int *)(p + 4); p += 64;
        rep = (unsigned *)p; p += kPatMax * 4;
        ids = (uint8_t *)p;
        cudaError_t e = cudaMemsetAsync(keys, 0xFF, kPatSlots * 8, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(nkeys, 0, 64, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(rep, 0xFF, kPatMax * 4, s);
        const unsigned grid = (unsigned)std::min<uint64_t>(4096, (rows + 255) / 256);
        if (e == cudaSuccess)
        {
            pat_insert_kernel<<<grid, 256, 0, s>>>(A->code, A->delta, A->ld, A->K, rows, sig, keys, nkeys, flag);
            count_launches(1);
            e = cudaGetLastError();
        }
        std::vector<unsigned long long> hk(kPatSlots);
        unsigned hn[2] = {0, 0};
        if (e == cudaSuccess) e = cudaMemcpyAsync(hk.data(), keys, kPatSlots * 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hn, nkeys, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        bool ok = e == cudaSuccess && hn[1] == 0 && hn[0] >= 1 && hn[0] <= (unsigned)kPatMax;
        std::vector<uint8_t> id_of_slot(kPatSlots, 0);
        uint32_t np = 0;
        if (ok)
        {
            for (uint32_t h = 0; h < kPatSlots; ++h)
                if (hk[h] != kPatEmptyKey) id_of_slot[h] = (uint8_t)np++;
            e = cudaMemcpyAsync(ids, id_of_slot.data(), kPatSlots, cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaMalloc(&A->pat, std::max<uint64_t>(rows, 16));
            if (e == cudaSuccess)
            {
                pat_encode_kernel<<<grid, 256, 0, s>>>(sig, rows, keys, ids, A->pat, rep, flag);
                pat_verify_kernel<<<grid, 256, 0, s>>>(A->code, A->delta, A->ld, A->K, rows, A->pat, rep, flag);
                count_launches(2);
                e = cudaGetLastError();
            }
            std::vector<unsigned> hrep(np);
            int hflag = 0;
            if (e == cudaSuccess) e = cudaMemcpyAsync(hrep.data(), rep, np * 4, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(&hflag, flag, 4, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            ok = e == cudaSuccess && hflag == 0;
            if (ok)
            {
                // the pattern table from the representative rows
                std::vector<T> vtab(A->ntable);
                e = cudaMemcpy(vtab.data(), A->table, A->ntable * sizeof(T), cudaMemcpyDeviceToHost);
                std::vector<PatEnt<T>> tab((size_t)np * A->K);
                for (uint32_t q = 0; q < np && e == cudaSuccess; ++q)
                    for (uint32_t k = 0; k < A->K && e == cudaSuccess; ++k)
                    {
                        uint8_t c = 0;
                        int16_t d = 0;
                        e = cudaMemcpy(&c, A->code + (uint64_t)k * A->ld + hrep[q], 1, cudaMemcpyDeviceToHost);
                        if (e == cudaSuccess) e = cudaMemcpy(&d, A->delta + (uint64_t)k * A->ld + hrep[q], 2, cudaMemcpyDeviceToHost);
                        PatEnt<T> & t = tab[(size_t)q * A->K + k];
                        t.val = vtab.empty() ? T(0) : vtab[c];
                        t.off = d == (int16_t)-32768 ? kPatEmpty : (int32_t)d;
                    }
                if (e == cudaSuccess) e = cudaMalloc(&A->ptab, tab.size() * sizeof(PatEnt<T>));
                if (e == cudaSuccess) e = cudaMemcpy(A->ptab, tab.data(), tab.size() * sizeof(PatEnt<T>), cudaMemcpyHostToDevice);
                ok = e == cudaSuccess;
                A->npat = np;
            }
        }
        cudaFree(tmp);
        if (! ok)
        {
            ell_free_pattern(A);
            cudaGetLastError();
            return e == cudaSuccess ? HB2_OK : cuda_status(e, "ELL row patterns");
        }
        A->pattern_bytes = rows + (uint64_t)np * A->K * sizeof(PatEnt<T>);
        // the windowed kernel applies when every offset lies in the bands around -m, 0, +m
        {
            std::vector<PatEnt<T>> htab((size_t)np * A->K);
            A->pat_win_m = 0;
            int64_t mm = 1;
            while (mm * mm < (int64_t)rows) ++mm;
            if (A->K == 9 && mm * mm == (int64_t)rows && mm >= 3 && (int64_t)rows < (1ll << 31) &&
                cudaMemcpy(htab.data(), A->ptab, htab.size() * sizeof(PatEnt<T>), cudaMemcpyDeviceToHost) == cudaSuccess)
            {
                bool ok_win = true;
                for (const auto & e : htab)
                {
                    if (e.off == kPatEmpty) continue;
                    const int64_t o = e.off;
                    if (! ((o >= -mm - 1 && o <= -mm + 1) || (o >= -1 && o <= 1) || (o >= mm - 1 && o <= mm + 1)))
                        ok_win = false;
                }
                if (ok_win) A->pat_win_m = mm;
            }
        }
        ell_find_q1_stencil(A);
        return HB2_OK;
    }

    int ell_build_pattern(hb2_ell_s * A, cudaStream_t stream)
    {
        if (! A->code || A->rows != A->cols || A->rows == 0 || A->K > (uint32_t)kPatMaxK) return HB2_OK;
        return A->dtype == HB2_F64 ? build_pattern_typed<double>(A, stream) : build_pattern_typed<float>(A, stream);
    }

    // Host-side row patterns of a small square matrix (K <= 9 slots, at most
    // kSubPatMax distinct rows): the fused small-level kernels keep the table in
    // shared memory and each row's pattern id in shared memory, so a row's
    // product needs one memory round trip (the gathers), not two.
    template <typename T>
    static int small_patterns_typed(hb2_ell_s * A)
    {
        const uint64_t n = A->rows, ld = A->ld;
        const uint32_t K = A->K;
        std::vector<T> val((size_t)K * ld);
        std::vector<int32_t> col((size_t)K * ld);
        HB2_CUDA(cudaMemcpy(val.data(), A->val, val.size() * sizeof(T), cudaMemcpyDeviceToHost));
        HB2_CUDA(cudaMemcpy(col.data(), A->col, col.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
        std::vector<PatEnt<T>> tab;
        std::vector<uint8_t> pat(n);
        std::vector<PatEnt<T>> row(K);
        for (uint64_t r = 0; r < n; ++r)
        {
            for (uint32_t k = 0; k < K; ++k)
            {
                const int32_t c = col[(size_t)k * ld + r];
                row[k].val = c >= 0 ? val[(size_t)k * ld + r] : T(0);
                row[k].off = c >= 0 ? (int32_t)(c - (int64_t)r) : kPatEmpty;
            }
            uint32_t q = 0;
            const uint32_t np = (uint32_t)(tab.size() / K);
            for (; q < np; ++q)
            {
                bool same = true;
                for (uint32_t k = 0; k < K && same; ++k)
                    same = tab[(size_t)q * K + k].off == row[k].off &&
                           memcmp(&tab[(size_t)q * K + k].val, &row[k].val, sizeof(T)) == 0;
                if (same) break;
            }
            if (q == np)
            {
                if (np == (uint32_t)kSubPatMax) return HB2_OK;   // too many distinct rows: none
                tab.insert(tab.end(), row.begin(), row.end());
            }
            pat[r] = (uint8_t)q;
        }
        HB2_CUDA(cudaMalloc(&A->spat, std::max<uint64_t>(n, 16)));
        HB2_CUDA(cudaMemcpy(A->spat, pat.data(), n, cudaMemcpyHostToDevice));
        HB2_CUDA(cudaMalloc(&A->sptab, tab.size() * sizeof(PatEnt<T>)));
        HB2_CUDA(cudaMemcpy(A->sptab, tab.data(), tab.size() * sizeof(PatEnt<T>), cudaMemcpyHostToDevice));
        A->snpat = (uint32_t)(tab.size() / K);
        return HB2_OK;
    }

    int ell_small_patterns(hb2_ell_s * A)
    {
        if (A->spat || A->rows != A->cols || A->rows == 0 || A->K != 9 || A->rows > (1u << 20)) return HB2_OK;
        return A->dtype == HB2_F64 ? small_patterns_typed<double>(A) : small_patterns_typed<float>(A);
    }

    void ell_free_pattern(hb2_ell_s * A)
    {
        cudaFree(A->pat);
        cudaFree(A->ptab);
        A->pat = 0;
        A->ptab = 0;
        A->npat = 0;
        A->pattern_bytes = 0;
    }
}
