// BF16-stored ELL matrices for the FP32 inner solve of mixed-precision iterative
// refinement: hb2_ell_create_bf16.
//
// Storage.  Every stored entry a becomes q = bf16(s * a), rounded once to the
// nearest BF16 value (ties to even) from the double s * a, with one scale s per
// matrix from {1, 3, 5, ..., 15}: the first with the smallest largest relative
// rounding error over the stored entries (the Q1 operator's 8/3, -1/3 and the
// Dirichlet 1 are 8, -1 and 3 at s = 3: exact).  Square matrices whose column
// offsets fit 16 bits (form 0): per slot one 32-bit word, BF16 value and offset
// from the row, 4 bytes per slot instead of 8 for an FP32 matrix; the words of 32
// consecutive rows lie slot after slot in one run of 128 K bytes, so a warp's
// loads of a row chunk read one contiguous run (slot-major arrays would give it
// 2 K separate streams).  Otherwise (form 1): BF16 values and int32 columns,
// slot-major like the plain layout, 6 bytes per slot.
//
// Row-sum compensated form.  Rounding every entry of a diffusion operator on its
// own breaks its zero row sums; the error then reaches the smooth modes that the
// operator barely damps, and the outer refinement stalls as the grid is refined.
// The compensated form gives the diagonal (the row's first slot with column ==
// row) the rounding errors of the row's off-diagonal entries (in double, slot
// order):  d = (float)(s * a_ii + sum_j!=i (s * a_ij - q_ij)),
// so s * A and the stored matrix have the same row sums up to d's one rounding.
// d is stored as its BF16 part h = bf16(d) in the diagonal's slot (an ordinary
// slot) and the rest l = d - h (exact in FP32) in a per-row FP32 array.
//
// Products.  acc = fmaf chain over the row's slots in order (v = q, exact in
// FP32), then acc = fmaf(l, x_i, acc) in the compensated form, then
// y_i = acc * fl(1/s) (the factor 1/s once per row, in the accumulator; no
// multiply for s = 1).  The plain arrays of the new matrix hold (float)(q / s)
// (and (float)(d / s) at the diagonal) for the paths that read FP32 values
// (small fused levels, CG, export).
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace hb2
{
    constexpr int16_t kBfEmpty = -32768;          // offset of a slot past the row's length
    constexpr uint32_t kBfEmptyWord = 0x80000000u;  // form 0: that slot's word (value 0)
    constexpr int kBfScales = 8;                  // s = 1, 3, ..., 15

    // double -> BF16 bits, rounded to nearest, ties to even, in one rounding:
    // truncate to float, record any discarded bits in the last place (round to
    // odd: float keeps 16 bits more than BF16, so the final rounding sees the
    // exact tie / non-tie), then round the float's upper 16 bits to nearest even.
    __device__ __forceinline__ uint16_t bf16_rne(double t)
    {
        const float f = __double2float_rz(t);
        uint32_t u = __float_as_uint(f);
        if ((double)f != t) u |= 1u;
        if ((u & 0x7f800000u) == 0x7f800000u)                      // inf stays inf, NaN stays NaN
            return (uint16_t)((u >> 16) | ((u & 0xffffu) ? 0x40u : 0u));
        u += 0x7fffu + ((u >> 16) & 1u);
        return (uint16_t)(u >> 16);
    }

    __device__ __forceinline__ float bf16_float(uint32_t b) { return __uint_as_float(b << 16); }

    __device__ __forceinline__ double warp_max(double v)
    {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        return v;
    }

    // slot k of row r is the row's diagonal: the first slot with column == row
    __device__ __forceinline__ bool diag_slot(const int32_t * col, uint64_t ld, uint64_t r, uint32_t k)
    {
        if (col[(uint64_t)k * ld + r] != (int32_t)r) return false;
        for (uint32_t j = 0; j < k; ++j)
            if (col[(uint64_t)j * ld + r] == (int32_t)r) return false;
        return true;
    }

    // per candidate scale the largest relative rounding error of the entries stored
    // in BF16 (err[c] as the bits of a non-negative double); flag: an offset that
    // does not fit 16 bits
    template <typename T>
    __global__ void bf16_scale_kernel(const T * __restrict__ val, const int32_t * __restrict__ col, uint64_t rows,
                                      uint64_t ld, uint32_t K, int compensate, unsigned long long * err, int * wide)
    {
        const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        double e[kBfScales];
#pragma unroll
        for (int c = 0; c < kBfScales; ++c) e[c] = 0.0;
        if (r < rows)
            for (uint32_t k = 0; k < K; ++k)
            {
                const int32_t cj = col[(uint64_t)k * ld + r];
                if (cj < 0) continue;
                const int64_t d = (int64_t)cj - (int64_t)r;
                if (d < -32767 || d > 32767) *wide = 1;
                if (compensate && diag_slot(col, ld, r, k)) continue;
                const double a = (double)val[(uint64_t)k * ld + r];
                if (a == 0.0) continue;
#pragma unroll
                for (int c = 0; c < kBfScales; ++c)
                {
                    const double t = a * (double)(2 * c + 1);
                    const double q = (double)bf16_float(bf16_rne(t));
                    e[c] = fmax(e[c], fabs(q - t) / fabs(t));
                }
            }
        __shared__ double part[kBfScales][kEllThreads / 32];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
        for (int c = 0; c < kBfScales; ++c)
        {
            const double m = warp_max(e[c]);
            if (lane == 0) part[c][w] = m;
        }
        __syncthreads();
        if (threadIdx.x < kBfScales)
        {
            double m = 0.0;
            for (int j = 0; j < (int)(blockDim.x >> 5); ++j) m = fmax(m, part[threadIdx.x][j]);
            atomicMax(err + threadIdx.x, (unsigned long long)__double_as_longlong(m));
        }
    }

    // one thread per row: BF16 values, indices, the compensated diagonal's FP32
    // remainder and the FP32 rendering (val32 / col32 of the new matrix, same
    // layout as the source)
    // form 0: word index of (row r, slot k) in the chunked layout
    __host__ __device__ __forceinline__ uint64_t bf16_word(uint64_t r, uint32_t k, uint32_t K)
    {
        return (r >> 5) * ((uint64_t)K << 5) + ((uint64_t)k << 5) + (r & 31);
    }

    __device__ __forceinline__ void bf16_put(int form, void * bval, void * bidx, uint64_t r, uint32_t k, uint32_t K,
                                             uint64_t i, uint16_t q, int16_t off, int32_t col)
    {
        if (form == 0) ((uint32_t *)bval)[bf16_word(r, k, K)] = (uint32_t)q | ((uint32_t)(uint16_t)off << 16);   // empty: q = 0, off = kBfEmpty
        else
        {
            ((uint16_t *)bval)[i] = q;
            ((int32_t *)bidx)[i] = col;
        }
    }

    template <typename T>
    __global__ void bf16_build_kernel(const T * __restrict__ val, const int32_t * __restrict__ col, uint64_t rows,
                                      uint64_t ld, uint32_t K, double s, int compensate, int form, void * bval,
                                      void * bidx, float * bdlo, float * val32, int32_t * col32)
    {
        const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (r >= ld) return;
        double comp = 0.0;
        int64_t dslot = -1;
        double dval = 0.0;
        for (uint32_t k = 0; k < K; ++k)
        {
            const uint64_t i = (uint64_t)k * ld + r;
            const int32_t cj = r < rows ? col[i] : -1;
            col32[i] = cj;
            if (cj < 0)
            {
                bf16_put(form, bval, bidx, r, k, K, i, 0, kBfEmpty, -1);
                val32[i] = 0.f;
                continue;
            }
            const double t = (double)val[i] * s;
            if (compensate && dslot < 0 && cj == (int32_t)r)
            {
                dslot = (int64_t)k;      // written once the row's errors are summed
                dval = t;
                continue;
            }
            const uint16_t q = bf16_rne(t);
            const double qd = (double)bf16_float(q);
            comp += t - qd;
            bf16_put(form, bval, bidx, r, k, K, i, q, (int16_t)((int64_t)cj - (int64_t)r), cj);
            val32[i] = (float)(qd / s);
        }
        if (bdlo)
        {
            float lo = 0.f;
            if (dslot >= 0)
            {
                const float d = (float)(dval + comp);
                const uint16_t h = bf16_rne((double)d);
                lo = d - bf16_float(h);           // exact: h is d to 8 bits
                const uint64_t i = (uint64_t)dslot * ld + r;
                bf16_put(form, bval, bidx, r, (uint32_t)dslot, K, i, h, 0, (int32_t)r);
                val32[i] = (float)((double)d / s);
            }
            bdlo[r] = lo;
        }
    }

    // ------------------------------------------------------------------ products
    struct EllBf16View
    {
        const void * val;     // form 0: packed words; form 1: BF16 values
        const int32_t * idx;  // form 1: columns
        const float * dlo;    // compensated form: the diagonal's FP32 remainder per row (else null)
        uint64_t rows, ld;
        uint32_t K;
        float inv;            // fl(1 / s); 1: no multiply
    };

    template <int R> struct BfWide;
    template <> struct BfWide<2> { typedef uint32_t V; typedef int2 C; };
    template <> struct BfWide<4> { typedef uint2 V; typedef int4 C; };
    template <> struct BfWide<8> { typedef uint4 V; typedef int4 C; };   // columns: two loads

    // slot k of rows r0 .. r0 + R - 1: BF16 bits and column (-1: empty)
    template <int R, int FORM>
    __device__ __forceinline__ void bf16_slot(const EllBf16View & A, uint32_t K, uint32_t k, uint64_t r0, bool keep,
                                              uint32_t (&q)[R], int (&c)[R])
    {
        if constexpr (FORM == 0)
        {
            // rows r0 .. r0 + R - 1 lie in one chunk (R divides 32), their words adjacent
            const unsigned * p = (const unsigned *)A.val + bf16_word(r0, k, K);
            uint32_t w[R];
            if constexpr (R == 1) w[0] = keep ? __ldcg(p) : __ldcs(p);
            else if constexpr (R == 2)
            {
                const uint2 t = keep ? __ldcg((const uint2 *)p) : __ldcs((const uint2 *)p);
                w[0] = t.x;
                w[1] = t.y;
            }
            else
            {
#pragma unroll
                for (int h = 0; h < R / 4; ++h)
                {
                    const uint4 t = keep ? __ldcg((const uint4 *)p + h) : __ldcs((const uint4 *)p + h);
                    w[4 * h] = t.x;
                    w[4 * h + 1] = t.y;
                    w[4 * h + 2] = t.z;
                    w[4 * h + 3] = t.w;
                }
            }
#pragma unroll
            for (int j = 0; j < R; ++j)
            {
                q[j] = w[j] & 0xffffu;
                c[j] = w[j] == kBfEmptyWord ? -1 : (int)r0 + j + (int)(int16_t)(w[j] >> 16);
            }
        }
        else
        {
            const uint64_t i = (uint64_t)k * A.ld + r0;
            const uint16_t * vp = (const uint16_t *)A.val + i;
            const int32_t * cp = A.idx + i;
            if constexpr (R == 1)
            {
                q[0] = keep ? __ldcg((const unsigned short *)vp) : __ldcs((const unsigned short *)vp);
                c[0] = keep ? __ldcg(cp) : __ldcs(cp);
            }
            else
            {
                typedef typename BfWide<R>::V V;
                union { V v; uint16_t h[R]; } u;
                u.v = keep ? __ldcg((const V *)vp) : __ldcs((const V *)vp);
#pragma unroll
                for (int j = 0; j < R; ++j) q[j] = u.h[j];
                if constexpr (R == 2)
                {
                    const int2 t = keep ? __ldcg((const int2 *)cp) : __ldcs((const int2 *)cp);
                    c[0] = t.x;
                    c[1] = t.y;
                }
                else
                {
#pragma unroll
                    for (int h = 0; h < R / 4; ++h)
                    {
                        const int4 t = keep ? __ldcg((const int4 *)cp + h) : __ldcs((const int4 *)cp + h);
                        c[4 * h] = t.x;
                        c[4 * h + 1] = t.y;
                        c[4 * h + 2] = t.z;
                        c[4 * h + 3] = t.w;
                    }
                }
            }
        }
    }

    // One thread: R consecutive rows; KT = compile-time slot count (0: runtime);
    // FORM 0: chunked words, 1: BF16 values + int32 columns.
    // The mode epilogues are those of the plain kernel, in FP32.
    template <int KT, int MODE, int R, int FORM>
    __global__ void __launch_bounds__(kEllMaxThreads)
    ell_bf16_kernel(EllBf16View A, const float * __restrict__ x_, float * __restrict__ y_,
                    const float * __restrict__ aux_, const float * __restrict__ aux2, float * __restrict__ zero_,
                    ReduceSlot rs, double * red_, int want_sqrt, int flags, Batch bt)
    {
        typedef Arith<float> M;
        pdl_entry();
        const bool listed = bt.list != nullptr;
        const uint32_t total = listed ? *bt.count * bt.gx : 1;
        for (uint32_t item = listed ? blockIdx.x : 0; item < total; item += listed ? gridDim.x : 1)
        {
        const uint32_t j = listed ? bt.list[item / bt.gx] : blockIdx.y;
        if (! listed && bt.active && ! bt.active[j]) return;
        const uint64_t vo = (uint64_t)j * bt.vstride;
        const float * __restrict__ x = x_ + (uint64_t)j * (bt.xstride ? bt.xstride : bt.vstride);
        float * __restrict__ y = y_ + vo;
        const float * __restrict__ aux = aux_ ? aux_ + vo : aux_;
        float * __restrict__ zero = zero_ ? zero_ + (uint64_t)j * bt.zstride : zero_;
        double * red = red_ ? red_ + j : red_;
        const uint64_t bx = listed ? item % bt.gx : blockIdx.x;
        const uint64_t blk = (flags & kReverse) ? (gridDim.x - 1 - bx) : bx;
        const bool keep = (flags & kKeepL2) != 0;
        const uint64_t r0 = (blk * blockDim.x + threadIdx.x) * R;
        const int K = KT > 0 ? KT : (int)A.K;
        float acc[R];
#pragma unroll
        for (int i = 0; i < R; ++i) acc[i] = 0.f;
        if (r0 < A.rows)
        {
            float lo[R];
#pragma unroll
            for (int i = 0; i < R; ++i) lo[i] = A.dlo ? A.dlo[r0 + i] : 0.f;
            auto slot = [&](const uint32_t (&q)[R], const int (&c)[R]) {
#pragma unroll
                for (int i = 0; i < R; ++i)
                    if (c[i] >= 0) acc[i] = M::fma(bf16_float(q[i]), __ldg(x + c[i]), acc[i]);
            };
            if constexpr (KT > 0)
            {
                uint32_t q[KT][R];
                int c[KT][R];
#pragma unroll
                for (int k = 0; k < KT; ++k) bf16_slot<R, FORM>(A, KT, k, r0, keep, q[k], c[k]);
#pragma unroll
                for (int k = 0; k < KT; ++k) slot(q[k], c[k]);
            }
            else
            {
                for (int k = 0; k < K; ++k)
                {
                    uint32_t q[R];
                    int c[R];
                    bf16_slot<R, FORM>(A, (uint32_t)K, (uint32_t)k, r0, keep, q, c);
                    slot(q, c);
                }
            }
            if (A.dlo)
#pragma unroll
                for (int i = 0; i < R; ++i) acc[i] = M::fma(lo[i], __ldg(x + r0 + i), acc[i]);
            if (A.inv != 1.f)
#pragma unroll
                for (int i = 0; i < R; ++i) acc[i] = M::mul(acc[i], A.inv);
        }
        double part = 0.0;
#pragma unroll
        for (int i = 0; i < R; ++i)
        {
            const uint64_t r = r0 + i;
            if (r >= A.rows) break;
            if (MODE == kPlain) y[r] = acc[i];
            else if (MODE == kDefect)
            {
                const float dd = M::sub(aux[r], acc[i]);
                y[r] = dd;
                part = fma((double)dd, (double)dd, part);
            }
            else if (MODE == kDot)
            {
                y[r] = acc[i];
                part = fma((double)acc[i], (double)x[r], part);
            }
            else if (MODE == kAdd) y[r] = M::add(y[r], acc[i]);
            else if (is_jacobi(MODE))
            {
                const float d = M::sub(aux[r], acc[i]);
                y[r] = M::add(x[r], M::mul(aux2[r], d));
                part = fma((double)d, (double)d, part);
            }
            else if (MODE == kRestrict) { y[r] = acc[i]; zero[r] = 0.f; }
        }
        if ((MODE == kDefect || MODE == kDot || MODE == kJacobiNorm) && red != 0)
        {
            __shared__ double scratch[32];
            ell_block_reduce(part, rs, red, want_sqrt, flags, scratch);
        }
        }
    }

    template <int MODE, int FORM>
    static void bf16_launch(const hb2_ell_s * A, const void * x, void * y, const void * aux, const void * aux2,
                            void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid, cudaStream_t s,
                            int flags, Batch b, unsigned bs, int R)
    {
        EllBf16View v;
        v.val = A->bval;
        v.idx = (const int32_t *)A->bidx;
        v.dlo = A->bdiag;
        v.rows = A->rows;
        v.ld = A->ld;
        v.K = A->K;
        v.inv = A->bscale == 1.f ? 1.f : (float)(1.0 / (double)A->bscale);
        const float * xp = (const float *)x;
        float * yp = (float *)y;
        const float * ap = (const float *)aux;
        const float * a2 = (const float *)aux2;
        float * zp = (float *)zero;
#define HB2_BF_LAUNCH(KT_, R_)                                                                                  \
        launch_pdl(ell_bf16_kernel<KT_, MODE, R_, FORM>, grid, dim3(bs), 0, s, v, xp, yp, ap, a2, zp, rs, red, \
                   want_sqrt, flags, b)
        if (A->K == 9)
        {
            if (R == 1) HB2_BF_LAUNCH(9, 1);
            else if (R == 2) HB2_BF_LAUNCH(9, 2);
            else if (R == 4) HB2_BF_LAUNCH(9, 4);
            else HB2_BF_LAUNCH(9, 8);
        }
        else
        {
            if (R == 1) HB2_BF_LAUNCH(0, 1);
            else if (R == 2) HB2_BF_LAUNCH(0, 2);
            else if (R == 4) HB2_BF_LAUNCH(0, 4);
            else HB2_BF_LAUNCH(0, 8);
        }
#undef HB2_BF_LAUNCH
    }

    template <int MODE>
    static void bf16_mode(const hb2_ell_s * A, const void * x, void * y, const void * aux, const void * aux2,
                          void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid, cudaStream_t s,
                          int flags, Batch b, unsigned bs, int R)
    {
        if (A->bform == 0) bf16_launch<MODE, 0>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, flags, b, bs, R);
        else bf16_launch<MODE, 1>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, flags, b, bs, R);
    }

    void launch_ell_bf16(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux,
                         const void * aux2, void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid,
                         cudaStream_t s, int f, Batch b, unsigned bs)
    {
        const int R = A->rpt[red ? 1 : 0];
        switch (mode)
        {
            case kPlain: bf16_mode<kPlain>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, R); break;
            case kDefect: bf16_mode<kDefect>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, R); break;
            case kDot: bf16_mode<kDot>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, R); break;
            case kAdd: bf16_mode<kAdd>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, R); break;
            case kJacobi:
                if (red) bf16_mode<kJacobiNorm>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, R);
                else bf16_mode<kJacobi>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, R);
                break;
            case kRestrict: bf16_mode<kRestrict>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs, R); break;
        }
    }

    void ell_free_bf16(hb2_ell_s * A)
    {
        cudaFree(A->bval);
        cudaFree(A->bidx);
        cudaFree(A->bdiag);
        A->bval = nullptr;
        A->bidx = nullptr;
        A->bdiag = nullptr;
    }

    template <typename T>
    static int build_bf16(const hb2_ell_s * A, hb2_ell_s * B, int compensate, double * scale_out, double * err_out,
                          cudaStream_t s)
    {
        const uint64_t slots = (uint64_t)A->K * A->ld;
        unsigned long long * err = 0;
        int * wide = 0;
        HB2_CUDA(cudaMalloc(&err, kBfScales * sizeof(unsigned long long) + sizeof(int)));
        wide = (int *)(err + kBfScales);
        cudaError_t e = cudaMemsetAsync(err, 0, kBfScales * sizeof(unsigned long long) + sizeof(int), s);
        const unsigned grid = ceil_div(std::max<uint64_t>(A->rows, 1), kEllThreads);
        if (e == cudaSuccess && A->rows > 0)
        {
            bf16_scale_kernel<T><<<grid, kEllThreads, 0, s>>>((const T *)A->val, A->col, A->rows, A->ld, A->K,
                                                              compensate, err, wide);
            count_launches(1);
            e = cudaGetLastError();
        }
        unsigned long long herr[kBfScales];
        int hwide = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(herr, err, sizeof(herr), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&hwide, wide, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFree(err);
        if (e != cudaSuccess) return cuda_status(e, "hb2_ell_create_bf16 (scale)");
        int best = 0;
        double be = 0.0;
        for (int c = 0; c < kBfScales; ++c)
        {
            double v;
            memcpy(&v, herr + c, sizeof(double));
            if (c == 0 || v < be) { be = v; best = c; }
        }
        const double sc = (double)(2 * best + 1);
        B->bscale = (float)sc;
        B->bform = (A->rows == A->cols && ! hwide) ? 0 : 1;
        e = cudaMalloc(&B->bval, std::max<size_t>(slots * (B->bform == 0 ? 4 : 2), 16));
        if (e == cudaSuccess && B->bform == 1) e = cudaMalloc(&B->bidx, std::max<size_t>(slots * 4, 16));
        if (e == cudaSuccess && compensate) e = cudaMalloc(&B->bdiag, std::max<size_t>(A->ld * 4, 16));
        if (e == cudaSuccess && A->ld > 0)
        {
            bf16_build_kernel<T><<<ceil_div(A->ld, kEllThreads), kEllThreads, 0, s>>>(
                (const T *)A->val, A->col, A->rows, A->ld, A->K, sc, compensate, B->bform, B->bval, B->bidx,
                B->bdiag, (float *)B->val, B->col);
            count_launches(1);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) return cuda_status(e, "hb2_ell_create_bf16 (build)");
        B->bf16_bytes = slots * (B->bform == 0 ? 4 : 6) + (compensate ? A->ld * 4 : 0);
        if (scale_out) *scale_out = sc;
        if (err_out) *err_out = be;
        return HB2_OK;
    }
}

using namespace hb2;

extern "C" int hb2_ell_create_bf16(hb2_ell * out, hb2_ell A, int compensate, double * scale, double * max_rel_error,
                                   cudaStream_t stream)
{
    if (! out || ! A) return fail(HB2_ERR_ARG, "hb2_ell_create_bf16: null argument");
    if (compensate != 0 && compensate != 1) return fail(HB2_ERR_ARG, "hb2_ell_create_bf16: compensate must be 0 or 1");
    if (compensate && A->rows != A->cols)
        return fail(HB2_ERR_ARG, "hb2_ell_create_bf16: the compensated form needs a square matrix");
    if (A->rows >= (1ull << 31)) return fail(HB2_ERR_UNSUPPORTED, "hb2_ell_create_bf16: 2^31 rows or more");
    hb2_ell_s * B = new hb2_ell_s();
    B->dtype = HB2_F32;
    B->device = A->device;
    B->rows = A->rows;
    B->cols = A->cols;
    B->K = A->K;
    B->ld = A->ld;
    B->ref_stride = A->ref_stride;
    B->ref_K = A->ref_K;
    B->ref_T = A->ref_T;
    const size_t nslots = (size_t)A->K * A->ld;
    cudaError_t e = cudaMalloc(&B->val, std::max<size_t>(nslots * 4, 16));
    if (e == cudaSuccess) e = cudaMalloc(&B->col, std::max<size_t>(nslots * 4, 16));
    if (e != cudaSuccess)
    {
        hb2_ell_destroy(B);
        return cuda_status(e, "hb2_ell_create_bf16 cudaMalloc");
    }
    B->bytes = nslots * 8;
    int st = A->dtype == HB2_F64 ? build_bf16<double>(A, B, compensate, scale, max_rel_error, stream)
                                 : build_bf16<float>(A, B, compensate, scale, max_rel_error, stream);
    if (! st)
    {
        B->layout[0] = B->layout[1] = kLayoutBF16;
        B->rpt[0] = B->rpt[1] = 1;
        st = ell_autotune(B, stream);
    }
    if (st)
    {
        hb2_ell_destroy(B);
        return st;
    }
    *out = B;
    return HB2_OK;
}
