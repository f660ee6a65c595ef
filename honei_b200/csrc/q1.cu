// BandedMatrixQx<Q1Type, DT> SpMV and defect (la/product.hh:370-403,
// math/defect.hh:194-198) with the x row-windows staged in shared memory by
// TMA bulk copies (cp.async.bulk, no multicast, completion on an mbarrier).
//
// A block owns B consecutive rows [r0, r0+B).  The nine bands touch three
// windows of x: [r0-m-1, r0+B-m+1), [r0-1, r0+B+1), [r0+m-1, r0+B+m+1).  Each is
// clamped to [0, n), rounded to 16-byte boundaries for the bulk copy, and a
// ragged tail (n is odd) is fetched with plain loads.  Band values stream with
// evict-first loads issued before the wait for the windows (rows interleaved
// across the block's threads, so they are coalesced).  Summation: DD*x first, then LL LD LU DL DU UL UD UU with
// the reference's bounds tests, each product and sum separately rounded, so
// the result is bit-identical to the reference.
#include "hb2_common.cuh"
#include "hb2_internal.hh"
#include "tma.cuh"

namespace hb2
{
    constexpr int kQ1Threads = 256;


    template <typename T>
    struct Window
    {
        int64_t base;   // global index of smem element 0
        int64_t lo, hi; // valid global range [lo, hi)
    };

    // MODE 0: y = A x; 1: y = rhs - A x; 2 (Jacobi, math/jacobi.hh MG variant):
    // y = x + (rhs - A x) (.) dinv, each product, sum and difference rounded
    template <typename T, int MODE>
    __global__ void __launch_bounds__(kQ1Threads)
    q1_kernel(const T * __restrict__ bands, const T * __restrict__ x, T * __restrict__ y, const T * __restrict__ rhs,
              const T * __restrict__ dinv, int64_t n, int64_t m, int * err)
    {
        typedef Arith<T> M;
        constexpr int R = RowsPerThread<T>::value;
        constexpr int B = kQ1Threads * R;
        constexpr int E = 16 / sizeof(T);
        constexpr int W = (B + 2 + 2 * E + E - 1) / E * E;   // each window 16-byte aligned
        __shared__ alignas(128) T win[3][W];
        __shared__ alignas(8) uint64_t bar;
        __shared__ int64_t base[3];

        const int64_t r0 = (int64_t)blockIdx.x * B;
        // rows r0 + k * kQ1Threads + threadIdx.x: the band (and rhs, dinv) loads are
        // coalesced and independent of x, so every thread issues them before the
        // block waits for its x windows
        T bv[R][9], rh[R], dv[R];
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int64_t i = r0 + (int64_t)k * kQ1Threads + threadIdx.x;
            const bool ok = i < n;
#pragma unroll
            for (int b = 0; b < 9; ++b) bv[k][b] = ok ? __ldcs(bands + b * n + i) : T(0);
            rh[k] = (MODE != 0 && ok) ? rhs[i] : T(0);
            dv[k] = (MODE == 2 && ok) ? dinv[i] : T(0);
        }
        if (threadIdx.x == 0)
        {
            mbar_init(&bar, 1);
            const int64_t starts[3] = {r0 - m - 1, r0 - 1, r0 + m - 1};
            unsigned total = 0;
            int64_t lo[3], ahi[3], alo[3], hi[3];
            for (int w = 0; w < 3; ++w)
            {
                lo[w] = starts[w] < 0 ? 0 : starts[w];
                hi[w] = starts[w] + B + 2 > n ? n : starts[w] + B + 2;
                alo[w] = lo[w] - (lo[w] % E);
                ahi[w] = hi[w] - (hi[w] % E);
                if (ahi[w] < alo[w]) ahi[w] = alo[w];
                base[w] = alo[w];
                total += (unsigned)((ahi[w] - alo[w]) * sizeof(T));
            }
            mbar_expect_tx(&bar, total);
            for (int w = 0; w < 3; ++w)
            {
                if (ahi[w] > alo[w])
                    bulk_g2s(&win[w][0], x + alo[w], (unsigned)((ahi[w] - alo[w]) * sizeof(T)), &bar);
                for (int64_t j = (ahi[w] > lo[w] ? ahi[w] : lo[w]); j < hi[w]; ++j)
                    win[w][j - alo[w]] = x[j];
            }
        }
        __syncthreads();
        if (! mbar_wait_bounded(&bar, 0, 1000000000ull))
        {
            // the copies never completed: flag it, give them one more bounded
            // chance to land before the block's shared memory is released
            atomicExch(err, 1);
            mbar_wait_bounded(&bar, 0, 1000000000ull);
            return;
        }
        const int64_t off[9] = {-m - 1, -m, -m + 1, -1, 0, 1, m - 1, m, m + 1};
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int64_t i = r0 + (int64_t)k * kQ1Threads + threadIdx.x;
            if (i >= n) break;
            T s = M::mul(bv[k][4], win[1][i - base[1]]);
#pragma unroll
            for (int b = 0; b < 9; ++b)
            {
                if (b == 4) continue;
                const int64_t j = i + off[b];
                if (j < 0 || j >= n) continue;
                const int w = b / 3;
                s = M::add(s, M::mul(bv[k][b], win[w][j - base[w]]));
            }
            if (MODE == 0) y[i] = s;
            else if (MODE == 1) y[i] = M::sub(rh[k], s);
            else y[i] = M::add(win[1][i - base[1]], M::mul(M::sub(rh[k], s), dv[k]));
        }
    }

    // plain-load variant for x pointers that are not 16-byte aligned
    template <typename T, int MODE>
    __global__ void q1_kernel_direct(const T * __restrict__ bands, const T * __restrict__ x, T * __restrict__ y,
                                     const T * __restrict__ rhs, const T * __restrict__ dinv, int64_t n, int64_t m)
    {
        typedef Arith<T> M;
        const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n) return;
        const int64_t off[9] = {-m - 1, -m, -m + 1, -1, 0, 1, m - 1, m, m + 1};
        T s = M::mul(bands[4 * n + i], x[i]);
        for (int b = 0; b < 9; ++b)
        {
            if (b == 4) continue;
            const int64_t j = i + off[b];
            if (j < 0 || j >= n) continue;
            s = M::add(s, M::mul(bands[b * n + i], __ldg(x + j)));
        }
        if (MODE == 0) y[i] = s;
        else if (MODE == 1) y[i] = M::sub(rhs[i], s);
        else y[i] = M::add(x[i], M::mul(M::sub(rhs[i], s), dinv[i]));
    }

    template <typename T>
    __global__ void q1_fill_kernel(T * bands, uint64_t M_, double aniso)
    {
        const uint64_t N = M_ * M_;
        const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (r >= N) return;
        const uint64_t i = r + 1;
        const bool dir = (i <= M_ || i > N - M_ || (i % M_) == 1 || (i % M_) == 0);
        for (int b = 0; b < 9; ++b)
        {
            T v = T(0);
            if (dir) v = b == 4 ? T(1.0) : T(0.0);
            else if (b == 4) v = aniso == 1.0 ? T(8.0 / 3.0) : T((6.0 + 2.0 * aniso) / 3.0);
            else if ((b == 3 || b == 5) && aniso != 1.0) v = T(-aniso / 3.0);
            else v = T(-1.0 / 3.0);
            bands[b * N + r] = v;
        }
    }

    template <typename T, int MODE>
    static void q1_launch_typed(const hb2_q1_s * A, const void * x, void * y, const void * rhs, const void * dinv,
                                int * err, cudaStream_t stream)
    {
        const int64_t n = (int64_t)A->n, m = (int64_t)A->m;
        const T * b = (const T *)A->bands;
        if (((uintptr_t)x % 16) == 0)
        {
            const unsigned grid = ceil_div(A->n, kQ1Threads * RowsPerThread<T>::value);
            q1_kernel<T, MODE><<<grid, kQ1Threads, 0, stream>>>(b, (const T *)x, (T *)y, (const T *)rhs,
                                                                (const T *)dinv, n, m, err);
        }
        else
        {
            const unsigned grid = ceil_div(A->n, 256);
            q1_kernel_direct<T, MODE><<<grid, 256, 0, stream>>>(b, (const T *)x, (T *)y, (const T *)rhs,
                                                                (const T *)dinv, n, m);
        }
    }

    // mode 0: y = A x, 1: y = rhs - A x, 2: y = x + (rhs - A x) (.) dinv (y != x);
    // err: device flag set when a block's bulk copies of x never completed
    int launch_q1(const hb2_q1_s * A, int mode, const void * x, void * y, const void * rhs, const void * dinv,
                  int * err, cudaStream_t stream)
    {
        if (A->n == 0) return HB2_OK;
        if (A->dtype == HB2_F64)
        {
            if (mode == 0) q1_launch_typed<double, 0>(A, x, y, rhs, dinv, err, stream);
            else if (mode == 1) q1_launch_typed<double, 1>(A, x, y, rhs, dinv, err, stream);
            else q1_launch_typed<double, 2>(A, x, y, rhs, dinv, err, stream);
        }
        else
        {
            if (mode == 0) q1_launch_typed<float, 0>(A, x, y, rhs, dinv, err, stream);
            else if (mode == 1) q1_launch_typed<float, 1>(A, x, y, rhs, dinv, err, stream);
            else q1_launch_typed<float, 2>(A, x, y, rhs, dinv, err, stream);
        }
        count_launches(1);
        HB2_LAUNCH_CHECK("q1 kernel launch");
        return HB2_OK;
    }

    static int q1_launch(const hb2_q1_s * A, const void * x, void * y, const void * rhs, bool defect,
                         cudaStream_t stream)
    {
        if (A->n == 0) return HB2_OK;
        Workspace * ws = 0;
        int st = stream_workspace(stream, &ws);
        if (st) return st;
        return launch_q1(A, defect ? 1 : 0, x, y, rhs, nullptr, ws->error, stream);
    }
}

using namespace hb2;

static int q1_alloc(hb2_q1 * out, hb2_dtype dtype, uint64_t n)
{
    uint64_t m = 1;
    while (m * m < n) ++m;
    if (m * m != n || m < 3 || ((m - 1) & (m - 2)) != 0)
        return fail(HB2_ERR_SIZE, "BandedMatrixQx: size must be (2^L+1)^2");
    hb2_q1_s * A = new hb2_q1_s();
    A->dtype = dtype;
    A->n = n;
    A->m = m;
    cudaError_t e = cudaMalloc(&A->bands, 9 * n * dtype_size(dtype));
    if (e != cudaSuccess) { delete A; return cuda_status(e, "BandedMatrixQx cudaMalloc"); }
    *out = A;
    return HB2_OK;
}

extern "C" int hb2_q1_create(hb2_q1 * out, hb2_dtype dtype, uint64_t n, const void * bands, int host_ptrs,
                             cudaStream_t stream)
{
    if (! out || ! bands) return fail(HB2_ERR_ARG, "hb2_q1_create: null argument");
    int st = q1_alloc(out, dtype, n);
    if (st) return st;
    cudaError_t e = cudaMemcpyAsync((*out)->bands, bands, 9 * n * dtype_size(dtype),
                                    host_ptrs ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess && host_ptrs) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) { hb2_q1_destroy(*out); *out = 0; return cuda_status(e, "hb2_q1_create"); }
    return HB2_OK;
}

extern "C" int hb2_q1_create_poisson(hb2_q1 * out, hb2_dtype dtype, unsigned level, double aniso, cudaStream_t stream)
{
    if (! out || level < 1 || level > 14 || ! (aniso > 0.0)) return fail(HB2_ERR_ARG, "hb2_q1_create_poisson: bad argument");
    uint64_t M_ = (1ULL << level) + 1;
    int st = q1_alloc(out, dtype, M_ * M_);
    if (st) return st;
    unsigned grid = ceil_div(M_ * M_, 256);
    if (dtype == HB2_F64) q1_fill_kernel<double><<<grid, 256, 0, stream>>>((double *)(*out)->bands, M_, aniso);
    else q1_fill_kernel<float><<<grid, 256, 0, stream>>>((float *)(*out)->bands, M_, aniso);
    count_launches(1);
    HB2_LAUNCH_CHECK("hb2_q1_create_poisson");
    return HB2_OK;
}

extern "C" int hb2_q1_destroy(hb2_q1 A)
{
    if (! A) return HB2_OK;
    cudaFree(A->bands);
    delete A;
    return HB2_OK;
}

extern "C" int hb2_product_q1(hb2_q1 A, const void * x, void * y, cudaStream_t stream)
{
    if (! A || ! x || ! y) return fail(HB2_ERR_ARG, "hb2_product_q1: null argument");
    return q1_launch(A, x, y, 0, false, stream);
}

extern "C" int hb2_defect_q1(hb2_q1 A, const void * rhs, const void * x, void * r, cudaStream_t stream)
{
    if (! A || ! x || ! r || ! rhs) return fail(HB2_ERR_ARG, "hb2_defect_q1: null argument");
    return q1_launch(A, x, r, rhs, true, stream);
}
