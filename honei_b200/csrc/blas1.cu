// BLAS-1 on DenseVector<DT>: ScaledSum, Sum, Difference, Scale, ElementProduct,
// fill, copy, convert, and the deterministic DotProduct / Norm.
//
// Element-wise updates round exactly like the reference's compiled tags::CPU
// loops (la/scaled_sum.hh:73-110, la/sum.hh, la/difference.hh, la/scale.hh,
// la/element_product.hh): multiply and add are separately rounded.
// Reductions accumulate in double with a fixed assignment of elements to
// threads and a fixed combination tree, so results are reproducible bit for
// bit (but not in the reference's sequential order).
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <algorithm>

namespace hb2
{
    enum Blas1Op { kAxpy, kAxpy3, kSum, kDiff, kDiff3, kScale, kEprod, kFill };

    template <typename T, int OP>
    __global__ void blas1_kernel(T * __restrict__ out, const T * __restrict__ a, const T * __restrict__ b, T s,
                                 uint64_t n)
    {
        typedef Arith<T> M;
        pdl_entry();
        const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        {
            if (OP == kAxpy) out[i] = M::add(out[i], M::mul(s, a[i]));          // x += s*y
            else if (OP == kAxpy3) out[i] = M::add(M::mul(s, b[i]), a[i]);      // r = s*y + x
            else if (OP == kSum) out[i] = M::add(out[i], a[i]);                 // x += y
            else if (OP == kDiff) out[i] = M::sub(out[i], a[i]);                // x -= y
            else if (OP == kDiff3) out[i] = M::sub(a[i], b[i]);                 // r = x - y
            else if (OP == kScale) out[i] = M::mul(out[i], s);                  // x *= s
            else if (OP == kEprod) out[i] = M::mul(a[i], b[i]);                 // r = a (.) b
            else if (OP == kFill) out[i] = s;
        }
    }

    static unsigned stream_grid(uint64_t n)
    {
        uint64_t g = (n + 255) / 256;
        uint64_t cap = (uint64_t)num_sms() * 16;
        return (unsigned)std::max<uint64_t>(1, std::min(g, cap));
    }

    template <int OP>
    static int launch_blas1(int dt, void * out, const void * a, const void * b, double s, uint64_t n, cudaStream_t st)
    {
        if (n == 0) return HB2_OK;
        if (! out) return fail(HB2_ERR_ARG, "BLAS-1: null output vector");
        unsigned grid = stream_grid(n);
        if (dt == HB2_F64)
            launch_pdl(blas1_kernel<double, OP>, grid, dim3(256), 0, st, (double *)out, (const double *)a, (const double *)b, s, n);
        else
            launch_pdl(blas1_kernel<float, OP>, grid, dim3(256), 0, st, (float *)out, (const float *)a, (const float *)b, (float)s, n);
        count_launches(1);
        HB2_LAUNCH_CHECK("BLAS-1 launch");
        return HB2_OK;
    }

    int launch_fill(int dt, void * x, double value, uint64_t n, cudaStream_t stream)
    {
        return launch_blas1<kFill>(dt, x, 0, 0, value, n, stream);
    }

    int launch_copy(int dt, void * dst, const void * src, uint64_t n, cudaStream_t stream)
    {
        if (n == 0 || dst == src) return HB2_OK;
        HB2_CUDA(cudaMemcpyAsync(dst, src, n * dtype_size(dt), cudaMemcpyDeviceToDevice, stream));
        return HB2_OK;
    }

    template <typename S, typename D>
    __global__ void convert_kernel(D * __restrict__ dst, const S * __restrict__ src, uint64_t n)
    {
        const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = D(src[i]);
    }

    int launch_convert(int dst_dt, void * dst, int src_dt, const void * src, uint64_t n, cudaStream_t stream)
    {
        if (n == 0) return HB2_OK;
        if (dst_dt == src_dt) return launch_copy(dst_dt, dst, src, n, stream);
        unsigned grid = stream_grid(n);
        if (src_dt == HB2_F64) convert_kernel<double, float><<<grid, 256, 0, stream>>>((float *)dst, (const double *)src, n);
        else convert_kernel<float, double><<<grid, 256, 0, stream>>>((double *)dst, (const float *)src, n);
        count_launches(1);
        HB2_LAUNCH_CHECK("convert launch");
        return HB2_OK;
    }

    // x64 += (double)c: convert<OuterTag>(c, x_inner) followed by Sum<OuterTag>(x, c)
    // (math/ir.hh:73-75) in one pass.
    template <typename S>
    __global__ void add_converted_kernel(double * __restrict__ x, const S * __restrict__ c, uint64_t n)
    {
        const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
            x[i] = __dadd_rn(x[i], (double)c[i]);
    }

    int launch_add_converted(void * x64, int c_dt, const void * c, uint64_t n, cudaStream_t stream)
    {
        if (n == 0) return HB2_OK;
        unsigned grid = stream_grid(n);
        if (c_dt == HB2_F32) add_converted_kernel<float><<<grid, 256, 0, stream>>>((double *)x64, (const float *)c, n);
        else add_converted_kernel<double><<<grid, 256, 0, stream>>>((double *)x64, (const double *)c, n);
        count_launches(1);
        HB2_LAUNCH_CHECK("add_converted launch");
        return HB2_OK;
    }

    // Deterministic dot: element i goes to thread (i / 4) % (grid*256) in a
    // fixed pattern; per-thread sums, a fixed block tree, a fixed final tree.
    template <typename T>
    __global__ void dot_kernel(const T * __restrict__ x, const T * __restrict__ y, uint64_t n, ReduceSlot rs,
                               double * out, int want_sqrt)
    {
        __shared__ double scratch[32];
        const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
        double s = 0.0;
        for (uint64_t i = tid; i < n; i += nthreads) s = fma((double)x[i], (double)y[i], s);
        s = block_sum(s, scratch);
        grid_sum_finish(s, rs, out, want_sqrt, scratch);
    }

    static unsigned reduce_grid(uint64_t n)
    {
        uint64_t g = (n + 1023) / 1024;
        uint64_t cap = (uint64_t)num_sms() * 4;
        return (unsigned)std::max<uint64_t>(1, std::min(g, cap));
    }

    int launch_dot(int dt, const void * x, const void * y, uint64_t n, int root, double * dev_out,
                   const Workspace * ws, cudaStream_t stream)
    {
        if (n == 0) { HB2_CUDA(cudaMemsetAsync(dev_out, 0, sizeof(double), stream)); return HB2_OK; }
        unsigned grid = reduce_grid(n);
        if (dt == HB2_F64) dot_kernel<double><<<grid, 256, 0, stream>>>((const double *)x, (const double *)y, n, ws->slot(), dev_out, root);
        else dot_kernel<float><<<grid, 256, 0, stream>>>((const float *)x, (const float *)y, n, ws->slot(), dev_out, root);
        count_launches(1);
        HB2_LAUNCH_CHECK("dot launch");
        return HB2_OK;
    }

    int launch_norm(int dt, const void * x, uint64_t n, int root, double * dev_out, const Workspace * ws,
                    cudaStream_t stream)
    {
        return launch_dot(dt, x, x, n, root, dev_out, ws, stream);
    }

    // The dot in the reference's tags::CPU order (la/dot_product.hh:72-89: one
    // sequential chain result += x[i] * y[i], contracted to fma by its compiler, in
    // the element type), sqrt in the element type for the rooted norm
    // (la/norm.hh:363-381).  One thread: for callers that need the reference's bits
    // (the tag binding's exact mode), not for speed.
    template <typename T>
    __global__ void dot_ordered_kernel(const T * __restrict__ x, const T * __restrict__ y, uint64_t n, double * out,
                                       int root)
    {
        if (threadIdx.x != 0 || blockIdx.x != 0) return;
        T s = T(0);
        uint64_t i = 0;
        for (; i + 8 <= n; i += 8)
        {
            T a[8], b[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) { a[k] = x[i + k]; b[k] = y[i + k]; }
#pragma unroll
            for (int k = 0; k < 8; ++k) s = Arith<T>::fma(a[k], b[k], s);
        }
        for (; i < n; ++i) s = Arith<T>::fma(x[i], y[i], s);
        *out = root ? (double)sqrt(s) : (double)s;
    }

    static int reduce_api(int dt, const void * x, const void * y, uint64_t n, int root, double * dev_out,
                          double * host_out, cudaStream_t stream, bool ordered = false)
    {
        if ((n > 0 && (! x || ! y)) || (! dev_out && ! host_out)) return fail(HB2_ERR_ARG, "reduction: null argument");
        Workspace * ws = 0;
        int st = stream_workspace(stream, &ws);
        if (st) return st;
        double * target = dev_out ? dev_out : ws->scalars;
        if (ordered)
        {
            if (dt == HB2_F64) dot_ordered_kernel<double><<<1, 32, 0, stream>>>((const double *)x, (const double *)y, n, target, root);
            else dot_ordered_kernel<float><<<1, 32, 0, stream>>>((const float *)x, (const float *)y, n, target, root);
            count_launches(1);
            HB2_LAUNCH_CHECK("ordered dot launch");
        }
        else st = launch_dot(dt, x, y, n, root, target, ws, stream);
        if (st) return st;
        if (host_out)
        {
            HB2_CUDA(cudaMemcpyAsync(ws->host_scalars, target, sizeof(double), cudaMemcpyDeviceToHost, stream));
            HB2_CUDA(cudaStreamSynchronize(stream));
            *host_out = ws->host_scalars[0];
        }
        return HB2_OK;
    }
}

using namespace hb2;

extern "C" int hb2_scaled_sum(hb2_dtype dt, void * x, const void * y, double b, uint64_t n, cudaStream_t s)
{ return launch_blas1<kAxpy>(dt, x, y, 0, b, n, s); }

extern "C" int hb2_scaled_sum3(hb2_dtype dt, void * r, const void * x, const void * y, double b, uint64_t n,
                               cudaStream_t s)
{ return launch_blas1<kAxpy3>(dt, r, x, y, b, n, s); }

extern "C" int hb2_sum(hb2_dtype dt, void * x, const void * y, uint64_t n, cudaStream_t s)
{ return launch_blas1<kSum>(dt, x, y, 0, 0.0, n, s); }

extern "C" int hb2_difference(hb2_dtype dt, void * x, const void * y, uint64_t n, cudaStream_t s)
{ return launch_blas1<kDiff>(dt, x, y, 0, 0.0, n, s); }

extern "C" int hb2_difference3(hb2_dtype dt, void * r, const void * x, const void * y, uint64_t n, cudaStream_t s)
{ return launch_blas1<kDiff3>(dt, r, x, y, 0.0, n, s); }

extern "C" int hb2_scale(hb2_dtype dt, void * x, double a, uint64_t n, cudaStream_t s)
{ return launch_blas1<kScale>(dt, x, 0, 0, a, n, s); }

extern "C" int hb2_element_product(hb2_dtype dt, void * r, const void * a, const void * b, uint64_t n, cudaStream_t s)
{ return launch_blas1<kEprod>(dt, r, a, b, 0.0, n, s); }

extern "C" int hb2_fill(hb2_dtype dt, void * x, double value, uint64_t n, cudaStream_t s)
{ return launch_fill(dt, x, value, n, s); }

extern "C" int hb2_copy(hb2_dtype dt, void * dst, const void * src, uint64_t n, cudaStream_t s)
{ return launch_copy(dt, dst, src, n, s); }

extern "C" int hb2_convert(hb2_dtype dst_dt, void * dst, hb2_dtype src_dt, const void * src, uint64_t n, cudaStream_t s)
{ return launch_convert(dst_dt, dst, src_dt, src, n, s); }

extern "C" int hb2_dot(hb2_dtype dt, const void * x, const void * y, uint64_t n, double * dev_out, double * host_out,
                       cudaStream_t s)
{ return reduce_api(dt, x, y, n, 0, dev_out, host_out, s); }

extern "C" int hb2_norm_l2(hb2_dtype dt, const void * x, uint64_t n, int root, double * dev_out, double * host_out,
                           cudaStream_t s)
{ return reduce_api(dt, x, x, n, root, dev_out, host_out, s); }

extern "C" int hb2_dot_ordered(hb2_dtype dt, const void * x, const void * y, uint64_t n, int root, double * dev_out,
                               double * host_out, cudaStream_t s)
{ return reduce_api(dt, x, y, n, root, dev_out, host_out, s, true); }
