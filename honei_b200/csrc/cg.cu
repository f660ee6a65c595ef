// CGSolver<Tag, methods::NONE> (math/cg.hh:64-135) on the device.
//
// Two executions of the same recurrence:
//  * cg_small_kernel -- one thread block, vectors (and the matrix when it fits)
//    in shared memory; used for the MG coarsest level and small systems.  With
//    `exact` the dot products run in the reference's sequential fma order, so
//    the iterates are bit-identical to the reference's tags::CPU solver.
//  * cg_coop_kernel -- one cooperative launch over the whole GPU; each
//    iteration is SpMV+dot | axpy,axpy+norm | p-update separated by bounded
//    grid barriers, all scalars stay on the device, reductions are in a fixed
//    order (reproducible, tree-ordered rather than sequential).
//
// The stop test is the reference's: sqrt(r.r) < eps * sqrt(r0.r0) or
// sqrt(r.r) < eps, checked after the p update; lambda and the p scaling guard
// their divisors with machine epsilon exactly like cg.hh:99 and :106.
#include "cg_warp.cuh"
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <algorithm>
#include <cfloat>
#include <cstring>

namespace hb2
{
    // ------------------------------------------------------------------ small
    template <typename T>
    struct SmallMat
    {
        const T * val;
        const int32_t * col;
        uint64_t ld;
    };

    template <typename T>
    __device__ __forceinline__ T row_product(const SmallMat<T> & A, uint32_t K, int r, const T * x)
    {
        typedef Arith<T> M;
        T s = T(0);
        for (uint32_t k = 0; k < K; ++k)
        {
            int c = A.col[(uint64_t)k * A.ld + r];
            if (c >= 0) s = M::add(s, M::mul(A.val[(uint64_t)k * A.ld + r], x[c]));
        }
        return s;
    }

    // dot of two shared-memory vectors, identical result in every thread
    template <typename T>
    __device__ __forceinline__ T small_dot(const T * a, const T * b, int n, bool exact, double * scratch, T * bcast)
    {
        if (exact)
        {
            __syncthreads();
            if (threadIdx.x == 0)
            {
                T s = T(0);
                for (int i = 0; i < n; ++i) s = Arith<T>::fma(a[i], b[i], s);
                *bcast = s;
            }
            __syncthreads();
            return *bcast;
        }
        double s = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) s = fma((double)a[i], (double)b[i], s);
        return (T)block_sum(s, scratch);
    }

    template <typename T>
    __global__ void cg_small_kernel(EllView<T> Ag, const T * __restrict__ b, T * __restrict__ xg, uint64_t max_iters,
                                    double eps_d, int exact, int mat_in_smem, uint64_t * used_out, double * defect_out)
    {
        typedef Arith<T> M;
        extern __shared__ __align__(16) unsigned char smem_raw[];
        __shared__ double scratch[32];
        __shared__ T bcast;
        const int n = (int)Ag.rows;
        T * x = (T *)smem_raw;
        T * r = x + n;
        T * p = r + n;
        T * v = p + n;
        SmallMat<T> A;
        if (mat_in_smem)
        {
            T * sval = v + n;
            int32_t * scol = (int32_t *)(sval + (size_t)Ag.K * n);
            for (int i = threadIdx.x; i < (int)(Ag.K * n); i += blockDim.x)
            {
                int k = i / n, row = i % n;
                sval[i] = Ag.val[(uint64_t)k * Ag.ld + row];
                scol[i] = Ag.col[(uint64_t)k * Ag.ld + row];
            }
            A.val = sval;
            A.col = scol;
            A.ld = n;
        }
        else
        {
            A.val = Ag.val;
            A.col = Ag.col;
            A.ld = Ag.ld;
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = xg[i];
        __syncthreads();
        // Defect(r, b, A, x); copy(r, p)
        for (int i = threadIdx.x; i < n; i += blockDim.x)
        {
            T d = M::sub(b[i], row_product(A, Ag.K, i, x));
            r[i] = d;
            p[i] = d;
        }
        __syncthreads();
        const T eps = T(eps_d);
        T alpha = small_dot(r, r, n, exact, scratch, &bcast);
        const T initial = sqrt(alpha);
        T current = initial;
        uint64_t it = 0, used = 0;
        while (it < max_iters)
        {
            for (int i = threadIdx.x; i < n; i += blockDim.x) v[i] = row_product(A, Ag.K, i, p);
            __syncthreads();
            const T temp = small_dot(v, p, n, exact, scratch, &bcast);
            const T lambda = M::div(alpha, guard(temp));
            const T mlambda = -lambda;
            for (int i = threadIdx.x; i < n; i += blockDim.x)
            {
                x[i] = M::add(x[i], M::mul(lambda, p[i]));
                r[i] = M::add(r[i], M::mul(mlambda, v[i]));
            }
            __syncthreads();
            const T alpha_old = alpha;
            alpha = small_dot(r, r, n, exact, scratch, &bcast);
            const T talpha = M::div(alpha, guard(alpha_old));
            for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = M::add(M::mul(p[i], talpha), r[i]);
            __syncthreads();
            ++it;
            current = sqrt(alpha);
            if (current < M::mul(eps, initial) || current < eps) { used = it; break; }
            if (it == max_iters) used = it;
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x) xg[i] = x[i];
        if (threadIdx.x == 0)
        {
            if (used_out) *used_out = used;
            if (defect_out) *defect_out = (double)current;
        }
    }

    template <typename T>
    __device__ __forceinline__ T warp_dot_tree(const T * a, const T * b, int n)
    {
        double s = 0.0;
        for (int i = threadIdx.x; i < n; i += 32) s = fma((double)a[i], (double)b[i], s);
        return (T)warp_sum(s);   // xor butterfly: every lane ends with the same bits
    }

    template <typename T>
    __global__ void __launch_bounds__(32)
    cg_warp_kernel(EllView<T> Ag, const T * __restrict__ b, T * __restrict__ xg, uint64_t max_iters, double eps_d,
                   int exact, int mat_in_smem, uint64_t * used_out, double * defect_out)
    {
        typedef Arith<T> M;
        extern __shared__ __align__(16) unsigned char smem_raw[];
        const int n = (int)Ag.rows, lane = threadIdx.x;
        T * x = (T *)smem_raw;
        T * r = x + n;
        T * p = r + n;
        T * v = p + n;
        SmallMat<T> A;
        if (mat_in_smem)
        {
            T * sval = v + n;
            int32_t * scol = (int32_t *)(sval + (size_t)Ag.K * n);
            for (uint32_t k = 0; k < Ag.K; ++k)
                for (int i = lane; i < n; i += 32)
                {
                    sval[k * n + i] = Ag.val[(uint64_t)k * Ag.ld + i];
                    scol[k * n + i] = Ag.col[(uint64_t)k * Ag.ld + i];
                }
            A.val = sval;
            A.col = scol;
            A.ld = n;
        }
        else
        {
            A.val = Ag.val;
            A.col = Ag.col;
            A.ld = Ag.ld;
        }
        for (int i = lane; i < n; i += 32) x[i] = xg[i];
        __syncwarp();
        for (int i = lane; i < n; i += 32)
        {
            T d = M::sub(b[i], row_product(A, Ag.K, i, x));
            r[i] = d;
            p[i] = d;
        }
        __syncwarp();
        const T eps = T(eps_d);
        T alpha = exact ? warp_dot_exact(r, r, n) : warp_dot_tree(r, r, n);
        const T initial = sqrt(alpha);
        T current = initial;
        uint64_t it = 0, used = 0;
        while (it < max_iters)
        {
            for (int i = lane; i < n; i += 32) v[i] = row_product(A, Ag.K, i, p);
            __syncwarp();
            const T temp = exact ? warp_dot_exact(v, p, n) : warp_dot_tree(v, p, n);
            const T lambda = M::div(alpha, guard(temp));
            const T mlambda = -lambda;
            for (int i = lane; i < n; i += 32)
            {
                x[i] = M::add(x[i], M::mul(lambda, p[i]));
                r[i] = M::add(r[i], M::mul(mlambda, v[i]));
            }
            __syncwarp();
            const T alpha_old = alpha;
            alpha = exact ? warp_dot_exact(r, r, n) : warp_dot_tree(r, r, n);
            const T talpha = M::div(alpha, guard(alpha_old));
            for (int i = lane; i < n; i += 32) p[i] = M::add(M::mul(p[i], talpha), r[i]);
            __syncwarp();
            ++it;
            current = sqrt(alpha);
            if (current < M::mul(eps, initial) || current < eps) { used = it; break; }
            if (it == max_iters) used = it;
        }
        for (int i = lane; i < n; i += 32) xg[i] = x[i];
        if (lane == 0)
        {
            if (used_out) *used_out = used;
            if (defect_out) *defect_out = (double)current;
        }
    }

    template <typename T, typename S>
    static bool launch_warp_reg(const hb2_ell_s * A, const void * b, void * x, uint64_t max_iters, double eps, int exact,
                                uint64_t * used_dev, double * defect_dev, cudaStream_t stream, uint32_t nvec = 1,
                                uint64_t vstride = 0, const uint8_t * active = nullptr,
                                const uint32_t * list = nullptr, const uint32_t * count = nullptr, uint64_t cap = 0)
    {
        if (A->K == 0 || A->K > 9 || A->rows > 128) return false;
        const int rpl = (int)((A->rows + 31) / 32);
        const size_t smem = 3 * A->rows * sizeof(T) + 16;
        EllView<T> v = A->view<T>();
        const S * bp = (const S *)b;
        S * xp = (S *)x;
        const unsigned grid = list ? (unsigned)std::min<uint64_t>(nvec, cap ? cap : list_grid_cap()) : nvec;
        switch (rpl)
        {
            case 1: launch_pdl(cg_warp_reg_kernel<T, S, 1>, dim3(grid), dim3(32), smem, stream, v, bp, xp, max_iters, eps, exact, used_dev, defect_dev, vstride, active, list, count); break;
            case 2: launch_pdl(cg_warp_reg_kernel<T, S, 2>, dim3(grid), dim3(32), smem, stream, v, bp, xp, max_iters, eps, exact, used_dev, defect_dev, vstride, active, list, count); break;
            case 3: launch_pdl(cg_warp_reg_kernel<T, S, 3>, dim3(grid), dim3(32), smem, stream, v, bp, xp, max_iters, eps, exact, used_dev, defect_dev, vstride, active, list, count); break;
            default: launch_pdl(cg_warp_reg_kernel<T, S, 4>, dim3(grid), dim3(32), smem, stream, v, bp, xp, max_iters, eps, exact, used_dev, defect_dev, vstride, active, list, count); break;
        }
        return true;
    }

    // nvec independent coarse systems with one operator, one warp each: FP64
    // arithmetic on FP32 vectors (A64 FP64) or in the operator's own type
    int launch_cg_warp_batched(const hb2_ell_s * A, int vec_dtype, const void * b, void * x, uint32_t nvec,
                               uint64_t vstride, const uint8_t * active, uint64_t max_iters, double eps,
                               cudaStream_t stream, const uint32_t * list, const uint32_t * count, uint64_t cap)
    {
        if (nvec == 0) return HB2_OK;
        bool ok;
        // the batched preconditioner keeps the standard recurrence: inside the outer
        // PCG the one-reduction form left some right-hand sides of the 512-system
        // batch short of their tolerance after 100 steps
        const int mode = kCgTreeStandard;
        if (A->dtype == HB2_F64 && vec_dtype == HB2_F32)
            ok = launch_warp_reg<double, float>(A, b, x, max_iters, eps, mode, 0, 0, stream, nvec, vstride, active, list, count, cap);
        else if (A->dtype == HB2_F64 && vec_dtype == HB2_F64)
            ok = launch_warp_reg<double, double>(A, b, x, max_iters, eps, mode, 0, 0, stream, nvec, vstride, active, list, count, cap);
        else if (A->dtype == HB2_F32 && vec_dtype == HB2_F32)
            ok = launch_warp_reg<float, float>(A, b, x, max_iters, eps, mode, 0, 0, stream, nvec, vstride, active, list, count, cap);
        else return fail(HB2_ERR_ARG, "batched coarse CG: unsupported element types");
        if (! ok) return fail(HB2_ERR_UNSUPPORTED, "batched coarse CG: the coarsest level needs <= 128 rows and 9 slots");
        count_launches(1);
        HB2_LAUNCH_CHECK("cg_warp_reg_kernel (batched)");
        return HB2_OK;
    }

    bool cg_mixed_supported(const hb2_ell_s * A64)
    {
        return A64->dtype == HB2_F64 && A64->K >= 1 && A64->K <= 9 && A64->rows <= 128;
    }

    // coarsest solve of an FP32 level in FP64: A64 is the FP64 operator, b / x are FP32
    int launch_cg_small_f32io(const hb2_ell_s * A64, const void * b32, void * x32, uint64_t max_iters, double eps,
                              int exact, uint64_t * used_dev, double * defect_dev, cudaStream_t stream)
    {
        if (! launch_warp_reg<double, float>(A64, b32, x32, max_iters, eps, exact, used_dev, defect_dev, stream))
            return fail(HB2_ERR_UNSUPPORTED, "FP64 coarse solve of an FP32 level needs <= 128 rows and 1-9 slots");
        count_launches(1);
        HB2_LAUNCH_CHECK("cg_warp_reg_kernel (FP32 vectors, FP64 arithmetic)");
        return HB2_OK;
    }

    constexpr uint64_t kWarpCgMaxRows = 1024;

    static size_t small_smem(const hb2_ell_s * A, bool with_matrix)
    {
        size_t es = dtype_size(A->dtype), n = A->rows;
        size_t bytes = 4 * n * es;
        if (with_matrix) bytes += (size_t)A->K * n * (es + 4);
        return bytes + 16;
    }

    constexpr size_t kSmallSmemLimit = 200 * 1024;

    bool cg_small_fits(const hb2_ell_s * A)
    {
        return A->rows == A->cols && A->rows > 0 && small_smem(A, false) <= kSmallSmemLimit;
    }

    int launch_cg_small(const hb2_ell_s * A, const void * b, void * x, uint64_t max_iters, double eps, int exact,
                        uint64_t * used_dev, double * defect_dev, cudaStream_t stream)
    {
        if (! cg_small_fits(A)) return fail(HB2_ERR_UNSUPPORTED, "system too large for the one-block CG");
        const bool mat = small_smem(A, true) <= kSmallSmemLimit;
        const size_t smem = small_smem(A, mat);
        int threads = (int)std::min<uint64_t>(1024, (A->rows + 31) / 32 * 32);
        static bool attr_set = false;   // once per process, never inside a stream capture
        if (! attr_set)
        {
            HB2_CUDA(cudaFuncSetAttribute(cg_small_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmemLimit + 64));
            HB2_CUDA(cudaFuncSetAttribute(cg_small_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmemLimit + 64));
            HB2_CUDA(cudaFuncSetAttribute(cg_warp_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmemLimit + 64));
            HB2_CUDA(cudaFuncSetAttribute(cg_warp_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmemLimit + 64));
            attr_set = true;
        }
        // the register kernel for the 9-slot operators; others take the shared-memory one
        const bool reg = A->K != 9 ? false
                       : A->dtype == HB2_F64
                             ? launch_warp_reg<double, double>(A, b, x, max_iters, eps, exact, used_dev, defect_dev, stream)
                             : launch_warp_reg<float, float>(A, b, x, max_iters, eps, exact, used_dev, defect_dev, stream);
        if (reg)
        {
            count_launches(1);
            HB2_LAUNCH_CHECK("cg_warp_reg_kernel");
            return HB2_OK;
        }
        if (A->rows <= kWarpCgMaxRows)
        {
            if (A->dtype == HB2_F64)
                cg_warp_kernel<double><<<1, 32, smem, stream>>>(A->view<double>(), (const double *)b, (double *)x,
                                                                max_iters, eps, exact, mat, used_dev, defect_dev);
            else
                cg_warp_kernel<float><<<1, 32, smem, stream>>>(A->view<float>(), (const float *)b, (float *)x,
                                                               max_iters, eps, exact, mat, used_dev, defect_dev);
            count_launches(1);
            HB2_LAUNCH_CHECK("cg_warp_kernel");
            return HB2_OK;
        }
        if (A->dtype == HB2_F64)
        {
            cg_small_kernel<double><<<1, threads, smem, stream>>>(A->view<double>(), (const double *)b, (double *)x,
                                                                  max_iters, eps, exact, mat, used_dev, defect_dev);
        }
        else
        {
            cg_small_kernel<float><<<1, threads, smem, stream>>>(A->view<float>(), (const float *)b, (float *)x,
                                                                 max_iters, eps, exact, mat, used_dev, defect_dev);
        }
        count_launches(1);
        HB2_LAUNCH_CHECK("cg_small_kernel");
        return HB2_OK;
    }

    // ------------------------------------------------------------------ cooperative
    constexpr int kCoopThreads = 256;

    // every block reduces the G block partials in the same fixed order
    __device__ __forceinline__ double reduce_partials(const double * partials, unsigned G, double * scratch)
    {
        double s = 0.0;
        for (unsigned i = threadIdx.x; i < G; i += blockDim.x) s += ((volatile const double *)partials)[i];
        return block_sum(s, scratch);
    }

    template <typename T>
    __global__ void __launch_bounds__(kCoopThreads)
    cg_coop_kernel(EllView<T> A, const T * __restrict__ b, T * __restrict__ x, T * __restrict__ r, T * __restrict__ p,
                   T * __restrict__ v, uint64_t max_iters, double eps_d, double * partials0, double * partials1,
                   GridBarrier bar, uint64_t * used_out, double * defect_out)
    {
        typedef Arith<T> M;
        __shared__ double scratch[32];
        const uint64_t n = A.rows;
        const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
        const unsigned G = gridDim.x;

        // r = b - A x, p = r, partial r.r
        double part = 0.0;
        for (uint64_t i = tid; i < n; i += nth)
        {
            T s = T(0);
            for (uint32_t k = 0; k < A.K; ++k)
            {
                int c = A.col[(uint64_t)k * A.ld + i];
                if (c >= 0) s = M::add(s, M::mul(A.val[(uint64_t)k * A.ld + i], x[c]));
            }
            T d = M::sub(b[i], s);
            r[i] = d;
            p[i] = d;
            part = fma((double)d, (double)d, part);
        }
        part = block_sum(part, scratch);
        if (threadIdx.x == 0) partials1[blockIdx.x] = part;
        if (! grid_sync(bar)) return;
        T alpha = (T)reduce_partials(partials1, G, scratch);
        const T eps = T(eps_d);
        const T initial = sqrt(alpha);
        T current = initial;
        uint64_t it = 0, used = 0;
        while (it < max_iters)
        {
            // v = A p, partial v.p
            part = 0.0;
            for (uint64_t i = tid; i < n; i += nth)
            {
                T s = T(0);
                for (uint32_t k = 0; k < A.K; ++k)
                {
                    int c = A.col[(uint64_t)k * A.ld + i];
                    if (c >= 0) s = M::add(s, M::mul(A.val[(uint64_t)k * A.ld + i], p[c]));
                }
                v[i] = s;
                part = fma((double)s, (double)p[i], part);
            }
            part = block_sum(part, scratch);
            if (threadIdx.x == 0) partials0[blockIdx.x] = part;
            if (! grid_sync(bar)) return;
            const T temp = (T)reduce_partials(partials0, G, scratch);
            const T lambda = M::div(alpha, guard(temp));
            const T mlambda = -lambda;
            part = 0.0;
            for (uint64_t i = tid; i < n; i += nth)
            {
                x[i] = M::add(x[i], M::mul(lambda, p[i]));
                T ri = M::add(r[i], M::mul(mlambda, v[i]));
                r[i] = ri;
                part = fma((double)ri, (double)ri, part);
            }
            part = block_sum(part, scratch);
            if (threadIdx.x == 0) partials1[blockIdx.x] = part;
            if (! grid_sync(bar)) return;
            const T alpha_old = alpha;
            alpha = (T)reduce_partials(partials1, G, scratch);
            const T talpha = M::div(alpha, guard(alpha_old));
            for (uint64_t i = tid; i < n; i += nth) p[i] = M::add(M::mul(p[i], talpha), r[i]);
            ++it;
            current = sqrt(alpha);
            bool stop = current < M::mul(eps, initial) || current < eps;
            if (stop) used = it;
            else if (it == max_iters) used = it;
            if (stop) break;
            if (! grid_sync(bar)) return;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0)
        {
            *used_out = used;
            *defect_out = (double)current;
        }
    }
}

using namespace hb2;

extern "C" int hb2_cg_solve(hb2_ell A, const void * b, void * x, uint64_t max_iters, double eps, uint64_t * used_iters,
                            double * final_defect, cudaStream_t stream)
{
    if (! A || ! b || ! x) return fail(HB2_ERR_ARG, "hb2_cg_solve: null argument");
    if (A->rows != A->cols) return fail(HB2_ERR_SIZE, "hb2_cg_solve: VectorSizeDoesNotMatch (square system required)");
    Workspace * ws = 0;
    int st = stream_workspace(stream, &ws);
    if (st) return st;
    uint64_t * used_dev = (uint64_t *)(ws->scalars + 8);
    double * def_dev = ws->scalars + 9;
    HB2_CUDA(cudaMemsetAsync(ws->scalars + 8, 0, 2 * sizeof(double), stream));
    const size_t es = dtype_size(A->dtype), n = A->rows;
    if (n == 0) { if (used_iters) *used_iters = 0; if (final_defect) *final_defect = 0; return HB2_OK; }
    if (cg_small_fits(A) && n <= 4096)
    {
        st = launch_cg_small(A, b, x, max_iters, eps, 0, used_dev, def_dev, stream);
        if (st) return st;
    }
    else
    {
        void * tmp = 0;
        const size_t vb = (n * es + 255) / 256 * 256;   // each vector 256-byte aligned
        HB2_CUDA(cudaMallocAsync(&tmp, 3 * vb + 64, stream));
        char * base = (char *)tmp;
        void * r = base, * p = base + vb, * v = base + 2 * vb;
        int dev = 0, per_sm = 0;
        cudaGetDevice(&dev);
        if (A->dtype == HB2_F64) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_coop_kernel<double>, kCoopThreads, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_coop_kernel<float>, kCoopThreads, 0);
        uint64_t want = (n + kCoopThreads * 2 - 1) / (kCoopThreads * 2);
        uint64_t cap = (uint64_t)std::max(1, per_sm) * num_sms();
        unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(std::min<uint64_t>(want, cap), ws->max_blocks / 2));
        double * partials0 = ws->partials, * partials1 = ws->partials + ws->max_blocks / 2;
        GridBarrier bar = ws->barrier();
        HB2_CUDA(cudaMemsetAsync(ws->bar_words, 0, 3 * sizeof(unsigned) + 2 * sizeof(int), stream));
        HB2_CUDA(cudaMemsetAsync(ws->error, 0, sizeof(int), stream));
        cudaError_t e;
        if (A->dtype == HB2_F64)
        {
            EllView<double> Av = A->view<double>();
            const double * bp = (const double *)b;
            double * xp = (double *)x, * rp = (double *)r, * pp = (double *)p, * vp = (double *)v;
            void * args[] = {&Av, &bp, &xp, &rp, &pp, &vp, &max_iters, &eps, &partials0, &partials1, &bar, &used_dev, &def_dev};
            e = cudaLaunchCooperativeKernel((const void *)cg_coop_kernel<double>, grid, kCoopThreads, args, 0, stream);
        }
        else
        {
            EllView<float> Av = A->view<float>();
            const float * bp = (const float *)b;
            float * xp = (float *)x, * rp = (float *)r, * pp = (float *)p, * vp = (float *)v;
            void * args[] = {&Av, &bp, &xp, &rp, &pp, &vp, &max_iters, &eps, &partials0, &partials1, &bar, &used_dev, &def_dev};
            e = cudaLaunchCooperativeKernel((const void *)cg_coop_kernel<float>, grid, kCoopThreads, args, 0, stream);
        }
        count_launches(1);
        cudaFreeAsync(tmp, stream);
        if (e != cudaSuccess) return cuda_status(e, "cg_coop_kernel cooperative launch");
    }
    HB2_CUDA(cudaMemcpyAsync(ws->host_scalars, ws->scalars + 8, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    int herr = 0;
    HB2_CUDA(cudaMemcpyAsync(ws->host_scalars + 2, ws->error, sizeof(int), cudaMemcpyDeviceToHost, stream));
    HB2_CUDA(cudaStreamSynchronize(stream));
    memcpy(&herr, ws->host_scalars + 2, sizeof(int));
    if (herr) return fail(HB2_ERR_TIMEOUT, "hb2_cg_solve: a grid barrier wait expired");
    uint64_t used = 0;
    memcpy(&used, ws->host_scalars, sizeof(uint64_t));
    if (used_iters) *used_iters = used;
    if (final_defect) *final_defect = ws->host_scalars[1];
    if (final_defect && ! (ws->host_scalars[1] == ws->host_scalars[1])) return fail(HB2_ERR_NOT_FINITE, "hb2_cg_solve: NaN defect");
    return HB2_OK;
}
