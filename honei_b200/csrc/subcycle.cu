// The small levels of a V-cycle in two thread-block-cluster launches.
//
// Below a few ten thousand rows every ELL pass of the V-cycle is bound by
// launch latency, not bandwidth (a kernel costs ~4 us whatever its size).  The
// levels 1..top of the hierarchy (top: the largest level with at most
// kSubMaxRows rows) therefore run as
//   down  : for each level top..1: pre-smoothing sweeps, defect, restriction
//           + clear of the next coarser correction
//   (coarsest-level CG: the one-warp kernel of cg.cu)
//   up    : for each level 1..top: prolongation + add, post-smoothing sweeps
// each as ONE kernel on one cluster of CTAs (16 on B200, 8 where 16 cannot be
// co-scheduled).  Phases are separated by the cluster's hardware barrier
// (barrier.cluster arrive/wait with release/acquire semantics); vectors
// written in one phase are read in the next with L2 loads (ld.cg), so no CTA
// can see a stale L1 line.  Each row is computed with exactly the arithmetic
// of the per-operator kernels (ell.cu), so results are bit-identical.
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace hb2
{
    template <typename T>
    struct SubLevel
    {
        EllView<T> A;      // this level's operator
        EllView<T> R;      // restriction to the next coarser level (levels > 0)
        EllView<T> P;      // prolongation from the next coarser level (levels > 0)
        T * x;
        T * b;
        T * store;
        T * tmp;
        const T * jac;
        uint32_t n;
    };

    constexpr int kSubMaxLevels = 10;

    template <typename T>
    struct SubCycle
    {
        SubLevel<T> lev[kSubMaxLevels];   // lev[0]: coarsest
        int top;                          // highest level index handled here
        int n_pre, n_post;
    };

    // sum_k A(r, k) * v(col(r, k)), slot order, separately rounded
    template <typename T, int KT>
    __device__ __forceinline__ T row_sum(const EllView<T> & A, uint32_t r, const T * v)
    {
        typedef Arith<T> M;
        T s = T(0);
#pragma unroll
        for (int k = 0; k < KT; ++k)
        {
            const int c = __ldg(A.col + (uint64_t)k * A.ld + r);
            if (c >= 0) s = M::add(s, M::mul(__ldg(A.val + (uint64_t)k * A.ld + r), __ldcg(v + c)));
        }
        return s;
    }

    template <typename T>
    __device__ __forceinline__ T row_sum_any(const EllView<T> & A, uint32_t r, const T * v)
    {
        if (A.K == 9) return row_sum<T, 9>(A, r, v);
        if (A.K == 4) return row_sum<T, 4>(A, r, v);
        typedef Arith<T> M;
        T s = T(0);
        for (uint32_t k = 0; k < A.K; ++k)
        {
            const int c = __ldg(A.col + (uint64_t)k * A.ld + r);
            if (c >= 0) s = M::add(s, M::mul(__ldg(A.val + (uint64_t)k * A.ld + r), __ldcg(v + c)));
        }
        return s;
    }

    // damped Jacobi sweeps with ping-pong (math/ri.hh:110-133), result back in x
    template <typename T>
    __device__ void sub_smooth(const SubLevel<T> & L, int sweeps, uint32_t tid, uint32_t nth)
    {
        typedef Arith<T> M;
        cg::cluster_group cluster = cg::this_cluster();
        T * cur = L.x, * nxt = L.tmp;
        for (int s = 0; s < sweeps; ++s)
        {
            for (uint32_t r = tid; r < L.n; r += nth)
            {
                const T acc = row_sum_any(L.A, r, cur);
                nxt[r] = M::add(__ldcg(cur + r), M::mul(__ldg(L.jac + r), M::sub(__ldcg(L.b + r), acc)));
            }
            cluster.sync();
            T * t = cur;
            cur = nxt;
            nxt = t;
        }
        if (cur != L.x)
        {
            for (uint32_t r = tid; r < L.n; r += nth) L.x[r] = __ldcg(cur + r);
            cluster.sync();
        }
    }

    template <typename T>
    __global__ void __launch_bounds__(1024) mg_sub_down_kernel(const __grid_constant__ SubCycle<T> sc)
    {
        typedef Arith<T> M;
        cg::cluster_group cluster = cg::this_cluster();
        const uint32_t tid = cluster.block_rank() * blockDim.x + threadIdx.x;
        const uint32_t nth = cluster.num_blocks() * blockDim.x;
        for (int i = sc.top; i >= 1; --i)
        {
            const SubLevel<T> & L = sc.lev[i];
            const SubLevel<T> & C = sc.lev[i - 1];
            sub_smooth(L, sc.n_pre, tid, nth);
            for (uint32_t r = tid; r < L.n; r += nth)
                L.store[r] = M::sub(__ldcg(L.b + r), row_sum_any(L.A, r, L.x));
            cluster.sync();
            for (uint32_t r = tid; r < C.n; r += nth)
            {
                C.b[r] = row_sum_any(L.R, r, L.store);
                C.x[r] = T(0);
            }
            cluster.sync();
        }
    }

    template <typename T>
    __global__ void __launch_bounds__(1024) mg_sub_up_kernel(const __grid_constant__ SubCycle<T> sc)
    {
        typedef Arith<T> M;
        cg::cluster_group cluster = cg::this_cluster();
        const uint32_t tid = cluster.block_rank() * blockDim.x + threadIdx.x;
        const uint32_t nth = cluster.num_blocks() * blockDim.x;
        for (int i = 1; i <= sc.top; ++i)
        {
            const SubLevel<T> & L = sc.lev[i];
            const SubLevel<T> & C = sc.lev[i - 1];
            for (uint32_t r = tid; r < L.n; r += nth)
                L.x[r] = M::add(__ldcg(L.x + r), row_sum_any(L.P, r, C.x));
            cluster.sync();
            sub_smooth(L, sc.n_post, tid, nth);
        }
    }

    template <typename T>
    static SubLevel<T> sub_level(const SubLevelDesc & d)
    {
        SubLevel<T> s;
        s.A = d.A->view<T>();
        if (d.R) s.R = d.R->view<T>(); else s.R = s.A;
        if (d.P) s.P = d.P->view<T>(); else s.P = s.A;
        s.x = (T *)d.x;
        s.b = (T *)d.b;
        s.store = (T *)d.store;
        s.tmp = (T *)d.tmp;
        s.jac = (const T *)d.jac;
        s.n = (uint32_t)d.A->rows;
        return s;
    }

    static int cluster_width(const void * fn)
    {
        static int width = 0;
        if (width) return width;
        cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        for (int w : {16, 8})
        {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(w);
            cfg.blockDim = dim3(1024);
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = w;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg) == cudaSuccess && nclusters > 0)
            {
                width = w;
                return width;
            }
            cudaGetLastError();
        }
        width = 1;
        return width;
    }

    template <typename T>
    static int launch_sub_typed(const SubLevelDesc * lev, int top, int n_pre, int n_post, bool down, cudaStream_t s)
    {
        SubCycle<T> sc;
        for (int i = 0; i <= top; ++i) sc.lev[i] = sub_level<T>(lev[i]);
        sc.top = top;
        sc.n_pre = n_pre;
        sc.n_post = n_post;
        // the cluster width and the non-portable-size attributes were set up
        // by subcycle_prepare(), outside any stream capture
        const int w = cluster_width((const void *)mg_sub_down_kernel<double>);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(w);
        cfg.blockDim = dim3(1024);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = w;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaError_t e = down ? cudaLaunchKernelEx(&cfg, mg_sub_down_kernel<T>, sc)
                             : cudaLaunchKernelEx(&cfg, mg_sub_up_kernel<T>, sc);
        count_launches(1);
        if (e != cudaSuccess) return cuda_status(e, "cluster sub-cycle launch");
        return HB2_OK;
    }

    int launch_subcycle(int dtype, const SubLevelDesc * lev, int top, int n_pre, int n_post, bool down,
                        cudaStream_t stream)
    {
        if (top < 1 || top >= kSubMaxLevels) return fail(HB2_ERR_UNSUPPORTED, "sub-cycle: bad level range");
        return dtype == HB2_F64 ? launch_sub_typed<double>(lev, top, n_pre, n_post, down, stream)
                                : launch_sub_typed<float>(lev, top, n_pre, n_post, down, stream);
    }

    // prime the cluster attributes outside any stream capture
    int subcycle_prepare()
    {
        cluster_width((const void *)mg_sub_down_kernel<double>);
        cudaFuncSetAttribute((const void *)mg_sub_down_kernel<float>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaFuncSetAttribute((const void *)mg_sub_up_kernel<double>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaFuncSetAttribute((const void *)mg_sub_up_kernel<float>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_status(e, "sub-cycle attributes");
        return HB2_OK;
    }
}
