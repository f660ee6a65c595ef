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
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>

#include "cg_warp.cuh"

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
        // row patterns of A (host-built, ell_small_patterns): a row's product
        // then reads its nine (value, offset) pairs from shared memory
        const uint8_t * pat;
        const PatEnt<T> * ptab;
        uint32_t npat;
        // R and P are the Q1 transfer matrices of grid level q1l (mf, mc points per
        // line): their rows come from q1_restrict_row / q1_prolong_row; 0: read R, P
        uint32_t q1l, mf, mc;
    };

    constexpr int kSubMaxLevels = 10;
    constexpr int kSubRowsPerThread = 3;   // kSubMaxRows / (8 CTAs x 1024 threads), rounded up

    template <typename T>
    struct SubCycle
    {
        SubLevel<T> lev[kSubMaxLevels];   // lev[0]: coarsest
        int top;                          // highest level index handled here
        int t1;                           // levels 1..t1 run in CTA 0 alone (block barriers)
        int n_pre, n_post;
    };

    // sum_k A(r, k) * v(col(r, k)), slot order, separately rounded.  Every
    // index, value and vector load of the row is issued before the first
    // product, so a row costs one memory round trip, not K.  L2: vector loads
    // through L2 (other CTAs of the cluster wrote them); otherwise plain loads,
    // coherent within the block (block-local phases).
    template <typename T, int KT, bool L2>
    __device__ __forceinline__ T row_sum(const EllView<T> & A, uint32_t r, const T * v)
    {
        typedef Arith<T> M;
        int c[KT];
        T a[KT], xv[KT];
#pragma unroll
        for (int k = 0; k < KT; ++k)
        {
            c[k] = __ldg(A.col + (uint64_t)k * A.ld + r);
            a[k] = __ldg(A.val + (uint64_t)k * A.ld + r);
        }
#pragma unroll
        for (int k = 0; k < KT; ++k) xv[k] = c[k] >= 0 ? (L2 ? __ldcg(v + c[k]) : v[c[k]]) : T(0);
        T s = T(0);
#pragma unroll
        for (int k = 0; k < KT; ++k)
            if (c[k] >= 0) s = M::add(s, M::mul(a[k], xv[k]));
        return s;
    }

    template <typename T, bool L2 = true>
    __device__ __forceinline__ T row_sum_any(const EllView<T> & A, uint32_t r, const T * v)
    {
        if (A.K == 9) return row_sum<T, 9, L2>(A, r, v);
        if (A.K == 4) return row_sum<T, 4, L2>(A, r, v);
        typedef Arith<T> M;
        T s = T(0);
        for (uint32_t k = 0; k < A.K; ++k)
        {
            const int c = __ldg(A.col + (uint64_t)k * A.ld + r);
            if (c >= 0) s = M::add(s, M::mul(__ldg(A.val + (uint64_t)k * A.ld + r), L2 ? __ldcg(v + c) : v[c]));
        }
        return s;
    }

    // the same product from a row pattern: (value, offset) pairs from shared
    // memory, every vector load issued before the first product
    template <typename T, bool L2>
    __device__ __forceinline__ T row_sum_pat(const PatEnt<T> * e, uint32_t r, const T * v)
    {
        typedef Arith<T> M;
        T a[9], xv[9];
        int32_t off[9];
#pragma unroll
        for (int k = 0; k < 9; ++k)
        {
            off[k] = e[k].off;
            a[k] = e[k].val;
        }
#pragma unroll
        for (int k = 0; k < 9; ++k)
            xv[k] = off[k] != kPatEmpty ? (L2 ? __ldcg(v + (uint32_t)((int32_t)r + off[k])) : v[(uint32_t)((int32_t)r + off[k])]) : T(0);
        T s = T(0);
#pragma unroll
        for (int k = 0; k < 9; ++k)
            if (off[k] != kPatEmpty) s = M::add(s, M::mul(a[k], xv[k]));
        return s;
    }

    // Shared-memory copies of a level's pattern table and of the pattern ids
    // of the rows this thread owns (row tid + j * nth in slot j); ids null:
    // read the id from global memory.
    template <typename T>
    struct SubPat
    {
        const PatEnt<T> * tab;
        const uint8_t * ids;
    };

    template <typename T, bool L2>
    __device__ __forceinline__ T row_A(const SubLevel<T> & L, const SubPat<T> & sp, uint32_t r, uint32_t j, const T * v)
    {
        if (! sp.tab) return row_sum_any<T, L2>(L.A, r, v);
        const uint32_t p = sp.ids ? sp.ids[j * 1024 + threadIdx.x] : __ldg(L.pat + r);
        return row_sum_pat<T, L2>(sp.tab + p * 9, r, v);
    }

    // The threads that share the work of one phase: the whole cluster (phases
    // end with the cluster barrier; vectors are read through L2 because other
    // CTAs wrote them) or one CTA (block barrier; plain loads, coherent within
    // the CTA).
    //
    // Cluster phases may also use plain loads (PL): the cluster barrier has
    // acquire semantics, so loads after it observe every store released before
    // it by the cluster's threads, and plain loads can hit L1 (the nine gathers
    // of a row share cache lines with the neighbouring rows').
    template <bool LOCAL, bool PL = false>
    struct Team
    {
        uint32_t tid, nth;
        static constexpr bool plain = LOCAL || PL;
        __device__ __forceinline__ void sync() const
        {
            if constexpr (LOCAL) __syncthreads();
            else cg::this_cluster().sync();
        }
        template <typename T> __device__ __forceinline__ T ld(const T * p) const
        {
            if constexpr (plain) return *p;
            else return __ldcg(p);
        }
    };

    // damped Jacobi sweeps with ping-pong (math/ri.hh:110-133), result back in x
    template <typename T, bool LOCAL, bool PL>
    __device__ void sub_smooth(const SubLevel<T> & L, int sweeps, const Team<LOCAL, PL> & tm, const SubPat<T> & sp)
    {
        typedef Arith<T> M;
        T * cur = L.x, * nxt = L.tmp;
        for (int s = 0; s < sweeps; ++s)
        {
            uint32_t j = 0;
            for (uint32_t r = tm.tid; r < L.n; r += tm.nth, ++j)
            {
                const T acc = row_A<T, ! Team<LOCAL, PL>::plain>(L, sp, r, j, cur);
                nxt[r] = M::add(tm.ld(cur + r), M::mul(__ldg(L.jac + r), M::sub(tm.ld(L.b + r), acc)));
            }
            tm.sync();
            T * t = cur;
            cur = nxt;
            nxt = t;
        }
        if (cur != L.x)
        {
            for (uint32_t r = tm.tid; r < L.n; r += tm.nth) L.x[r] = tm.ld(cur + r);
            tm.sync();
        }
    }

    // pre-smoothing, defect, restriction + clear of the coarser correction
    template <typename T, bool LOCAL, bool PL>
    __device__ void down_level(const SubLevel<T> & L, const SubLevel<T> & C, int n_pre, const Team<LOCAL, PL> & tm,
                               const SubPat<T> & sp)
    {
        typedef Arith<T> M;
        sub_smooth(L, n_pre, tm, sp);
        uint32_t j = 0;
        for (uint32_t r = tm.tid; r < L.n; r += tm.nth, ++j)
            L.store[r] = M::sub(tm.ld(L.b + r), row_A<T, ! Team<LOCAL, PL>::plain>(L, sp, r, j, L.x));
        tm.sync();
        for (uint32_t r = tm.tid; r < C.n; r += tm.nth)
        {
            C.b[r] = L.q1l ? q1_restrict_row<T, ! Team<LOCAL, PL>::plain>(r, L.store, L.mf, L.mc)
                           : row_sum_any<T, ! Team<LOCAL, PL>::plain>(L.R, r, L.store);
            C.x[r] = T(0);
        }
        tm.sync();
    }

    // prolongation + add, post-smoothing
    template <typename T, bool LOCAL, bool PL>
    __device__ void up_level(const SubLevel<T> & L, const SubLevel<T> & C, int n_post, const Team<LOCAL, PL> & tm,
                             const SubPat<T> & sp)
    {
        typedef Arith<T> M;
        for (uint32_t r = tm.tid; r < L.n; r += tm.nth)
            L.x[r] = M::add(tm.ld(L.x + r), L.q1l ? q1_prolong_row<T, ! Team<LOCAL, PL>::plain>(r, C.x, L.mf, L.mc)
                                                  : row_sum_any<T, ! Team<LOCAL, PL>::plain>(L.P, r, C.x));
        tm.sync();
        sub_smooth(L, n_post, tm, sp);
    }

    // Shared memory of the split kernels: the pattern tables of every level and,
    // for the levels that run over the whole cluster, the pattern ids of the
    // rows each thread owns.  Loaded once per launch (the data are constant).
    template <typename T>
    struct SubShared
    {
        PatEnt<T> tab[kSubMaxLevels][kSubPatMax * 9];
        uint8_t ids[kSubMaxLevels][kSubRowsPerThread * 1024];
    };

    template <typename T>
    __device__ void sub_load_patterns(const SubCycle<T> & sc, SubShared<T> & sh, uint32_t tid, uint32_t nth)
    {
        for (int i = 1; i <= sc.top; ++i)
        {
            const SubLevel<T> & L = sc.lev[i];
            if (! L.ptab) continue;
            for (uint32_t e = threadIdx.x; e < L.npat * 9; e += blockDim.x) sh.tab[i][e] = L.ptab[e];
            if (i > sc.t1)
            {
                uint32_t j = 0;
                for (uint32_t r = tid; j < (uint32_t)kSubRowsPerThread; r += nth, ++j)
                    sh.ids[i][j * 1024 + threadIdx.x] = r < L.n ? __ldg(L.pat + r) : (uint8_t)0;
            }
        }
        __syncthreads();
    }

    template <typename T>
    __device__ __forceinline__ SubPat<T> sub_pat(const SubCycle<T> & sc, const SubShared<T> & sh, int i, bool cluster_wide)
    {
        SubPat<T> p;
        p.tab = sc.lev[i].ptab ? sh.tab[i] : nullptr;
        p.ids = cluster_wide ? sh.ids[i] : nullptr;
        return p;
    }

    // down: levels top..t1+1 over the cluster, then levels t1..1 in CTA 0 alone
    // (the smallest levels have too few rows to need more than one CTA, and a
    // block barrier is far cheaper than a cluster barrier)
    template <typename T, bool PL>
    __global__ void __launch_bounds__(1024, 1) mg_sub_down_kernel(const __grid_constant__ SubCycle<T> sc)
    {
        __shared__ SubShared<T> sh;
        pdl_entry();
        cg::cluster_group cluster = cg::this_cluster();
        const Team<false, PL> all = {cluster.block_rank() * blockDim.x + threadIdx.x, cluster.num_blocks() * blockDim.x};
        sub_load_patterns(sc, sh, all.tid, all.nth);
        for (int i = sc.top; i > sc.t1; --i) down_level(sc.lev[i], sc.lev[i - 1], sc.n_pre, all, sub_pat(sc, sh, i, true));
        if (sc.t1 < 1 || cluster.block_rank() != 0) return;
        const Team<true> blk = {threadIdx.x, blockDim.x};
        for (int i = sc.t1; i >= 1; --i) down_level(sc.lev[i], sc.lev[i - 1], sc.n_pre, blk, sub_pat(sc, sh, i, false));
    }

    // up: levels 1..t1 in CTA 0 alone, then t1+1..top over the cluster
    template <typename T, bool PL>
    __global__ void __launch_bounds__(1024, 1) mg_sub_up_kernel(const __grid_constant__ SubCycle<T> sc)
    {
        __shared__ SubShared<T> sh;
        pdl_entry();
        cg::cluster_group cluster = cg::this_cluster();
        const Team<false, PL> all = {cluster.block_rank() * blockDim.x + threadIdx.x, cluster.num_blocks() * blockDim.x};
        sub_load_patterns(sc, sh, all.tid, all.nth);
        if (sc.t1 >= 1)
        {
            if (cluster.block_rank() == 0)
            {
                const Team<true> blk = {threadIdx.x, blockDim.x};
                for (int i = 1; i <= sc.t1; ++i) up_level(sc.lev[i], sc.lev[i - 1], sc.n_post, blk, sub_pat(sc, sh, i, false));
            }
            cluster.sync();
        }
        for (int i = sc.t1 + 1; i <= sc.top; ++i) up_level(sc.lev[i], sc.lev[i - 1], sc.n_post, all, sub_pat(sc, sh, i, true));
    }

    // ------------------------------------------------------------------
    // The whole bottom of the V-cycle in one launch: levels t1+1..top phase by
    // phase over the cluster; then CTA 0 alone runs levels t1..1 down, the
    // coarsest CG (its first warp: cg_warp.cuh) and levels 1..t1 up with block
    // barriers only, while the other CTAs wait at the cluster barrier; then the
    // cluster runs levels t1+1..top up.  A block barrier costs a small fraction
    // of a cluster barrier, and the smallest levels have too few rows to keep
    // more than one CTA busy anyway.
    template <typename T>
    struct SubVCycle
    {
        SubLevel<T> lev[kSubMaxLevels];
        int top, t1, n_pre, n_post;
        EllView<T> C;            // coarsest operator
        EllView<double> C64;     // its FP64 copy (FP32 hierarchies with an FP64 coarse solve)
        int mixed, exact;
        uint64_t max_iters;
        double eps;
        uint64_t * used;
        double * defect;
    };

    template <typename TA, typename S, typename T>
    __device__ __forceinline__ void coarse_dispatch(const EllView<TA> & A, const SubVCycle<T> & sc, TA * smem)
    {
        const SubLevel<T> & L0 = sc.lev[0];
        const S * b = (const S *)L0.b;
        S * x = (S *)L0.x;
        switch ((L0.n + 31) / 32)
        {
            case 1: cg_warp_reg<TA, S, 1>(A, b, x, sc.max_iters, sc.eps, sc.exact, sc.used, sc.defect, smem); break;
            case 2: cg_warp_reg<TA, S, 2>(A, b, x, sc.max_iters, sc.eps, sc.exact, sc.used, sc.defect, smem); break;
            default: cg_warp_reg<TA, S, 3>(A, b, x, sc.max_iters, sc.eps, sc.exact, sc.used, sc.defect, smem); break;
        }
    }

    constexpr int kSubVThreads = 512;   // 128 registers per thread: the coarse CG stays in registers

    template <typename T, bool PL>
    __global__ void __launch_bounds__(kSubVThreads, 1) mg_sub_vcycle_kernel(const __grid_constant__ SubVCycle<T> sc)
    {
        pdl_entry();
        __shared__ double cg_smem[3 * 96];
        cg::cluster_group cluster = cg::this_cluster();
        const Team<false, PL> all = {cluster.block_rank() * blockDim.x + threadIdx.x, cluster.num_blocks() * blockDim.x};
        const SubPat<T> none = {nullptr, nullptr};
        for (int i = sc.top; i > sc.t1; --i) down_level(sc.lev[i], sc.lev[i - 1], sc.n_pre, all, none);
        if (cluster.block_rank() == 0)
        {
            const Team<true> blk = {threadIdx.x, blockDim.x};
            for (int i = sc.t1; i >= 1; --i) down_level(sc.lev[i], sc.lev[i - 1], sc.n_pre, blk, none);
            if (threadIdx.x < 32)
            {
                if constexpr (std::is_same<T, float>::value)
                {
                    if (sc.mixed) coarse_dispatch<double, float>(sc.C64, sc, cg_smem);
                    else coarse_dispatch<float, float>(sc.C, sc, (float *)cg_smem);
                }
                else coarse_dispatch<double, double>(sc.C, sc, cg_smem);
            }
            __syncthreads();
            for (int i = 1; i <= sc.t1; ++i) up_level(sc.lev[i], sc.lev[i - 1], sc.n_post, blk, none);
        }
        cluster.sync();
        for (int i = sc.t1 + 1; i <= sc.top; ++i) up_level(sc.lev[i], sc.lev[i - 1], sc.n_post, all, none);
    }

    // HB2_Q1_TRANSFER=0: the fused small levels read the transfer matrices too
    static bool q1_transfer_rows_enabled()
    {
        const char * v = getenv("HB2_Q1_TRANSFER");
        return ! (v && strcmp(v, "0") == 0);
    }

    // HB2_SUB_PATTERNS=0: the fused small levels read the plain ELL arrays
    static bool sub_patterns_enabled()
    {
        static const bool on = ! (getenv("HB2_SUB_PATTERNS") && strcmp(getenv("HB2_SUB_PATTERNS"), "0") == 0);
        return on;
    }

    template <typename T>
    static SubLevel<T> sub_level(const SubLevelDesc & d)
    {
        SubLevel<T> s;
        s.A = d.A->view<T>();
        if (d.R) s.R = d.R->view<T>(); else s.R = s.A;
        if (d.P) s.P = d.P->view<T>(); else s.P = s.A;
        s.q1l = s.mf = s.mc = 0;
        if (d.R && d.P && d.P->q1_transfer > 1 && d.R->q1_transfer == -d.P->q1_transfer && q1_transfer_rows_enabled())
        {
            s.q1l = (uint32_t)d.P->q1_transfer;
            s.mf = (1u << s.q1l) + 1;
            s.mc = (1u << (s.q1l - 1)) + 1;
        }
        s.x = (T *)d.x;
        s.b = (T *)d.b;
        s.store = (T *)d.store;
        s.tmp = (T *)d.tmp;
        s.jac = (const T *)d.jac;
        s.n = (uint32_t)d.A->rows;
        const bool pat = d.A->sptab && d.A->snpat > 0 && d.A->snpat <= (uint32_t)kSubPatMax && sub_patterns_enabled();
        s.pat = pat ? d.A->spat : nullptr;
        s.ptab = pat ? (const PatEnt<T> *)d.A->sptab : nullptr;
        s.npat = pat ? d.A->snpat : 0;
        return s;
    }

    // HB2_SUB_LDCG=1: cluster phases read vectors with L2-only loads
    static bool plain_loads()
    {
        static const bool pl = ! (getenv("HB2_SUB_LDCG") && strcmp(getenv("HB2_SUB_LDCG"), "1") == 0);
        return pl;
    }

    // widest cluster (16 CTAs of 1024 threads, else 8) that can be resident,
    // per kernel, computed once outside any stream capture (subcycle_prepare)
    static int cluster_width(const void * fn, int threads = 1024)
    {
        static std::mutex mu;
        static std::map<const void *, int> widths;
        std::lock_guard<std::mutex> lock(mu);
        auto it = widths.find(fn);
        if (it != widths.end()) return it->second;
        cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        int width = 1;
        // HB2_SUB_CLUSTER=<w> caps the width (16, 8, 4, 2)
        const char * cap = getenv("HB2_SUB_CLUSTER");
        const int wmax = cap && *cap ? atoi(cap) : 16;
        for (int w : {16, 8, 4, 2})
        {
            if (w > wmax) continue;
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(w);
            cfg.blockDim = dim3(threads);
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
                break;
            }
            cudaGetLastError();
        }
        widths[fn] = width;
        return width;
    }

    template <typename K, typename P>
    static int launch_cluster(K kernel, const P & param, int w, cudaStream_t s, const char * what, int threads = 1024)
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(w);
        cfg.blockDim = dim3(threads);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cudaLaunchAttribute at[2];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = w;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = pdl_enabled() ? 2 : 1;
        cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, param);
        count_launches(1);
        if (e != cudaSuccess) return cuda_status(e, what);
        return HB2_OK;
    }

    template <typename T>
    static int launch_sub_typed(const SubLevelDesc * lev, int top, int t1, int n_pre, int n_post, bool down,
                                cudaStream_t s)
    {
        SubCycle<T> sc;
        for (int i = 0; i <= top; ++i) sc.lev[i] = sub_level<T>(lev[i]);
        sc.top = top;
        sc.t1 = t1;
        sc.n_pre = n_pre;
        sc.n_post = n_post;
        const int w = cluster_width((const void *)mg_sub_down_kernel<T, true>);
        if (plain_loads())
            return down ? launch_cluster(mg_sub_down_kernel<T, true>, sc, w, s, "cluster sub-cycle launch (down)")
                        : launch_cluster(mg_sub_up_kernel<T, true>, sc, w, s, "cluster sub-cycle launch (up)");
        return down ? launch_cluster(mg_sub_down_kernel<T, false>, sc, w, s, "cluster sub-cycle launch (down)")
                    : launch_cluster(mg_sub_up_kernel<T, false>, sc, w, s, "cluster sub-cycle launch (up)");
    }

    int launch_subcycle(int dtype, const SubLevelDesc * lev, int top, int t1, int n_pre, int n_post, bool down,
                        cudaStream_t stream)
    {
        if (top < 1 || top >= kSubMaxLevels || t1 < 0 || t1 > top) return fail(HB2_ERR_UNSUPPORTED, "sub-cycle: bad level range");
        return dtype == HB2_F64 ? launch_sub_typed<double>(lev, top, t1, n_pre, n_post, down, stream)
                                : launch_sub_typed<float>(lev, top, t1, n_pre, n_post, down, stream);
    }

    bool subvcycle_supported(const hb2_ell_s * coarse, const hb2_ell_s * coarse64)
    {
        const hb2_ell_s * C = coarse64 ? coarse64 : coarse;
        return C->K == 9 && C->rows <= 96 && C->rows > 0;   // up to 3 rows per lane in the coarse CG
    }

    template <typename T>
    static int launch_subv_typed(const SubLevelDesc * lev, int top, int t1, int n_pre, int n_post,
                                 const hb2_ell_s * coarse, const hb2_ell_s * coarse64, uint64_t max_iters, double eps,
                                 int exact, uint64_t * used, double * defect, cudaStream_t s)
    {
        SubVCycle<T> sc;
        memset(&sc, 0, sizeof(sc));
        for (int i = 0; i <= top; ++i) sc.lev[i] = sub_level<T>(lev[i]);
        sc.top = top;
        sc.t1 = t1;
        sc.n_pre = n_pre;
        sc.n_post = n_post;
        sc.C = coarse->view<T>();
        sc.mixed = coarse64 != 0;
        if (coarse64) sc.C64 = coarse64->view<double>();
        sc.exact = exact;
        sc.max_iters = max_iters;
        sc.eps = eps;
        sc.used = used;
        sc.defect = defect;
        const int w = top > t1 ? cluster_width((const void *)mg_sub_vcycle_kernel<T, true>, kSubVThreads) : 1;
        if (plain_loads())
            return launch_cluster(mg_sub_vcycle_kernel<T, true>, sc, w, s, "fused small-level V-cycle launch", kSubVThreads);
        return launch_cluster(mg_sub_vcycle_kernel<T, false>, sc, w, s, "fused small-level V-cycle launch", kSubVThreads);
    }

    int launch_subvcycle(int dtype, const SubLevelDesc * lev, int top, int t1, int n_pre, int n_post,
                         const hb2_ell_s * coarse, const hb2_ell_s * coarse64, uint64_t max_iters, double eps, int exact,
                         uint64_t * used, double * defect, cudaStream_t stream)
    {
        if (top < 1 || top >= kSubMaxLevels || t1 < 0 || t1 > top || ! subvcycle_supported(coarse, coarse64))
            return fail(HB2_ERR_UNSUPPORTED, "fused small-level V-cycle: bad level range or coarse operator");
        if (coarse64 && dtype != HB2_F32) return fail(HB2_ERR_ARG, "fused small-level V-cycle: FP64 coarse copy of an FP64 level");
        return dtype == HB2_F64 ? launch_subv_typed<double>(lev, top, t1, n_pre, n_post, coarse, coarse64, max_iters, eps,
                                                           exact, used, defect, stream)
                                : launch_subv_typed<float>(lev, top, t1, n_pre, n_post, coarse, coarse64, max_iters, eps,
                                                          exact, used, defect, stream);
    }

    // prime the cluster attributes and widths outside any stream capture
    int subcycle_prepare()
    {
        plain_loads();
        for (bool pl : {false, true})
        {
            cluster_width(pl ? (const void *)mg_sub_down_kernel<double, true> : (const void *)mg_sub_down_kernel<double, false>);
            cluster_width(pl ? (const void *)mg_sub_down_kernel<float, true> : (const void *)mg_sub_down_kernel<float, false>);
            cluster_width(pl ? (const void *)mg_sub_up_kernel<double, true> : (const void *)mg_sub_up_kernel<double, false>);
            cluster_width(pl ? (const void *)mg_sub_up_kernel<float, true> : (const void *)mg_sub_up_kernel<float, false>);
            cluster_width(pl ? (const void *)mg_sub_vcycle_kernel<double, true> : (const void *)mg_sub_vcycle_kernel<double, false>,
                          kSubVThreads);
            cluster_width(pl ? (const void *)mg_sub_vcycle_kernel<float, true> : (const void *)mg_sub_vcycle_kernel<float, false>,
                          kSubVThreads);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_status(e, "sub-cycle attributes");
        return HB2_OK;
    }
}
