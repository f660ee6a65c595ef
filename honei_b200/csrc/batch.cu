// Batched solves: many Q1 Poisson systems of different sizes, each with one or
// more right-hand sides, solved together by MG-preconditioned CG
// (CGSolver<Tag, methods::VAR>, math/cg.hh:142-210) in mixed precision.
//
// Vectors.  Every right-hand side is one "vector" j.  Vectors are numbered by
// finest level, largest first, so the vectors that own a level-l copy (finest
// level >= l) are a prefix 0 .. nv(l)-1 of the numbering.  All systems at level
// l share one operator, so each stage of the V-cycle -- one Jacobi sweep on
// level l, one restriction, ... -- is ONE launch over the (row block, vector)
// pairs of every vector that is at that level at that moment, whatever its
// finest level: the systems whose finest level is l start their cycle there
// while the larger systems pass through on their way down.  One PCG step of
// the whole batch is therefore a fixed sequence of launches whose length is set
// by the deepest hierarchy, not by the number of systems.
//
// Precision.  The outer CG recurrence (x, r, p, v, the dots and norms, the stop
// test) is FP64 on the FP64 operator.  The preconditioner z = M r is one
// V-cycle (Jacobi omega, n_pre / n_post sweeps, bilinear transfers) on FP32
// operators and vectors, with the coarsest-level CG in FP64 arithmetic.
//
// Work lists.  Each step starts with a one-block kernel that lists the vectors
// with work (ascending, so each group's -- each finest level's -- vectors form
// one segment), and the stop test ends with one that lists the vectors the
// preconditioner runs for, with the number of them present on each level (a
// prefix of the list).  Every other kernel of the step is a persistent grid
// walking the (vector, row block) items of a list, so a step costs what its
// live vectors need, not what the batch could hold.  Each vector's fused dot /
// norm is reduced over its own row blocks in a fixed order: a vector's iterates
// do not depend on which other systems share the batch or when they started.
//
// Per-vector state machine: kNew (start requested) -> first step computes
// r = b - A x and ||r0||; kRun -> each step updates x, r and tests
// ||r|| < eps ||r0|| or ||r|| < eps or max_iters; then kDone.  New systems can
// be started between steps while others are in flight: that is how the
// serving loop interleaves requests.
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <numeric>
#include <vector>

namespace hb2
{
    enum SlotState : uint8_t
    {
        kIdle = 0,
        kNew = 1,
        kRun = 2,
        kDone = 3
    };

    constexpr int kMaxGroups = 14;
    constexpr int kOuterThreads = 256;
    constexpr int kOuterRows = 2;   // rows per thread: one 128-bit load of FP64 values per slot

    constexpr int kMaxLevels = 16;

    // Work lists of one step, built on the device (one block): the ascending
    // list of vectors with work, with each group's segment of it (a group's
    // vectors are consecutive, so its listed vectors are too) and the first
    // work item (vector x row block) of each group; for the V-cycle, the number
    // of listed vectors present on each level (a prefix of the list).
    struct Plan
    {
        uint32_t live_start[kMaxGroups], live_n[kMaxGroups], live_item0[kMaxGroups + 1];
        uint32_t prec_start[kMaxGroups], prec_n[kMaxGroups], prec_item0[kMaxGroups + 1];
        uint32_t vcount[kMaxLevels];
        uint32_t nactive;
    };

    // per-vector device scalars and the work lists
    struct SlotScalars
    {
        double * red_a;     // phase A: ||r0||^2 (kNew) or v.p (kRun)
        double * red_u;     // update: ||r||^2
        double * red_z;     // preconditioner: r.z
        double * d0;        // ||r0||
        double * cur;       // ||r||
        double * an;        // alpha_new = r.z
        double * tco;       // alpha_new / alpha for the p update
        double * eps;       // per-vector relative tolerance
        uint32_t * iters;
        uint8_t * state;
        uint8_t * fresh;    // first preconditioner application of this vector
        uint8_t * prec;     // preconditioner runs for this vector in this step
        uint32_t * live;    // list: vectors in kNew / kRun at the start of the step
        uint32_t * plist;   // list: vectors the preconditioner runs for
        Plan * plan;
        uint64_t * steps;
    };

    struct OuterGroup
    {
        EllView<double> A;            // FP64 operator of the finest level (plain layout)
        uint64_t n, vs;               // rows, stride of the FP64 vectors
        uint64_t vs32;                // stride of the level's FP32 vectors
        uint32_t first, count;        // vector range
        uint32_t gx;                  // row blocks per vector
        double * x, * b, * r, * p, * v;   // count vectors each, index j - first
        float * b32, * x32;           // the level's inner rhs / correction, index j
        double * partials, * gpart;   // reduction scratch: gx and gx/32 per vector
        unsigned * ticket;            // gx/32 + 1 per vector
    };

    struct OuterPlan
    {
        OuterGroup g[kMaxGroups];
        int ngroups;
        uint32_t nv[kMaxLevels];      // vectors present on each level (index level - coarse)
        int nlev;
    };

    __device__ __forceinline__ double guard_signed(double d)
    {
        // math/cg.hh:173 and :203: |d| > eps ? d : eps * sign(d)
        return fabs(d) > DBL_EPSILON ? d : __dmul_rn(DBL_EPSILON, __ddiv_rn(d, fabs(d)));
    }

    // acc[i] = sum_k A(r0 + i, k) * x(col), slot order, separately rounded
    // (la/product.hh:148-206)
    template <int KT>
    __device__ __forceinline__ void rows_product(const EllView<double> & A, uint64_t r0, const double * x,
                                                 double (&acc)[kOuterRows])
    {
        acc[0] = acc[1] = 0.0;
        if (r0 >= A.rows) return;
        const int K = KT > 0 ? KT : (int)A.K;
        if constexpr (KT > 0)
        {
            double2 v[KT];
            int2 c[KT];
#pragma unroll
            for (int k = 0; k < KT; ++k)
            {
                v[k] = __ldg((const double2 *)(A.val + (uint64_t)k * A.ld + r0));
                c[k] = __ldg((const int2 *)(A.col + (uint64_t)k * A.ld + r0));
            }
#pragma unroll
            for (int k = 0; k < KT; ++k)
            {
                if (c[k].x >= 0) acc[0] = __dadd_rn(acc[0], __dmul_rn(v[k].x, __ldg(x + c[k].x)));
                if (c[k].y >= 0) acc[1] = __dadd_rn(acc[1], __dmul_rn(v[k].y, __ldg(x + c[k].y)));
            }
        }
        else
        {
            for (int k = 0; k < K; ++k)
            {
                const double2 vv = __ldg((const double2 *)(A.val + (uint64_t)k * A.ld + r0));
                const int2 cc = __ldg((const int2 *)(A.col + (uint64_t)k * A.ld + r0));
                if (cc.x >= 0) acc[0] = __dadd_rn(acc[0], __dmul_rn(vv.x, __ldg(x + cc.x)));
                if (cc.y >= 0) acc[1] = __dadd_rn(acc[1], __dmul_rn(vv.y, __ldg(x + cc.y)));
            }
        }
    }

    template <typename F>
    __device__ __forceinline__ void finish(const OuterGroup & G, uint32_t lj, uint32_t blk, double part, double * out,
                                           F && on_total)
    {
        __shared__ double scratch[32];
        const double s = block_sum(part, scratch);
        const unsigned ngr = (G.gx + kReduceGroup - 1) / kReduceGroup;
        if (sum_finish(s, G.partials + (uint64_t)lj * G.gx, G.gpart + (uint64_t)lj * ngr,
                       G.ticket + (uint64_t)lj * (ngr + 1), G.gx, blk, out, 0, scratch) && threadIdx.x == 0)
            on_total();
    }

    // Persistent walk over the work items (vector x row block) of one list:
    // body(G, j, lj, blk) for every item, the items of one block in turn.
    template <typename F>
    __device__ __forceinline__ void walk(const OuterPlan & P, const uint32_t * list, const uint32_t * start,
                                         const uint32_t * item0, F && body)
    {
        __shared__ uint32_t s_item0[kMaxGroups + 1], s_start[kMaxGroups];
        pdl_entry();
        if (threadIdx.x <= (unsigned)P.ngroups) s_item0[threadIdx.x] = item0[threadIdx.x];
        if (threadIdx.x < (unsigned)P.ngroups) s_start[threadIdx.x] = start[threadIdx.x];
        __syncthreads();
        const uint32_t total = s_item0[P.ngroups];
        for (uint32_t item = blockIdx.x; item < total; item += gridDim.x)
        {
            int g = 0;
            while (g + 1 < P.ngroups && item >= s_item0[g + 1]) ++g;
            const OuterGroup & G = P.g[g];
            const uint32_t local = item - s_item0[g];
            const uint32_t j = list[s_start[g] + local / G.gx];
            body(G, j, j - G.first, local % G.gx);
        }
    }

    // Phase A.  kNew: r = b - A x (math/cg.hh:161), ||r||^2; kRun: v = A p,
    // v.p (cg.hh:174-175).  Either way the inner rhs of the finest level gets
    // (float) r and the inner correction 0, ready for the preconditioner.
    template <int KT>
    __global__ void __launch_bounds__(kOuterThreads) bpcg_phase_a_kernel(const __grid_constant__ OuterPlan P, SlotScalars S)
    {
        walk(P, S.live, S.plan->live_start, S.plan->live_item0, [&](const OuterGroup & G, uint32_t j, uint32_t lj, uint32_t blk) {
            const bool init = S.state[j] == kNew;
            const uint64_t o = (uint64_t)lj * G.vs, o32 = (uint64_t)j * G.vs32;
            const uint64_t r0 = ((uint64_t)blk * kOuterThreads + threadIdx.x) * kOuterRows;
            double acc[kOuterRows];
            rows_product<KT>(G.A, r0, (init ? G.x : G.p) + o, acc);
            double part = 0.0;
#pragma unroll
            for (int i = 0; i < kOuterRows; ++i)
            {
                const uint64_t row = r0 + i;
                if (row >= G.n) break;
                if (init)
                {
                    const double d = __dsub_rn(G.b[o + row], acc[i]);
                    G.r[o + row] = d;
                    G.b32[o32 + row] = __double2float_rn(d);
                    G.x32[o32 + row] = 0.f;
                    part = fma(d, d, part);
                }
                else
                {
                    G.v[o + row] = acc[i];
                    part = fma(acc[i], G.p[o + row], part);
                }
            }
            finish(G, lj, blk, part, S.red_a + j, [] {});
        });
    }

    // kRun: lambda = alpha_new / temp; x += lambda p; r -= lambda v; ||r||^2
    // (math/cg.hh:173-183); the inner rhs gets (float) r.
    __global__ void __launch_bounds__(kOuterThreads) bpcg_update_kernel(const __grid_constant__ OuterPlan P, SlotScalars S)
    {
        walk(P, S.live, S.plan->live_start, S.plan->live_item0, [&](const OuterGroup & G, uint32_t j, uint32_t lj, uint32_t blk) {
            if (S.state[j] != kRun) return;
            const double lambda = __ddiv_rn(S.an[j], guard_signed(S.red_a[j]));
            const double mlambda = -lambda;
            const uint64_t o = (uint64_t)lj * G.vs, o32 = (uint64_t)j * G.vs32;
            const uint64_t r0 = ((uint64_t)blk * kOuterThreads + threadIdx.x) * kOuterRows;
            double part = 0.0;
#pragma unroll
            for (int i = 0; i < kOuterRows; ++i)
            {
                const uint64_t row = r0 + i;
                if (row >= G.n) break;
                G.x[o + row] = __dadd_rn(G.x[o + row], __dmul_rn(lambda, G.p[o + row]));
                const double rr = __dadd_rn(G.r[o + row], __dmul_rn(mlambda, G.v[o + row]));
                G.r[o + row] = rr;
                G.b32[o32 + row] = __double2float_rn(rr);
                G.x32[o32 + row] = 0.f;
                part = fma(rr, rr, part);
            }
            finish(G, lj, blk, part, S.red_u + j, [] {});
        });
    }

    // one block: ascending list of the j < n with flag(j); returns the count
    template <typename F>
    __device__ uint32_t block_compact(uint32_t n, F && flag, uint32_t * list)
    {
        __shared__ uint32_t wsum[32];
        __shared__ uint32_t total;
        const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
        const uint32_t lo = min(n, threadIdx.x * per), hi = min(n, lo + per);
        uint32_t c = 0;
        for (uint32_t j = lo; j < hi; ++j) c += flag(j) ? 1u : 0u;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        uint32_t incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        if (warp == 0)
        {
            const int nw = (blockDim.x + 31) >> 5;
            uint32_t w = lane < nw ? wsum[lane] : 0u, wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1)
            {
                const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += t;
            }
            if (lane < nw) wsum[lane] = wi - w;   // exclusive prefix of the warps
            if (lane == 31) total = wi;
        }
        __syncthreads();
        uint32_t pos = wsum[warp] + incl - c;
        for (uint32_t j = lo; j < hi; ++j)
            if (flag(j)) list[pos++] = j;
        __syncthreads();
        return total;
    }

    __device__ __forceinline__ uint32_t lower_bound(const uint32_t * list, uint32_t n, uint32_t v)
    {
        uint32_t lo = 0, hi = n;
        while (lo < hi)
        {
            const uint32_t mid = (lo + hi) >> 1;
            if (list[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    }

    // group segments and item offsets of a list
    __device__ void segments(const OuterPlan & P, const uint32_t * list, uint32_t n, uint32_t * start, uint32_t * cnt,
                             uint32_t * item0)
    {
        if (threadIdx.x == 0)
        {
            uint32_t items = 0;
            for (int g = 0; g < P.ngroups; ++g)
            {
                const uint32_t a = lower_bound(list, n, P.g[g].first);
                const uint32_t b = lower_bound(list, n, P.g[g].first + P.g[g].count);
                start[g] = a;
                cnt[g] = b - a;
                item0[g] = items;
                items += (b - a) * P.g[g].gx;
            }
            item0[P.ngroups] = items;
        }
        __syncthreads();
    }

    // start of a step: the vectors with work (kNew, kRun)
    __global__ void __launch_bounds__(1024) bpcg_plan_kernel(const __grid_constant__ OuterPlan P, SlotScalars S, uint32_t nvec)
    {
        pdl_entry();
        const uint32_t n = block_compact(nvec, [&](uint32_t j) { const uint8_t st = S.state[j]; return st == kNew || st == kRun; },
                                         S.live);
        segments(P, S.live, n, S.plan->live_start, S.plan->live_n, S.plan->live_item0);
    }

    // Stop tests (math/cg.hh:185-200), then the preconditioner's work list.
    __global__ void __launch_bounds__(1024) bpcg_decide_kernel(const __grid_constant__ OuterPlan P, SlotScalars S,
                                                               uint32_t nvec, uint64_t max_iters)
    {
        pdl_entry();
        for (uint32_t j = threadIdx.x; j < nvec; j += blockDim.x)
        {
            const uint8_t st = S.state[j];
            uint8_t prec = 0;
            if (st == kNew)
            {
                const double d0 = sqrt(S.red_a[j]);
                S.d0[j] = d0;
                S.cur[j] = d0;
                S.iters[j] = 0;
                // a zero right-hand side is solved by x = 0 as it stands (the
                // reference would divide 0 by 0 here); so is max_iters = 0
                if (! (d0 > 0.0) || max_iters == 0) S.state[j] = kDone;
                else
                {
                    S.state[j] = kRun;
                    S.fresh[j] = 1;
                    prec = 1;
                }
            }
            else if (st == kRun)
            {
                const uint32_t it = S.iters[j] + 1;
                S.iters[j] = it;
                const double cur = sqrt(S.red_u[j]);
                S.cur[j] = cur;
                const double eps = S.eps[j];
                if (cur < __dmul_rn(eps, S.d0[j]) || cur < eps || it >= max_iters || ! (cur == cur)) S.state[j] = kDone;
                else
                {
                    S.fresh[j] = 0;
                    prec = 1;
                }
            }
            S.prec[j] = prec;
        }
        __syncthreads();
        const uint32_t n = block_compact(nvec, [&](uint32_t j) { return S.prec[j] != 0; }, S.plist);
        segments(P, S.plist, n, S.plan->prec_start, S.plan->prec_n, S.plan->prec_item0);
        if (threadIdx.x < (unsigned)P.nlev) S.plan->vcount[threadIdx.x] = lower_bound(S.plist, n, P.nv[threadIdx.x]);
        if (threadIdx.x == 0) S.plan->nactive = n;
    }

    // alpha_new = r.z with z = (double) inner correction (cg.hh:202-204)
    __global__ void __launch_bounds__(kOuterThreads) bpcg_dot_z_kernel(const __grid_constant__ OuterPlan P, SlotScalars S)
    {
        walk(P, S.plist, S.plan->prec_start, S.plan->prec_item0, [&](const OuterGroup & G, uint32_t j, uint32_t lj, uint32_t blk) {
            const uint64_t o = (uint64_t)lj * G.vs, o32 = (uint64_t)j * G.vs32;
            const uint64_t r0 = ((uint64_t)blk * kOuterThreads + threadIdx.x) * kOuterRows;
            double part = 0.0;
#pragma unroll
            for (int i = 0; i < kOuterRows; ++i)
            {
                const uint64_t row = r0 + i;
                if (row >= G.n) break;
                part = fma(G.r[o + row], (double)G.x32[o32 + row], part);
            }
            finish(G, lj, blk, part, S.red_z + j, [&] {
                const double an_new = S.red_z[j];
                const double an_old = S.an[j];
                S.tco[j] = S.fresh[j] ? 0.0 : __ddiv_rn(an_new, guard_signed(an_old));
                S.an[j] = an_new;
            });
        });
    }

    // p = z (first application, cg.hh:163) or p = talpha p + z (cg.hh:205-207)
    __global__ void __launch_bounds__(kOuterThreads) bpcg_p_kernel(const __grid_constant__ OuterPlan P, SlotScalars S)
    {
        walk(P, S.plist, S.plan->prec_start, S.plan->prec_item0, [&](const OuterGroup & G, uint32_t j, uint32_t lj, uint32_t blk) {
            const bool fresh = S.fresh[j] != 0;
            const double t = S.tco[j];
            const uint64_t o = (uint64_t)lj * G.vs, o32 = (uint64_t)j * G.vs32;
            const uint64_t r0 = ((uint64_t)blk * kOuterThreads + threadIdx.x) * kOuterRows;
#pragma unroll
            for (int i = 0; i < kOuterRows; ++i)
            {
                const uint64_t row = r0 + i;
                if (row >= G.n) break;
                const double z = (double)G.x32[o32 + row];
                G.p[o + row] = fresh ? z : __dadd_rn(__dmul_rn(G.p[o + row], t), z);
            }
        });
    }

    __global__ void bpcg_start_kernel(SlotScalars S, uint32_t first, uint32_t count, double eps)
    {
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= count) return;
        S.state[first + i] = kNew;
        S.eps[first + i] = eps;
        S.iters[first + i] = 0;
    }

    __global__ void bpcg_loop_init_kernel(uint64_t * steps, cudaGraphConditionalHandle h)
    {
        *steps = 0;
        cudaGraphSetConditional(h, 1u);
    }

    __global__ void bpcg_loop_decide_kernel(const Plan * plan, uint64_t * steps, uint64_t max_steps,
                                            cudaGraphConditionalHandle h)
    {
        pdl_entry();
        const uint64_t s = *steps + 1;
        *steps = s;
        cudaGraphSetConditional(h, (plan->nactive > 0 && s < max_steps) ? 1u : 0u);
    }

    __global__ void bpcg_count_step_kernel(uint64_t * steps) { *steps += 1; }

    struct BLevel
    {
        unsigned level = 0;
        hb2_ell A = 0, P = 0, R = 0;    // FP32 operator; transfers to / from the next coarser level
        uint64_t n = 0, vs = 0;
        uint32_t nv = 0;                 // vectors with a copy on this level (a prefix)
        float * x = 0, * b = 0, * store = 0, * tmp = 0, * jac = 0;
    };

    struct BGroup
    {
        unsigned level = 0;
        hb2_ell A64 = 0;
        uint32_t first = 0, count = 0, gx = 0;
        uint64_t n = 0, vs = 0;
        double * x = 0, * b = 0, * r = 0, * p = 0, * v = 0;
    };
}

struct hb2_batch_s
{
    int device = 0;
    hb2_batch_params prm;
    unsigned coarse_level = 0, top_level = 0;
    uint32_t nsys = 0, nvec = 0;
    std::vector<unsigned> sys_level;
    std::vector<uint32_t> sys_nrhs, sys_first;
    std::vector<hb2::BLevel> lev;      // index level - coarse_level
    std::vector<hb2::BGroup> grp;
    hb2_ell coarse64 = 0;
    hb2::OuterPlan plan;
    uint64_t outer_items = 0;           // largest number of outer work items of a step
    bool outer_k9 = true;
    hb2::SlotScalars S;
    void * block = 0;                   // every device array of the batch
    uint64_t bytes = 0;
    cudaStream_t cap = 0, cap2 = 0;
    cudaGraph_t step_graph = 0, solve_graph = 0, light_graph = 0;
    cudaGraphExec_t step_exec = 0, solve_exec = 0, light_exec = 0;
    uint64_t step_kernels = 0;
    uint64_t grid_cap = 0;              // blocks of the work-list launches being recorded (0: default)
    uint64_t light_rows = 0;            // live rows up to which hb2_batch_step uses the light graph
    uint64_t started_rows = 0;          // rows of the vectors started since the last step
    std::vector<uint64_t> vec_rows;     // finest-level rows of each vector
    // pinned host mirror of the per-vector results
    uint8_t * h_state = 0;
    uint32_t * h_iters = 0;
    double * h_d0 = 0, * h_cur = 0;
    uint64_t * h_steps = 0;
    void * h_block = 0;
};

namespace hb2
{
    static uint64_t round64(uint64_t n) { return std::max<uint64_t>(64, (n + 63) / 64 * 64); }
    static uint64_t q1_rows(unsigned level) { const uint64_t m = (1ull << level) + 1; return m * m; }

    // outer kernels: a persistent grid (8 blocks of 256 threads per SM) over the work list
    static int outer_launch(hb2_batch_s * B, int which, cudaStream_t s)
    {
        const dim3 grid((unsigned)std::min<uint64_t>(B->outer_items, B->grid_cap ? B->grid_cap : list_grid_cap()));
        switch (which)
        {
            case 0:
                if (B->outer_k9) launch_pdl(bpcg_phase_a_kernel<9>, grid, dim3(kOuterThreads), 0, s, B->plan, B->S);
                else launch_pdl(bpcg_phase_a_kernel<0>, grid, dim3(kOuterThreads), 0, s, B->plan, B->S);
                break;
            case 1: launch_pdl(bpcg_update_kernel, grid, dim3(kOuterThreads), 0, s, B->plan, B->S); break;
            case 2: launch_pdl(bpcg_dot_z_kernel, grid, dim3(kOuterThreads), 0, s, B->plan, B->S); break;
            default: launch_pdl(bpcg_p_kernel, grid, dim3(kOuterThreads), 0, s, B->plan, B->S); break;
        }
        count_launches(1);
        HB2_LAUNCH_CHECK("batched PCG outer kernel");
        return HB2_OK;
    }

    static int b_smooth(hb2_batch_s * B, BLevel & L, uint64_t sweeps, cudaStream_t s)
    {
        Batch bt;
        bt.nvec = L.nv;
        bt.vstride = L.vs;
        bt.list = B->S.plist;
        bt.count = &B->S.plan->vcount[L.level - B->coarse_level];
        bt.cap = B->grid_cap;
        float * cur = L.x, * nxt = L.tmp;
        for (uint64_t k = 0; k < sweeps; ++k)
        {
            int st = launch_ell(L.A, kJacobi, cur, nxt, L.b, L.jac, 0, 0, 0, 0, s, 0, &bt);
            if (st) return st;
            std::swap(cur, nxt);
        }
        if (cur != L.x) return launch_copy(HB2_F32, L.x, cur, (uint64_t)L.nv * L.vs, s);
        return HB2_OK;
    }

    // z = M r: one V-cycle over every vector the mask selects (MGCycleCreation
    // V::STATIC order, math/mg.hh:577-640), level by level
    static int b_vcycle(hb2_batch_s * B, cudaStream_t s)
    {
        const int top = (int)B->lev.size() - 1;
        for (int i = top; i >= 1; --i)
        {
            BLevel & L = B->lev[i], & C = B->lev[i - 1];
            if (L.nv == 0) continue;
            int st = b_smooth(B, L, B->prm.n_pre_smooth, s);
            Batch bt;
            bt.nvec = L.nv;
            bt.vstride = L.vs;
            bt.list = B->S.plist;
            bt.count = &B->S.plan->vcount[i];
            bt.cap = B->grid_cap;
            if (! st) st = launch_ell(L.A, kDefect, L.x, L.store, L.b, 0, 0, 0, 0, 0, s, 0, &bt);
            Batch br = bt;
            br.vstride = C.vs;
            br.xstride = L.vs;
            br.zstride = C.vs;
            if (! st) st = launch_ell(L.R, kRestrict, L.store, C.b, 0, 0, C.x, 0, 0, 0, s, 0, &br);
            if (st) return st;
        }
        BLevel & C0 = B->lev[0];
        int st = launch_cg_warp_batched(B->coarse64, HB2_F32, C0.b, C0.x, C0.nv, C0.vs, 0,
                                        B->prm.max_iters_coarse, B->prm.coarse_eps, s, B->S.plist, &B->S.plan->vcount[0], B->grid_cap);
        if (st) return st;
        for (int i = 1; i <= top; ++i)
        {
            BLevel & L = B->lev[i], & C = B->lev[i - 1];
            if (L.nv == 0) continue;
            Batch bp;
            bp.nvec = L.nv;
            bp.vstride = L.vs;
            bp.xstride = C.vs;
            bp.list = B->S.plist;
            bp.count = &B->S.plan->vcount[i];
            bp.cap = B->grid_cap;
            st = launch_ell(L.P, kAdd, C.x, L.x, 0, 0, 0, 0, 0, 0, s, 0, &bp);
            if (! st) st = b_smooth(B, L, B->prm.n_post_smooth, s);
            if (st) return st;
        }
        return HB2_OK;
    }

    static int record_step(hb2_batch_s * B, cudaStream_t s)
    {
        launch_pdl(bpcg_plan_kernel, dim3(1), dim3(1024), 0, s, B->plan, B->S, B->nvec);
        count_launches(1);
        HB2_LAUNCH_CHECK("bpcg_plan_kernel");
        int st = outer_launch(B, 0, s);
        if (! st) st = outer_launch(B, 1, s);
        if (! st)
        {
            launch_pdl(bpcg_decide_kernel, dim3(1), dim3(1024), 0, s, B->plan, B->S, B->nvec, B->prm.max_iters);
            count_launches(1);
            HB2_LAUNCH_CHECK("bpcg_decide_kernel");
        }
        if (! st) st = b_vcycle(B, s);
        if (! st) st = outer_launch(B, 2, s);
        if (! st) st = outer_launch(B, 3, s);
        return st;
    }

    static int end_capture(cudaStream_t s, cudaGraph_t * g)
    {
        cudaGraph_t tmp = 0;
        cudaError_t e = cudaStreamEndCapture(s, &tmp);
        if (e != cudaSuccess) { if (tmp) cudaGraphDestroy(tmp); return cuda_status(e, "cudaStreamEndCapture (batch)"); }
        *g = tmp;
        return HB2_OK;
    }

    // The step graph with the work-list launches capped at `cap` blocks (0: the
    // default, 32 per SM).  A light copy with 2 blocks per SM serves steps with
    // few live vectors, where the full cap would mostly launch empty blocks.
    static int build_step_graph(hb2_batch_s * B, uint64_t cap, cudaGraph_t * graph_out, cudaGraphExec_t * exec_out)
    {
        B->grid_cap = cap;
        const uint64_t before = hb2_launch_count();
        HB2_CUDA(cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal));
        int st = record_step(B, B->cap);
        if (! st)
        {
            bpcg_count_step_kernel<<<1, 1, 0, B->cap>>>(B->S.steps);
            count_launches(1);
        }
        cudaGraph_t g = 0;
        const int st2 = end_capture(B->cap, &g);
        B->step_kernels = hb2_launch_count() - before;
        set_launch_count(before);
        B->grid_cap = 0;
        if (st) { if (g) cudaGraphDestroy(g); return st; }
        if (st2) return st2;
        *graph_out = g;
        HB2_CUDA(cudaGraphInstantiate(exec_out, g, 0));
        return HB2_OK;
    }

    static int build_solve_graph(hb2_batch_s * B)
    {
        const uint64_t before = hb2_launch_count();
        HB2_CUDA(cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal));
        cudaStreamCaptureStatus cs;
        cudaGraph_t capg = 0;
        const cudaGraphNode_t * deps = 0;
        size_t ndeps = 0;
        cudaGraph_t dummy = 0;
        cudaError_t e = cudaStreamGetCaptureInfo(B->cap, &cs, 0, &capg, &deps, &ndeps);
        cudaGraphConditionalHandle h;
        if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, capg, 1, cudaGraphCondAssignDefault);
        if (e == cudaSuccess)
        {
            bpcg_loop_init_kernel<<<1, 1, 0, B->cap>>>(B->S.steps, h);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(B->cap, &cs, 0, &capg, &deps, &ndeps);
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cudaGraphNode_t cnode;
        if (e == cudaSuccess)
        {
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            e = cudaGraphAddNode(&cnode, capg, deps, ndeps, &cp);
        }
        if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(B->cap, &cnode, 1, cudaStreamSetCaptureDependencies);
        cudaGraph_t body = e == cudaSuccess ? cp.conditional.phGraph_out[0] : 0;
        if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(B->cap2, body, 0, 0, 0, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess)
        {
            cudaStreamEndCapture(B->cap, &dummy);
            if (dummy) cudaGraphDestroy(dummy);
            return cuda_status(e, "batch solve graph");
        }
        int st = record_step(B, B->cap2);
        if (! st)
        {
            launch_pdl(bpcg_loop_decide_kernel, dim3(1), dim3(1), 0, B->cap2, B->S.plan, B->S.steps, B->prm.max_iters + 2, h);
            e = cudaGetLastError();
            if (e != cudaSuccess) st = cuda_status(e, "bpcg_loop_decide_kernel");
        }
        cudaGraph_t bodyg = 0;
        e = cudaStreamEndCapture(B->cap2, &bodyg);
        if (! st && e != cudaSuccess) st = cuda_status(e, "cudaStreamEndCapture (batch body)");
        cudaGraph_t g = 0;
        const int st2 = end_capture(B->cap, &g);
        set_launch_count(before);
        if (st) { if (g) cudaGraphDestroy(g); return st; }
        if (st2) return st2;
        B->solve_graph = g;
        HB2_CUDA(cudaGraphInstantiate(&B->solve_exec, g, 0));
        return HB2_OK;
    }

    static hb2_batch_params batch_defaults()
    {
        hb2_batch_params p;
        p.max_iters = 100;
        p.eps_relative = 1e-8;
        p.n_pre_smooth = 4;
        p.n_post_smooth = 4;
        p.max_iters_coarse = 100;
        p.coarse_eps = 1e-10;
        p.omega = 0.7;
        return p;
    }

    // copies the per-vector results into the pinned host mirror
    static int mirror(hb2_batch_s * B, cudaStream_t s)
    {
        const size_t nv = B->nvec;
        HB2_CUDA(cudaMemcpyAsync(B->h_state, B->S.state, nv, cudaMemcpyDeviceToHost, s));
        HB2_CUDA(cudaMemcpyAsync(B->h_iters, B->S.iters, nv * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        HB2_CUDA(cudaMemcpyAsync(B->h_d0, B->S.d0, nv * sizeof(double), cudaMemcpyDeviceToHost, s));
        HB2_CUDA(cudaMemcpyAsync(B->h_cur, B->S.cur, nv * sizeof(double), cudaMemcpyDeviceToHost, s));
        HB2_CUDA(cudaMemcpyAsync(B->h_steps, B->S.steps, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        return HB2_OK;
    }

    static const BGroup * group_of(const hb2_batch_s * B, uint32_t sys)
    {
        for (const BGroup & g : B->grp)
            if (g.level == B->sys_level[sys]) return &g;
        return 0;
    }

    static int start_range(hb2_batch_s * B, uint32_t first, uint32_t count, double eps, cudaStream_t s)
    {
        if (count == 0) return HB2_OK;
        bpcg_start_kernel<<<(count + 255) / 256, 256, 0, s>>>(B->S, first, count, eps > 0 ? eps : B->prm.eps_relative);
        count_launches(1);
        HB2_LAUNCH_CHECK("bpcg_start_kernel");
        return HB2_OK;
    }

    static int batch_create(hb2_batch_s * B, cudaStream_t stream)
    {
        const unsigned c = B->coarse_level, t = B->top_level;
        // vector numbering: systems by finest level, largest first, then by index
        std::vector<uint32_t> order(B->nsys);
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(),
                         [&](uint32_t a, uint32_t b) { return B->sys_level[a] > B->sys_level[b]; });
        B->sys_first.assign(B->nsys, 0);
        uint32_t next = 0;
        for (uint32_t s : order)
        {
            B->sys_first[s] = next;
            next += B->sys_nrhs[s];
        }
        B->nvec = next;
        // levels and groups
        B->lev.resize(t - c + 1);
        for (unsigned l = c; l <= t; ++l)
        {
            BLevel & L = B->lev[l - c];
            L.level = l;
            L.n = q1_rows(l);
            L.vs = round64(L.n);
            for (uint32_t s = 0; s < B->nsys; ++s)
                if (B->sys_level[s] >= l) L.nv += B->sys_nrhs[s];
        }
        for (unsigned l = t + 1; l-- > c;)
        {
            uint32_t first = UINT32_MAX, count = 0;
            for (uint32_t s = 0; s < B->nsys; ++s)
                if (B->sys_level[s] == l)
                {
                    first = std::min(first, B->sys_first[s]);
                    count += B->sys_nrhs[s];
                }
            if (! count) continue;
            BGroup g;
            g.level = l;
            g.first = first;
            g.count = count;
            g.n = q1_rows(l);
            g.vs = round64(g.n);
            g.gx = ceil_div(g.n, (uint64_t)kOuterThreads * kOuterRows);
            B->grp.push_back(g);
        }
        if (B->grp.size() > (size_t)kMaxGroups) return fail(HB2_ERR_ARG, "hb2_batch_create_q1: too many distinct levels");
        // operators
        int st = HB2_OK;
        for (size_t i = 0; i < B->lev.size() && ! st; ++i)
        {
            BLevel & L = B->lev[i];
            st = hb2_ell_create_q1(&L.A, HB2_F32, L.level, 1.0, stream);
            if (! st && i > 0) st = hb2_ell_create_transfer(&L.P, &L.R, HB2_F32, L.level, stream);
        }
        if (! st) st = hb2_ell_create_q1(&B->coarse64, HB2_F64, c, 1.0, stream);
        for (BGroup & g : B->grp)
            if (! st) st = hb2_ell_create_q1(&g.A64, HB2_F64, g.level, 1.0, stream);
        if (st) return st;
        if (! cg_mixed_supported(B->coarse64))
            return fail(HB2_ERR_UNSUPPORTED, "hb2_batch_create_q1: the coarsest level needs <= 128 rows (level <= 3)");
        // one device block: level vectors | group vectors | reduction scratch | scalars
        size_t total = 0;
        auto take = [&](size_t bytes) { size_t o = total; total += (bytes + 255) / 256 * 256; return o; };
        std::vector<size_t> lo(B->lev.size() * 5), go(B->grp.size() * 8);
        for (size_t i = 0; i < B->lev.size(); ++i)
        {
            const BLevel & L = B->lev[i];
            const size_t vb = (size_t)std::max<uint32_t>(L.nv, 1) * L.vs * sizeof(float);
            for (int k = 0; k < 4; ++k) lo[i * 5 + k] = take(vb);
            lo[i * 5 + 4] = take(L.vs * sizeof(float));
        }
        for (size_t i = 0; i < B->grp.size(); ++i)
        {
            const BGroup & g = B->grp[i];
            const size_t vb = (size_t)g.count * g.vs * sizeof(double);
            for (int k = 0; k < 5; ++k) go[i * 8 + k] = take(vb);
            const uint64_t ngr = (g.gx + kReduceGroup - 1) / kReduceGroup;
            go[i * 8 + 5] = take((size_t)g.count * g.gx * sizeof(double));
            go[i * 8 + 6] = take((size_t)g.count * ngr * sizeof(double));
            go[i * 8 + 7] = take((size_t)g.count * (ngr + 1) * sizeof(unsigned));
        }
        const size_t nv = B->nvec;
        const size_t so = take(nv * sizeof(double) * 8 + nv * sizeof(uint32_t) * 3 + nv * 3 + sizeof(Plan) + 256);
        cudaError_t e = cudaMalloc(&B->block, total);
        if (e != cudaSuccess) return cuda_status(e, "hb2_batch_create_q1: device memory");
        B->bytes = total;
        HB2_CUDA(cudaMemsetAsync(B->block, 0, total, stream));
        char * base = (char *)B->block;
        for (size_t i = 0; i < B->lev.size(); ++i)
        {
            BLevel & L = B->lev[i];
            L.x = (float *)(base + lo[i * 5 + 0]);
            L.b = (float *)(base + lo[i * 5 + 1]);
            L.store = (float *)(base + lo[i * 5 + 2]);
            L.tmp = (float *)(base + lo[i * 5 + 3]);
            L.jac = (float *)(base + lo[i * 5 + 4]);
            st = hb2_jacobi_precon(L.A, B->prm.omega, L.jac, stream);
            if (st) return st;
        }
        char * sp = base + so;
        B->S.red_a = (double *)sp; sp += nv * 8;
        B->S.red_u = (double *)sp; sp += nv * 8;
        B->S.red_z = (double *)sp; sp += nv * 8;
        B->S.d0 = (double *)sp; sp += nv * 8;
        B->S.cur = (double *)sp; sp += nv * 8;
        B->S.an = (double *)sp; sp += nv * 8;
        B->S.tco = (double *)sp; sp += nv * 8;
        B->S.eps = (double *)sp; sp += nv * 8;
        B->S.steps = (uint64_t *)sp; sp += 8;
        B->S.plan = (Plan *)sp; sp += (sizeof(Plan) + 15) / 16 * 16;
        B->S.iters = (uint32_t *)sp; sp += nv * 4;
        B->S.live = (uint32_t *)sp; sp += nv * 4;
        B->S.plist = (uint32_t *)sp; sp += nv * 4;
        B->S.state = (uint8_t *)sp; sp += nv;
        B->S.fresh = (uint8_t *)sp; sp += nv;
        B->S.prec = (uint8_t *)sp;
        // the outer work list
        memset(&B->plan, 0, sizeof(B->plan));
        B->plan.ngroups = (int)B->grp.size();
        uint64_t blocks = 0;
        B->outer_k9 = true;
        for (size_t i = 0; i < B->grp.size(); ++i)
        {
            BGroup & g = B->grp[i];
            g.x = (double *)(base + go[i * 8 + 0]);
            g.b = (double *)(base + go[i * 8 + 1]);
            g.r = (double *)(base + go[i * 8 + 2]);
            g.p = (double *)(base + go[i * 8 + 3]);
            g.v = (double *)(base + go[i * 8 + 4]);
            OuterGroup & o = B->plan.g[i];
            o.A = g.A64->view<double>();
            if (g.A64->K != 9) B->outer_k9 = false;
            o.n = g.n;
            o.vs = g.vs;
            const BLevel & L = B->lev[g.level - c];
            o.vs32 = L.vs;
            o.b32 = L.b;
            o.x32 = L.x;
            o.first = g.first;
            o.count = g.count;
            o.gx = g.gx;
            o.x = g.x;
            o.b = g.b;
            o.r = g.r;
            o.p = g.p;
            o.v = g.v;
            o.partials = (double *)(base + go[i * 8 + 5]);
            o.gpart = (double *)(base + go[i * 8 + 6]);
            o.ticket = (unsigned *)(base + go[i * 8 + 7]);
            blocks += (uint64_t)g.count * g.gx;
        }
        if (blocks > 0x7fffffffull) return fail(HB2_ERR_UNSUPPORTED, "hb2_batch_create_q1: work list too long");
        B->outer_items = blocks;
        for (size_t i = 0; i < B->lev.size(); ++i) B->plan.nv[i] = B->lev[i].nv;
        B->plan.nlev = (int)B->lev.size();
        // pinned host mirror
        const size_t hb = nv * (1 + 4 + 8 + 8) + 64;
        HB2_CUDA(cudaMallocHost(&B->h_block, hb));
        memset(B->h_block, 0, hb);
        char * hp = (char *)B->h_block;
        B->h_d0 = (double *)hp; hp += nv * 8;
        B->h_cur = (double *)hp; hp += nv * 8;
        B->h_steps = (uint64_t *)hp; hp += 8;
        B->h_iters = (uint32_t *)hp; hp += nv * 4;
        B->h_state = (uint8_t *)hp;
        HB2_CUDA(cudaStreamSynchronize(stream));
        HB2_CUDA(cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking));
        HB2_CUDA(cudaStreamCreateWithFlags(&B->cap2, cudaStreamNonBlocking));
        st = build_step_graph(B, 0, &B->step_graph, &B->step_exec);
        if (! st) st = build_step_graph(B, (uint64_t)num_sms() * 2, &B->light_graph, &B->light_exec);
        // the light graph (2 blocks per SM) serves up to about two row blocks of
        // work per block: ~150k live rows (a few systems of level 8 and below)
        B->light_rows = (uint64_t)num_sms() * 2 * kEllThreads * 2;
        B->vec_rows.assign(B->nvec, 0);
        for (uint32_t s = 0; s < B->nsys; ++s)
            for (uint32_t k = 0; k < B->sys_nrhs[s]; ++k) B->vec_rows[B->sys_first[s] + k] = q1_rows(B->sys_level[s]);
        if (! st) st = build_solve_graph(B);
        return st;
    }
}

using namespace hb2;

extern "C" int hb2_batch_create_q1(hb2_batch * out, uint32_t num_systems, const uint32_t * levels,
                                   const uint32_t * nrhs, unsigned coarse_level, const hb2_batch_params * params,
                                   cudaStream_t stream)
{
    if (! out || num_systems == 0 || ! levels) return fail(HB2_ERR_ARG, "hb2_batch_create_q1: bad argument");
    if (coarse_level < 1 || coarse_level > 3) return fail(HB2_ERR_ARG, "hb2_batch_create_q1: coarse level must be 1..3");
    uint64_t nvec = 0;
    unsigned top = coarse_level;
    for (uint32_t s = 0; s < num_systems; ++s)
    {
        if (levels[s] < coarse_level || levels[s] > 12)
            return fail(HB2_ERR_ARG, "hb2_batch_create_q1: system level outside coarse_level..12");
        const uint32_t k = nrhs ? nrhs[s] : 1;
        if (k == 0) return fail(HB2_ERR_ARG, "hb2_batch_create_q1: a system without right-hand sides");
        nvec += k;
        top = std::max(top, levels[s]);
    }
    if (nvec > 65535) return fail(HB2_ERR_UNSUPPORTED, "hb2_batch_create_q1: more than 65535 right-hand sides");
    hb2_batch_s * B = new hb2_batch_s();
    cudaGetDevice(&B->device);
    B->prm = params ? *params : batch_defaults();
    B->coarse_level = coarse_level;
    B->top_level = top;
    B->nsys = num_systems;
    B->sys_level.assign(levels, levels + num_systems);
    B->sys_nrhs.resize(num_systems);
    for (uint32_t s = 0; s < num_systems; ++s) B->sys_nrhs[s] = nrhs ? nrhs[s] : 1;
    const int st = batch_create(B, stream);
    if (st)
    {
        const std::string msg = hb2_last_error();
        hb2_batch_destroy(B);
        set_error(msg);
        return st;
    }
    *out = B;
    return HB2_OK;
}

extern "C" int hb2_batch_destroy(hb2_batch B)
{
    if (! B) return HB2_OK;
    if (B->step_exec) cudaGraphExecDestroy(B->step_exec);
    if (B->step_graph) cudaGraphDestroy(B->step_graph);
    if (B->light_exec) cudaGraphExecDestroy(B->light_exec);
    if (B->light_graph) cudaGraphDestroy(B->light_graph);
    if (B->solve_exec) cudaGraphExecDestroy(B->solve_exec);
    if (B->solve_graph) cudaGraphDestroy(B->solve_graph);
    if (B->cap) cudaStreamDestroy(B->cap);
    if (B->cap2) cudaStreamDestroy(B->cap2);
    for (BLevel & L : B->lev)
    {
        hb2_ell_destroy(L.A);
        hb2_ell_destroy(L.P);
        hb2_ell_destroy(L.R);
    }
    for (BGroup & g : B->grp) hb2_ell_destroy(g.A64);
    hb2_ell_destroy(B->coarse64);
    if (B->block) cudaFree(B->block);
    if (B->h_block) cudaFreeHost(B->h_block);
    delete B;
    return HB2_OK;
}

extern "C" int hb2_batch_info(hb2_batch B, uint32_t * num_vectors, uint64_t * device_bytes, uint64_t * launches_per_step)
{
    if (! B) return fail(HB2_ERR_ARG, "hb2_batch_info: null handle");
    if (num_vectors) *num_vectors = B->nvec;
    if (device_bytes) *device_bytes = B->bytes;
    if (launches_per_step) *launches_per_step = B->step_kernels;
    return HB2_OK;
}

extern "C" int hb2_batch_copy(hb2_batch B, uint32_t system, int which, void * buf, cudaStream_t stream)
{
    if (! B || ! buf || system >= B->nsys || which < 0 || which > 2) return fail(HB2_ERR_ARG, "hb2_batch_copy: bad argument");
    const BGroup * g = group_of(B, system);
    const size_t row = g->n * sizeof(double), pitch = g->vs * sizeof(double);
    double * dev = (which == 0 ? g->b : g->x) + (uint64_t)(B->sys_first[system] - g->first) * g->vs;
    cudaError_t e = which == 2 ? cudaMemcpy2DAsync(buf, row, dev, pitch, row, B->sys_nrhs[system], cudaMemcpyDefault, stream)
                               : cudaMemcpy2DAsync(dev, pitch, buf, row, row, B->sys_nrhs[system], cudaMemcpyDefault, stream);
    if (e != cudaSuccess) return cuda_status(e, "hb2_batch_copy");
    return HB2_OK;
}

extern "C" int hb2_batch_start(hb2_batch B, uint32_t system, double eps_relative, int zero_guess, cudaStream_t stream)
{
    if (! B || system >= B->nsys) return fail(HB2_ERR_ARG, "hb2_batch_start: bad argument");
    const BGroup * g = group_of(B, system);
    if (zero_guess)
        HB2_CUDA(cudaMemsetAsync(g->x + (uint64_t)(B->sys_first[system] - g->first) * g->vs, 0,
                                 (size_t)B->sys_nrhs[system] * g->vs * sizeof(double), stream));
    B->started_rows += (uint64_t)B->sys_nrhs[system] * q1_rows(B->sys_level[system]);
    return start_range(B, B->sys_first[system], B->sys_nrhs[system], eps_relative, stream);
}

extern "C" int hb2_batch_step(hb2_batch B, uint32_t steps, uint8_t * done, cudaStream_t stream)
{
    if (! B) return fail(HB2_ERR_ARG, "hb2_batch_step: null handle");
    // little work in flight (rows of the live vectors as of the last step, plus
    // those started since): the light graph
    uint64_t rows = B->started_rows;
    for (uint32_t j = 0; j < B->nvec; ++j)
        if (B->h_state[j] == kNew || B->h_state[j] == kRun) rows += B->vec_rows[j];
    cudaGraphExec_t exec = rows <= B->light_rows ? B->light_exec : B->step_exec;
    for (uint32_t i = 0; i < steps; ++i)
    {
        HB2_CUDA(cudaGraphLaunch(exec, stream));
        count_launches(B->step_kernels);
    }
    B->started_rows = 0;
    int st = mirror(B, stream);
    if (st) return st;
    HB2_CUDA(cudaStreamSynchronize(stream));
    if (done)
        for (uint32_t s = 0; s < B->nsys; ++s)
        {
            uint8_t d = 1;
            for (uint32_t k = 0; k < B->sys_nrhs[s]; ++k)
            {
                const uint8_t state = B->h_state[B->sys_first[s] + k];
                if (state == kNew || state == kRun) d = 0;
            }
            done[s] = d;
        }
    return HB2_OK;
}

extern "C" int hb2_batch_solve(hb2_batch B, int zero_guess, uint64_t * steps, cudaStream_t stream)
{
    if (! B) return fail(HB2_ERR_ARG, "hb2_batch_solve: null handle");
    if (zero_guess)
        for (const BGroup & g : B->grp)
            HB2_CUDA(cudaMemsetAsync(g.x, 0, (size_t)g.count * g.vs * sizeof(double), stream));
    int st = start_range(B, 0, B->nvec, 0.0, stream);
    if (st) return st;
    HB2_CUDA(cudaGraphLaunch(B->solve_exec, stream));
    st = mirror(B, stream);
    if (st) return st;
    HB2_CUDA(cudaStreamSynchronize(stream));
    const uint64_t used = *B->h_steps;
    count_launches(1 + used * (B->step_kernels));   // the loop kernels replace the step counter
    if (steps) *steps = used;
    for (uint32_t j = 0; j < B->nvec; ++j)
        if (! (B->h_cur[j] == B->h_cur[j])) return fail(HB2_ERR_NOT_FINITE, "hb2_batch_solve: NaN defect norm");
    return HB2_OK;
}

extern "C" int hb2_batch_result(hb2_batch B, uint32_t system, uint32_t rhs, uint64_t * iters, double * rel_defect)
{
    if (! B || system >= B->nsys || rhs >= B->sys_nrhs[system]) return fail(HB2_ERR_ARG, "hb2_batch_result: bad argument");
    const uint32_t j = B->sys_first[system] + rhs;
    if (iters) *iters = B->h_iters[j];
    if (rel_defect) *rel_defect = B->h_d0[j] > 0 ? B->h_cur[j] / B->h_d0[j] : 0.0;
    return HB2_OK;
}
