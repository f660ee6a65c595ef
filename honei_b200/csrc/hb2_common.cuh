// Common device/host helpers for the B200 backend of the HONEI sparse solver path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/honei_b200.h"

namespace hb2
{
    // Status plumbing: every C-ABI entry point returns an int status; the message
    // of the last failure on this host thread is kept for hb2_last_error().
    void set_error(const std::string & msg);
    int fail(int status, const std::string & msg);
    int cuda_status(cudaError_t e, const char * where);

#define HB2_CUDA(call)                                                       \
    do {                                                                     \
        cudaError_t e_ = (call);                                             \
        if (e_ != cudaSuccess) return ::hb2::cuda_status(e_, #call);         \
    } while (0)

#define HB2_LAUNCH_CHECK(where)                                              \
    do {                                                                     \
        cudaError_t e_ = cudaGetLastError();                                 \
        if (e_ != cudaSuccess) return ::hb2::cuda_status(e_, where);         \
    } while (0)

    inline size_t dtype_size(int dt) { return dt == HB2_F64 ? 8 : 4; }

    // ------------------------------------------------------------------
    // Arithmetic with explicit rounding.  The reference's compiled CPU loops
    // round a*b and then the sum separately (no fma) in the ELL and banded
    // products and the element-wise updates, and contract to fma in the dot
    // product and the CSR product; the kernels reproduce each exactly so
    // results are bit-identical.
    template <typename T> struct Arith;
    template <> struct Arith<double>
    {
        static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
        static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
        static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
        static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
        static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    };
    template <> struct Arith<float>
    {
        static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
        static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
        static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
        static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
        static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    };

    // ------------------------------------------------------------------
    // Programmatic dependent launch.  A kernel launched with
    // cudaLaunchAttributeProgrammaticStreamSerialization (launch_pdl) may be
    // scheduled while its predecessor in the stream is still finishing; it
    // waits here until the predecessor has completed and its writes are
    // visible, then lets its own successor start launching.  Without the
    // attribute both instructions return at once.  Every kernel launched with
    // the attribute calls this before it reads anything a predecessor wrote.
    __device__ __forceinline__ void pdl_entry()
    {
        asm volatile("griddepcontrol.wait;" ::: "memory");
        asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    }

    // ------------------------------------------------------------------
    // Deterministic reductions.  A block reduces its threads' partials with a
    // fixed shuffle tree, writes one partial per block, and the last block to
    // finish (ticket counter) reduces the partials in a fixed order.  The result
    // depends only on the data and the launch shape, never on timing.
    __device__ __forceinline__ double warp_sum(double v)
    {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        return v;
    }

    // block-wide sum; every thread gets the result.  scratch: >= 32 doubles.
    __device__ __forceinline__ double block_sum(double v, double * scratch)
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
        v = warp_sum(v);
        __syncthreads();
        if (lane == 0) scratch[warp] = v;
        __syncthreads();
        double t = (threadIdx.x < nwarps) ? scratch[threadIdx.x] : 0.0;
        if (warp == 0) t = warp_sum(t);
        if (threadIdx.x == 0) scratch[0] = t;
        __syncthreads();
        double r = scratch[0];
        __syncthreads();
        return r;
    }

    // Workspace used by the fused reductions of one stream: block partials,
    // group partials and ticket counters.
    struct ReduceSlot
    {
        double * partials;      // >= blocks * vectors
        double * gpart;         // >= groups * vectors
        unsigned * ticket;      // >= (groups + 1) * vectors, zero between launches
        uint32_t max_blocks;
    };

    constexpr unsigned kReduceGroup = 32;

    // Called by every block after it computed `v` (valid in all threads).  Two
    // levels: the last block of each group of kReduceGroup blocks sums the
    // group's partials, the last group sums the group partials -- each in a
    // fixed order, so the result depends only on the data and the launch
    // shape, and no counter takes more than kReduceGroup atomics.  Vector
    // blockIdx.y of a batched launch uses its own partials and counters.  The
    // finishing block writes *out (sqrt when asked) and re-arms the counters.
    //
    // sum_finish is the same reduction over G blocks of one vector whose block
    // index `blk` (0..G-1) and scratch (partials: G doubles, gpart: groups
    // doubles, ticket: groups + 1 counters) the caller chose, for launches that
    // map blocks to vectors through a work list.
    __device__ __forceinline__ bool sum_finish(double v, double * partials, double * gpart, unsigned * ticket,
                                               unsigned G, unsigned blk, double * out, int want_sqrt, double * scratch)
    {
        __shared__ int stage;
        const unsigned ngroups = (G + kReduceGroup - 1) / kReduceGroup;
        const unsigned group = blk / kReduceGroup;
        const unsigned gsize = min(kReduceGroup, G - group * kReduceGroup);
        if (threadIdx.x == 0)
        {
            partials[blk] = v;
            __threadfence();
            const unsigned t = atomicAdd(ticket + 1 + group, 1u);
            stage = (t == gsize - 1);
        }
        __syncthreads();
        if (! stage) return false;
        __threadfence();
        double s = threadIdx.x < gsize ? ((volatile double *)partials)[group * kReduceGroup + threadIdx.x] : 0.0;
        s = block_sum(s, scratch);
        if (threadIdx.x == 0)
        {
            gpart[group] = s;
            ticket[1 + group] = 0;
            __threadfence();
            const unsigned t = atomicAdd(ticket, 1u);
            stage = (t == ngroups - 1);
        }
        __syncthreads();
        if (! stage) return false;
        __threadfence();
        s = 0.0;
        for (unsigned i = threadIdx.x; i < ngroups; i += blockDim.x) s += ((volatile double *)gpart)[i];
        s = block_sum(s, scratch);
        if (threadIdx.x == 0)
        {
            out[0] = want_sqrt ? sqrt(s) : s;
            ticket[0] = 0;
        }
        return true;
    }

    __device__ __forceinline__ bool grid_sum_finish(double v, ReduceSlot rs, double * out, int want_sqrt,
            double * scratch)
    {
        const unsigned G = gridDim.x, ngroups = (G + kReduceGroup - 1) / kReduceGroup;
        return sum_finish(v, rs.partials + (uint64_t)blockIdx.y * G, rs.gpart + (uint64_t)blockIdx.y * ngroups,
                          rs.ticket + (uint64_t)blockIdx.y * (ngroups + 1), G, blockIdx.x, out, want_sqrt, scratch);
    }

    // ------------------------------------------------------------------
    // Grid-wide barrier for cooperative (co-resident) launches, with a bounded
    // wait: after `limit_ns` of spinning it records an error and returns false
    // instead of hanging.  count/gen live in device memory, zero-initialised.
    struct GridBarrier
    {
        unsigned * count;
        unsigned * gen;
        int * error;
    };

    __device__ __forceinline__ unsigned long long global_ns()
    {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        return t;
    }

    __device__ __forceinline__ bool grid_sync(GridBarrier b, unsigned long long limit_ns = 2000000000ull)
    {
        __shared__ int ok;
        __syncthreads();
        if (threadIdx.x == 0)
        {
            ok = 1;
            volatile unsigned * vgen = b.gen;
            unsigned g = *vgen;
            __threadfence();
            unsigned arrived = atomicAdd(b.count, 1u);
            if (arrived == gridDim.x - 1)
            {
                *b.count = 0;
                __threadfence();
                atomicAdd(b.gen, 1u);
            }
            else
            {
                unsigned long long t0 = global_ns();
                while (*vgen == g)
                {
                    if (*((volatile int *)b.error) != 0) { ok = 0; break; }
                    if (global_ns() - t0 > limit_ns)
                    {
                        atomicExch(b.error, 1);
                        ok = 0;
                        break;
                    }
                    __nanosleep(20);
                }
            }
            __threadfence();
        }
        __syncthreads();
        return ok != 0;
    }

    // ------------------------------------------------------------------
    // device workspace: reduction slots, barrier words, scalar slots.
    struct Workspace
    {
        int device;
        double * partials;       // max_blocks doubles
        double * gpart;          // max_blocks / kReduceGroup + 4096 doubles
        unsigned * ticket;       // max_tickets
        unsigned * bar_words;    // 2 (count, gen)
        int * error;             // 1
        double * scalars;        // 64 doubles of solver scalars
        uint32_t max_blocks;
        uint32_t max_tickets;
        double * host_scalars;   // pinned, 64 doubles
        ReduceSlot slot() const
        {
            ReduceSlot r;
            r.partials = partials;
            r.gpart = gpart;
            r.ticket = ticket;
            r.max_blocks = max_blocks;
            return r;
        }
        GridBarrier barrier() const { GridBarrier g; g.count = bar_words; g.gen = bar_words + 1; g.error = error; return g; }
    };

    // Per-device default workspace, created on first use (cudaMalloc) and kept
    // until process exit.  Not thread-safe across concurrent streams: calls
    // that use the default workspace must be stream-ordered.
    int default_workspace(Workspace ** out);
    int workspace_create(Workspace ** out, uint32_t max_blocks);
    void workspace_destroy(Workspace * w);

    inline unsigned ceil_div(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

    // Rows of the Q1 transfer matrices of the identity index maps, from the grid (mf,
    // mc points per fine / coarse line): the products and slot-ordered sums of the
    // matrix rows, bit-identical to an ELL row sum over them.  Prolongation row of fine
    // node (i, j), coarse (I, J) = (i/2, j/2): (I,J) x 1; (I,J), (I,J+1) or (I,J),
    // (I+1,J) x 1/2; (I,J), (I,J+1), (I+1,J), (I+1,J+1) x 1/4.  Restriction row of coarse
    // node (I, J): the fine nodes (2I+di, 2J+dj) inside the grid, di, dj = -1, 0, 1 in
    // that order, x (1 or 1/2)(1 or 1/2).  L2: vector loads through L2 (data written
    // by other blocks of the same launch).
    template <typename T, bool L2>
    __device__ __forceinline__ T q1_load(const T * p)
    {
        return L2 ? __ldcg(p) : *p;
    }

    template <typename T, bool L2>
    __device__ __forceinline__ T q1_prolong_row(uint64_t r, const T * c, uint32_t mf, uint32_t mc)
    {
        typedef Arith<T> M;
        const uint32_t i = (uint32_t)(r / mf), j = (uint32_t)(r - (uint64_t)i * mf);
        const T * cp = c + (uint64_t)(i >> 1) * mc + (j >> 1);
        const T h = T(0.5), q = T(0.25);
        if (! (i & 1) && ! (j & 1)) return M::add(T(0), M::mul(T(1), q1_load<T, L2>(cp)));
        if (! (i & 1)) return M::add(M::add(T(0), M::mul(h, q1_load<T, L2>(cp))), M::mul(h, q1_load<T, L2>(cp + 1)));
        if (! (j & 1)) return M::add(M::add(T(0), M::mul(h, q1_load<T, L2>(cp))), M::mul(h, q1_load<T, L2>(cp + mc)));
        const T a0 = q1_load<T, L2>(cp), a1 = q1_load<T, L2>(cp + 1), a2 = q1_load<T, L2>(cp + mc),
                a3 = q1_load<T, L2>(cp + mc + 1);
        return M::add(M::add(M::add(M::add(T(0), M::mul(q, a0)), M::mul(q, a1)), M::mul(q, a2)), M::mul(q, a3));
    }

    template <typename T, bool L2>
    __device__ __forceinline__ T q1_restrict_row(uint64_t r, const T * x, uint32_t mf, uint32_t mc)
    {
        typedef Arith<T> M;
        const int I = (int)(r / mc), J = (int)(r - (uint64_t)I * mc);
        T acc = T(0);
#pragma unroll
        for (int di = -1; di <= 1; ++di)
        {
            const int i = 2 * I + di;
            if (i < 0 || i >= (int)mf) continue;
            const T * xr = x + (uint64_t)i * mf;
            const T wi = di == 0 ? T(1) : T(0.5);
#pragma unroll
            for (int dj = -1; dj <= 1; ++dj)
            {
                const int jj = 2 * J + dj;
                if (jj < 0 || jj >= (int)mf) continue;
                const T w = dj == 0 ? wi : (di == 0 ? T(0.5) : T(0.25));
                acc = M::add(acc, M::mul(w, q1_load<T, L2>(xr + jj)));
            }
        }
        return acc;
    }

    extern int g_num_sms;
    int num_sms();

    // a hint: the line of `p` (a generic address of global memory) into L2
    __device__ __forceinline__ void prefetch_l2(const void * p)
    {
        asm volatile("prefetch.L2 [%0];" :: "l"(p));
    }

    // L2 prefetch distance of the streaming one-row-per-thread kernels (the Q1 stencil
    // kernel's gather form, the Q1 transfer kernels), in rows: HB2_Q1_PREFETCH=<waves>
    // of resident rows (2,048 per SM) ahead, read at each launch (runtime.cu); none by
    // default.  Measured: with every launch reading its vectors from DRAM (graph-timed,
    // vector sets of more than twice L2) half a wave ahead takes the level-11 FP64
    // sweep from 25.9 to 23.7 us (0.82 -> 0.90 of measured HBM; no gain in FP32) and
    // the prolongation from 26.2 to 23.0 us; inside the MG solve, where a level's
    // vectors partly stay in L2 from pass to pass and the kernels are issue-bound, it
    // made the solves 1-4 % slower at levels 9-11.
    int64_t l2_prefetch_rows(size_t elem);
}
