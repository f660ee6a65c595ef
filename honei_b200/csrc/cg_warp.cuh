// One-warp CG (CGSolver<Tag, methods::NONE>, math/cg.hh:64-135) for the
// smallest systems -- the MG coarsest level -- shared by the stand-alone
// coarse-solve kernels (cg.cu) and the fused small-level V-cycle (subcycle.cu).
#pragma once

#include <cfloat>

#include "hb2_common.cuh"
#include "hb2_internal.hh"

namespace hb2
{
    template <typename T> struct Eps;
    template <> struct Eps<double> { static __device__ __forceinline__ double v() { return DBL_EPSILON; } };
    template <> struct Eps<float> { static __device__ __forceinline__ float v() { return FLT_EPSILON; } };

    // the `exact` argument of the coarse CG: the reference's sequential fma order
    // (bit-identical to it); the standard recurrence with tree-ordered dots; the
    // Chronopoulos-Gear recurrence with one fused reduction per iteration
    constexpr int kCgTreeOneReduction = 0;
    constexpr int kCgExact = 1;
    constexpr int kCgTreeStandard = 2;

    template <typename T> struct Recip;
    template <> struct Recip<double> { static __device__ __forceinline__ double rn(double v) { return __drcp_rn(v); } };
    template <> struct Recip<float> { static __device__ __forceinline__ float rn(float v) { return __frcp_rn(v); } };

    template <typename T>
    __device__ __forceinline__ T guard(T d)
    {
        return fabs(d) > Eps<T>::v() ? d : Eps<T>::v();
    }

    // ------------------------------------------------------------------ one warp
    // Latency-bound coarse solves (the MG coarsest level has 81 unknowns and runs
    // a hundred iterations per V-cycle): one warp, no block barriers, reductions
    // by shuffles.  The reference-order dot is one fma chain in lane 0 with the
    // operands fetched ahead of the chain.
    template <typename T>
    __device__ __forceinline__ T warp_dot_exact(const T * a, const T * b, int n)
    {
        T s = T(0);
        if ((threadIdx.x & 31) == 0)
        {
            int i = 0;
            for (; i + 8 <= n; i += 8)
            {
                T a0 = a[i], a1 = a[i + 1], a2 = a[i + 2], a3 = a[i + 3], a4 = a[i + 4], a5 = a[i + 5], a6 = a[i + 6],
                  a7 = a[i + 7];
                T b0 = b[i], b1 = b[i + 1], b2 = b[i + 2], b3 = b[i + 3], b4 = b[i + 4], b5 = b[i + 5], b6 = b[i + 6],
                  b7 = b[i + 7];
                s = Arith<T>::fma(a0, b0, s);
                s = Arith<T>::fma(a1, b1, s);
                s = Arith<T>::fma(a2, b2, s);
                s = Arith<T>::fma(a3, b3, s);
                s = Arith<T>::fma(a4, b4, s);
                s = Arith<T>::fma(a5, b5, s);
                s = Arith<T>::fma(a6, b6, s);
                s = Arith<T>::fma(a7, b7, s);
            }
            for (; i < n; ++i) s = Arith<T>::fma(a[i], b[i], s);
        }
        return __shfl_sync(0xffffffffu, s, 0);
    }

    // Register-resident variant for the smallest systems (n <= 32 * RPL, K = 9):
    // each lane keeps its RPL rows of A and of x, r, p, v in registers; only p
    // (gathered by the SpMV) and, for the reference-order dots, the dot operands
    // go through shared memory.
    // T: arithmetic and matrix type; S: element type of b and x in memory (an
    // FP32 hierarchy can run its coarsest solve in FP64 on an FP64 copy of the
    // coarse operator: b is widened on load, x rounded on store).
    //
    // cg_warp_reg runs in one full warp (lane = threadIdx.x & 31) and needs 3n
    // elements of T in shared memory; it is called by cg_warp_reg_kernel and by
    // the fused small-level V-cycle kernel (subcycle.cu), which writes b earlier
    // in the same launch -- hence plain (coherent) loads of b, no __restrict__.
    template <typename T, typename S, int RPL>
    __device__ __forceinline__ void cg_warp_reg(const EllView<T> & Ag, const S * b, S * xg,
                                                uint64_t max_iters, double eps_d, int exact, uint64_t * used_out,
                                                double * defect_out, T * smem)
    {
        typedef Arith<T> M;
        constexpr int K = 9;
        const int n = (int)Ag.rows, lane = threadIdx.x & 31;
        T * sp = smem;            // p (and x for the initial defect)
        T * sa = sp + n;          // first dot operand (exact mode)
        T * sb = sa + n;          // second dot operand (exact mode)
        T av[RPL][K];
        int ac[RPL][K];
        T xr[RPL], rr[RPL], pr[RPL], vr[RPL];
#pragma unroll
        for (int j = 0; j < RPL; ++j)
        {
            const int row = lane + 32 * j;
            const bool ok = row < n;
#pragma unroll
            for (int k = 0; k < K; ++k)
            {
                const bool okk = ok && k < (int)Ag.K;     // up to 9 slots; the missing ones are skipped
                av[j][k] = okk ? Ag.val[(uint64_t)k * Ag.ld + row] : T(0);
                ac[j][k] = okk ? Ag.col[(uint64_t)k * Ag.ld + row] : -1;
            }
            xr[j] = ok ? T(xg[row]) : T(0);
            if (ok) sp[row] = xr[j];
        }
        __syncwarp();
        auto spmv = [&](T (&out)[RPL]) {
#pragma unroll
            for (int j = 0; j < RPL; ++j)
            {
                T s = T(0);
#pragma unroll
                for (int k = 0; k < K; ++k)
                    if (ac[j][k] >= 0) s = M::add(s, M::mul(av[j][k], sp[ac[j][k]]));
                out[j] = s;
            }
        };
        // dot of per-lane register vectors a, b over the valid rows
        auto dot = [&](const T (&a)[RPL], const T (&bb)[RPL]) -> T {
            if (exact == kCgExact)
            {
#pragma unroll
                for (int j = 0; j < RPL; ++j)
                {
                    const int row = lane + 32 * j;
                    if (row < n) { sa[row] = a[j]; sb[row] = bb[j]; }
                }
                __syncwarp();
                T s = warp_dot_exact(sa, sb, n);
                __syncwarp();
                return s;
            }
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < RPL; ++j)
                if (lane + 32 * j < n) s = fma((double)a[j], (double)bb[j], s);
            return (T)warp_sum(s);
        };
        T tmp[RPL];
        spmv(tmp);
        __syncwarp();
#pragma unroll
        for (int j = 0; j < RPL; ++j)
        {
            const int row = lane + 32 * j;
            rr[j] = row < n ? M::sub(T(b[row]), tmp[j]) : T(0);
            pr[j] = rr[j];
            if (row < n) sp[row] = pr[j];
        }
        __syncwarp();
        const T eps = T(eps_d);
        T alpha = dot(rr, rr);
        const T initial = sqrt(alpha);
        T current = initial;
        uint64_t it = 0, used = 0;
        if (exact == kCgTreeOneReduction && max_iters > 0)
        {
            // Chronopoulos-Gear recurrence (the same iterates as the loop below in
            // exact arithmetic): per iteration one product w = A r and both dots
            // (r, r), (w, r) in one shuffle tree, so the chain of an iteration holds
            // one reduction and one division instead of two of each; the
            // reciprocals the next iteration needs are formed off that chain.
            //   x += a p; r -= a s; w = A r; g = (r, r); d = (w, r);
            //   b = g / g_old; a = g / (d - b g / a_old); p = r + b p; s = w + b s
            T sr[RPL], wr[RPL];
            spmv(wr);   // w0 = A r0 (sp holds r0 = p0)
            T gam = alpha, del;
            {
                double s1 = 0.0;
#pragma unroll
                for (int j = 0; j < RPL; ++j)
                    if (lane + 32 * j < n) s1 = fma((double)wr[j], (double)rr[j], s1);
                del = (T)warp_sum(s1);
            }
            T a = M::div(gam, guard(del));
            T inv_a = Recip<T>::rn(guard(a)), inv_g = Recip<T>::rn(guard(gam));
            // the stop test on squared norms: no square root on the iteration's chain
            const T thr = M::mul(eps, initial), thr2 = M::mul(thr, thr), eps2 = M::mul(eps, eps);
#pragma unroll
            for (int j = 0; j < RPL; ++j) sr[j] = wr[j];
            while (it < max_iters)
            {
                const T ma = -a;
#pragma unroll
                for (int j = 0; j < RPL; ++j)
                {
                    xr[j] = M::add(xr[j], M::mul(a, pr[j]));
                    rr[j] = M::add(rr[j], M::mul(ma, sr[j]));
                }
                __syncwarp();   // every lane is done gathering the old r
#pragma unroll
                for (int j = 0; j < RPL; ++j)
                    if (lane + 32 * j < n) sp[lane + 32 * j] = rr[j];
                __syncwarp();
                spmv(wr);
                double s1 = 0.0, s2 = 0.0;
#pragma unroll
                for (int j = 0; j < RPL; ++j)
                    if (lane + 32 * j < n)
                    {
                        s1 = fma((double)rr[j], (double)rr[j], s1);
                        s2 = fma((double)wr[j], (double)rr[j], s2);
                    }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
                {
                    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
                }
                const T g = (T)s1;
                del = (T)s2;
                ++it;
                if (g < thr2 || g < eps2 || it == max_iters)
                {
                    current = sqrt(g);
                    used = it;
                    break;
                }
                // single-rounded reciprocals instead of IEEE divisions (this mode is
                // not the reference's order anyway)
                const T b = M::mul(g, inv_g);
                a = M::mul(g, Recip<T>::rn(guard(M::sub(del, M::mul(M::mul(b, g), inv_a)))));
#pragma unroll
                for (int j = 0; j < RPL; ++j)
                {
                    pr[j] = M::add(rr[j], M::mul(b, pr[j]));
                    sr[j] = M::add(wr[j], M::mul(b, sr[j]));
                }
                inv_a = Recip<T>::rn(guard(a));
                inv_g = Recip<T>::rn(guard(g));
                gam = g;
            }
            it = max_iters;   // done: skip the loop below
        }
        while (it < max_iters)
        {
            spmv(vr);
            const T temp = dot(vr, pr);
            const T lambda = M::div(alpha, guard(temp));
            const T mlambda = -lambda;
#pragma unroll
            for (int j = 0; j < RPL; ++j)
            {
                xr[j] = M::add(xr[j], M::mul(lambda, pr[j]));
                rr[j] = M::add(rr[j], M::mul(mlambda, vr[j]));
            }
            const T alpha_old = alpha;
            alpha = dot(rr, rr);
            const T talpha = M::div(alpha, guard(alpha_old));
            __syncwarp();   // every lane is done gathering the old p
#pragma unroll
            for (int j = 0; j < RPL; ++j)
            {
                const int row = lane + 32 * j;
                pr[j] = M::add(M::mul(pr[j], talpha), rr[j]);
                if (row < n) sp[row] = pr[j];
            }
            __syncwarp();
            ++it;
            current = sqrt(alpha);
            if (current < M::mul(eps, initial) || current < eps) { used = it; break; }
            if (it == max_iters) used = it;
        }
#pragma unroll
        for (int j = 0; j < RPL; ++j)
            if (lane + 32 * j < n) xg[lane + 32 * j] = S(xr[j]);
        if (lane == 0)
        {
            if (used_out) *used_out = used;
            if (defect_out) *defect_out = (double)current;
        }
    }

    template <typename T, typename S, int RPL>
    __global__ void __launch_bounds__(32)
    cg_warp_reg_kernel(EllView<T> Ag, const S * __restrict__ b, S * __restrict__ xg, uint64_t max_iters, double eps_d,
                       int exact, uint64_t * used_out, double * defect_out, uint64_t vstride, const uint8_t * active,
                       const uint32_t * list, const uint32_t * count)
    {
        extern __shared__ __align__(16) unsigned char smem_raw[];
        pdl_entry();
        if (list)
        {
            // work list: the systems of vectors list[0 .. *count - 1], one per warp in turn
            const uint32_t n = *count;
            for (uint32_t i = blockIdx.x; i < n; i += gridDim.x)
            {
                const uint64_t o = (uint64_t)list[i] * vstride;
                cg_warp_reg<T, S, RPL>(Ag, b + o, xg + o, max_iters, eps_d, exact, used_out, defect_out, (T *)smem_raw);
                __syncwarp();
            }
            return;
        }
        // batched launches: block j solves the system of vector j (b, x at j * vstride)
        if (active && ! active[blockIdx.x]) return;
        cg_warp_reg<T, S, RPL>(Ag, b + (uint64_t)blockIdx.x * vstride, xg + (uint64_t)blockIdx.x * vstride, max_iters,
                               eps_d, exact, used_out, defect_out, (T *)smem_raw);
    }
}
