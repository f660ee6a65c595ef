// Krylov solvers with a variable preconditioner on the device:
// CGSolver<Tag, methods::VAR> (math/cg.hh:142-210), CGSmoother (math/cg.hh:217-290)
// and BiCGStabSolver<Tag, methods::VAR> (math/bicgstab.hh:60-210).  P is a vector
// (Product of two DenseVectors: the element-wise product, la/product.hh:1198-1204)
// or an ELL matrix.
//
// A solve is one CUDA graph: a prefix (initial defect, first preconditioning),
// a conditional WHILE node whose body is one iteration, and the copy of the
// solver state to pinned host memory.  Every scalar of the recurrences lives in
// device memory (KState); one-thread decide kernels evaluate the reference's
// tests and set the loop's condition, so a solve costs one graph launch and one
// host synchronisation.  BiCGStab leaves its iteration early (a restart, or
// convergence right after the first half-step): its body is a flat sequence of
// IF nodes, each guarded by a condition that a decide kernel earlier in the
// same iteration sets -- a decide kernel that finds its segment skipped
// clears the conditions of the segments after it.
//
// Vector updates round every product and sum separately, as the reference's
// ScaledSum / Scale / Sum / ElementProduct do; the dot products and norms are
// deterministic two-level grid reductions (the reference sums sequentially, so
// iteration counts may differ by one).  FP64.
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <cfloat>
#include <cstring>

using namespace hb2;

namespace
{
    struct KState
    {
        double alpha_new, alpha, temp, init, cur;          // CG
        double alpha_next;                                 // CG, vector P: <r, d (.) r> of the new r
        double rho, rho_new, gamma, omega, ab, d0, d00, defnorm;   // BiCGStab
        unsigned long long iter, used;
        int stage, restart, first, converged;
    };

    constexpr int kVecThreads = 256;

    __device__ __forceinline__ double eps_guard(double t)
    {
        return fabs(t) > DBL_EPSILON ? t : DBL_EPSILON * (t / fabs(t));
    }

    // ScaledSum: b*y + x, product and sum each rounded
    __device__ __forceinline__ double axpy(double b, double y, double x) { return __dadd_rn(__dmul_rn(b, y), x); }

    // reductions k = 0 .. NRED-1 of one launch: each its own partials / counters
    template <int NRED>
    __device__ __forceinline__ void finish(const double (&acc)[2], ReduceSlot rs, double * out0, double * out1,
                                           double * scratch)
    {
        const unsigned G = gridDim.x, ng = (G + kReduceGroup - 1) / kReduceGroup;
        for (int k = 0; k < NRED; ++k)
        {
            const double v = block_sum(acc[k], scratch);
            sum_finish(v, rs.partials + k * G, rs.gpart + k * ng, rs.ticket + k * (ng + 1), G, blockIdx.x,
                       k ? out1 : out0, 0, scratch);
        }
    }

    // z = d (.) a when d (else z as given); c1 = c2 = z when given;
    // out0 = <z, w0>, out1 = <z, w1> (a null w: z itself)
    template <int NRED>
    __global__ void __launch_bounds__(kVecThreads) k_vec_dots(uint64_t n, const double * __restrict__ d,
                                                              const double * __restrict__ a, double * z, double * c1,
                                                              double * c2, const double * w0, const double * w1,
                                                              ReduceSlot rs, double * out0, double * out1)
    {
        __shared__ double scratch[32];
        double acc[2] = {0.0, 0.0};
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        {
            double zi;
            if (d)
            {
                zi = __dmul_rn(d[i], a[i]);
                z[i] = zi;
            }
            else zi = z[i];
            if (c1) c1[i] = zi;
            if (c2) c2[i] = zi;
            acc[0] = fma(zi, w0 ? w0[i] : zi, acc[0]);
            if (NRED == 2) acc[1] = fma(zi, w1 ? w1[i] : zi, acc[1]);
        }
        finish<NRED>(acc, rs, out0, out1, scratch);
    }

    // CG: lambda = alpha_new / guard(temp); x += lambda p; r += (-lambda) v; (||r||^2)
    template <bool NORM>
    __global__ void __launch_bounds__(kVecThreads) k_cg_update(uint64_t n, double * x, double * r, const double * p,
                                                               const double * v, const KState * st, ReduceSlot rs,
                                                               double * out)
    {
        __shared__ double scratch[32];
        const double lambda = st->alpha_new / eps_guard(st->temp), ml = -lambda;
        double acc[2] = {0.0, 0.0};
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        {
            x[i] = axpy(lambda, p[i], x[i]);
            const double ri = axpy(ml, v[i], r[i]);
            r[i] = ri;
            if (NORM) acc[0] = fma(ri, ri, acc[0]);
        }
        if (NORM) finish<1>(acc, rs, out, nullptr, scratch);
    }

    // CG: talpha = alpha_new / guard(alpha); p = p * talpha; p = p + z
    __global__ void __launch_bounds__(kVecThreads) k_cg_p(uint64_t n, double * p, const double * z, const KState * st)
    {
        const double ta = st->alpha_new / eps_guard(st->alpha);
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
            p[i] = __dadd_rn(__dmul_rn(p[i], ta), z[i]);
    }

    // CG with a vector P: the update also forms z = d (.) r of the new r and
    // alpha_next = <z, r> (plus ||r||^2 unless smoothing); z is not stored
    template <bool NORM>
    __global__ void __launch_bounds__(kVecThreads) k_cg_update_diag(uint64_t n, double * x, double * r,
                                                                    const double * p, const double * v,
                                                                    const double * d, const KState * st,
                                                                    ReduceSlot rs, double * out_z, double * out_n)
    {
        __shared__ double scratch[32];
        const double lambda = st->alpha_new / eps_guard(st->temp), ml = -lambda;
        double acc[2] = {0.0, 0.0};
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        {
            x[i] = axpy(lambda, p[i], x[i]);
            const double ri = axpy(ml, v[i], r[i]);
            r[i] = ri;
            const double zi = __dmul_rn(d[i], ri);
            acc[0] = fma(zi, ri, acc[0]);
            if (NORM) acc[1] = fma(ri, ri, acc[1]);
        }
        if (NORM) finish<2>(acc, rs, out_z, out_n, scratch);
        else finish<1>(acc, rs, out_z, nullptr, scratch);
    }

    // CG with a vector P: p = p * talpha + d (.) r (z formed again, each step rounded)
    __global__ void __launch_bounds__(kVecThreads) k_cg_p_diag(uint64_t n, double * p, const double * d,
                                                               const double * r, const KState * st)
    {
        const double ta = st->alpha_new / eps_guard(st->alpha);
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
            p[i] = __dadd_rn(__dmul_rn(p[i], ta), __dmul_rn(d[i], r[i]));
    }

    __global__ void k_cg_init(KState * st, uint64_t max_iters, cudaGraphConditionalHandle h)
    {
        st->iter = 0;
        st->used = 0;
        cudaGraphSetConditional(h, max_iters > 0 ? 1u : 0u);
    }

    // math/cg.hh:178-198 (smoother: math/cg.hh:263-267); fused: the next alpha_new
    // was already reduced by the update (vector P)
    __global__ void k_cg_decide(KState * st, uint64_t max_iters, double eps, int smoother, int fused,
                                cudaGraphConditionalHandle h)
    {
        const unsigned long long it = st->iter + 1;
        st->iter = it;
        bool stop;
        if (smoother) stop = it == max_iters;
        else
        {
            const double cur = sqrt(st->cur);
            st->cur = cur;
            stop = cur < eps * st->init || cur < eps || it == max_iters;
        }
        if (stop) st->used = it;
        st->alpha = st->alpha_new;
        if (fused) st->alpha_new = st->alpha_next;
        cudaGraphSetConditional(h, stop ? 0u : 1u);
    }

    // BiCGStab vector steps (math/bicgstab.hh:143-194)
    __global__ void __launch_bounds__(kVecThreads) k_bicg_s(uint64_t n, double * s, const double * r, const double * v,
                                                            double * st_, const double * rt, const double * vt,
                                                            const KState * st, ReduceSlot rs, double * out)
    {
        __shared__ double scratch[32];
        const double ma = -st->ab;
        double acc[2] = {0.0, 0.0};
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        {
            const double si = axpy(ma, v[i], r[i]);
            s[i] = si;
            st_[i] = axpy(ma, vt[i], rt[i]);
            acc[0] = fma(si, si, acc[0]);
        }
        finish<1>(acc, rs, out, nullptr, scratch);
    }

    __global__ void __launch_bounds__(kVecThreads) k_axpy_ab(uint64_t n, double * x, const double * y, const KState * st)
    {
        const double a = st->ab;
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
            x[i] = axpy(a, y[i], x[i]);
    }

    // x += omega s~; x += alpha p~; r = (-omega) t + s; ||r||^2
    __global__ void __launch_bounds__(kVecThreads) k_bicg_u(uint64_t n, double * x, const double * st_, const double * pt,
                                                            double * r, const double * s, const double * t,
                                                            const KState * st, ReduceSlot rs, double * out)
    {
        __shared__ double scratch[32];
        const double om = st->omega, a = st->ab, mo = -om;
        double acc[2] = {0.0, 0.0};
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        {
            x[i] = axpy(a, pt[i], axpy(om, st_[i], x[i]));
            const double ri = axpy(mo, t[i], s[i]);
            r[i] = ri;
            acc[0] = fma(ri, ri, acc[0]);
        }
        finish<1>(acc, rs, out, nullptr, scratch);
    }

    // r~ = (-omega) t~ + s~; rho_new = <r~, r~0>
    __global__ void __launch_bounds__(kVecThreads) k_bicg_w1(uint64_t n, double * rt, const double * st_,
                                                             const double * tt, const double * rt0, const KState * st,
                                                             ReduceSlot rs, double * out)
    {
        __shared__ double scratch[32];
        const double mo = -st->omega;
        double acc[2] = {0.0, 0.0};
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        {
            const double v = axpy(mo, tt[i], st_[i]);
            rt[i] = v;
            acc[0] = fma(v, rt0[i], acc[0]);
        }
        finish<1>(acc, rs, out, nullptr, scratch);
    }

    // beta = (alpha / omega) * (rho_new / rho); p~ += (-omega) v~; p~ *= beta; p~ += r~
    __global__ void __launch_bounds__(kVecThreads) k_bicg_w2(uint64_t n, double * pt, const double * vt, const double * rt,
                                                             const KState * st)
    {
        const double beta = (st->ab / st->omega) * (st->rho_new / st->rho), mo = -st->omega;
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
            pt[i] = __dadd_rn(__dmul_rn(axpy(mo, vt[i], pt[i]), beta), rt[i]);
    }

    // ---- BiCGStab control (math/bicgstab.hh:100-198) ------------------------
    // stage: 1 after the first half-step is due, 2 the second, 3 the update, 4 the
    // direction update; 0 = the iteration has ended
    __global__ void k_bi_init(KState * st, cudaGraphConditionalHandle h_loop)
    {
        st->iter = 0;
        st->restart = 1;
        st->first = 1;
        st->converged = 0;
        st->stage = 0;
        st->d00 = 1e14;
        cudaGraphSetConditional(h_loop, 1u);
    }
    __global__ void k_bi_d0(const KState * st, cudaGraphConditionalHandle h_restart)
    {
        cudaGraphSetConditional(h_restart, st->restart ? 1u : 0u);
    }
    // after the restart block: the squared defect, defnorm_00 on the first pass
    __global__ void k_bi_restarted(KState * st)
    {
        st->defnorm = st->d0;
        if (st->first) st->d00 = st->d0;
        st->first = 0;
        st->restart = 0;
    }
    __global__ void k_bi_d1(KState * st, uint64_t max_iters, cudaGraphConditionalHandle h_loop,
                            cudaGraphConditionalHandle h_s)
    {
        const unsigned long long it = st->iter + 1;
        st->iter = it;
        if (fabs(st->gamma) < fabs(st->rho) * 1e-14)
        {
            st->restart = 1;
            st->stage = 0;
            cudaGraphSetConditional(h_s, 0u);
            cudaGraphSetConditional(h_loop, it < max_iters ? 1u : 0u);
            return;
        }
        st->ab = st->rho / st->gamma;
        st->stage = 1;
        cudaGraphSetConditional(h_s, 1u);
    }
    __global__ void k_bi_d2(KState * st, double eps, cudaGraphConditionalHandle h_loop,
                            cudaGraphConditionalHandle h_conv, cudaGraphConditionalHandle h_t)
    {
        if (st->stage != 1)
        {
            cudaGraphSetConditional(h_conv, 0u);
            cudaGraphSetConditional(h_t, 0u);
            return;
        }
        if (st->defnorm < eps * st->d00)
        {
            st->converged = 1;
            st->stage = 0;
            cudaGraphSetConditional(h_conv, 1u);
            cudaGraphSetConditional(h_t, 0u);
            cudaGraphSetConditional(h_loop, 0u);
            return;
        }
        st->stage = 2;
        cudaGraphSetConditional(h_conv, 0u);
        cudaGraphSetConditional(h_t, 1u);
    }
    __global__ void k_bi_d3(KState * st, uint64_t max_iters, cudaGraphConditionalHandle h_loop,
                            cudaGraphConditionalHandle h_u)
    {
        if (st->stage != 2) { cudaGraphSetConditional(h_u, 0u); return; }
        if (fabs(st->gamma) < fabs(st->omega) * 1e-14)
        {
            st->restart = 1;
            st->stage = 0;
            cudaGraphSetConditional(h_u, 0u);
            cudaGraphSetConditional(h_loop, st->iter < max_iters ? 1u : 0u);
            return;
        }
        st->omega = st->omega / st->gamma;
        st->stage = 3;
        cudaGraphSetConditional(h_u, 1u);
    }
    __global__ void k_bi_d4(KState * st, double eps, cudaGraphConditionalHandle h_loop, cudaGraphConditionalHandle h_w)
    {
        if (st->stage != 3) { cudaGraphSetConditional(h_w, 0u); return; }
        if (st->defnorm < eps * st->d00)
        {
            st->converged = 1;
            st->stage = 0;
            cudaGraphSetConditional(h_w, 0u);
            cudaGraphSetConditional(h_loop, 0u);
            return;
        }
        st->stage = 4;
        cudaGraphSetConditional(h_w, 1u);
    }
    __global__ void k_bi_d5(KState * st, uint64_t max_iters, cudaGraphConditionalHandle h_loop)
    {
        if (st->stage != 4) return;
        st->rho = st->rho_new;
        st->stage = 0;
        cudaGraphSetConditional(h_loop, st->iter <= max_iters ? 1u : 0u);
    }
}

struct hb2_krylov_s
{
    int method;
    int device;
    hb2_ell A = nullptr, P = nullptr;
    double * pdiag = nullptr;      // own copy of a vector preconditioner
    uint64_t n = 0, max_iters = 0;
    double eps = 0;
    double * vec = nullptr;
    int nvec = 0;
    KState * st = nullptr;
    KState * host_st = nullptr;    // pinned
    Workspace * ws = nullptr;
    cudaStream_t cap = nullptr, cap2 = nullptr, cap3 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t prefix_kernels = 0, body_kernels = 0;

    double * v(int i) const { return vec + (uint64_t)i * n; }
};

namespace
{
    uint32_t vgrid(uint64_t n)
    {
        const uint64_t g = (n + kVecThreads - 1) / kVecThreads;
        return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(g, 8ull * num_sms()));
    }

    // z = P a with out0 = <z, w0> (and out1 = <z, w1>; a null w: z itself);
    // copies c1 = c2 = z when given.  A matrix P: the ELL product, then one pass
    // for the dots and copies; a vector P: one fused pass.
    int precond(hb2_krylov_s * K, const double * a, double * z, const double * w0, double * out0, const double * w1,
                double * out1, double * c1, double * c2, cudaStream_t s)
    {
        const uint64_t n = K->n;
        if (! K->pdiag)
        {
            int st = launch_ell(K->P, kPlain, a, z, 0, 0, 0, 0, 0, K->ws, s);
            if (st) return st;
        }
        if (out1)
            k_vec_dots<2><<<vgrid(n), kVecThreads, 0, s>>>(n, K->pdiag, a, z, c1, c2, w0, w1, K->ws->slot(), out0, out1);
        else
            k_vec_dots<1><<<vgrid(n), kVecThreads, 0, s>>>(n, K->pdiag, a, z, c1, c2, w0, nullptr, K->ws->slot(), out0,
                                                            nullptr);
        count_launches(1);
        HB2_LAUNCH_CHECK("krylov vector kernel");
        return HB2_OK;
    }

    int capture_fail(hb2_krylov_s * K, cudaError_t e, const char * what)
    {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(K->cap3, &g);
        cudaStreamEndCapture(K->cap2, &g);
        cudaStreamEndCapture(K->cap, &g);
        if (g) cudaGraphDestroy(g);
        return cuda_status(e == cudaSuccess ? cudaErrorUnknown : e, what);
    }

    // an IF node at the end of the body being captured on cap2, its body captured
    // on cap3 by `fill`
    template <typename F>
    int add_if(hb2_krylov_s * K, cudaGraphConditionalHandle h, F fill)
    {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t * deps = nullptr;
        size_t ndeps = 0;
        cudaError_t e = cudaStreamGetCaptureInfo(K->cap2, &cs, 0, &g, &deps, &ndeps);
        if (e != cudaSuccess) return capture_fail(K, e, "cudaStreamGetCaptureInfo (if)");
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        e = cudaGraphAddNode(&node, g, deps, ndeps, &cp);
        if (e != cudaSuccess) return capture_fail(K, e, "cudaGraphAddNode (if)");
        e = cudaStreamUpdateCaptureDependencies(K->cap2, &node, 1, cudaStreamSetCaptureDependencies);
        if (e == cudaSuccess)
            e = cudaStreamBeginCaptureToGraph(K->cap3, cp.conditional.phGraph_out[0], 0, 0, 0,
                                              cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return capture_fail(K, e, "capture of an if body");
        int st = fill(K->cap3);
        cudaGraph_t body = nullptr;
        e = cudaStreamEndCapture(K->cap3, &body);
        if (st) return st;
        if (e != cudaSuccess) return capture_fail(K, e, "cudaStreamEndCapture (if body)");
        return HB2_OK;
    }

    int body_cg(hb2_krylov_s * K, cudaGraphConditionalHandle h_loop)
    {
        const uint64_t n = K->n;
        const bool smoother = K->method == HB2_CG_SMOOTHER;
        double * x = K->v(1), * r = K->v(2), * p = K->v(3), * v = K->v(4), * z = K->v(5);
        KState * st = K->st;
        cudaStream_t s = K->cap2;
        int e = launch_ell(K->A, kDot, p, v, 0, 0, 0, &st->temp, 0, K->ws, s);
        if (e) return e;
        if (K->pdiag)
        {
            // vector P: z = d (.) r and <z, r> fused into the update, z formed again in
            // the direction update -- four kernels per iteration
            if (smoother)
                k_cg_update_diag<false><<<vgrid(n), kVecThreads, 0, s>>>(n, x, r, p, v, K->pdiag, st, K->ws->slot(),
                                                                          &st->alpha_next, nullptr);
            else
                k_cg_update_diag<true><<<vgrid(n), kVecThreads, 0, s>>>(n, x, r, p, v, K->pdiag, st, K->ws->slot(),
                                                                         &st->alpha_next, &st->cur);
            k_cg_decide<<<1, 1, 0, s>>>(st, K->max_iters, K->eps, smoother ? 1 : 0, 1, h_loop);
            k_cg_p_diag<<<vgrid(n), kVecThreads, 0, s>>>(n, p, K->pdiag, r, st);
            count_launches(3);
            HB2_LAUNCH_CHECK("krylov CG (vector P)");
            return HB2_OK;
        }
        if (smoother) k_cg_update<false><<<vgrid(n), kVecThreads, 0, s>>>(n, x, r, p, v, st, K->ws->slot(), nullptr);
        else k_cg_update<true><<<vgrid(n), kVecThreads, 0, s>>>(n, x, r, p, v, st, K->ws->slot(), &st->cur);
        k_cg_decide<<<1, 1, 0, s>>>(st, K->max_iters, K->eps, smoother ? 1 : 0, 0, h_loop);
        count_launches(2);
        HB2_LAUNCH_CHECK("krylov CG update");
        if (K->pdiag) e = precond(K, r, z, r, &st->alpha_new, nullptr, nullptr, nullptr, nullptr, s);
        else e = launch_ell(K->P, kDot, r, z, 0, 0, 0, &st->alpha_new, 0, K->ws, s);
        if (e) return e;
        k_cg_p<<<vgrid(n), kVecThreads, 0, s>>>(n, p, z, st);
        count_launches(1);
        HB2_LAUNCH_CHECK("krylov CG direction");
        return HB2_OK;
    }

    int body_bicg(hb2_krylov_s * K, cudaGraphConditionalHandle h_loop)
    {
        const uint64_t n = K->n;
        KState * st = K->st;
        cudaStream_t s = K->cap2;
        double * b = K->v(0), * x = K->v(1), * r = K->v(2), * rt = K->v(3), * rt0 = K->v(4), * pt = K->v(5),
               * v = K->v(6), * vt = K->v(7), * sv = K->v(8), * stv = K->v(9), * t = K->v(10), * tt = K->v(11);
        cudaGraph_t body = nullptr;
        {
            cudaStreamCaptureStatus cs;
            const cudaGraphNode_t * deps = nullptr;
            size_t ndeps = 0;
            cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, 0, &body, &deps, &ndeps);
            if (e != cudaSuccess) return capture_fail(K, e, "cudaStreamGetCaptureInfo (body)");
        }
        cudaGraphConditionalHandle h_restart, h_s, h_conv, h_t, h_u, h_w;
        cudaError_t ce = cudaGraphConditionalHandleCreate(&h_restart, body, 0, 0);
        if (ce == cudaSuccess) ce = cudaGraphConditionalHandleCreate(&h_s, body, 0, 0);
        if (ce == cudaSuccess) ce = cudaGraphConditionalHandleCreate(&h_conv, body, 0, 0);
        if (ce == cudaSuccess) ce = cudaGraphConditionalHandleCreate(&h_t, body, 0, 0);
        if (ce == cudaSuccess) ce = cudaGraphConditionalHandleCreate(&h_u, body, 0, 0);
        if (ce == cudaSuccess) ce = cudaGraphConditionalHandleCreate(&h_w, body, 0, 0);
        if (ce != cudaSuccess) return capture_fail(K, ce, "cudaGraphConditionalHandleCreate (bicgstab)");
        const uint32_t G = vgrid(n);
        int e;
        // restart: r = b - A x, ||r||^2; r~0 = P r; r~ = p~ = r~0; rho = <r~0, r~0>
        k_bi_d0<<<1, 1, 0, s>>>(st, h_restart);
        count_launches(1);
        e = add_if(K, h_restart, [&](cudaStream_t s3) {
            int q = launch_ell(K->A, kDefect, x, r, b, 0, 0, &st->d0, 0, K->ws, s3);
            if (! q) q = precond(K, r, rt0, nullptr, &st->rho, nullptr, nullptr, rt, pt, s3);
            if (q) return q;
            k_bi_restarted<<<1, 1, 0, s3>>>(st);
            count_launches(1);
            HB2_LAUNCH_CHECK("krylov restart");
            return (int)HB2_OK;
        });
        if (e) return e;
        // v = A p~; v~ = P v; gamma = <v~, r~0>
        e = launch_ell(K->A, kPlain, pt, v, 0, 0, 0, 0, 0, K->ws, s);
        if (! e) e = precond(K, v, vt, rt0, &st->gamma, nullptr, nullptr, nullptr, nullptr, s);
        if (e) return e;
        k_bi_d1<<<1, 1, 0, s>>>(st, K->max_iters, h_loop, h_s);
        count_launches(1);
        // s = r - alpha v; s~ = r~ - alpha v~; ||s||^2
        e = add_if(K, h_s, [&](cudaStream_t s3) {
            k_bicg_s<<<G, kVecThreads, 0, s3>>>(n, sv, r, v, stv, rt, vt, st, K->ws->slot(), &st->defnorm);
            count_launches(1);
            HB2_LAUNCH_CHECK("krylov bicgstab s");
            return (int)HB2_OK;
        });
        if (e) return e;
        k_bi_d2<<<1, 1, 0, s>>>(st, K->eps, h_loop, h_conv, h_t);
        count_launches(1);
        e = add_if(K, h_conv, [&](cudaStream_t s3) {
            k_axpy_ab<<<G, kVecThreads, 0, s3>>>(n, x, pt, st);
            count_launches(1);
            HB2_LAUNCH_CHECK("krylov bicgstab x");
            return (int)HB2_OK;
        });
        if (e) return e;
        // t = A s~; t~ = P t; gamma = <t~, t~>, omega = <t~, s~>
        e = add_if(K, h_t, [&](cudaStream_t s3) {
            int q = launch_ell(K->A, kPlain, stv, t, 0, 0, 0, 0, 0, K->ws, s3);
            if (! q) q = precond(K, t, tt, nullptr, &st->gamma, stv, &st->omega, nullptr, nullptr, s3);
            return q;
        });
        if (e) return e;
        k_bi_d3<<<1, 1, 0, s>>>(st, K->max_iters, h_loop, h_u);
        count_launches(1);
        e = add_if(K, h_u, [&](cudaStream_t s3) {
            k_bicg_u<<<G, kVecThreads, 0, s3>>>(n, x, stv, pt, r, sv, t, st, K->ws->slot(), &st->defnorm);
            count_launches(1);
            HB2_LAUNCH_CHECK("krylov bicgstab update");
            return (int)HB2_OK;
        });
        if (e) return e;
        k_bi_d4<<<1, 1, 0, s>>>(st, K->eps, h_loop, h_w);
        count_launches(1);
        e = add_if(K, h_w, [&](cudaStream_t s3) {
            k_bicg_w1<<<G, kVecThreads, 0, s3>>>(n, rt, stv, tt, rt0, st, K->ws->slot(), &st->rho_new);
            k_bicg_w2<<<G, kVecThreads, 0, s3>>>(n, pt, vt, rt, st);
            count_launches(2);
            HB2_LAUNCH_CHECK("krylov bicgstab direction");
            return (int)HB2_OK;
        });
        if (e) return e;
        k_bi_d5<<<1, 1, 0, s>>>(st, K->max_iters, h_loop);
        count_launches(1);
        HB2_LAUNCH_CHECK("krylov bicgstab control");
        return HB2_OK;
    }

    int build_graph(hb2_krylov_s * K)
    {
        const uint64_t before = hb2_launch_count();
        HB2_CUDA(cudaStreamBeginCapture(K->cap, cudaStreamCaptureModeThreadLocal));
        KState * st = K->st;
        const uint64_t n = K->n;
        double * b = K->v(0), * x = K->v(1), * r = K->v(2), * p = K->v(3);
        int e = HB2_OK;
        cudaStreamCaptureStatus cs;
        cudaGraph_t capg = nullptr;
        const cudaGraphNode_t * deps = nullptr;
        size_t ndeps = 0;
        cudaError_t ce = cudaStreamGetCaptureInfo(K->cap, &cs, 0, &capg, &deps, &ndeps);
        if (ce != cudaSuccess) return capture_fail(K, ce, "cudaStreamGetCaptureInfo");
        cudaGraphConditionalHandle h_loop;
        ce = cudaGraphConditionalHandleCreate(&h_loop, capg, 0, 0);
        if (ce != cudaSuccess) return capture_fail(K, ce, "cudaGraphConditionalHandleCreate");
        if (K->method == HB2_BICGSTAB_VAR)
        {
            k_bi_init<<<1, 1, 0, K->cap>>>(st, h_loop);
            count_launches(1);
        }
        else
        {
            // r = b - A x (||r||); p = P r; alpha_new = <r, p>
            e = launch_ell(K->A, kDefect, x, r, b, 0, 0, &st->init, 1, K->ws, K->cap);
            if (! e)
            {
                if (K->pdiag) e = precond(K, r, p, r, &st->alpha_new, nullptr, nullptr, nullptr, nullptr, K->cap);
                else e = launch_ell(K->P, kDot, r, p, 0, 0, 0, &st->alpha_new, 0, K->ws, K->cap);
            }
            if (e) { capture_fail(K, cudaSuccess, ""); return e; }
            k_cg_init<<<1, 1, 0, K->cap>>>(st, K->max_iters, h_loop);
            count_launches(1);
        }
        ce = cudaGetLastError();
        if (ce == cudaSuccess) ce = cudaStreamGetCaptureInfo(K->cap, &cs, 0, &capg, &deps, &ndeps);
        if (ce != cudaSuccess) return capture_fail(K, ce, "capture (prefix)");
        K->prefix_kernels = hb2_launch_count() - before;
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = h_loop;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        ce = cudaGraphAddNode(&cnode, capg, deps, ndeps, &cp);
        if (ce != cudaSuccess) return capture_fail(K, ce, "cudaGraphAddNode (while)");
        ce = cudaStreamUpdateCaptureDependencies(K->cap, &cnode, 1, cudaStreamSetCaptureDependencies);
        if (ce == cudaSuccess)
            ce = cudaStreamBeginCaptureToGraph(K->cap2, cp.conditional.phGraph_out[0], 0, 0, 0,
                                               cudaStreamCaptureModeThreadLocal);
        if (ce != cudaSuccess) return capture_fail(K, ce, "capture of the loop body");
        const uint64_t body0 = hb2_launch_count();
        e = K->method == HB2_BICGSTAB_VAR ? body_bicg(K, h_loop) : body_cg(K, h_loop);
        if (e) { capture_fail(K, cudaSuccess, ""); return e; }
        K->body_kernels = hb2_launch_count() - body0;
        cudaGraph_t body = nullptr;
        ce = cudaStreamEndCapture(K->cap2, &body);
        if (ce != cudaSuccess) return capture_fail(K, ce, "cudaStreamEndCapture (body)");
        ce = cudaMemcpyAsync(K->host_st, st, sizeof(KState), cudaMemcpyDeviceToHost, K->cap);
        if (ce != cudaSuccess) return capture_fail(K, ce, "state copy");
        (void)n;
        (void)p;
        cudaGraph_t g = nullptr;
        ce = cudaStreamEndCapture(K->cap, &g);
        set_launch_count(before);
        if (ce != cudaSuccess) return cuda_status(ce, "cudaStreamEndCapture (krylov)");
        K->graph = g;
        ce = cudaGraphInstantiate(&K->exec, g, 0);
        if (ce != cudaSuccess) return cuda_status(ce, "cudaGraphInstantiate (krylov)");
        return HB2_OK;
    }

    void krylov_free(hb2_krylov_s * K)
    {
        if (! K) return;
        if (K->exec) cudaGraphExecDestroy(K->exec);
        if (K->graph) cudaGraphDestroy(K->graph);
        if (K->cap) cudaStreamDestroy(K->cap);
        if (K->cap2) cudaStreamDestroy(K->cap2);
        if (K->cap3) cudaStreamDestroy(K->cap3);
        cudaFree(K->vec);
        cudaFree(K->pdiag);
        cudaFree(K->st);
        if (K->host_st) cudaFreeHost(K->host_st);
        workspace_destroy(K->ws);
        delete K;
    }
}

extern "C" int hb2_krylov_create(hb2_krylov * out, int method, hb2_ell A, hb2_ell P, const double * pdiag,
                                 uint64_t max_iters, double eps, cudaStream_t stream)
{
    if (! out || ! A) return fail(HB2_ERR_ARG, "hb2_krylov_create: null argument");
    *out = nullptr;
    if (method != HB2_CG_VAR && method != HB2_BICGSTAB_VAR && method != HB2_CG_SMOOTHER)
        return fail(HB2_ERR_ARG, "hb2_krylov_create: unknown method");
    if ((P == nullptr) == (pdiag == nullptr))
        return fail(HB2_ERR_ARG, "hb2_krylov_create: give exactly one preconditioner (matrix or vector)");
    if (A->dtype != HB2_F64 || (P && P->dtype != HB2_F64))
        return fail(HB2_ERR_UNSUPPORTED, "hb2_krylov_create: FP64 matrices only");
    if (A->rows != A->cols) return fail(HB2_ERR_SIZE, "hb2_krylov_create: MatrixIsNotSquare");
    if (P && (P->rows != A->rows || P->cols != A->rows))
        return fail(HB2_ERR_SIZE, "hb2_krylov_create: MatrixRowsDoNotMatch (preconditioner)");
    hb2_krylov_s * K = new hb2_krylov_s();
    K->method = method;
    cudaGetDevice(&K->device);
    K->A = A;
    K->P = P;
    K->n = A->rows;
    K->max_iters = max_iters;
    K->eps = eps;
    K->nvec = method == HB2_BICGSTAB_VAR ? 12 : 6;
    const uint64_t n = std::max<uint64_t>(K->n, 1);
    cudaError_t e = cudaMalloc(&K->vec, sizeof(double) * n * K->nvec);
    if (e == cudaSuccess) e = cudaMemsetAsync(K->vec, 0, sizeof(double) * n * K->nvec, stream);
    if (e == cudaSuccess) e = cudaMalloc(&K->st, sizeof(KState));
    if (e == cudaSuccess) e = cudaMemsetAsync(K->st, 0, sizeof(KState), stream);
    if (e == cudaSuccess) e = cudaMallocHost(&K->host_st, sizeof(KState));
    if (e == cudaSuccess && pdiag)
    {
        e = cudaMalloc(&K->pdiag, sizeof(double) * n);
        if (e == cudaSuccess) e = cudaMemcpyAsync(K->pdiag, pdiag, sizeof(double) * K->n, cudaMemcpyDefault, stream);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&K->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&K->cap2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&K->cap3, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) { krylov_free(K); return cuda_status(e, "hb2_krylov_create"); }
    int st = workspace_create(&K->ws, kMaxReduceBlocks);
    if (! st) st = build_graph(K);
    if (st) { krylov_free(K); return st; }
    *out = K;
    return HB2_OK;
}

extern "C" int hb2_krylov_destroy(hb2_krylov K)
{
    krylov_free(K);
    return HB2_OK;
}

extern "C" int hb2_krylov_solve(hb2_krylov K, const void * b, void * x, uint64_t * used_iters, double * final_defect,
                                cudaStream_t stream)
{
    if (! K || ! b || ! x) return fail(HB2_ERR_ARG, "hb2_krylov_solve: null argument");
    int st = launch_copy(HB2_F64, K->v(0), b, K->n, stream);
    if (! st) st = launch_copy(HB2_F64, K->v(1), x, K->n, stream);
    if (st) return st;
    HB2_CUDA(cudaGraphLaunch(K->exec, stream));
    st = launch_copy(HB2_F64, x, K->v(1), K->n, stream);
    if (st) return st;
    HB2_CUDA(cudaStreamSynchronize(stream));
    const KState & h = *K->host_st;
    uint64_t used;
    double defect;
    if (K->method == HB2_BICGSTAB_VAR)
    {
        used = h.iter + 1;            // math/bicgstab.hh:201
        defect = h.defnorm;           // squared, as the reference's Norm<vnt_l_two, false>
    }
    else if (K->method == HB2_CG_SMOOTHER)
    {
        used = h.iter;
        defect = 0.0;
    }
    else
    {
        used = h.used;
        defect = h.iter ? h.cur : h.init;
    }
    count_launches(K->prefix_kernels + (uint64_t)h.iter * K->body_kernels);
    if (used_iters) *used_iters = used;
    if (final_defect) *final_defect = defect;
    return HB2_OK;
}
