// The legacy multigrid solver Multigrid<Tag, OuterTag, methods::NONE, methods::JAC,
// methods::CYCLE::V, methods::FIXED> on BandedMatrixQx (math/multigrid.hh:151-466,
// 781-825), with its MGInfo configuration (math/multigrid.hh:65-149).
//
// The whole solve is one CUDA graph: the prefix (the initial guess with the
// right-hand side's Dirichlet values, the initial defect and its norm, the start
// test), a conditional WHILE node whose body is one V-cycle plus the defect norm
// and a one-thread decide kernel, and the copy of the solver state to the host.
// A cycle, level by level (the reference's restriction and prolongation loops):
//   finest level:  c = dinv (.) d, n_pre - 1 Jacobi sweeps on A c = d, x += c;
//   coarser levels: x = dinv (.) rhs, n_pre - 1 sweeps on A x = rhs;
//   then d = rhs - A x and rhs(coarser) = R d (matrix-free, Dirichlet mask);
//   coarsest level: the banded ConjugateGradients (math/conjugate_gradients.hh:491-560)
//     in one thread -- its dot products in the reference's sequential order;
//   upwards: c = P x(coarser), x += alpha c, n_pre Jacobi sweeps (the reference's
//     kernel uses n_pre_smooth for the post-smoothing too), d = rhs - A x.
// A Jacobi sweep is one fused banded kernel y = x + (rhs - A x) (.) dinv with the
// reference's rounding; every kernel but the finest norm is bit-identical to the
// reference, and the norm (a tree reduction) only decides when to stop.
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

using namespace hb2;

namespace
{
    struct LState
    {
        double d2;          // ||d||^2 of the finest level (this cycle)
        double defect, initial;
        unsigned long long cycles;
        int err;            // coarse CG step cap reached
        int bc;             // 1: value()'s initial guess (b's Dirichlet values), 0: x as given
        double dots[32][2]; // adaptive correction: <d, c>, <A c, c> per level
    };

    template <typename T>
    __global__ void k_bc_init(T * x, const T * x_in, const T * rhs, uint64_t n, uint64_t sq, const LState * st)
    {
        const bool bc = st ? st->bc != 0 : true;
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
            x[i] = (bc && (i < sq || i >= n - sq || i % sq == 0)) ? rhs[i] : x_in[i];
    }

    // out0 = <a, b>, out1 = <c, b> (the adaptive correction's two dots)
    template <typename T>
    __global__ void __launch_bounds__(256) k_dot2(const T * a, const T * b, const T * c, uint64_t n, ReduceSlot rs,
                                                  double * out)
    {
        __shared__ double scratch[32];
        double acc0 = 0.0, acc1 = 0.0;
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        {
            acc0 = fma((double)a[i], (double)b[i], acc0);
            acc1 = fma((double)c[i], (double)b[i], acc1);
        }
        const unsigned G = gridDim.x, ng = (G + kReduceGroup - 1) / kReduceGroup;
        double v = block_sum(acc0, scratch);
        sum_finish(v, rs.partials, rs.gpart, rs.ticket, G, blockIdx.x, out, 0, scratch);
        v = block_sum(acc1, scratch);
        sum_finish(v, rs.partials + G, rs.gpart + ng, rs.ticket + ng + 1, G, blockIdx.x, out + 1, 0, scratch);
    }

    // x = x + alpha c with alpha = <d, c> / <A c, c> in the vectors' type
    template <typename T>
    __global__ void k_axpy_adaptive(T * x, const T * c, const double * dots, uint64_t n)
    {
        const T alpha = Arith<T>::div((T)dots[0], (T)dots[1]);
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
            x[i] = Arith<T>::add(x[i], Arith<T>::mul(alpha, c[i]));
    }

    template <typename T>
    __global__ void k_eprod(T * out, const T * a, const T * b, uint64_t n)
    {
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
            out[i] = Arith<T>::mul(a[i], b[i]);
    }

    // x = x + alpha c (ScaledSum, alpha of the vectors' type; alpha == 1: Sum)
    template <typename T>
    __global__ void k_axpy(T * x, const T * c, T alpha, uint64_t n)
    {
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
            x[i] = Arith<T>::add(x[i], Arith<T>::mul(alpha, c[i]));
    }

    template <typename T>
    __global__ void __launch_bounds__(256) k_norm2(const T * d, uint64_t n, ReduceSlot rs, double * out)
    {
        __shared__ double scratch[32];
        double acc = 0.0;
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
            acc = fma((double)d[i], (double)d[i], acc);
        const double v = block_sum(acc, scratch);
        grid_sum_finish(v, rs, out, 0, scratch);
    }

    // ---- the banded ConjugateGradients, one thread ------------------------
    template <typename T>
    __device__ void seq_spmv(const T * bands, uint64_t n, uint64_t m, const T * x, T * y)
    {
        const int64_t N = (int64_t)n, r = (int64_t)m;
        const int64_t off[9] = {-r - 1, -r, -r + 1, -1, 0, 1, r - 1, r, r + 1};
        for (int64_t i = 0; i < N; ++i)
        {
            T s = Arith<T>::mul(bands[4 * N + i], x[i]);
            for (int b = 0; b < 9; ++b)
            {
                if (b == 4) continue;
                const int64_t j = i + off[b];
                if (j >= 0 && j < N) s = Arith<T>::add(s, Arith<T>::mul(bands[b * N + i], x[j]));
            }
            y[i] = s;
        }
    }
    template <typename T>
    __device__ T seq_dot(const T * x, const T * y, uint64_t n)
    {
        T s = T(0);
        for (uint64_t i = 0; i < n; ++i) s = Arith<T>::fma(x[i], y[i], s);
        return s;
    }
    template <typename T> struct Eps;
    template <> struct Eps<double> { static __device__ double v() { return DBL_EPSILON; } };
    template <> struct Eps<float> { static __device__ float v() { return FLT_EPSILON; } };

    // math/conjugate_gradients.hh:491-560 with the banded cg_kernel (:108-151); the
    // loop runs while ||x||^2 grows by more than konv_rad (at most `cap` steps)
    template <typename T>
    __global__ void k_coarse_cg(const T * bands, uint64_t n, uint64_t m, const T * rhs, T * x, T * g, T * u, T * e,
                                T * ng, double konv_rad, uint64_t cap, LState * st)
    {
        typedef Arith<T> M;
        const T eps = Eps<T>::v();
        for (uint64_t i = 0; i < n; ++i) x[i] = T(0);
        seq_spmv(bands, n, m, x, g);
        for (uint64_t i = 0; i < n; ++i) g[i] = M::sub(g[i], rhs[i]);
        for (uint64_t i = 0; i < n; ++i) u[i] = M::mul(g[i], T(-1));
        T norm_x = seq_dot(x, x, n), norm_x_last = M::sub(norm_x, T(1));
        uint64_t it = 0;
        while ((double)M::sub(norm_x, norm_x_last) > konv_rad)
        {
            if (it == cap) { st->err = 1; break; }
            T upper = seq_dot(g, g, n);
            seq_spmv(bands, n, m, u, e);
            T lower = seq_dot(e, u, n);
            T f = fabs(lower) >= eps ? M::div(upper, lower) : M::div(upper, eps);
            for (uint64_t i = 0; i < n; ++i) e[i] = M::add(M::mul(u[i], f), x[i]);
            lower = upper;
            seq_spmv(bands, n, m, e, ng);
            for (uint64_t i = 0; i < n; ++i) ng[i] = M::sub(ng[i], rhs[i]);
            upper = seq_dot(ng, ng, n);
            f = fabs(lower) >= eps ? M::div(upper, lower) : M::div(upper, eps);
            for (uint64_t i = 0; i < n; ++i) u[i] = M::sub(M::mul(u[i], f), ng[i]);
            for (uint64_t i = 0; i < n; ++i) { g[i] = ng[i]; x[i] = e[i]; }
            norm_x_last = norm_x;
            norm_x = seq_dot(x, x, n);
            ++it;
        }
    }

    // ---- control -----------------------------------------------------------
    template <typename T>
    __global__ void k_lmg_init(LState * st, uint64_t n_max_iter, int is_smoother, int convergence_check,
                               double tolerance, cudaGraphConditionalHandle h)
    {
        st->cycles = 0;
        st->err = 0;
        const T defect = is_smoother ? T(1e8) : (T)sqrt(st->d2);
        st->initial = (double)defect;
        st->defect = (double)defect;
        const bool nothing = convergence_check && defect <= (T)tolerance;
        cudaGraphSetConditional(h, (! nothing && n_max_iter > 0) ? 1u : 0u);
    }

    // math/multigrid.hh:443-460: after a cycle, stop when ||d|| <= initial * tolerance
    // (not in smoother mode), after n_max_iter cycles, or after the single cycle of a
    // one-level hierarchy
    template <typename T>
    __global__ void k_lmg_decide(LState * st, uint64_t n_max_iter, int is_smoother, int one_level, double tolerance,
                                 cudaGraphConditionalHandle h)
    {
        const unsigned long long c = st->cycles + 1;
        st->cycles = c;
        bool stop = one_level || c >= n_max_iter;
        if (! one_level && ! is_smoother)
        {
            const T defect = (T)sqrt(st->d2);
            st->defect = (double)defect;
            if (defect <= (T)st->initial * (T)tolerance) stop = true;
        }
        cudaGraphSetConditional(h, stop ? 0u : 1u);
    }

    uint32_t grid_of(uint64_t n) { return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 8ull * num_sms())); }

    // host sources of the bc flag copy (static storage: valid while a copy is in flight)
    const int kOne = 1, kZero = 0;
}

struct hb2_lmg_s
{
    int dtype;
    int device;
    unsigned lmin, lmax;
    hb2_lmg_params prm;
    struct Level
    {
        hb2_q1 A;
        uint64_t n, m;
        void * x, * c, * d, * rhs, * tmp, * dinv;
    };
    std::vector<Level> lev;          // index l - lmin
    void * xin = nullptr;            // initial guess (finest)
    void * cg = nullptr;             // 4 scratch vectors of the coarse CG
    void * block = nullptr;          // all level vectors
    LState * st = nullptr;
    LState * host_st = nullptr;
    Workspace * ws = nullptr;
    cudaStream_t cap = nullptr, cap2 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t prefix_kernels = 0, body_kernels = 0;
};

namespace
{
    template <typename T>
    int sweeps(hb2_lmg_s * G, hb2_lmg_s::Level & L, void * v, const void * rhs, uint64_t k, cudaStream_t s)
    {
        void * cur = v, * nxt = L.tmp;
        for (uint64_t i = 0; i < k; ++i)
        {
            int st = launch_q1(L.A, 2, cur, nxt, rhs, L.dinv, G->ws->error, s);
            if (st) return st;
            std::swap(cur, nxt);
        }
        if (cur != v) return launch_copy(G->dtype, v, cur, L.n, s);
        return HB2_OK;
    }

    template <typename T>
    int record_cycle(hb2_lmg_s * G, cudaStream_t s)
    {
        const unsigned nl = G->lmax - G->lmin + 1;
        const uint64_t npre = G->prm.n_pre_smooth;
        const T alpha = (T)G->prm.adapt_correction_factor;
        auto & C = G->lev[0];
        T * cgv = (T *)G->cg;
        const uint64_t nc = C.n;
        int st = HB2_OK;
        if (nl == 1)
        {
            k_coarse_cg<T><<<1, 1, 0, s>>>((const T *)C.A->bands, C.n, C.m, (const T *)C.d, (T *)C.x, cgv, cgv + nc,
                                           cgv + 2 * nc, cgv + 3 * nc, (double)std::numeric_limits<T>::epsilon(),
                                           100000, G->st);
            count_launches(1);
            HB2_LAUNCH_CHECK("lmg coarse cg");
            return launch_q1(C.A, 1, C.x, C.d, C.rhs, nullptr, G->ws->error, s);
        }
        for (int i = (int)nl - 1; i >= 1 && ! st; --i)
        {
            auto & L = G->lev[i];
            const uint32_t g = grid_of(L.n);
            if (i == (int)nl - 1)
            {
                k_eprod<T><<<g, 256, 0, s>>>((T *)L.c, (const T *)L.dinv, (const T *)L.d, L.n);
                count_launches(1);
                HB2_LAUNCH_CHECK("lmg jacobi start");
                st = sweeps<T>(G, L, L.c, L.d, npre - 1, s);
                if (st) break;
                k_axpy<T><<<g, 256, 0, s>>>((T *)L.x, (const T *)L.c, T(1), L.n);
                count_launches(1);
                HB2_LAUNCH_CHECK("lmg sum");
            }
            else
            {
                k_eprod<T><<<g, 256, 0, s>>>((T *)L.x, (const T *)L.dinv, (const T *)L.rhs, L.n);
                count_launches(1);
                HB2_LAUNCH_CHECK("lmg jacobi start");
                st = sweeps<T>(G, L, L.x, L.rhs, npre - 1, s);
                if (st) break;
            }
            st = launch_q1(L.A, 1, L.x, L.d, L.rhs, nullptr, G->ws->error, s);
            if (! st)
                st = hb2_restriction((hb2_dtype)G->dtype, G->lev[i - 1].rhs, G->lev[i - 1].n, L.d, L.n,
                                     G->prm.macro_border_mask, s);
        }
        if (st) return st;
        k_coarse_cg<T><<<1, 1, 0, s>>>((const T *)C.A->bands, C.n, C.m, (const T *)C.rhs, (T *)C.x, cgv, cgv + nc,
                                       cgv + 2 * nc, cgv + 3 * nc, (double)std::numeric_limits<T>::epsilon(), 100000,
                                       G->st);
        count_launches(1);
        HB2_LAUNCH_CHECK("lmg coarse cg");
        for (unsigned i = 1; i < nl && ! st; ++i)
        {
            auto & L = G->lev[i];
            st = hb2_prolongation((hb2_dtype)G->dtype, L.c, L.n, G->lev[i - 1].x, G->lev[i - 1].n,
                                  G->prm.macro_border_mask, s);
            if (st) break;
            if (G->prm.adaptive && G->prm.adapt_correction_factor == 0.0)
            {
                // math/multigrid.hh:1712-1721 (the MIXED kernel): alpha = <d, c> / <A c, c>
                double * dots = G->st->dots[G->lmin + i];
                st = launch_q1(L.A, 0, L.c, L.tmp, nullptr, nullptr, G->ws->error, s);
                if (st) break;
                k_dot2<T><<<grid_of(L.n), 256, 0, s>>>((const T *)L.d, (const T *)L.c, (const T *)L.tmp, L.n,
                                                       G->ws->slot(), dots);
                k_axpy_adaptive<T><<<grid_of(L.n), 256, 0, s>>>((T *)L.x, (const T *)L.c, dots, L.n);
                count_launches(2);
            }
            else
            {
                k_axpy<T><<<grid_of(L.n), 256, 0, s>>>((T *)L.x, (const T *)L.c, alpha, L.n);
                count_launches(1);
            }
            HB2_LAUNCH_CHECK("lmg correction");
            st = sweeps<T>(G, L, L.x, L.rhs, npre, s);
            if (! st) st = launch_q1(L.A, 1, L.x, L.d, L.rhs, nullptr, G->ws->error, s);
        }
        return st;
    }

    int capture_fail(hb2_lmg_s * G, cudaError_t e, const char * what)
    {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(G->cap2, &g);
        cudaStreamEndCapture(G->cap, &g);
        if (g) cudaGraphDestroy(g);
        return cuda_status(e == cudaSuccess ? cudaErrorUnknown : e, what);
    }

    template <typename T>
    int build_graph(hb2_lmg_s * G)
    {
        const uint64_t before = hb2_launch_count();
        auto & F = G->lev.back();
        const hb2_lmg_params & p = G->prm;
        HB2_CUDA(cudaStreamBeginCapture(G->cap, cudaStreamCaptureModeThreadLocal));
        cudaStreamCaptureStatus cs;
        cudaGraph_t capg = nullptr;
        const cudaGraphNode_t * deps = nullptr;
        size_t ndeps = 0;
        cudaError_t ce = cudaStreamGetCaptureInfo(G->cap, &cs, 0, &capg, &deps, &ndeps);
        if (ce != cudaSuccess) return capture_fail(G, ce, "cudaStreamGetCaptureInfo");
        cudaGraphConditionalHandle h;
        ce = cudaGraphConditionalHandleCreate(&h, capg, 0, 0);
        if (ce != cudaSuccess) return capture_fail(G, ce, "cudaGraphConditionalHandleCreate");
        // value(): the initial guess with b's values on the first row, the last row and
        // the first column; then d = b (initial_zero) or b - A x, and ||d||
        k_bc_init<T><<<grid_of(F.n), 256, 0, G->cap>>>((T *)F.x, (const T *)G->xin, (const T *)F.rhs, F.n, F.m, G->st);
        count_launches(1);
        int st;
        if (p.initial_zero) st = launch_copy(G->dtype, F.d, F.rhs, F.n, G->cap);
        else st = launch_q1(F.A, 1, F.x, F.d, F.rhs, nullptr, G->ws->error, G->cap);
        if (st) { capture_fail(G, cudaSuccess, ""); return st; }
        k_norm2<T><<<grid_of(F.n), 256, 0, G->cap>>>((const T *)F.d, F.n, G->ws->slot(), &G->st->d2);
        k_lmg_init<T><<<1, 1, 0, G->cap>>>(G->st, p.n_max_iter, p.is_smoother, p.convergence_check, p.tolerance, h);
        count_launches(2);
        ce = cudaGetLastError();
        if (ce == cudaSuccess) ce = cudaStreamGetCaptureInfo(G->cap, &cs, 0, &capg, &deps, &ndeps);
        if (ce != cudaSuccess) return capture_fail(G, ce, "capture (prefix)");
        G->prefix_kernels = hb2_launch_count() - before;
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        ce = cudaGraphAddNode(&cnode, capg, deps, ndeps, &cp);
        if (ce != cudaSuccess) return capture_fail(G, ce, "cudaGraphAddNode (while)");
        ce = cudaStreamUpdateCaptureDependencies(G->cap, &cnode, 1, cudaStreamSetCaptureDependencies);
        if (ce == cudaSuccess)
            ce = cudaStreamBeginCaptureToGraph(G->cap2, cp.conditional.phGraph_out[0], 0, 0, 0,
                                               cudaStreamCaptureModeThreadLocal);
        if (ce != cudaSuccess) return capture_fail(G, ce, "capture of the loop body");
        const uint64_t body0 = hb2_launch_count();
        st = record_cycle<T>(G, G->cap2);
        if (st) { capture_fail(G, cudaSuccess, ""); return st; }
        const bool one_level = G->lmin == G->lmax;
        if (! one_level && ! p.is_smoother)
        {
            k_norm2<T><<<grid_of(F.n), 256, 0, G->cap2>>>((const T *)F.d, F.n, G->ws->slot(), &G->st->d2);
            count_launches(1);
        }
        k_lmg_decide<T><<<1, 1, 0, G->cap2>>>(G->st, p.n_max_iter, p.is_smoother, one_level ? 1 : 0, p.tolerance, h);
        count_launches(1);
        ce = cudaGetLastError();
        if (ce != cudaSuccess) return capture_fail(G, ce, "capture (body)");
        G->body_kernels = hb2_launch_count() - body0;
        cudaGraph_t body = nullptr;
        ce = cudaStreamEndCapture(G->cap2, &body);
        if (ce != cudaSuccess) return capture_fail(G, ce, "cudaStreamEndCapture (body)");
        ce = cudaMemcpyAsync(G->host_st, G->st, sizeof(LState), cudaMemcpyDeviceToHost, G->cap);
        if (ce != cudaSuccess) return capture_fail(G, ce, "state copy");
        cudaGraph_t g = nullptr;
        ce = cudaStreamEndCapture(G->cap, &g);
        set_launch_count(before);
        if (ce != cudaSuccess) return cuda_status(ce, "cudaStreamEndCapture (lmg)");
        G->graph = g;
        ce = cudaGraphInstantiate(&G->exec, g, 0);
        if (ce != cudaSuccess) return cuda_status(ce, "cudaGraphInstantiate (lmg)");
        return HB2_OK;
    }

    // diags_inverted as the reference's tests build them: ElementInverse(DD) (0 stays 0),
    // then Scale by the double omega
    template <typename T>
    __global__ void k_dinv(T * dinv, const T * bands, uint64_t n, double omega)
    {
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        {
            const T dd = bands[4 * n + i];
            const T inv = dd == T(0) ? T(0) : Arith<T>::div(T(1), dd);
            // Scale<tags::CPU> with a double factor: the product formed in double
            dinv[i] = (T)__dmul_rn((double)inv, omega);
        }
    }

    void lmg_free(hb2_lmg_s * G)
    {
        if (! G) return;
        if (G->exec) cudaGraphExecDestroy(G->exec);
        if (G->graph) cudaGraphDestroy(G->graph);
        if (G->cap) cudaStreamDestroy(G->cap);
        if (G->cap2) cudaStreamDestroy(G->cap2);
        cudaFree(G->block);
        cudaFree(G->st);
        if (G->host_st) cudaFreeHost(G->host_st);
        workspace_destroy(G->ws);
        delete G;
    }
}

extern "C" int hb2_lmg_create(hb2_lmg * out, unsigned min_level, unsigned max_level, const hb2_q1 * A,
                              const hb2_lmg_params * params, cudaStream_t stream)
{
    if (! out || ! A || ! params) return fail(HB2_ERR_ARG, "hb2_lmg_create: null argument");
    *out = nullptr;
    if (min_level < 1 || max_level < min_level || max_level > 14) return fail(HB2_ERR_ARG, "hb2_lmg_create: levels");
    if (params->n_pre_smooth < 1) return fail(HB2_ERR_ARG, "hb2_lmg_create: n_pre_smooth must be at least 1");
    const unsigned nl = max_level - min_level + 1;
    for (unsigned i = 0; i < nl; ++i)
    {
        if (! A[i]) return fail(HB2_ERR_ARG, "hb2_lmg_create: null matrix");
        const uint64_t m = (1ULL << (min_level + i)) + 1;
        if (A[i]->n != m * m) return fail(HB2_ERR_SIZE, "hb2_lmg_create: matrix i must be of level min_level + i");
        if (A[i]->dtype != A[0]->dtype) return fail(HB2_ERR_ARG, "hb2_lmg_create: mixed element types");
    }
    hb2_lmg_s * G = new hb2_lmg_s();
    G->dtype = A[0]->dtype;
    cudaGetDevice(&G->device);
    G->lmin = min_level;
    G->lmax = max_level;
    G->prm = *params;
    const size_t es = dtype_size(G->dtype);
    uint64_t total = 0;
    G->lev.resize(nl);
    for (unsigned i = 0; i < nl; ++i)
    {
        G->lev[i].A = A[i];
        G->lev[i].n = A[i]->n;
        G->lev[i].m = A[i]->m;
        total += 6 * ((A[i]->n + 31) / 32 * 32);
    }
    const uint64_t nf = G->lev.back().n, nc = G->lev[0].n;
    total += (nf + 31) / 32 * 32 + 4 * ((nc + 31) / 32 * 32);
    cudaError_t e = cudaMalloc(&G->block, es * total);
    if (e == cudaSuccess) e = cudaMemsetAsync(G->block, 0, es * total, stream);
    if (e == cudaSuccess) e = cudaMalloc(&G->st, sizeof(LState));
    if (e == cudaSuccess) e = cudaMemsetAsync(G->st, 0, sizeof(LState), stream);
    if (e == cudaSuccess) e = cudaMallocHost(&G->host_st, sizeof(LState));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&G->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&G->cap2, cudaStreamNonBlocking);
    if (e != cudaSuccess) { lmg_free(G); return cuda_status(e, "hb2_lmg_create"); }
    char * p = (char *)G->block;
    auto take = [&](uint64_t n) { void * q = p; p += es * ((n + 31) / 32 * 32); return q; };
    for (auto & L : G->lev)
    {
        L.x = take(L.n); L.c = take(L.n); L.d = take(L.n); L.rhs = take(L.n); L.tmp = take(L.n); L.dinv = take(L.n);
        if (G->dtype == HB2_F64)
            k_dinv<double><<<grid_of(L.n), 256, 0, stream>>>((double *)L.dinv, (const double *)L.A->bands, L.n,
                                                              params->omega);
        else
            k_dinv<float><<<grid_of(L.n), 256, 0, stream>>>((float *)L.dinv, (const float *)L.A->bands, L.n,
                                                             params->omega);
        count_launches(1);
    }
    G->xin = take(nf);
    G->cg = take(4 * nc);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) { lmg_free(G); return cuda_status(e, "hb2_lmg_create (setup)"); }
    int st = workspace_create(&G->ws, kMaxReduceBlocks);
    if (! st) st = G->dtype == HB2_F64 ? build_graph<double>(G) : build_graph<float>(G);
    if (st) { lmg_free(G); return st; }
    *out = G;
    return HB2_OK;
}

extern "C" int hb2_lmg_destroy(hb2_lmg G)
{
    lmg_free(G);
    return HB2_OK;
}

namespace
{
    // one run of the graph: bc = 1 applies value()'s initial guess, 0 runs the kernel
    // on x as given (the MIXED driver's persistent inner iterate)
    int lmg_run(hb2_lmg G, const void * b, void * x, int bc, uint64_t * cycles, double * defect, cudaStream_t stream);
}

extern "C" int hb2_lmg_solve(hb2_lmg G, const void * b, void * x, uint64_t * cycles, double * defect,
                             cudaStream_t stream)
{
    if (! G || ! b || ! x) return fail(HB2_ERR_ARG, "hb2_lmg_solve: null argument");
    return lmg_run(G, b, x, 1, cycles, defect, stream);
}

namespace
{
    __global__ void k_res_update(double * res, const float * xi, double scale, uint64_t n)
    {
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
            res[i] = __dadd_rn(res[i], __dmul_rn(scale, (double)xi[i]));
    }
    __global__ void k_scale64(double * v, double a, uint64_t n)
    {
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
            v[i] = __dmul_rn(v[i], a);
    }
    __global__ void k_to_f32(float * o, const double * v, uint64_t n)
    {
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
            o[i] = (float)v[i];
    }

    double host_norm(hb2_lmg G, const double * v, uint64_t n, cudaStream_t stream, int * st)
    {
        double * out = &G->st->dots[0][0];
        k_norm2<double><<<grid_of(n), 256, 0, stream>>>(v, n, G->ws->slot(), out);
        count_launches(1);
        double h = 0;
        cudaError_t e = cudaMemcpyAsync(&h, out, sizeof(double), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) *st = cuda_status(e, "hb2_lmg_solve_mixed (norm)");
        return sqrt(h);
    }
}

extern "C" int hb2_lmg_solve_mixed(hb2_lmg G, hb2_q1 A, const void * b, void * x, uint64_t max_outer,
                                   uint64_t * outer_steps, uint64_t * inner_cycles, double * final_defect,
                                   cudaStream_t stream)
{
    if (! G || ! A || ! b || ! x) return fail(HB2_ERR_ARG, "hb2_lmg_solve_mixed: null argument");
    if (G->dtype != HB2_F32 || A->dtype != HB2_F64)
        return fail(HB2_ERR_ARG, "hb2_lmg_solve_mixed: an F32 hierarchy and an F64 matrix");
    auto & F = G->lev.back();
    if (A->n != F.n) return fail(HB2_ERR_SIZE, "hb2_lmg_solve_mixed: MatrixRowsDoNotMatch (finest level)");
    const uint64_t n = F.n;
    double * buf = nullptr;
    // ig, od, res (F64), then two 256-byte aligned F32 vectors padded to 64 elements
    const size_t bytes = 3 * n * sizeof(double) + 256 + 2 * ((n + 63) / 64 * 64) * sizeof(float);
    HB2_CUDA(cudaMallocAsync((void **)&buf, bytes, stream));
    double * ig = buf, * od = buf + n, * res = buf + 2 * n;
    float * x32 = (float *)(((uintptr_t)(buf + 3 * n) + 255) & ~(uintptr_t)255);
    float * r32 = x32 + ((n + 63) / 64) * 64;
    const uint32_t g = grid_of(n);
    int st = HB2_OK;
    uint64_t outer = 0, inner = 0;
    double def = 0.0;
    // value(): the initial guess with b's Dirichlet values; the inner iterate starts at it
    k_bc_init<double><<<g, 256, 0, stream>>>(ig, (const double *)x, (const double *)b, n, F.m, nullptr);
    k_to_f32<<<g, 256, 0, stream>>>(x32, ig, n);
    cudaError_t ce = cudaMemsetAsync(res, 0, n * sizeof(double), stream);
    count_launches(2);
    if (ce != cudaSuccess) st = cuda_status(ce, "hb2_lmg_solve_mixed");
    if (! st) st = launch_q1(A, 1, ig, od, b, nullptr, G->ws->error, stream);
    const double initial = st ? 0.0 : host_norm(G, od, n, stream, &st);
    const double outer_eps = (double)(float)G->prm.tolerance;
    double scale = 1.0;
    while (! st && outer < max_outer)
    {
        k_to_f32<<<g, 256, 0, stream>>>(r32, od, n);
        count_launches(1);
        uint64_t c = 0;
        st = lmg_run(G, r32, x32, 0, &c, nullptr, stream);
        if (st) break;
        inner += c;
        ++outer;
        k_res_update<<<g, 256, 0, stream>>>(res, x32, scale, n);
        count_launches(1);
        st = launch_q1(A, 1, res, od, b, nullptr, G->ws->error, stream);
        if (st) break;
        def = host_norm(G, od, n, stream, &st);
        if (st || def < outer_eps * initial) break;
        scale = def;
        k_scale64<<<g, 256, 0, stream>>>(od, 1.0 / scale, n);
        count_launches(1);
    }
    if (! st) st = launch_copy(HB2_F64, x, res, n, stream);
    cudaFreeAsync(buf, stream);
    ce = cudaStreamSynchronize(stream);
    if (! st && ce != cudaSuccess) st = cuda_status(ce, "hb2_lmg_solve_mixed");
    if (outer_steps) *outer_steps = outer;
    if (inner_cycles) *inner_cycles = inner;
    if (final_defect) *final_defect = def;
    if (! st && outer == max_outer && ! (def < outer_eps * initial))
        return fail(HB2_ERR_NOT_FINITE, "hb2_lmg_solve_mixed: no convergence within max_outer steps");
    return st;
}

namespace
{
int lmg_run(hb2_lmg G, const void * b, void * x, int bc, uint64_t * cycles, double * defect, cudaStream_t stream)
{
    auto & F = G->lev.back();
    int st = launch_copy(G->dtype, F.rhs, b, F.n, stream);
    if (! st) st = launch_copy(G->dtype, G->xin, x, F.n, stream);
    if (st) return st;
    HB2_CUDA(cudaMemcpyAsync(&G->st->bc, bc ? &kOne : &kZero, sizeof(int), cudaMemcpyHostToDevice, stream));
    HB2_CUDA(cudaGraphLaunch(G->exec, stream));
    st = launch_copy(G->dtype, x, F.x, F.n, stream);
    if (st) return st;
    HB2_CUDA(cudaStreamSynchronize(stream));
    const LState & h = *G->host_st;
    count_launches(G->prefix_kernels + h.cycles * G->body_kernels);
    if (cycles) *cycles = h.cycles;
    if (defect) *defect = h.defect;
    int err = 0;
    HB2_CUDA(cudaMemcpy(&err, G->ws->error, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return fail(HB2_ERR_TIMEOUT, "hb2_lmg_solve: a banded kernel's copy wait expired");
    if (h.err) return fail(HB2_ERR_TIMEOUT, "hb2_lmg_solve: the coarse CG reached its step cap");
    return HB2_OK;
}
}
