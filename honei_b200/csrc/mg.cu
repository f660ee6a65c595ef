// Geometric multigrid on the device: MGData + MGCycleCreation<V::STATIC,
// CGSolver<NONE>, RISmoother, Restriction<PROLMAT>, Prolongation<PROLMAT>>
// (math/mg.hh:57-240, 567-656), MGSolver (math/mg.hh:1094-1127) and IRSolver
// (math/ir.hh:31-80).
//
// The reference walks a vector of virtual Operator objects per cycle, each a
// tag-dispatched call (math/operator_list.hh:69-76).  Here the same operator
// sequence is recorded once into a CUDA graph with fused kernels:
//   smoother sweep  = Defect + ElementProduct + Sum     -> one Jacobi pass
//   Defect + Restriction + Fill(c = 0)                  -> defect pass + restrict pass
//   Prolongation + Sum                                  -> one SpMV-add pass
//   coarsest CGSolver                                   -> one thread block, shared memory
//   convergence Defect + Norm                           -> one pass
// and the MGSolver loop itself runs on the device: the solve graph is the
// initial defect, a conditional WHILE node whose body is one V-cycle plus the
// convergence defect and a one-thread decision kernel, and the copy of the
// statistics to pinned host memory -- one graph launch and one host
// synchronisation per solve.  Each kernel is bit-identical to the
// reference's operator; with coarse_exact the coarse CG is too, so the MG
// iterates match the reference's tags::CPU solver bit for bit.
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace hb2
{
    struct MgLevel
    {
        hb2_ell_s * A = 0;
        hb2_ell_s * P = 0;   // prolongation from the next coarser level (levels > 0)
        hb2_ell_s * R = 0;   // restriction to the next coarser level
        uint64_t n = 0;
        void * x = 0;        // finest: solution; coarser: c
        void * b = 0;        // finest: rhs; coarser: d
        void * store = 0;
        void * tmp = 0;      // Jacobi ping-pong
        void * jac = 0;      // omega / diag(A)
        int keep = 0;        // kKeepL2 when the level's working set is near the L2 size
        bool rev_A = false, rev_R = false, rev_P = false;   // direction of the next pass

        int pass(bool & rev)
        {
            int f = keep | (rev ? kReverse : 0);
            rev = ! rev;
            return f;
        }
    };
}

struct hb2_mg_s
{
    int dtype;
    int device;
    uint32_t nlev;
    std::vector<hb2::MgLevel> lev;
    hb2_mg_params prm;
    bool owns_matrices;
    hb2::Workspace * ws;
    void * vec_block;        // one allocation for all level vectors
    void * rfine;            // finest-level defect
    cudaStream_t cap, cap2;
    cudaGraph_t graph;       // one V-cycle + convergence defect (hb2_mg_cycle)
    cudaGraphExec_t exec;
    uint64_t graph_kernels;
    cudaGraph_t solve_graph; // the whole MGSolver loop
    cudaGraphExec_t solve_exec;
    uint64_t body_kernels;
    double * norm_dev;       // sqrt(r.r) after the cycle
    uint64_t * coarse_used_dev;
    double * coarse_def_dev;
    double * r0_dev;         // sqrt(r0.r0)
    uint64_t * iters_dev;    // cycles done
    int sub_top;             // levels 1..sub_top run as cluster kernels (-1: none)
    int sub_t1;              // of those, levels 1..sub_t1 run in one CTA
    bool sub_fused;          // levels 0..sub_top, coarse CG included, in one launch
    hb2_ell_s * coarse64;    // FP64 copy of the coarsest operator (F32 hierarchies with coarse_fp64)
    double * ir_r;           // outer FP64 defect of hb2_ir_solve (allocated on first use, kept)
    // hb2_ir_solve as one CUDA graph, built for the outer operator and vectors of
    // the last call (rebuilt when any of them or the loop parameters change)
    cudaStream_t cap3 = 0, cap4 = 0;
    cudaGraph_t ir_graph = 0;
    cudaGraphExec_t ir_exec = 0;
    const void * ir_key_A = 0, * ir_key_b = 0, * ir_key_x = 0;
    double ir_key_eps = 0;
    uint64_t ir_key_max = 0;
    int ir_key_reset = -1;
    uint64_t ir_body_kernels = 0, ir_inner_body_kernels = 0;
    // The convergence test's norm ||b - A x|| fused into the next cycle's first
    // finest-level Jacobi sweep, which computes that defect anyway (fused_norm: the
    // finest level outside the cluster kernels, at least one pre-smoothing sweep):
    // the loop body is that sweep with its norm, the decision, and the rest of the
    // cycle under a conditional IF node.  When the loop stops, x is the last cycle's
    // (the sweep wrote the other Jacobi buffer).  One finest-level defect pass less
    // per cycle, one discarded sweep per solve.  The host loop runs the two parts as
    // graphs of their own.  Off by default (HB2_MG_FUSED_NORM=1 turns it on): measured
    // on B200 the second conditional node per cycle costs about what the defect pass
    // saves (level 9 +5 us, level 10 +2 us, level 11 -6 us per cycle).
    bool fused_norm = false;
    cudaGraph_t first_graph = 0, rest_graph = 0;
    cudaGraphExec_t first_exec = 0, rest_exec = 0;
    uint64_t pro_kernels = 0, first_kernels = 0, rest_kernels = 0;
    uint64_t ir_first_kernels = 0, ir_rest_kernels = 0;
};

namespace hb2
{
    static uint64_t env_u64(const char * name, uint64_t dflt)
    {
        const char * v = getenv(name);
        return v && *v ? strtoull(v, 0, 10) : dflt;
    }

    // `sweeps` Jacobi sweeps on level L; done = 1: the first one already ran (x -> tmp)
    static int smooth(hb2_mg_s * mg, MgLevel & L, uint64_t sweeps, cudaStream_t s, uint64_t done = 0)
    {
        void * cur = done ? L.tmp : L.x, * nxt = done ? L.x : L.tmp;
        for (uint64_t k = done; k < sweeps; ++k)
        {
            int st = launch_ell(L.A, kJacobi, cur, nxt, L.b, L.jac, 0, 0, 0, mg->ws, s, L.pass(L.rev_A));
            if (st) return st;
            std::swap(cur, nxt);
        }
        if (cur != L.x) return launch_copy(mg->dtype, L.x, cur, L.n, s);
        return HB2_OK;
    }

    // the coarsest-level CG (math/mg.hh:585-594); FP64 arithmetic for an FP32
    // hierarchy when coarse_fp64 is set
    static int coarse_solve(hb2_mg_s * mg, cudaStream_t s)
    {
        MgLevel & C = mg->lev[0];
        if (mg->coarse64)
            return launch_cg_small_f32io(mg->coarse64, C.b, C.x, mg->prm.max_iters_coarse, mg->prm.coarse_eps,
                                         mg->prm.coarse_exact, mg->coarse_used_dev, mg->coarse_def_dev, s);
        return launch_cg_small(C.A, C.b, C.x, mg->prm.max_iters_coarse, mg->prm.coarse_eps, mg->prm.coarse_exact,
                               mg->coarse_used_dev, mg->coarse_def_dev, s);
    }

    // levels 0..sub_top: down leg (cluster kernel), coarse CG, up leg (cluster kernel)
    static int record_small_levels(hb2_mg_s * mg, cudaStream_t s)
    {
        SubLevelDesc d[16];
        for (int i = 0; i <= mg->sub_top; ++i)
        {
            MgLevel & L = mg->lev[i];
            d[i].A = L.A;
            d[i].R = L.R;
            d[i].P = L.P;
            d[i].x = L.x;
            d[i].b = L.b;
            d[i].store = L.store;
            d[i].tmp = L.tmp;
            d[i].jac = L.jac;
        }
        if (mg->sub_fused)
            return launch_subvcycle(mg->dtype, d, mg->sub_top, mg->sub_t1, (int)mg->prm.n_pre_smooth,
                                    (int)mg->prm.n_post_smooth, mg->lev[0].A, mg->coarse64, mg->prm.max_iters_coarse,
                                    mg->prm.coarse_eps, mg->prm.coarse_exact, mg->coarse_used_dev, mg->coarse_def_dev, s);
        int st = launch_subcycle(mg->dtype, d, mg->sub_top, mg->sub_t1, (int)mg->prm.n_pre_smooth,
                                 (int)mg->prm.n_post_smooth, true, s);
        if (! st) st = coarse_solve(mg, s);
        if (! st) st = launch_subcycle(mg->dtype, d, mg->sub_top, mg->sub_t1, (int)mg->prm.n_pre_smooth,
                                       (int)mg->prm.n_post_smooth, false, s);
        return st;
    }

    // MGCycleCreation::_build_cycle (math/mg.hh:577-640); first_done: the level's
    // first pre-smoothing sweep already ran (the fused loop)
    static int record_cycle(hb2_mg_s * mg, uint32_t i, cudaStream_t s, bool first_done = false)
    {
        MgLevel & L = mg->lev[i];
        if ((int)i == mg->sub_top) return record_small_levels(mg, s);
        if (i == 0) return coarse_solve(mg, s);
        MgLevel & C = mg->lev[i - 1];
        int st = smooth(mg, L, mg->prm.n_pre_smooth, s, first_done ? 1 : 0);
        if (! st) st = launch_ell(L.A, kDefect, L.x, L.store, L.b, 0, 0, 0, 0, mg->ws, s, L.pass(L.rev_A));
        if (! st) st = launch_ell(L.R, kRestrict, L.store, C.b, 0, 0, C.x, 0, 0, mg->ws, s, L.pass(L.rev_R));
        if (! st) st = record_cycle(mg, i - 1, s);
        // W-cycle (math/mg.hh:720-722): the coarser level's cycle twice, except
        // directly above the coarsest level
        if (! st && mg->prm.cycle == 1 && i - 1 != 0) st = record_cycle(mg, i - 1, s);
        if (! st) st = launch_ell(L.P, kAdd, C.x, L.x, 0, 0, 0, 0, 0, mg->ws, s, L.pass(L.rev_P));
        if (! st) st = smooth(mg, L, mg->prm.n_post_smooth, s);
        return st;
    }

    static int finest_norm(hb2_mg_s * mg, cudaStream_t s)
    {
        MgLevel & F = mg->lev[mg->nlev - 1];
        return launch_ell(F.A, kDefect, F.x, mg->rfine, F.b, 0, 0, mg->norm_dev, 1, mg->ws, s, F.pass(F.rev_A));
    }

    // the fused loop's first part: the finest level's first pre-smoothing sweep
    // (x -> tmp) with the norm of its defect b - A x into norm_dev
    static int first_sweep_norm(hb2_mg_s * mg, cudaStream_t s)
    {
        MgLevel & F = mg->lev[mg->nlev - 1];
        return launch_ell(F.A, kJacobi, F.x, F.tmp, F.b, F.jac, 0, mg->norm_dev, 1, mg->ws, s, F.pass(F.rev_A));
    }

    static void reset_directions(hb2_mg_s * mg)
    {
        for (MgLevel & L : mg->lev) L.rev_A = L.rev_R = L.rev_P = false;
    }

    // MGSolver loop control (math/mg.hh:1109-1121): after each cycle, stop when
    // ||r|| < eps ||r0|| or max_iters cycles are done (also on a NaN norm).
    __global__ void mg_loop_init_kernel(uint64_t * iters, uint64_t max_iters, cudaGraphConditionalHandle h)
    {
        *iters = 0;
        cudaGraphSetConditional(h, max_iters > 0 ? 1u : 0u);
    }

    __global__ void mg_loop_decide_kernel(const double * norm, const double * r0, uint64_t * iters, uint64_t max_iters,
                                          double eps, cudaGraphConditionalHandle h)
    {
        pdl_entry();
        const uint64_t it = *iters + 1;
        *iters = it;
        const double rc = *norm;
        const bool stop = rc < eps * *r0 || ! (rc == rc) || it >= max_iters;
        cudaGraphSetConditional(h, stop ? 0u : 1u);
    }

    // the fused loop's decision, after the first sweep of the cycle that would be
    // number k + 1 (k = cycles done): for k >= 1 the sweep's norm is ||b - A x|| after
    // cycle k, and the stop test of mg_loop_decide_kernel applies to it; k = 0 always
    // runs (the loop is entered only when max_iters > 0).  Sets both the IF node over
    // the rest of the cycle and the loop's WHILE node.
    __global__ void mg_loop_decide_pre_kernel(const double * norm, const double * r0, uint64_t * iters,
                                              uint64_t max_iters, double eps, cudaGraphConditionalHandle hw,
                                              cudaGraphConditionalHandle hif)
    {
        pdl_entry();
        const uint64_t k = *iters;
        const double rc = *norm;
        const bool run = k == 0 || ! (rc < eps * *r0 || ! (rc == rc) || k >= max_iters);
        if (run) *iters = k + 1;
        cudaGraphSetConditional(hif, run ? 1u : 0u);
        cudaGraphSetConditional(hw, run ? 1u : 0u);
    }

    static int capture_error(cudaError_t e, const char * what, hb2_mg_s * mg)
    {
        cudaGraph_t g = 0;
        if (mg->cap3) { cudaStreamEndCapture(mg->cap3, &g); if (g) { cudaGraphDestroy(g); g = 0; } }
        cudaStreamEndCapture(mg->cap2, &g);
        if (g) { cudaGraphDestroy(g); g = 0; }
        cudaStreamEndCapture(mg->cap, &g);
        if (g) cudaGraphDestroy(g);
        return cuda_status(e, what);
    }

    static cudaError_t new_handle(cudaStream_t s, cudaGraphConditionalHandle * h);
    static cudaError_t add_conditional(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType t,
                                       cudaGraph_t * body);

    // the fused loop body on `s` (capturing into the WHILE node's body graph, handle
    // hw): first sweep + norm, decision, IF (rest of the cycle), the IF body captured
    // on mg->cap3; the kernel counts of the two parts into *first / *rest
    static int record_fused_body(hb2_mg_s * mg, cudaStream_t s, cudaGraphConditionalHandle hw, uint64_t * first,
                                 uint64_t * rest)
    {
        if (! mg->cap3) HB2_CUDA(cudaStreamCreateWithFlags(&mg->cap3, cudaStreamNonBlocking));
        const uint64_t c0 = hb2_launch_count();
        int st = first_sweep_norm(mg, s);
        if (st) return st;
        cudaGraphConditionalHandle hif;
        cudaError_t e = new_handle(s, &hif);
        if (e != cudaSuccess) return cuda_status(e, "MG loop: IF handle");
        launch_pdl(mg_loop_decide_pre_kernel, dim3(1), dim3(1), 0, s, mg->norm_dev, mg->r0_dev, mg->iters_dev,
                   mg->prm.max_iters, mg->prm.eps_relative, hw, hif);
        count_launches(1);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_status(e, "MG loop: decide kernel");
        *first = hb2_launch_count() - c0;
        cudaGraph_t ifbody = 0;
        e = add_conditional(s, hif, cudaGraphCondTypeIf, &ifbody);
        if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(mg->cap3, ifbody, 0, 0, 0, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_status(e, "MG loop: IF node");
        const uint64_t c1 = hb2_launch_count();
        st = record_cycle(mg, mg->nlev - 1, mg->cap3, true);
        *rest = hb2_launch_count() - c1;
        cudaGraph_t g = ifbody;
        e = cudaStreamEndCapture(mg->cap3, &g);
        if (st) return st;
        if (e != cudaSuccess) return cuda_status(e, "MG loop: IF body");
        return HB2_OK;
    }

    static int build_solve_graph(hb2_mg_s * mg)
    {
        MgLevel & F = mg->lev[mg->nlev - 1];
        HB2_CUDA(cudaStreamBeginCapture(mg->cap, cudaStreamCaptureModeThreadLocal));
        const uint64_t before = hb2_launch_count();
        cudaStreamCaptureStatus cs;
        cudaGraph_t capg = 0;
        const cudaGraphNode_t * deps = 0;
        size_t ndeps = 0;
        cudaError_t e = cudaStreamGetCaptureInfo(mg->cap, &cs, 0, &capg, &deps, &ndeps);
        if (e != cudaSuccess) return capture_error(e, "cudaStreamGetCaptureInfo", mg);
        cudaGraphConditionalHandle h;
        e = cudaGraphConditionalHandleCreate(&h, capg, 1, cudaGraphCondAssignDefault);
        if (e != cudaSuccess) return capture_error(e, "cudaGraphConditionalHandleCreate", mg);
        reset_directions(mg);
        int st = launch_ell(F.A, kDefect, F.x, mg->rfine, F.b, 0, 0, mg->r0_dev, 1, mg->ws, mg->cap, F.pass(F.rev_A));
        if (st) { capture_error(cudaSuccess, "", mg); return st; }
        mg_loop_init_kernel<<<1, 1, 0, mg->cap>>>(mg->iters_dev, mg->prm.max_iters, h);
        count_launches(1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(mg->cap, &cs, 0, &capg, &deps, &ndeps);
        if (e != cudaSuccess) return capture_error(e, "capture (loop init)", mg);
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        e = cudaGraphAddNode(&cnode, capg, deps, ndeps, &cp);
        if (e != cudaSuccess) return capture_error(e, "cudaGraphAddNode (while)", mg);
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        e = cudaStreamUpdateCaptureDependencies(mg->cap, &cnode, 1, cudaStreamSetCaptureDependencies);
        if (e == cudaSuccess)
            e = cudaStreamBeginCaptureToGraph(mg->cap2, body, 0, 0, 0, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return capture_error(e, "capture of the loop body", mg);
        mg->pro_kernels = hb2_launch_count() - before;
        const uint64_t body0 = hb2_launch_count();
        if (mg->fused_norm)
        {
            st = record_fused_body(mg, mg->cap2, h, &mg->first_kernels, &mg->rest_kernels);
            if (st) { capture_error(cudaSuccess, "", mg); return st; }
        }
        else
        {
            st = record_cycle(mg, mg->nlev - 1, mg->cap2);
            if (! st) st = finest_norm(mg, mg->cap2);
            if (! st)
            {
                launch_pdl(mg_loop_decide_kernel, dim3(1), dim3(1), 0, mg->cap2, mg->norm_dev, mg->r0_dev,
                           mg->iters_dev, mg->prm.max_iters, mg->prm.eps_relative, h);
                count_launches(1);
                e = cudaGetLastError();
                if (e != cudaSuccess) return capture_error(e, "decide kernel", mg);
            }
            if (st) { capture_error(cudaSuccess, "", mg); return st; }
        }
        mg->body_kernels = hb2_launch_count() - body0;
        e = cudaStreamEndCapture(mg->cap2, &body);
        if (e != cudaSuccess) return capture_error(e, "cudaStreamEndCapture (body)", mg);
        // statistics: norm, coarse iterations, coarse defect, r0, iterations
        e = cudaMemcpyAsync(mg->ws->host_scalars, mg->ws->scalars, 5 * sizeof(double), cudaMemcpyDeviceToHost, mg->cap);
        if (e != cudaSuccess) return capture_error(e, "stats copy", mg);
        cudaGraph_t g = 0;
        e = cudaStreamEndCapture(mg->cap, &g);
        set_launch_count(before);
        if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture (solve)");
        mg->solve_graph = g;
        e = cudaGraphInstantiate(&mg->solve_exec, g, 0);
        if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate (solve)");
        return HB2_OK;
    }

    static int build_graph(hb2_mg_s * mg)
    {
        HB2_CUDA(cudaStreamBeginCapture(mg->cap, cudaStreamCaptureModeThreadLocal));
        uint64_t before = hb2_launch_count();
        reset_directions(mg);
        int st = record_cycle(mg, mg->nlev - 1, mg->cap);
        if (! st) st = finest_norm(mg, mg->cap);
        if (! st)
        {
            cudaError_t e = cudaMemcpyAsync(mg->ws->host_scalars, mg->norm_dev, sizeof(double), cudaMemcpyDeviceToHost, mg->cap);
            if (e != cudaSuccess) st = cuda_status(e, "capture D2H");
        }
        cudaGraph_t g = 0;
        cudaError_t e = cudaStreamEndCapture(mg->cap, &g);
        if (st) { if (g) cudaGraphDestroy(g); return st; }
        if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
        mg->graph_kernels = hb2_launch_count() - before;
        set_launch_count(before);
        mg->graph = g;
        e = cudaGraphInstantiate(&mg->exec, g, 0);
        if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate");
        if (! mg->fused_norm) return HB2_OK;
        // the fused loop on the host: (first sweep + norm, its copy to the host) and
        // (the rest of the cycle) as two graphs, the pass directions continuing from
        // one to the other as in the device loop's body
        reset_directions(mg);
        HB2_CUDA(cudaStreamBeginCapture(mg->cap, cudaStreamCaptureModeThreadLocal));
        st = first_sweep_norm(mg, mg->cap);
        if (! st)
        {
            e = cudaMemcpyAsync(mg->ws->host_scalars, mg->norm_dev, sizeof(double), cudaMemcpyDeviceToHost, mg->cap);
            if (e != cudaSuccess) st = cuda_status(e, "capture D2H");
        }
        g = 0;
        e = cudaStreamEndCapture(mg->cap, &g);
        if (st) { if (g) cudaGraphDestroy(g); set_launch_count(before); return st; }
        if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture (first sweep)");
        mg->first_graph = g;
        HB2_CUDA(cudaStreamBeginCapture(mg->cap, cudaStreamCaptureModeThreadLocal));
        st = record_cycle(mg, mg->nlev - 1, mg->cap, true);
        g = 0;
        e = cudaStreamEndCapture(mg->cap, &g);
        set_launch_count(before);
        if (st) { if (g) cudaGraphDestroy(g); return st; }
        if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture (rest of the cycle)");
        mg->rest_graph = g;
        e = cudaGraphInstantiate(&mg->first_exec, mg->first_graph, 0);
        if (e == cudaSuccess) e = cudaGraphInstantiate(&mg->rest_exec, mg->rest_graph, 0);
        if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate (fused loop)");
        return HB2_OK;
    }

    static int mg_alloc(hb2_mg_s * mg, cudaStream_t stream)
    {
        const size_t es = dtype_size(mg->dtype);
        size_t total = 0;
        for (uint32_t i = 0; i < mg->nlev; ++i) total += 5 * ((mg->lev[i].n * es + 255) / 256 * 256);
        total += (mg->lev[mg->nlev - 1].n * es + 255) / 256 * 256;
        HB2_CUDA(cudaMalloc(&mg->vec_block, total));
        HB2_CUDA(cudaMemsetAsync(mg->vec_block, 0, total, stream));
        char * p = (char *)mg->vec_block;
        for (uint32_t i = 0; i < mg->nlev; ++i)
        {
            size_t sz = (mg->lev[i].n * es + 255) / 256 * 256;
            MgLevel & L = mg->lev[i];
            L.x = p; p += sz;
            L.b = p; p += sz;
            L.store = p; p += sz;
            L.tmp = p; p += sz;
            L.jac = p; p += sz;
            int st = hb2_jacobi_precon(L.A, mg->prm.omega, L.jac, stream);
            if (st) return st;
        }
        mg->rfine = p;
        // L2 policy per level: keep the matrix stream in L2 when the level's
        // working set (matrix + five vectors) is at most twice the L2 size
        int l2 = 0;
        cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, mg->device);
        if (l2 <= 0) l2 = 126 << 20;
        for (uint32_t i = 0; i < mg->nlev; ++i)
        {
            MgLevel & L = mg->lev[i];
            uint64_t ws_bytes = L.A->bytes + 5 * L.n * es;
            L.keep = ws_bytes <= 2ull * (uint64_t)l2 ? kKeepL2 : 0;
        }
        int st = workspace_create(&mg->ws, kMaxReduceBlocks);
        if (st) return st;
        mg->norm_dev = mg->ws->scalars + 0;
        mg->coarse_used_dev = (uint64_t *)(mg->ws->scalars + 1);
        mg->coarse_def_dev = mg->ws->scalars + 2;
        mg->r0_dev = mg->ws->scalars + 3;
        mg->iters_dev = (uint64_t *)(mg->ws->scalars + 4);
        HB2_CUDA(cudaStreamCreateWithFlags(&mg->cap, cudaStreamNonBlocking));
        HB2_CUDA(cudaStreamCreateWithFlags(&mg->cap2, cudaStreamNonBlocking));
        return HB2_OK;
    }

    static int mg_finish_create(hb2_mg_s * mg, cudaStream_t stream)
    {
        int st = mg_alloc(mg, stream);
        if (st) return st;
        // the small levels (at most kSubMaxRows rows, above the coarsest) run as
        // cluster kernels unless disabled
        // (HB2_SUB_MAX_ROWS / HB2_SUB_LOCAL_ROWS override the two row limits;
        // HB2_SUB_FUSED=1 runs the small levels and the coarse CG as one launch,
        // measured slower on B200 than down / coarse CG / up as three)
        mg->sub_top = -1;
        mg->sub_t1 = 0;
        const uint64_t max_rows = env_u64("HB2_SUB_MAX_ROWS", kSubMaxRows);
        const uint64_t local_rows = env_u64("HB2_SUB_LOCAL_ROWS", kSubLocalRows);
        if (! mg->prm.no_fused_levels && mg->prm.cycle == 0 && mg->prm.n_pre_smooth < (1u << 20) &&
            mg->prm.n_post_smooth < (1u << 20))
            for (uint32_t i = 1; i < mg->nlev && i < 10; ++i)
                if (mg->lev[i].n <= max_rows) mg->sub_top = (int)i;
        if (mg->sub_top >= 1)
        {
            for (int i = 1; i <= mg->sub_top; ++i)
            {
                if (mg->lev[i].n <= local_rows) mg->sub_t1 = i;
                st = ell_small_patterns(mg->lev[i].A);
                if (st) return st;
            }
            st = subcycle_prepare();
            if (st) return st;
        }
        if (mg->dtype == HB2_F32 && mg->prm.coarse_fp64)
        {
            hb2_ell c64 = 0;
            st = hb2_ell_convert(&c64, mg->lev[0].A, HB2_F64, stream);
            if (st) return st;
            mg->coarse64 = c64;
            if (! cg_mixed_supported(c64)) return fail(HB2_ERR_UNSUPPORTED, "coarse_fp64: the coarsest level needs <= 128 rows and 1-9 slots");
            HB2_CUDA(cudaStreamSynchronize(stream));
        }
        HB2_CUDA(cudaStreamSynchronize(stream));
        mg->fused_norm = mg->nlev >= 2 && mg->sub_top < (int)mg->nlev - 1 && mg->prm.n_pre_smooth >= 1 &&
                         env_u64("HB2_MG_FUSED_NORM", 0) != 0;
        mg->sub_fused = mg->sub_top >= 1 && env_u64("HB2_SUB_FUSED", 0) != 0 &&
                        subvcycle_supported(mg->lev[0].A, mg->coarse64);
        // prime the coarse kernel's shared-memory attribute outside the capture
        MgLevel & C = mg->lev[0];
        st = launch_cg_small(C.A, C.b, C.x, 0, mg->prm.coarse_eps, mg->prm.coarse_exact, mg->coarse_used_dev,
                             mg->coarse_def_dev, mg->cap);
        if (st) return st;
        HB2_CUDA(cudaStreamSynchronize(mg->cap));
        st = build_graph(mg);
        if (! st) st = build_solve_graph(mg);
        return st;
    }

    static hb2_mg_params default_params()
    {
        hb2_mg_params p;
        p.n_pre_smooth = 4;
        p.n_post_smooth = 4;
        p.max_iters = 100;
        p.max_iters_coarse = 100;
        p.eps_relative = 1e-10;
        p.coarse_eps = 1e-10;
        p.omega = 0.7;
        p.coarse_exact = 1;
        p.no_fused_levels = 0;
        p.coarse_fp64 = 0;
        p.cycle = 0;
        return p;
    }

    static int validate(uint32_t nlev, const hb2_ell * A, const hb2_ell * prol, const hb2_ell * res)
    {
        if (nlev < 1 || ! A) return fail(HB2_ERR_ARG, "hb2_mg_create: no levels");
        for (uint32_t i = 0; i < nlev; ++i)
        {
            if (! A[i] || A[i]->rows != A[i]->cols) return fail(HB2_ERR_SIZE, "hb2_mg_create: level matrix not square");
            if (A[i]->dtype != A[0]->dtype) return fail(HB2_ERR_ARG, "hb2_mg_create: mixed element types");
            if (i > 0)
            {
                const hb2_ell_s * P = prol[i - 1], * R = res[i - 1];
                if (! P || ! R) return fail(HB2_ERR_ARG, "hb2_mg_create: missing transfer matrix");
                if (P->rows != A[i]->rows || P->cols != A[i - 1]->rows || R->rows != A[i - 1]->rows || R->cols != A[i]->rows)
                    return fail(HB2_ERR_SIZE, "hb2_mg_create: MatrixRowsDoNotMatch (transfer vs level sizes)");
                if (P->dtype != A[0]->dtype || R->dtype != A[0]->dtype) return fail(HB2_ERR_ARG, "hb2_mg_create: mixed element types");
            }
        }
        if (! cg_small_fits(A[0])) return fail(HB2_ERR_UNSUPPORTED, "hb2_mg_create: coarsest level too large for the one-block CG");
        return HB2_OK;
    }

    // The same solve with the loop on the host: one launch of the plain cycle
    // graph per V-cycle and a synchronisation to read its norm.  Identical
    // kernels and results; selected with HB2_MG_LOOP=host, for profilers that
    // do not descend into conditional graph bodies.
    static int solve_host_loop(hb2_mg_s * mg, double * stats, cudaStream_t stream)
    {
        MgLevel & F = mg->lev[mg->nlev - 1];
        int st = launch_ell(F.A, kDefect, F.x, mg->rfine, F.b, 0, 0, mg->norm_dev, 1, mg->ws, stream);
        if (st) return st;
        HB2_CUDA(cudaMemcpyAsync(mg->ws->host_scalars, mg->norm_dev, sizeof(double), cudaMemcpyDeviceToHost, stream));
        HB2_CUDA(cudaStreamSynchronize(stream));
        const double r0 = mg->ws->host_scalars[0];
        double rc = 1e16;
        uint64_t used = 0;
        if (mg->fused_norm)
        {
            // the device loop's steps: first sweep + norm, decision, rest of the cycle
            for (uint64_t k = 0; mg->prm.max_iters > 0; ++k)
            {
                HB2_CUDA(cudaGraphLaunch(mg->first_exec, stream));
                count_launches(mg->first_kernels - 1);
                HB2_CUDA(cudaStreamSynchronize(stream));
                rc = mg->ws->host_scalars[0];
                if (k > 0 && (rc < mg->prm.eps_relative * r0 || ! (rc == rc) || k >= mg->prm.max_iters)) break;
                HB2_CUDA(cudaGraphLaunch(mg->rest_exec, stream));
                count_launches(mg->rest_kernels);
                used = k + 1;
            }
        }
        else
            for (uint64_t i = 0; i < mg->prm.max_iters; ++i)
            {
                HB2_CUDA(cudaGraphLaunch(mg->exec, stream));
                count_launches(mg->graph_kernels);
                HB2_CUDA(cudaStreamSynchronize(stream));
                rc = mg->ws->host_scalars[0];
                used = i + 1;
                if (rc < mg->prm.eps_relative * r0 || ! (rc == rc)) break;
            }
        if (stats)
        {
            uint64_t cu = 0;
            HB2_CUDA(cudaMemcpy(&cu, mg->coarse_used_dev, sizeof(uint64_t), cudaMemcpyDeviceToHost));
            stats[0] = (double)used;
            stats[1] = r0;
            stats[2] = rc;
            stats[3] = (double)cu;
        }
        if (! (rc == rc) || ! (r0 == r0)) return fail(HB2_ERR_NOT_FINITE, "MG solve: NaN defect norm");
        return HB2_OK;
    }

    static bool host_loop_requested()
    {
        const char * v = getenv("HB2_MG_LOOP");
        return v && strcmp(v, "host") == 0;
    }

    // MGSolver::value on the hierarchy's own finest vectors (b, x already in
    // place): one launch of the solve graph, one synchronisation.
    static int solve_internal(hb2_mg_s * mg, double * stats, cudaStream_t stream)
    {
        if (host_loop_requested()) return solve_host_loop(mg, stats, stream);
        HB2_CUDA(cudaGraphLaunch(mg->solve_exec, stream));
        HB2_CUDA(cudaStreamSynchronize(stream));
        const double * h = mg->ws->host_scalars;
        uint64_t used = 0, cu = 0;
        memcpy(&used, h + 4, sizeof(uint64_t));
        memcpy(&cu, h + 1, sizeof(uint64_t));
        const double r0 = h[3], rc = used ? h[0] : 1e16;
        if (! mg->fused_norm) count_launches(mg->pro_kernels + used * mg->body_kernels);
        else if (mg->prm.max_iters > 0)
            count_launches(mg->pro_kernels + (used + 1) * mg->first_kernels + used * mg->rest_kernels);
        else count_launches(mg->pro_kernels);
        if (stats)
        {
            stats[0] = (double)used;
            stats[1] = r0;
            stats[2] = rc;
            stats[3] = (double)cu;
        }
        if (! (rc == rc) || ! (r0 == r0)) return fail(HB2_ERR_NOT_FINITE, "MG solve: NaN defect norm");
        return HB2_OK;
    }
}

namespace hb2
{
    // IRSolver loop control (math/ir.hh:55-75) on the device.  Scalars (the
    // inner hierarchy's workspace): [16] ||r0||, [17] ||r|| at the last check,
    // [18] outer index i, [19] last checked i, [20] inner cycles in all.
    __global__ void ir_loop_init_kernel(double * sc, uint64_t max_iters, cudaGraphConditionalHandle h)
    {
        sc[17] = 1e16;
        uint64_t * u = (uint64_t *)sc;
        u[18] = 0;
        u[19] = 0;
        u[20] = 0;
        cudaGraphSetConditional(h, max_iters > 0 ? 1u : 0u);
    }

    // after an inner solve, the update and the next defect: i += 1; the defect of
    // index i is checked only while i < max_iters (the reference's loop runs its
    // i-th defect at the top of iteration i)
    __global__ void ir_loop_decide_kernel(double * sc, const double * norm, const uint64_t * inner_iters,
                                          uint64_t max_iters, double eps, cudaGraphConditionalHandle h)
    {
        pdl_entry();
        uint64_t * u = (uint64_t *)sc;
        const uint64_t i = u[18] + 1;
        u[18] = i;
        u[20] += *inner_iters;
        bool stop = i >= max_iters;
        if (! stop)
        {
            const double rc = *norm;
            sc[17] = rc;
            u[19] = i;
            stop = rc < eps * sc[16] || ! (rc == rc);
        }
        cudaGraphSetConditional(h, stop ? 0u : 1u);
    }

    // a conditional handle in the graph `s` is capturing into
    static cudaError_t new_handle(cudaStream_t s, cudaGraphConditionalHandle * h)
    {
        cudaStreamCaptureStatus cs;
        cudaGraph_t capg = 0;
        const cudaGraphNode_t * deps = 0;
        size_t ndeps = 0;
        cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, 0, &capg, &deps, &ndeps);
        if (e != cudaSuccess) return e;
        return cudaGraphConditionalHandleCreate(h, capg, 0, cudaGraphCondAssignDefault);
    }

    // a conditional node (WHILE or IF) on handle h at the capture position of `s`:
    // returns its body graph and makes the node `s`'s dependency
    static cudaError_t add_conditional(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType t,
                                       cudaGraph_t * body)
    {
        cudaStreamCaptureStatus cs;
        cudaGraph_t capg = 0;
        const cudaGraphNode_t * deps = 0;
        size_t ndeps = 0;
        cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, 0, &capg, &deps, &ndeps);
        if (e != cudaSuccess) return e;
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = h;
        cp.conditional.type = t;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        e = cudaGraphAddNode(&node, capg, deps, ndeps, &cp);
        if (e != cudaSuccess) return e;
        *body = cp.conditional.phGraph_out[0];
        return cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
    }

    static cudaError_t add_while(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraph_t * body)
    {
        return add_conditional(s, h, cudaGraphCondTypeWhile, body);
    }

    static int ir_capture_error(cudaError_t e, const char * what, hb2_mg_s * mg, int st = HB2_OK)
    {
        cudaGraph_t g = 0;
        if (mg->cap4) { cudaStreamEndCapture(mg->cap4, &g); if (g) { cudaGraphDestroy(g); g = 0; } }
        cudaStreamEndCapture(mg->cap3, &g);
        if (g) { cudaGraphDestroy(g); g = 0; }
        cudaStreamEndCapture(mg->cap2, &g);
        if (g) { cudaGraphDestroy(g); g = 0; }
        cudaStreamEndCapture(mg->cap, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (st) return st;
        return cuda_status(e == cudaSuccess ? cudaErrorUnknown : e, what);
    }

    // The whole IRSolver (math/ir.hh:31-80) as one graph:
    //   outer defect (FP64; fused: its FP32 copy into the inner rhs, the inner guess
    //   cleared when reset_inner, ||r0||)
    //   WHILE (outer):
    //     inner MGSolver: its initial defect, WHILE (inner): V-cycle, norm, decide
    //     x += (double) inner x
    //     outer defect (fused as above), decide
    //   statistics to pinned host memory
    static int build_ir_graph(hb2_mg_s * mg, const hb2_ell_s * A, const double * b, double * x, double eps,
                              uint64_t max_iters, int reset_inner)
    {
        if (mg->ir_exec) { cudaGraphExecDestroy(mg->ir_exec); mg->ir_exec = 0; }
        if (mg->ir_graph) { cudaGraphDestroy(mg->ir_graph); mg->ir_graph = 0; }
        if (! mg->cap3) HB2_CUDA(cudaStreamCreateWithFlags(&mg->cap3, cudaStreamNonBlocking));
        if (! mg->ir_r) HB2_CUDA(cudaMalloc(&mg->ir_r, A->rows * 8 + 16));
        MgLevel & F = mg->lev[mg->nlev - 1];
        double * sc = mg->ws->scalars;
        float * b32 = (float *)F.b, * x32 = reset_inner ? (float *)F.x : nullptr;
        const uint64_t before = hb2_launch_count();
        HB2_CUDA(cudaStreamBeginCapture(mg->cap, cudaStreamCaptureModeThreadLocal));
        cudaGraphConditionalHandle ho, hi;
        cudaGraph_t obody = 0, ibody = 0;
        reset_directions(mg);
        cudaError_t e = new_handle(mg->cap, &ho);
        if (e != cudaSuccess) return ir_capture_error(e, "IR outer handle", mg);
        ir_loop_init_kernel<<<1, 1, 0, mg->cap>>>(sc, max_iters, ho);
        count_launches(1);
        int st = launch_ir_defect(A, x, b, b32, x32, mg->ir_r, sc + 16, mg->ws, mg->cap);
        if (st) return ir_capture_error(cudaSuccess, "", mg, st);
        e = add_while(mg->cap, ho, &obody);
        if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(mg->cap2, obody, 0, 0, 0, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return ir_capture_error(e, "IR outer loop", mg);
        const uint64_t obody0 = hb2_launch_count();
        // the inner MGSolver on (F.b, F.x)
        st = launch_ell(F.A, kDefect, F.x, mg->rfine, F.b, 0, 0, mg->r0_dev, 1, mg->ws, mg->cap2, F.pass(F.rev_A));
        if (st) return ir_capture_error(cudaSuccess, "", mg, st);
        e = new_handle(mg->cap2, &hi);
        if (e != cudaSuccess) return ir_capture_error(e, "IR inner handle", mg);
        mg_loop_init_kernel<<<1, 1, 0, mg->cap2>>>(mg->iters_dev, mg->prm.max_iters, hi);
        count_launches(1);
        e = add_while(mg->cap2, hi, &ibody);
        if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(mg->cap3, ibody, 0, 0, 0, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return ir_capture_error(e, "IR inner loop", mg);
        const uint64_t ibody0 = hb2_launch_count();
        if (mg->fused_norm)
        {
            // the inner body captured on cap3, its IF body on cap4
            if (! mg->cap4) HB2_CUDA(cudaStreamCreateWithFlags(&mg->cap4, cudaStreamNonBlocking));
            std::swap(mg->cap3, mg->cap4);
            st = record_fused_body(mg, mg->cap4, hi, &mg->ir_first_kernels, &mg->ir_rest_kernels);
            std::swap(mg->cap3, mg->cap4);
            if (st) return ir_capture_error(cudaSuccess, "", mg, st);
        }
        else
        {
            st = record_cycle(mg, mg->nlev - 1, mg->cap3);
            if (! st) st = finest_norm(mg, mg->cap3);
            if (st) return ir_capture_error(cudaSuccess, "", mg, st);
            launch_pdl(mg_loop_decide_kernel, dim3(1), dim3(1), 0, mg->cap3, mg->norm_dev, mg->r0_dev, mg->iters_dev,
                       mg->prm.max_iters, mg->prm.eps_relative, hi);
            count_launches(1);
            e = cudaGetLastError();
            if (e != cudaSuccess) return ir_capture_error(e, "IR inner decide", mg);
        }
        mg->ir_inner_body_kernels = hb2_launch_count() - ibody0;
        e = cudaStreamEndCapture(mg->cap3, &ibody);
        if (e != cudaSuccess) return ir_capture_error(e, "IR inner body", mg);
        // x += (double) inner x; the next outer defect; the decision
        st = launch_add_converted(x, mg->dtype, F.x, F.n, mg->cap2);
        if (! st) st = launch_ir_defect(A, x, b, b32, x32, mg->ir_r, sc + 21, mg->ws, mg->cap2);
        if (st) return ir_capture_error(cudaSuccess, "", mg, st);
        launch_pdl(ir_loop_decide_kernel, dim3(1), dim3(1), 0, mg->cap2, sc, (const double *)(sc + 21),
                   (const uint64_t *)mg->iters_dev, max_iters, eps, ho);
        count_launches(1);
        e = cudaGetLastError();
        if (e != cudaSuccess) return ir_capture_error(e, "IR decide", mg);
        mg->ir_body_kernels = hb2_launch_count() - obody0 - mg->ir_inner_body_kernels;
        e = cudaStreamEndCapture(mg->cap2, &obody);
        if (e != cudaSuccess) return ir_capture_error(e, "IR outer body", mg);
        e = cudaMemcpyAsync(mg->ws->host_scalars + 16, sc + 16, 5 * sizeof(double), cudaMemcpyDeviceToHost, mg->cap);
        if (e != cudaSuccess) return ir_capture_error(e, "IR statistics copy", mg);
        cudaGraph_t g = 0;
        e = cudaStreamEndCapture(mg->cap, &g);
        set_launch_count(before);
        if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture (IR)");
        mg->ir_graph = g;
        e = cudaGraphInstantiate(&mg->ir_exec, g, 0);
        if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate (IR)");
        mg->ir_key_A = A;
        mg->ir_key_b = b;
        mg->ir_key_x = x;
        mg->ir_key_eps = eps;
        mg->ir_key_max = max_iters;
        mg->ir_key_reset = reset_inner;
        return HB2_OK;
    }
}

using namespace hb2;

extern "C" int hb2_mg_create(hb2_mg * out, uint32_t num_levels, const hb2_ell * A, const hb2_ell * prol,
                             const hb2_ell * res, const hb2_mg_params * params, cudaStream_t stream)
{
    if (! out) return fail(HB2_ERR_ARG, "hb2_mg_create: null output");
    int st = validate(num_levels, A, prol, res);
    if (st) return st;
    if (params && (params->cycle < 0 || params->cycle > 1)) return fail(HB2_ERR_ARG, "hb2_mg_create: cycle must be 0 (V) or 1 (W)");
    hb2_mg_s * mg = new hb2_mg_s();
    mg->dtype = A[0]->dtype;
    cudaGetDevice(&mg->device);
    mg->nlev = num_levels;
    mg->prm = params ? *params : default_params();
    mg->owns_matrices = false;
    mg->lev.resize(num_levels);
    for (uint32_t i = 0; i < num_levels; ++i)
    {
        mg->lev[i].A = A[i];
        mg->lev[i].n = A[i]->rows;
        if (i > 0) { mg->lev[i].P = prol[i - 1]; mg->lev[i].R = res[i - 1]; }
    }
    st = mg_finish_create(mg, stream);
    if (st) { hb2_mg_destroy(mg); return st; }
    *out = mg;
    return HB2_OK;
}

extern "C" int hb2_mg_create_q1(hb2_mg * out, hb2_dtype dtype, unsigned min_level, unsigned max_level, double aniso,
                                const hb2_mg_params * params, cudaStream_t stream)
{
    if (! out || min_level < 1 || max_level < min_level || max_level > 14) return fail(HB2_ERR_ARG, "hb2_mg_create_q1: bad levels");
    const uint32_t nlev = max_level - min_level + 1;
    std::vector<hb2_ell> A(nlev, (hb2_ell)0), P(nlev, (hb2_ell)0), R(nlev, (hb2_ell)0);
    int st = HB2_OK;
    for (uint32_t i = 0; i < nlev && ! st; ++i)
    {
        st = hb2_ell_create_q1(&A[i], dtype, min_level + i, aniso, stream);
        if (! st && i > 0) st = hb2_ell_create_transfer(&P[i - 1], &R[i - 1], dtype, min_level + i, stream);
    }
    hb2_mg mg = 0;
    if (! st) st = hb2_mg_create(&mg, nlev, A.data(), P.data(), R.data(), params, stream);
    if (st)
    {
        for (uint32_t i = 0; i < nlev; ++i) { hb2_ell_destroy(A[i]); hb2_ell_destroy(P[i]); hb2_ell_destroy(R[i]); }
        return st;
    }
    mg->owns_matrices = true;
    *out = mg;
    return HB2_OK;
}

extern "C" int hb2_mg_destroy(hb2_mg mg)
{
    if (! mg) return HB2_OK;
    if (mg->exec) cudaGraphExecDestroy(mg->exec);
    if (mg->graph) cudaGraphDestroy(mg->graph);
    if (mg->solve_exec) cudaGraphExecDestroy(mg->solve_exec);
    if (mg->solve_graph) cudaGraphDestroy(mg->solve_graph);
    if (mg->cap) cudaStreamDestroy(mg->cap);
    if (mg->cap2) cudaStreamDestroy(mg->cap2);
    if (mg->ir_exec) cudaGraphExecDestroy(mg->ir_exec);
    if (mg->ir_graph) cudaGraphDestroy(mg->ir_graph);
    if (mg->cap3) cudaStreamDestroy(mg->cap3);
    if (mg->cap4) cudaStreamDestroy(mg->cap4);
    if (mg->first_exec) cudaGraphExecDestroy(mg->first_exec);
    if (mg->rest_exec) cudaGraphExecDestroy(mg->rest_exec);
    if (mg->first_graph) cudaGraphDestroy(mg->first_graph);
    if (mg->rest_graph) cudaGraphDestroy(mg->rest_graph);
    if (mg->coarse64) hb2_ell_destroy(mg->coarse64);
    if (mg->ir_r) cudaFree(mg->ir_r);
    if (mg->vec_block) cudaFree(mg->vec_block);
    workspace_destroy(mg->ws);
    if (mg->owns_matrices)
        for (uint32_t i = 0; i < mg->nlev; ++i)
        {
            hb2_ell_destroy(mg->lev[i].A);
            hb2_ell_destroy(mg->lev[i].P);
            hb2_ell_destroy(mg->lev[i].R);
        }
    delete mg;
    return HB2_OK;
}

extern "C" int hb2_mg_solve(hb2_mg mg, const void * b, void * x, double * stats, cudaStream_t stream)
{
    if (! mg || ! b || ! x) return fail(HB2_ERR_ARG, "hb2_mg_solve: null argument");
    MgLevel & F = mg->lev[mg->nlev - 1];
    int st = launch_copy(mg->dtype, F.b, b, F.n, stream);
    if (! st) st = launch_copy(mg->dtype, F.x, x, F.n, stream);
    if (st) return st;
    int solve_st = solve_internal(mg, stats, stream);
    st = launch_copy(mg->dtype, x, F.x, F.n, stream);
    if (! st) { cudaError_t e = cudaStreamSynchronize(stream); if (e != cudaSuccess) st = cuda_status(e, "hb2_mg_solve"); }
    return solve_st ? solve_st : st;
}

extern "C" int hb2_mg_cycle(hb2_mg mg, const void * b, void * x, cudaStream_t stream)
{
    if (! mg || ! b || ! x) return fail(HB2_ERR_ARG, "hb2_mg_cycle: null argument");
    MgLevel & F = mg->lev[mg->nlev - 1];
    int st = launch_copy(mg->dtype, F.b, b, F.n, stream);
    if (! st) st = launch_copy(mg->dtype, F.x, x, F.n, stream);
    if (st) return st;
    HB2_CUDA(cudaGraphLaunch(mg->exec, stream));
    count_launches(mg->graph_kernels);
    return launch_copy(mg->dtype, x, F.x, F.n, stream);
}

extern "C" int hb2_ir_solve(hb2_ell A, hb2_mg inner, const void * b, void * x, double eps, uint64_t max_iters,
                            int reset_inner, double * stats, cudaStream_t stream)
{
    if (! A || ! inner || ! b || ! x) return fail(HB2_ERR_ARG, "hb2_ir_solve: null argument");
    if (A->dtype != HB2_F64) return fail(HB2_ERR_ARG, "hb2_ir_solve: the outer system must be F64");
    MgLevel & F = inner->lev[inner->nlev - 1];
    if (F.n != A->rows || A->rows != A->cols) return fail(HB2_ERR_SIZE, "hb2_ir_solve: VectorSizeDoesNotMatch (inner finest level)");
    const char * loop = getenv("HB2_IR_LOOP");
    if (! (loop && strcmp(loop, "host") == 0) && ! host_loop_requested())
    {
        // the whole solve as one graph launch and one synchronisation
        if (! inner->ir_exec || inner->ir_key_A != A || inner->ir_key_b != b || inner->ir_key_x != x ||
            inner->ir_key_eps != eps || inner->ir_key_max != max_iters || inner->ir_key_reset != reset_inner)
        {
            int st = build_ir_graph(inner, A, (const double *)b, (double *)x, eps, max_iters, reset_inner);
            if (st) return st;
        }
        HB2_CUDA(cudaGraphLaunch(inner->ir_exec, stream));
        HB2_CUDA(cudaStreamSynchronize(stream));
        const double * h = inner->ws->host_scalars + 16;
        uint64_t outer = 0, used = 0, inner_total = 0;
        memcpy(&outer, h + 2, sizeof(uint64_t));
        memcpy(&used, h + 3, sizeof(uint64_t));
        memcpy(&inner_total, h + 4, sizeof(uint64_t));
        count_launches(3 + outer * inner->ir_body_kernels + inner_total * inner->ir_inner_body_kernels);
        const double r0 = h[0], rc = used ? h[1] : 1e16;
        if (stats)
        {
            stats[0] = (double)used;
            stats[1] = r0;
            stats[2] = rc;
            stats[3] = (double)inner_total;
        }
        if (! (rc == rc) || ! (r0 == r0)) return fail(HB2_ERR_NOT_FINITE, "hb2_ir_solve: NaN defect norm");
        return HB2_OK;
    }
    Workspace * ws = 0;
    int st = stream_workspace(stream, &ws);
    if (st) return st;
    if (! inner->ir_r) HB2_CUDA(cudaMalloc(&inner->ir_r, A->rows * 8 + 16));
    void * r = inner->ir_r;
    double r0 = 1e16, rc = 1e16;
    uint64_t used = 0, inner_total = 0;
    for (uint64_t i = 0; i < max_iters && ! st; ++i)
    {
        // Defect<OuterTag>(r, b, A, x) with the norm fused in
        st = launch_ell(A, kDefect, x, r, b, 0, 0, ws->scalars + 16, 1, ws, stream);
        if (st) break;
        cudaError_t e = cudaMemcpyAsync(ws->host_scalars + 16, ws->scalars + 16, sizeof(double), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) { st = cuda_status(e, "hb2_ir_solve"); break; }
        const double nr = ws->host_scalars[16];
        if (i == 0) r0 = nr;
        else
        {
            rc = nr;
            used = i;
            if (rc < eps * r0) break;
            if (! (rc == rc)) break;
        }
        // convert<OuterTag>(inner b, r); inner MGSolver; convert + Sum
        st = launch_convert(inner->dtype, F.b, HB2_F64, r, F.n, stream);
        if (! st && reset_inner) st = launch_fill(inner->dtype, F.x, 0.0, F.n, stream);
        double ist[4] = {0, 0, 0, 0};
        if (! st) st = solve_internal(inner, ist, stream);
        inner_total += (uint64_t)ist[0];
        if (! st) st = launch_add_converted(x, inner->dtype, F.x, F.n, stream);
    }
    cudaError_t e = cudaStreamSynchronize(stream);
    if (! st && e != cudaSuccess) st = cuda_status(e, "hb2_ir_solve");
    if (stats)
    {
        stats[0] = (double)used;
        stats[1] = r0;
        stats[2] = rc;
        stats[3] = (double)inner_total;
    }
    if (! st && ! (rc == rc)) st = fail(HB2_ERR_NOT_FINITE, "hb2_ir_solve: NaN defect norm");
    return st;
}
