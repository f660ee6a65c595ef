// hb2_defect_ell_noalloc: the fused defect + squared-norm pass without any
// device allocation.
//
// hb2_defect_ell reduces ||r||^2 through per-block partial sums and a ticket
// counter that live in a workspace the library allocates with cudaMalloc the
// first time a stream is used.  Some callers cannot allow that allocation:
// code that runs under a hard device-memory budget where every byte is
// reserved up front, or a latency-critical loop where a cudaMalloc would stall
// the device.  This entry point keeps the reduction scratch in a fixed
// file-scope device array instead, so it allocates nothing.
//
// Limits and sharing:
//  * the scratch holds kNoAllocMaxBlocks block partials, so the matrix may have
//    at most kNoAllocMaxBlocks * 512 rows in FP64 (8,388,608) and
//    kNoAllocMaxBlocks * 1024 rows in FP32 (16,777,216); larger matrices are
//    rejected with HB2_ERR_UNSUPPORTED before anything is launched.  The
//    decision depends on the row count and element type only: where the
//    matrix's tuned layout would need more row blocks than that, the kernel
//    runs on the same layout with more rows per thread (same defect bits);
//  * every GPU that loads the library holds the array (about 134 KiB) until the
//    process exits;
//  * all calls on a device share the one array: calls whose kernels overlap on
//    the GPU (different streams without ordering between them) race on it and
//    give wrong norms.  Calls ordered on one stream are safe;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make that
//    first call before any stream capture on that device.
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <mutex>

namespace hb2
{
    constexpr uint32_t kNoAllocMaxBlocks = 16384;
    constexpr int kNoAllocMaxDevices = 64;

    // Layout (in doubles): [0, kNoAllocMaxBlocks) block partials, then
    // kNoAllocGroups group partials, then kNoAllocGroups + 1 ticket counters.
    constexpr uint32_t kNoAllocGroups = kNoAllocMaxBlocks / kReduceGroup;
    constexpr uint32_t kNoAllocTicketDoubles = (kNoAllocGroups + 1 + 1) / 2 + 1;
    static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxBlocks + kNoAllocGroups + kNoAllocTicketDoubles];

    static std::mutex g_noalloc_mutex;
    static void * g_noalloc_addr[kNoAllocMaxDevices];

    // Device address of g_noalloc_scratch on the current device.  In host code
    // the symbol's name is only a host-side stand-in, never a device address.
    static int noalloc_scratch(double ** out)
    {
        int dev = 0;
        HB2_CUDA(cudaGetDevice(&dev));
        if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(HB2_ERR_UNSUPPORTED, "hb2_defect_ell_noalloc: device ordinal out of range");
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (! g_noalloc_addr[dev])
        {
            void * p = 0;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return cuda_status(e, "hb2_defect_ell_noalloc: cudaGetSymbolAddress");
            g_noalloc_addr[dev] = p;
        }
        *out = (double *)g_noalloc_addr[dev];
        return HB2_OK;
    }
}

using namespace hb2;

extern "C" int hb2_defect_ell_noalloc(hb2_ell A, const void * rhs, const void * x, void * r, double * norm2_dev,
                                      cudaStream_t stream)
{
    if (! A || ! norm2_dev) return fail(HB2_ERR_ARG, "hb2_defect_ell_noalloc: null matrix or norm output");
    if (A->rows != A->cols) return fail(HB2_ERR_SIZE, "hb2_defect_ell_noalloc: VectorSizeDoesNotMatch (rhs vs columns)");
    if (A->rows > 0 && (! rhs || ! x || ! r)) return fail(HB2_ERR_ARG, "hb2_defect_ell_noalloc: null vector");
    // at most max_rows rows (512 per scratch partial in FP64, 1024 in FP32): the
    // only condition, so the answer depends on the row count and element type
    // alone, never on the layout the autotuner picked for this matrix
    const uint64_t rows_per_block = (uint64_t)kEllThreads *
                                    (A->dtype == HB2_F64 ? RowsPerThread<double>::value : RowsPerThread<float>::value);
    const uint64_t max_rows = (uint64_t)kNoAllocMaxBlocks * rows_per_block;
    if (A->rows > max_rows)
        return fail(HB2_ERR_UNSUPPORTED, "hb2_defect_ell_noalloc: " + std::to_string(A->rows) +
                    " rows exceed the static scratch limit of " + std::to_string(max_rows) +
                    " rows for this element type; use hb2_defect_ell");
    // The kernel runs on the matrix's tuned layout, in blocks of 256 threads,
    // unless that layout's row blocks outnumber the scratch partials (the row-pattern layout at one row
    // per thread, or the compressed one at two in FP32): then on the same layout
    // with enough rows per thread.  Every variant forms the same products and
    // slot-ordered sums, so the defect vector is the same bit for bit; the norm's
    // block partials follow the launch shape.
    hb2_ell_s V = *A;
    V.bs[1] = kEllThreads;   // the default launch shape: 256 threads, one per row
    V.tpr[1] = 1;
    const int base = V.rpt[1] & ~kPatFlags, kflags = V.rpt[1] & kPatFlags;
    for (int r = 2; r <= 8 && ell_grid(&V, true) > kNoAllocMaxBlocks; r *= 2)
    {
        if (V.layout[1] == kLayoutPattern && r > base && (r <= 4 || (kflags & kPatQ1)))
            V.rpt[1] = r | (kflags & (kPatQ1 | kPatQ1G | kPatQ1S)) | (r <= 2 ? (kflags & (kPatWin | kPatQ1P)) : 0);
        else if (V.layout[1] == kLayoutCompact && r > V.compact_rpt_red) V.compact_rpt_red = r;
        else if (V.layout[1] == kLayoutBF16 && r > V.rpt[1]) V.rpt[1] = r;
    }
    if (ell_grid(&V, true) > kNoAllocMaxBlocks)
        return fail(HB2_ERR_UNSUPPORTED, "hb2_defect_ell_noalloc: no layout variant fits the static scratch");
    double * scratch = 0;
    int st = noalloc_scratch(&scratch);
    if (st) return st;
    // The ticket counters must start at zero.  Every completed launch leaves them
    // at zero again, but a launch that stopped part-way (an error on the device,
    // or a call that raced with another on a second stream) would leave a
    // counter off by some tickets and every later norm wrong, so they are
    // cleared here each call.  The partials need no clearing: each block writes
    // its own before the last block reads them.
    unsigned * ticket = (unsigned *)(scratch + kNoAllocMaxBlocks + kNoAllocGroups);
    HB2_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned) * (kNoAllocGroups + 1), stream));
    Workspace ws;
    ws.device = 0;
    ws.partials = scratch;
    ws.gpart = scratch + kNoAllocMaxBlocks;
    ws.ticket = ticket;
    ws.bar_words = 0;
    ws.error = 0;
    ws.scalars = 0;
    ws.max_blocks = kNoAllocMaxBlocks;
    ws.max_tickets = kNoAllocGroups + 1;
    ws.host_scalars = 0;
    return launch_ell(&V, kDefect, x, r, rhs, 0, 0, norm2_dev, 0, &ws, stream);
}
