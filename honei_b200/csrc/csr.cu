// SparseMatrixCSR on the device: Product and Defect.
//
// The reference's CSR (la/sparse_matrix_csr-impl.hh:40-135) stores, per row,
// Ar[row]..Ar[row+1] blocks; block i starts at column Aj[i] and holds
// csr::blocksize (bs) consecutive values Ax[i*bs ..].  Its tags::CPU Product
// and Defect (la/product.hh:208-244, math/defect.hh:385-420) walk a row's
// blocks in order and accumulate sum = fma(Ax, x[col], sum), skipping a block
// value whose column is past the vector; its compiled loop contracts the
// multiply-add into one fma (unlike the ELL loop).  The result of a row is
// therefore one ordered fma chain over the row's entries -- its block values
// in order, minus those past the vector -- and the kernels reproduce it.
//
// Device layout (built on the host at creation).  Each row is expanded into
// its entries (column, value) in the reference's order.  Then:
//   * rows of at most kShortRow entries: SELL-C-sigma (Kreutzer et al., SIAM J.
//     Sci. Comput. 36(5), 2014) with C = 32 and sigma = kSigma -- inside each
//     window of kSigma rows the rows are ordered by decreasing length, cut
//     into slices of 32 rows, and a slice is stored slot-major (slot k of lane
//     l at offset + 32 k + l) to the length of its longest row, padding
//     columns -1.  One warp per slice, one lane per row: the loads of a slot
//     are coalesced across the rows like the ELL kernels', and each lane runs
//     its row's chain in registers.  The reordering changes which rows share a
//     warp, never the order inside a row.
//   * longer rows: chunks of W entries ("items") in a compact entry array,
//     run by warps that stage a chunk's (value, x[column]) pairs in shared
//     memory with cp.async while lane 0 runs the chain over the previous chunk
//     (two buffers); a row's chunks stay in one warp.
// One launch: the CTAs of the long rows first (their chains are the longest),
// then the slices.  The reference arrays are kept on the host for export.
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

using namespace hb2;

namespace
{
    constexpr int kCsrWarps = 4;                         // warps per CTA
    constexpr uint32_t kShortRow = 128;                  // longest row in the sliced part
    constexpr uint32_t kSigma = 512;                     // sorting window of the sliced part
    constexpr uint32_t kW = 128;                         // entries per long-row chunk
    constexpr uint32_t kFirstFlag = 0x80000000u;         // first chunk: the sum starts at 0
    constexpr uint32_t kLastFlag = 0x40000000u;          // last chunk: the sum is stored
    constexpr uint32_t kRowMask = 0x3fffffffu;
    constexpr uint64_t kMaxBlockSize = 1024;
}

struct hb2_csr_s
{
    int dtype;
    int device;
    uint64_t rows, cols, bs;
    uint64_t nblocks;              // Ar[rows]
    // the reference arrays (host), for export
    std::vector<uint64_t> hAr, hAj;
    std::vector<unsigned char> hAx;
    // sliced part
    uint2 * slices = nullptr;      // (first slot, width)
    uint32_t * perm = nullptr;     // row of each (slice, lane); 0xffffffff: none
    int32_t * scol = nullptr;      // slot columns, -1 past a row's end
    void * sval = nullptr;         // slot values
    uint32_t nslices = 0;
    uint64_t nslots = 0;
    int unroll = 8;                // slots per lane and round (8 or 16)
    // long rows
    uint4 * items = nullptr;       // (row | flags, 0, first entry, end entry)
    uint32_t * tasks = nullptr;    // nlong_warps + 1 item offsets
    int32_t * lcol = nullptr;      // entry columns
    void * lval = nullptr;         // entry values
    uint32_t nitems = 0, nlong_warps = 0, nlong_rows = 0;
    uint64_t nlong_entries = 0;
    uint64_t bytes = 0;
};

namespace
{
    // 4- or 8-byte asynchronous copy global -> shared
    template <int BYTES>
    __device__ __forceinline__ void cp_async(void * dst, const void * src)
    {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(BYTES) : "memory");
    }
    __device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
    __device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

    // one slice: lane = row, slots streamed U at a time (columns and values of
    // U slots in flight, then their x entries), the chain in order
    template <typename T, bool DEFECT, int U>
    __device__ __forceinline__ void run_slice(uint32_t slice, uint32_t lane, const uint2 * __restrict__ slices,
                                              const uint32_t * __restrict__ perm, const int32_t * __restrict__ scol,
                                              const T * __restrict__ sval, const T * __restrict__ x,
                                              const T * __restrict__ rhs, T * __restrict__ y)
    {
        const uint2 d = __ldg(slices + slice);
        const uint32_t row = __ldg(perm + 32 * slice + lane);
        if (row == 0xffffffffu) return;
        T rh = T(0);
        if (DEFECT) rh = __ldg(rhs + row);
        const int32_t * cp = scol + d.x + lane;
        const T * vp = sval + d.x + lane;
        T s = T(0);
        for (uint32_t k = 0; k < d.y; k += U)
        {
            int32_t c[U];
            T a[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
            {
                c[u] = -1;
                a[u] = T(0);
                if (k + u < d.y)
                {
                    c[u] = __ldcs(cp + 32 * (k + u));
                    a[u] = __ldcs(vp + 32 * (k + u));
                }
            }
            T xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) xv[u] = c[u] >= 0 ? __ldg(x + c[u]) : T(0);
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (c[u] >= 0) s = Arith<T>::fma(a[u], xv[u], s);
        }
        if (DEFECT) y[row] = Arith<T>::sub(rh, s);
        else y[row] = s;
    }

    // the long rows of one warp: items k0 .. k1-1, staged two buffers deep
    template <typename T, bool DEFECT>
    __device__ __forceinline__ void run_long(uint32_t k0, uint32_t k1, uint32_t lane, T (*buf)[2][kW],
                                             const uint4 * __restrict__ items, const int32_t * __restrict__ lcol,
                                             const T * __restrict__ lval, const T * __restrict__ x,
                                             const T * __restrict__ rhs, T * __restrict__ y)
    {
        if (k0 >= k1) return;
        auto stage = [&](const uint4 & it, T (*b)[kW]) {
            const uint32_t n = it.w - it.z;
            int32_t c[kW / 32];
#pragma unroll
            for (int u = 0; u < (int)(kW / 32); ++u)
            {
                const uint32_t i = lane + 32 * u;
                c[u] = i < n ? __ldg(lcol + it.z + i) : -1;
            }
#pragma unroll
            for (int u = 0; u < (int)(kW / 32); ++u)
            {
                const uint32_t i = lane + 32 * u;
                if (i < n)
                {
                    cp_async<sizeof(T)>(&b[0][i], lval + it.z + i);
                    cp_async<sizeof(T)>(&b[1][i], x + c[u]);
                }
            }
            cp_async_commit();
        };
        uint4 cur = __ldg(items + k0);
        stage(cur, buf[0]);
        T s = T(0);
        for (uint32_t k = k0; k < k1; ++k)
        {
            const uint32_t bsel = (k - k0) & 1;
            uint4 nxt = cur;
            if (k + 1 < k1) nxt = __ldg(items + k + 1);
            cp_async_wait_all();
            __syncwarp();
            if (lane == 0)
            {
                if (cur.x & kFirstFlag) s = T(0);
                const uint32_t n = cur.w - cur.z;
                const T * a = buf[bsel][0];
                const T * xv = buf[bsel][1];
                for (uint32_t i = 0; i < n; ++i) s = Arith<T>::fma(a[i], xv[i], s);
                if (cur.x & kLastFlag)
                {
                    const uint32_t row = cur.x & kRowMask;
                    if (DEFECT) y[row] = Arith<T>::sub(__ldg(rhs + row), s);
                    else y[row] = s;
                }
            }
            __syncwarp();
            if (k + 1 < k1)
            {
                stage(nxt, buf[bsel ^ 1]);
                cur = nxt;
            }
        }
    }

    template <typename T, bool DEFECT, int U>
    __global__ void __launch_bounds__(32 * kCsrWarps) csr_kernel(
        uint32_t long_ctas, const uint4 * __restrict__ items, const uint32_t * __restrict__ tasks,
        uint32_t nlong_warps, const int32_t * __restrict__ lcol, const T * __restrict__ lval,
        const uint2 * __restrict__ slices, uint32_t nslices, const uint32_t * __restrict__ perm,
        const int32_t * __restrict__ scol, const T * __restrict__ sval, const T * __restrict__ x,
        const T * __restrict__ rhs, T * __restrict__ y)
    {
        __shared__ __align__(16) T sbuf[kCsrWarps][2][2][kW];     // [warp][buffer][value | x][i]
        const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (blockIdx.x < long_ctas)
        {
            const uint32_t w = blockIdx.x * kCsrWarps + warp;
            if (w < nlong_warps)
                run_long<T, DEFECT>(__ldg(tasks + w), __ldg(tasks + w + 1), lane, sbuf[warp], items, lcol, lval, x,
                                    rhs, y);
            return;
        }
        const uint32_t slice = (blockIdx.x - long_ctas) * kCsrWarps + warp;
        if (slice < nslices) run_slice<T, DEFECT, U>(slice, lane, slices, perm, scol, sval, x, rhs, y);
    }

    int csr_free(hb2_csr_s * A)
    {
        if (! A) return HB2_OK;
        cudaFree(A->slices);
        cudaFree(A->perm);
        cudaFree(A->scol);
        cudaFree(A->sval);
        cudaFree(A->items);
        cudaFree(A->tasks);
        cudaFree(A->lcol);
        cudaFree(A->lval);
        delete A;
        return HB2_OK;
    }

    template <typename T, bool DEFECT>
    int launch(hb2_csr A, const void * rhs, const void * x, void * y, cudaStream_t stream)
    {
        const uint32_t long_ctas = (A->nlong_warps + kCsrWarps - 1) / kCsrWarps;
        const uint32_t slice_ctas = (A->nslices + kCsrWarps - 1) / kCsrWarps;
        if (long_ctas + slice_ctas == 0) return HB2_OK;
        auto k = A->unroll == 16 ? csr_kernel<T, DEFECT, 16> : csr_kernel<T, DEFECT, 8>;
        k<<<long_ctas + slice_ctas, 32 * kCsrWarps, 0, stream>>>(
            long_ctas, A->items, A->tasks, A->nlong_warps, A->lcol, (const T *)A->lval, A->slices, A->nslices,
            A->perm, A->scol, (const T *)A->sval, (const T *)x, (const T *)rhs, (T *)y);
        count_launches(1);
        HB2_LAUNCH_CHECK("csr_kernel");
        return HB2_OK;
    }

    // Slots loaded per lane and round in the sliced part: 8 or 16, whichever
    // runs the product faster on this matrix (timed at creation when it holds
    // at least 2^20 slots; bit-identical results either way).  Measured on the
    // level-11 Q1 operator: FP64 108.6 us (16) / 127.0 us (8), FP32 83.9 us (16)
    // / 75.0 us (8).  HB2_CSR_U=8|16 fixes it.
    template <typename T>
    int choose_unroll(hb2_csr_s * A, cudaStream_t stream)
    {
        A->unroll = 8;
        if (const char * env = getenv("HB2_CSR_U"))
        {
            A->unroll = atoi(env) == 16 ? 16 : 8;
            return HB2_OK;
        }
        if (A->nslots + A->nlong_entries < (1u << 20)) return HB2_OK;
        T * x = nullptr, * y = nullptr;
        HB2_CUDA(cudaMalloc(&x, sizeof(T) * std::max<uint64_t>(A->cols, 1)));
        cudaError_t e = cudaMalloc(&y, sizeof(T) * std::max<uint64_t>(A->rows, 1));
        if (e == cudaSuccess) e = cudaMemsetAsync(x, 0, sizeof(T) * std::max<uint64_t>(A->cols, 1), stream);
        cudaEvent_t ev[2] = {nullptr, nullptr};
        if (e == cudaSuccess) e = cudaEventCreate(&ev[0]);
        if (e == cudaSuccess) e = cudaEventCreate(&ev[1]);
        float best = 1e30f;
        int best_u = 8;
        for (int u : {8, 16})
        {
            if (e != cudaSuccess) break;
            A->unroll = u;
            int st = launch<T, false>(A, nullptr, x, y, stream);    // warm-up
            if (st) { e = cudaErrorUnknown; break; }
            e = cudaEventRecord(ev[0], stream);
            for (int i = 0; i < 3 && e == cudaSuccess; ++i)
                if (launch<T, false>(A, nullptr, x, y, stream)) e = cudaErrorUnknown;
            if (e == cudaSuccess) e = cudaEventRecord(ev[1], stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
            float ms = 0;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
            if (e == cudaSuccess && ms < best) { best = ms; best_u = u; }
        }
        A->unroll = best_u;
        if (ev[0]) cudaEventDestroy(ev[0]);
        if (ev[1]) cudaEventDestroy(ev[1]);
        cudaFree(x);
        cudaFree(y);
        if (e != cudaSuccess) return cuda_status(e, "hb2_csr_create: unroll timing");
        return HB2_OK;
    }

    template <typename T>
    cudaError_t upload(void ** dst, const std::vector<T> & v, cudaStream_t stream)
    {
        cudaError_t e = cudaMalloc(dst, sizeof(T) * std::max<size_t>(v.size(), 1));
        if (e == cudaSuccess && ! v.empty())
            e = cudaMemcpyAsync(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, stream);
        return e;
    }

    // Build both device parts from the reference arrays (host) and upload them.
    template <typename T>
    int build_device(hb2_csr_s * A, cudaStream_t stream)
    {
        const uint64_t rows = A->rows, bs = A->bs, ncols = A->cols;
        const T * Ax = (const T *)A->hAx.data();
        // entries of every row, in the reference's order, past-the-vector values dropped
        std::vector<uint64_t> start(rows + 1, 0);
        for (uint64_t r = 0; r < rows; ++r)
        {
            uint64_t n = 0;
            for (uint64_t i = A->hAr[r]; i < A->hAr[r + 1]; ++i)
                for (uint64_t o = 0; o < bs; ++o) n += A->hAj[i] + o < ncols;
            start[r + 1] = start[r] + n;
        }
        std::vector<int32_t> ecol(start[rows]);
        std::vector<T> eval(start[rows]);
        for (uint64_t r = 0, q = 0; r < rows; ++r)
            for (uint64_t i = A->hAr[r]; i < A->hAr[r + 1]; ++i)
                for (uint64_t o = 0; o < bs; ++o)
                    if (A->hAj[i] + o < ncols)
                    {
                        ecol[q] = (int32_t)(A->hAj[i] + o);
                        eval[q] = Ax[i * bs + o];
                        ++q;
                    }
        auto len = [&](uint64_t r) { return start[r + 1] - start[r]; };
        // long rows: chunks of kW entries in a compact entry array, tasks for
        // the warps of at most one wave (a row's chunks in one task)
        std::vector<int32_t> lcol;
        std::vector<T> lval;
        std::vector<uint4> items;
        std::vector<uint32_t> short_rows;
        uint32_t nlong_rows = 0;
        for (uint64_t r = 0; r < rows; ++r)
        {
            if (len(r) <= kShortRow) { short_rows.push_back((uint32_t)r); continue; }
            ++nlong_rows;
            const uint64_t base = lcol.size();
            lcol.insert(lcol.end(), ecol.begin() + start[r], ecol.begin() + start[r + 1]);
            lval.insert(lval.end(), eval.begin() + start[r], eval.begin() + start[r + 1]);
            for (uint64_t v = 0; v < len(r); v += kW)
            {
                const uint32_t fl = (v == 0 ? kFirstFlag : 0) | (v + kW >= len(r) ? kLastFlag : 0);
                items.push_back(make_uint4((uint32_t)r | fl, 0, (uint32_t)(base + v),
                                           (uint32_t)(base + std::min<uint64_t>(v + kW, len(r)))));
            }
        }
        std::vector<uint32_t> tasks;
        {
            int per_sm = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csr_kernel<T, false, 8>, 32 * kCsrWarps, 0) !=
                    cudaSuccess || per_sm < 1)
                per_sm = 1;
            const uint64_t nwarps = std::max<uint64_t>(1, std::min<uint64_t>(nlong_rows, (uint64_t)per_sm * num_sms() * kCsrWarps));
            const uint64_t share = items.empty() ? 1 : (items.size() + nwarps - 1) / nwarps;
            uint64_t k = 0;
            while (k < items.size())
            {
                tasks.push_back((uint32_t)k);
                uint64_t e = std::min<uint64_t>(items.size(), k + share);
                while (e < items.size() && ! (items[e].x & kFirstFlag)) ++e;
                k = e;
            }
            tasks.push_back((uint32_t)items.size());
        }
        // short rows: ordered by decreasing length inside windows of kSigma, slices of 32
        for (size_t w = 0; w < short_rows.size(); w += kSigma)
        {
            auto b = short_rows.begin() + w, e = short_rows.begin() + std::min<size_t>(short_rows.size(), w + kSigma);
            std::stable_sort(b, e, [&](uint32_t p, uint32_t q) { return len(p) > len(q); });
        }
        // slices of H = 32 rows; slot k of the slice's row j at first + H k + j
        const uint64_t H = 32;
        const uint64_t nslices = (short_rows.size() + H - 1) / H;
        std::vector<uint2> slices(nslices);
        std::vector<uint32_t> perm(nslices * H, 0xffffffffu);
        uint64_t nslots = 0;
        for (uint64_t sl = 0; sl < nslices; ++sl)
        {
            uint64_t width = 0;
            for (uint64_t j = 0; j < H && H * sl + j < short_rows.size(); ++j)
            {
                perm[H * sl + j] = short_rows[H * sl + j];
                width = std::max<uint64_t>(width, len(short_rows[H * sl + j]));
            }
            if (nslots + H * width >= 0xffffffffULL) return fail(HB2_ERR_UNSUPPORTED, "hb2_csr_create: more than 2^32 slots");
            slices[sl] = make_uint2((uint32_t)nslots, (uint32_t)width);
            nslots += H * width;
        }
        std::vector<int32_t> scol(nslots, -1);
        std::vector<T> sval(nslots, T(0));
        for (uint64_t sl = 0; sl < nslices; ++sl)
            for (uint64_t j = 0; j < H; ++j)
            {
                const uint32_t r = perm[H * sl + j];
                if (r == 0xffffffffu) continue;
                for (uint64_t k = 0; k < len(r); ++k)
                {
                    scol[slices[sl].x + H * k + j] = ecol[start[r] + k];
                    sval[slices[sl].x + H * k + j] = eval[start[r] + k];
                }
            }
        cudaError_t e = upload((void **)&A->slices, slices, stream);
        if (e == cudaSuccess) e = upload((void **)&A->perm, perm, stream);
        if (e == cudaSuccess) e = upload((void **)&A->scol, scol, stream);
        if (e == cudaSuccess) e = upload(&A->sval, sval, stream);
        if (e == cudaSuccess) e = upload((void **)&A->items, items, stream);
        if (e == cudaSuccess) e = upload((void **)&A->tasks, tasks, stream);
        if (e == cudaSuccess) e = upload((void **)&A->lcol, lcol, stream);
        if (e == cudaSuccess) e = upload(&A->lval, lval, stream);
        // the host vectors die with this call
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_status(e, "hb2_csr_create upload");
        A->nslices = (uint32_t)nslices;
        A->nslots = nslots;
        A->nitems = (uint32_t)items.size();
        A->nlong_warps = (uint32_t)tasks.size() - 1;
        A->nlong_rows = nlong_rows;
        A->nlong_entries = lcol.size();
        A->bytes = sizeof(uint2) * nslices + sizeof(uint32_t) * perm.size() + (sizeof(int32_t) + sizeof(T)) * nslots +
                   sizeof(uint4) * items.size() + sizeof(uint32_t) * tasks.size() +
                   (sizeof(int32_t) + sizeof(T)) * lcol.size();
        return HB2_OK;
    }
}

extern "C" int hb2_csr_create(hb2_csr * out, hb2_dtype dtype, uint64_t rows, uint64_t cols, uint64_t blocksize,
                              const uint64_t * Ar, const uint64_t * Aj, const void * Ax, int host_ptrs,
                              cudaStream_t stream)
{
    if (! out || ! Ar) return fail(HB2_ERR_ARG, "hb2_csr_create: null argument");
    *out = nullptr;
    if (dtype != HB2_F64 && dtype != HB2_F32) return fail(HB2_ERR_ARG, "hb2_csr_create: dtype");
    if (blocksize == 0 || blocksize > kMaxBlockSize) return fail(HB2_ERR_ARG, "hb2_csr_create: blocksize out of range");
    if (rows > kRowMask || cols > 0x7fffffffULL) return fail(HB2_ERR_UNSUPPORTED, "hb2_csr_create: too many rows or columns");
    const size_t es = dtype_size(dtype);
    hb2_csr_s * A = new hb2_csr_s();
    A->hAr.resize(rows + 1);
    if (host_ptrs) memcpy(A->hAr.data(), Ar, sizeof(uint64_t) * (rows + 1));
    else
    {
        cudaError_t e = cudaMemcpy(A->hAr.data(), Ar, sizeof(uint64_t) * (rows + 1), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { csr_free(A); return cuda_status(e, "hb2_csr_create: read Ar"); }
    }
    int st = HB2_OK;
    if (A->hAr[0] != 0) st = fail(HB2_ERR_ARG, "hb2_csr_create: Ar[0] != 0");
    for (uint64_t r = 0; ! st && r < rows; ++r)
        if (A->hAr[r + 1] < A->hAr[r]) st = fail(HB2_ERR_ARG, "hb2_csr_create: Ar not monotone");
    const uint64_t nblocks = st ? 0 : A->hAr[rows];
    if (! st && nblocks && (! Aj || ! Ax)) st = fail(HB2_ERR_ARG, "hb2_csr_create: null argument");
    if (! st && nblocks * blocksize >= 0xffffff00ULL) st = fail(HB2_ERR_UNSUPPORTED, "hb2_csr_create: more than 2^32 values");
    if (st) { csr_free(A); return st; }
    A->hAj.resize(nblocks);
    A->hAx.resize(es * nblocks * blocksize);
    if (nblocks)
    {
        cudaError_t e = cudaSuccess;
        if (host_ptrs)
        {
            memcpy(A->hAj.data(), Aj, sizeof(uint64_t) * nblocks);
            memcpy(A->hAx.data(), Ax, A->hAx.size());
        }
        else
        {
            e = cudaMemcpy(A->hAj.data(), Aj, sizeof(uint64_t) * nblocks, cudaMemcpyDeviceToHost);
            if (e == cudaSuccess) e = cudaMemcpy(A->hAx.data(), Ax, A->hAx.size(), cudaMemcpyDeviceToHost);
        }
        if (e != cudaSuccess) { csr_free(A); return cuda_status(e, "hb2_csr_create: read Aj / Ax"); }
    }
    for (uint64_t i = 0; i < nblocks; ++i)
        if (A->hAj[i] >= cols) { csr_free(A); return fail(HB2_ERR_ARG, "hb2_csr_create: column index out of range"); }
    A->dtype = dtype;
    cudaGetDevice(&A->device);
    A->rows = rows;
    A->cols = cols;
    A->bs = blocksize;
    A->nblocks = nblocks;
    st = dtype == HB2_F64 ? build_device<double>(A, stream) : build_device<float>(A, stream);
    if (! st) st = dtype == HB2_F64 ? choose_unroll<double>(A, stream) : choose_unroll<float>(A, stream);
    if (st) { csr_free(A); return st; }
    *out = A;
    return HB2_OK;
}

extern "C" int hb2_csr_from_ell(hb2_csr * out, hb2_ell E, uint64_t blocksize, cudaStream_t stream)
{
    if (! out || ! E) return fail(HB2_ERR_ARG, "hb2_csr_from_ell: null argument");
    if (blocksize == 0 || blocksize > kMaxBlockSize) return fail(HB2_ERR_ARG, "hb2_csr_from_ell: blocksize out of range");
    const uint64_t size = E->ref_K * E->ref_stride, T = E->ref_T;
    const size_t es = dtype_size(E->dtype);
    std::vector<uint64_t> Aj(size), Arl(std::max<uint64_t>(E->rows, 1));
    std::vector<unsigned char> Ax(es * size);
    int st = hb2_ell_export(E, Aj.data(), Ax.data(), Arl.data());
    if (st) return st;
    // SparseMatrix(SparseMatrixELL) (la/sparse_matrix.hh:157-185): every nonzero
    // slot, later slots overwriting earlier ones at the same column; rows in
    // ascending column order.  Then _create (la/sparse_matrix_csr-impl.hh:98-135).
    std::vector<uint64_t> cAr(1, 0), cAj;
    std::vector<unsigned char> cAx;
    std::vector<std::pair<uint64_t, uint64_t>> ent;   // (column, slot)
    for (uint64_t r = 0; r < E->rows; ++r)
    {
        ent.clear();
        for (uint64_t i = r * T; i < size; i += E->ref_stride)
            for (uint64_t t = 0; t < T; ++t)
            {
                const unsigned char * p = &Ax[es * (i + t)];
                const bool nz = es == 8 ? *(const double *)p != 0.0 : *(const float *)p != 0.0f;
                if (nz) ent.push_back(std::make_pair(Aj[i + t], i + t));
            }
        std::stable_sort(ent.begin(), ent.end(),
                         [](const std::pair<uint64_t, uint64_t> & a, const std::pair<uint64_t, uint64_t> & b) { return a.first < b.first; });
        // duplicates: keep the last slot written
        std::vector<std::pair<uint64_t, uint64_t>> uniq;
        for (const auto & q : ent)
        {
            if (! uniq.empty() && uniq.back().first == q.first) uniq.back() = q;
            else uniq.push_back(q);
        }
        for (size_t i = 0; i < uniq.size();)
        {
            const uint64_t base = uniq[i].first - uniq[i].first % blocksize;
            cAj.push_back(base);
            size_t d = 0;
            for (uint64_t b = 0; b < blocksize; ++b)
            {
                const size_t at = cAx.size();
                cAx.resize(at + es, 0);
                if (i + d < uniq.size() && base + b == uniq[i + d].first)
                {
                    memcpy(&cAx[at], &Ax[es * uniq[i + d].second], es);
                    ++d;
                }
            }
            i += d;
        }
        cAr.push_back(cAj.size());
    }
    return hb2_csr_create(out, (hb2_dtype)E->dtype, E->rows, E->cols, blocksize, cAr.data(),
                          cAj.empty() ? nullptr : cAj.data(), cAx.empty() ? nullptr : cAx.data(), 1, stream);
}

extern "C" int hb2_csr_destroy(hb2_csr A) { return csr_free(A); }

extern "C" int hb2_csr_info(hb2_csr A, uint64_t * rows, uint64_t * cols, uint64_t * blocksize, uint64_t * nblocks,
                            uint64_t * device_bytes)
{
    if (! A) return fail(HB2_ERR_ARG, "hb2_csr_info: null matrix");
    if (rows) *rows = A->rows;
    if (cols) *cols = A->cols;
    if (blocksize) *blocksize = A->bs;
    if (nblocks) *nblocks = A->nblocks;
    if (device_bytes) *device_bytes = A->bytes;
    return HB2_OK;
}

extern "C" int hb2_csr_layout(hb2_csr A, uint64_t * slots, uint64_t * long_rows, uint64_t * long_entries,
                              uint32_t * unroll)
{
    if (! A) return fail(HB2_ERR_ARG, "hb2_csr_layout: null matrix");
    if (slots) *slots = A->nslots;
    if (long_rows) *long_rows = A->nlong_rows;
    if (long_entries) *long_entries = A->nlong_entries;
    if (unroll) *unroll = (uint32_t)A->unroll;
    return HB2_OK;
}

extern "C" int hb2_csr_export(hb2_csr A, uint64_t * Ar, uint64_t * Aj, void * Ax)
{
    if (! A || ! Ar || (A->nblocks && (! Aj || ! Ax))) return fail(HB2_ERR_ARG, "hb2_csr_export: null argument");
    memcpy(Ar, A->hAr.data(), sizeof(uint64_t) * (A->rows + 1));
    if (A->nblocks)
    {
        memcpy(Aj, A->hAj.data(), sizeof(uint64_t) * A->nblocks);
        memcpy(Ax, A->hAx.data(), A->hAx.size());
    }
    return HB2_OK;
}

extern "C" int hb2_product_csr(hb2_csr A, const void * x, void * y, cudaStream_t stream)
{
    if (! A || (A->rows && (! x || ! y))) return fail(HB2_ERR_ARG, "hb2_product_csr: null argument");
    return A->dtype == HB2_F64 ? launch<double, false>(A, nullptr, x, y, stream)
                               : launch<float, false>(A, nullptr, x, y, stream);
}

extern "C" int hb2_defect_csr(hb2_csr A, const void * rhs, const void * x, void * r, cudaStream_t stream)
{
    if (! A || (A->rows && (! rhs || ! x || ! r))) return fail(HB2_ERR_ARG, "hb2_defect_csr: null argument");
    return A->dtype == HB2_F64 ? launch<double, true>(A, rhs, x, r, stream)
                               : launch<float, true>(A, rhs, x, r, stream);
}
