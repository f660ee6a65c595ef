// Compressed device layout for SparseMatrixELL: value dictionary + 16-bit
// column offsets.
//
// FEM and stencil operators have few distinct values and bounded column
// offsets.  When a matrix has at most 255 distinct value bit patterns and every
// column lies within +-32767 of its row's base column (base = row for square
// matrices, floor(row * cols / rows) otherwise), each slot is stored as a 1-byte
// index into a per-matrix value table plus a 2-byte offset: 3 bytes per slot
// instead of 12 (FP64 value + int32 column) or 8 (FP32).  The kernels look the
// value up in shared memory and perform exactly the products and sums of the
// plain layout, so results are bit-identical.  The plain arrays are kept (the
// small-level, CG and export paths read them); launch_ell uses the compressed
// arrays when present.  Set HB2_ELL_COMPACT=0 to keep matrices plain,
// HB2_ELL_COMPACT=force2|force4|force8 to skip the autotuner.
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace hb2
{
    constexpr int16_t kEmptyOffset = -32768;
    constexpr uint32_t kDictSlots = 4096;
    constexpr unsigned long long kEmptyKey = 0xFFFFFFFFFFFFFFFFull;
    constexpr int kCompactRowsMax = 8;                // rows per thread: 2, 4 or 8 (autotuned)
    constexpr uint64_t kCompactMinRows = 32768;       // smaller matrices stay plain
    constexpr uint64_t kShapeMinRows = 4096;          // smaller ones also keep the default launch shape

    template <typename T> __device__ __forceinline__ unsigned long long key_of(T v);
    template <> __device__ __forceinline__ unsigned long long key_of<double>(double v) { return (unsigned long long)__double_as_longlong(v); }
    template <> __device__ __forceinline__ unsigned long long key_of<float>(float v) { return (unsigned long long)__float_as_uint(v); }

    __device__ __forceinline__ uint32_t dict_hash(unsigned long long k)
    {
        k ^= k >> 33;
        k *= 0xff51afd7ed558ccdull;
        k ^= k >> 33;
        return (uint32_t)k & (kDictSlots - 1);
    }

    __device__ __forceinline__ int64_t row_base(uint64_t r, uint64_t rows, uint64_t cols)
    {
        return rows == cols ? (int64_t)r : (int64_t)((r * cols) / rows);
    }

    // row_base without the 64-bit division, for the kernels: ratio = cols / rows
    // rounded to double.  For r < rows < 2^32 and cols < 2^31 the estimate
    // r * ratio is within 2^-20 of r * cols / rows, so its truncation is off by at
    // most one, and the exact integer products settle which way.
    __device__ __forceinline__ int64_t row_base_est(uint64_t r, uint64_t rows, uint64_t cols, double ratio)
    {
        if (rows == cols) return (int64_t)r;
        const uint64_t num = r * cols;
        uint64_t q = (uint64_t)((double)r * ratio);
        if (q * rows > num) --q;
        else if ((q + 1) * rows <= num) ++q;
        return (int64_t)q;
    }

    // one insert per distinct value of a warp: matrices with few values would
    // otherwise send every slot's atomic to the same few addresses
    template <typename T>
    __global__ void dict_insert_kernel(const T * __restrict__ val, const int32_t * __restrict__ col, uint64_t n,
                                       unsigned long long * keys, int * flag)
    {
        const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
        for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride)
        {
            const uint64_t i = base + threadIdx.x;
            const bool live = i < n && col[i] >= 0;
            const unsigned long long k = live ? key_of(val[i]) : kEmptyKey;
            if (live && k == kEmptyKey) atomicExch(flag, 3);
            const unsigned peers = __match_any_sync(0xffffffffu, k);
            if (k == kEmptyKey || (threadIdx.x & 31) != (unsigned)(__ffs(peers) - 1)) continue;
            uint32_t h = dict_hash(k);
            bool placed = false;
            for (uint32_t p = 0; p < kDictSlots; ++p)
            {
                const unsigned long long prev = atomicCAS(keys + h, kEmptyKey, k);
                if (prev == kEmptyKey || prev == k) { placed = true; break; }
                h = (h + 1) & (kDictSlots - 1);
            }
            if (! placed) atomicExch(flag, 1);
        }
    }

    template <typename T>
    __global__ void ell_encode_kernel(const T * __restrict__ val, const int32_t * __restrict__ col, uint64_t rows,
                                      uint64_t cols, uint64_t ld, uint32_t K, const unsigned long long * __restrict__ keys,
                                      const uint16_t * __restrict__ code_of_slot, uint8_t * code, int16_t * delta,
                                      int * flag)
    {
        const uint64_t n = (uint64_t)K * ld;
        const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        {
            const uint64_t r = i % ld;
            const int32_t c = col[i];
            if (c < 0 || r >= rows)
            {
                code[i] = 0;
                delta[i] = kEmptyOffset;
                continue;
            }
            const unsigned long long k = key_of(val[i]);
            uint32_t h = dict_hash(k);
            uint32_t p = 0;
            while (keys[h] != k && p < kDictSlots) { h = (h + 1) & (kDictSlots - 1); ++p; }
            if (p == kDictSlots) { atomicExch(flag, 4); code[i] = 0; delta[i] = kEmptyOffset; continue; }
            code[i] = (uint8_t)code_of_slot[h];
            const int64_t d = (int64_t)c - row_base(r, rows, cols);
            if (d <= -32768 || d > 32767) { atomicExch(flag, 2); delta[i] = kEmptyOffset; continue; }
            delta[i] = (int16_t)d;
        }
    }

    template <typename T>
    struct EllCompactView
    {
        const uint8_t * code;
        const int16_t * delta;
        const T * table;
        uint64_t rows, cols, ld;
        uint32_t K, ntable;
        double ratio;   // cols / rows (row_base_est)
    };

    // one thread: R consecutive rows; per slot it loads R one-byte codes and R
    // 16-bit offsets (R = 2: 16 + 32 bits, 4: 32 + 64 bits, 8: 64 + 128 bits)
    template <int R> struct CodeWord;
    template <> struct CodeWord<2> { typedef uint16_t C; typedef int32_t D; };
    template <> struct CodeWord<4> { typedef uint32_t C; typedef int2 D; };
    template <> struct CodeWord<8> { typedef uint2 C; typedef int4 D; };

    template <int R>
    __device__ __forceinline__ void unpack(const typename CodeWord<R>::C & c, const typename CodeWord<R>::D & d,
                                           uint32_t (&code)[R], int (&off)[R])
    {
        uint32_t cw[(R + 3) / 4];
        int32_t dw[(R + 1) / 2];
        if constexpr (R == 2) { cw[0] = c; dw[0] = d; }
        else if constexpr (R == 4) { cw[0] = c; dw[0] = d.x; dw[1] = d.y; }
        else { cw[0] = c.x; cw[1] = c.y; dw[0] = d.x; dw[1] = d.y; dw[2] = d.z; dw[3] = d.w; }
#pragma unroll
        for (int i = 0; i < R; ++i)
        {
            code[i] = (cw[i >> 2] >> ((i & 3) * 8)) & 0xffu;
            off[i] = (int16_t)(dw[i >> 1] >> ((i & 1) * 16));
        }
    }

    template <typename V>
    __device__ __forceinline__ V ld_policy(const V * p, bool keep) { return keep ? __ldcg(p) : __ldcs(p); }
    template <>
    __device__ __forceinline__ uint16_t ld_policy<uint16_t>(const uint16_t * p, bool keep)
    {
        return keep ? __ldcg((const unsigned short *)p) : __ldcs((const unsigned short *)p);
    }

    template <typename T, int KT, int MODE, int R>
    __global__ void __launch_bounds__(kEllMaxThreads)
    ell_compact_kernel(EllCompactView<T> A, const T * __restrict__ x_, T * __restrict__ y_, const T * __restrict__ aux_,
                       const T * __restrict__ aux2, T * __restrict__ zero_, ReduceSlot rs, double * red_, int want_sqrt,
                       int flags, Batch bt)
    {
        typedef Arith<T> M;
        typedef typename CodeWord<R>::C CW;
        typedef typename CodeWord<R>::D DW;
        __shared__ T table[256];
        for (uint32_t i = threadIdx.x; i < A.ntable; i += blockDim.x) table[i] = A.table[i];
        __syncthreads();
        pdl_entry();   // the value table is constant: loaded before the wait
        // work items: (vector j, row block) -- the launch grid (blockIdx.x, blockIdx.y),
        // or, with a device work list, items 0 .. count * gx - 1 walked by a
        // persistent grid (vector list[item / gx], row block item % gx)
        const bool listed = bt.list != nullptr;
        const uint32_t total = listed ? *bt.count * bt.gx : 1;
        for (uint32_t item = listed ? blockIdx.x : 0; item < total; item += listed ? gridDim.x : 1)
        {
        const uint32_t j = listed ? bt.list[item / bt.gx] : blockIdx.y;
        if (! listed && bt.active && ! bt.active[j]) return;
        const uint64_t vo = (uint64_t)j * bt.vstride;
        const T * __restrict__ x = x_ + (uint64_t)j * (bt.xstride ? bt.xstride : bt.vstride);
        T * __restrict__ y = y_ + vo;
        const T * __restrict__ aux = aux_ ? aux_ + vo : aux_;
        T * __restrict__ zero = zero_ ? zero_ + (uint64_t)j * bt.zstride : zero_;
        double * red = red_ ? red_ + j : red_;   // the block reduction offsets its partials / counters itself
        const uint64_t bx = listed ? item % bt.gx : blockIdx.x;
        const uint64_t blk = (flags & kReverse) ? (gridDim.x - 1 - bx) : bx;
        const bool keep = (flags & kKeepL2) != 0;
        const uint64_t r0 = (blk * blockDim.x + threadIdx.x) * R;
        const int K = KT > 0 ? KT : (int)A.K;
        T acc[R];
#pragma unroll
        for (int i = 0; i < R; ++i) acc[i] = T(0);
        if (r0 < A.rows)
        {
            int64_t base[R];
#pragma unroll
            for (int i = 0; i < R; ++i) base[i] = row_base_est(r0 + i, A.rows, A.cols, A.ratio);
            if constexpr (KT > 0)
            {
                CW cw[KT];
                DW dw[KT];
#pragma unroll
                for (int k = 0; k < KT; ++k)
                {
                    cw[k] = ld_policy((const CW *)(A.code + (uint64_t)k * A.ld + r0), keep);
                    dw[k] = ld_policy((const DW *)(A.delta + (uint64_t)k * A.ld + r0), keep);
                }
#pragma unroll
                for (int k = 0; k < KT; ++k)
                {
                    uint32_t code[R];
                    int off[R];
                    unpack<R>(cw[k], dw[k], code, off);
#pragma unroll
                    for (int i = 0; i < R; ++i)
                        if (off[i] != kEmptyOffset) acc[i] = M::add(acc[i], M::mul(table[code[i]], __ldg(x + base[i] + off[i])));
                }
            }
            else
            {
                for (int k = 0; k < K; ++k)
                {
                    uint32_t code[R];
                    int off[R];
                    unpack<R>(ld_policy((const CW *)(A.code + (uint64_t)k * A.ld + r0), keep),
                              ld_policy((const DW *)(A.delta + (uint64_t)k * A.ld + r0), keep), code, off);
#pragma unroll
                    for (int i = 0; i < R; ++i)
                        if (off[i] != kEmptyOffset) acc[i] = M::add(acc[i], M::mul(table[code[i]], __ldg(x + base[i] + off[i])));
                }
            }
        }
        double part = 0.0;
#pragma unroll
        for (int i = 0; i < R; ++i)
        {
            const uint64_t r = r0 + i;
            if (r >= A.rows) break;
            if (MODE == kPlain) y[r] = acc[i];
            else if (MODE == kDefect)
            {
                T d = M::sub(aux[r], acc[i]);
                y[r] = d;
                part = fma((double)d, (double)d, part);
            }
            else if (MODE == kDot)
            {
                y[r] = acc[i];
                part = fma((double)acc[i], (double)x[r], part);
            }
            else if (MODE == kAdd) y[r] = M::add(y[r], acc[i]);
            else if (is_jacobi(MODE))
            {
                // the sweep's defect b - A x, and its square for a fused norm
                const T d = M::sub(aux[r], acc[i]);
                y[r] = M::add(x[r], M::mul(aux2[r], d));
                part = fma((double)d, (double)d, part);
            }
            else if (MODE == kRestrict) { y[r] = acc[i]; zero[r] = T(0); }
        }
        if ((MODE == kDefect || MODE == kDot || MODE == kJacobiNorm) && red != 0)
        {
            __shared__ double scratch[32];
            ell_block_reduce(part, rs, red, want_sqrt, flags, scratch);
        }
        }
    }

    template <typename T, int MODE>
    static void compact_mode(const hb2_ell_s * A, const void * x, void * y, const void * aux, const void * aux2,
                             void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid, cudaStream_t s,
                             int flags, Batch b, unsigned bs)
    {
        EllCompactView<T> v;
        v.code = A->code;
        v.delta = A->delta;
        v.table = (const T *)A->table;
        v.rows = A->rows;
        v.cols = A->cols;
        v.ld = A->ld;
        v.K = A->K;
        v.ntable = A->ntable;
        v.ratio = (double)A->cols / (double)A->rows;
        const T * xp = (const T *)x;
        T * yp = (T *)y;
        const T * ap = (const T *)aux;
        const T * a2 = (const T *)aux2;
        T * zp = (T *)zero;
#define HB2_COMPACT_LAUNCH(KT_, R_)                                                                          \
        launch_pdl(ell_compact_kernel<T, KT_, MODE, R_>, grid, dim3(bs), 0, s, v, xp, yp, ap, a2, zp, rs, \
                   red, want_sqrt, flags, b)
        const int R = red ? A->compact_rpt_red : A->compact_rpt;
        if (A->K == 9) { if (R == 2) HB2_COMPACT_LAUNCH(9, 2); else if (R == 4) HB2_COMPACT_LAUNCH(9, 4); else HB2_COMPACT_LAUNCH(9, 8); }
        else if (A->K == 4) { if (R == 2) HB2_COMPACT_LAUNCH(4, 2); else if (R == 4) HB2_COMPACT_LAUNCH(4, 4); else HB2_COMPACT_LAUNCH(4, 8); }
        else { if (R == 2) HB2_COMPACT_LAUNCH(0, 2); else if (R == 4) HB2_COMPACT_LAUNCH(0, 4); else HB2_COMPACT_LAUNCH(0, 8); }
#undef HB2_COMPACT_LAUNCH
    }

    template <typename T>
    static void compact_typed(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux,
                              const void * aux2, void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid,
                              cudaStream_t s, int f, Batch b, unsigned bs)
    {
        switch (mode)
        {
            case kPlain: compact_mode<T, kPlain>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs); break;
            case kDefect: compact_mode<T, kDefect>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs); break;
            case kDot: compact_mode<T, kDot>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs); break;
            case kAdd: compact_mode<T, kAdd>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs); break;
            case kJacobi:
                if (red) compact_mode<T, kJacobiNorm>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs);
                else compact_mode<T, kJacobi>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs);
                break;
            case kRestrict: compact_mode<T, kRestrict>(A, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, s, f, b, bs); break;
        }
    }

    void launch_ell_compact(const hb2_ell_s * A, int mode, const void * x, void * y, const void * aux,
                            const void * aux2, void * zero, double * red, int want_sqrt, ReduceSlot rs, dim3 grid,
                            cudaStream_t stream, int flags, Batch b, unsigned bs)
    {
        if (A->dtype == HB2_F64) compact_typed<double>(A, mode, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, stream, flags, b, bs);
        else compact_typed<float>(A, mode, x, y, aux, aux2, zero, red, want_sqrt, rs, grid, stream, flags, b, bs);
    }

    static bool compact_enabled()
    {
        const char * v = getenv("HB2_ELL_COMPACT");
        return ! (v && strcmp(v, "0") == 0);
    }

    template <typename T>
    static int build_compact_typed(hb2_ell_s * A, cudaStream_t s)
    {
        const uint64_t n = (uint64_t)A->K * A->ld;
        unsigned long long * keys = 0;
        int * flag = 0;
        uint16_t * cos = 0;
        HB2_CUDA(cudaMalloc(&keys, kDictSlots * sizeof(unsigned long long)));
        cudaError_t e = cudaMalloc(&flag, sizeof(int));
        if (e == cudaSuccess) e = cudaMemsetAsync(keys, 0xFF, kDictSlots * sizeof(unsigned long long), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(flag, 0, sizeof(int), s);
        const unsigned grid = (unsigned)std::min<uint64_t>(4096, (n + 255) / 256);
        if (e == cudaSuccess)
        {
            dict_insert_kernel<T><<<grid, 256, 0, s>>>((const T *)A->val, A->col, n, keys, flag);
            count_launches(1);
            e = cudaGetLastError();
        }
        std::vector<unsigned long long> hk(kDictSlots);
        int hflag = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(hk.data(), keys, kDictSlots * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        int st = e == cudaSuccess ? HB2_OK : cuda_status(e, "ELL compaction (dictionary)");
        std::vector<T> table;
        std::vector<uint16_t> code_of_slot(kDictSlots, 0);
        bool ok = st == HB2_OK && hflag == 0;
        if (ok)
            for (uint32_t h = 0; h < kDictSlots && ok; ++h)
                if (hk[h] != kEmptyKey)
                {
                    if (table.size() == 255) { ok = false; break; }
                    T v;
                    if (sizeof(T) == 8) { unsigned long long b = hk[h]; memcpy(&v, &b, 8); }
                    else { uint32_t b = (uint32_t)hk[h]; memcpy(&v, &b, 4); }
                    code_of_slot[h] = (uint16_t)table.size();
                    table.push_back(v);
                }
        if (ok && ! table.empty())
        {
            e = cudaMalloc(&cos, kDictSlots * sizeof(uint16_t));
            if (e == cudaSuccess) e = cudaMemcpyAsync(cos, code_of_slot.data(), kDictSlots * sizeof(uint16_t), cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaMalloc(&A->table, table.size() * sizeof(T));
            if (e == cudaSuccess) e = cudaMemcpyAsync(A->table, table.data(), table.size() * sizeof(T), cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaMalloc(&A->code, n);
            if (e == cudaSuccess) e = cudaMalloc(&A->delta, n * sizeof(int16_t));
            if (e == cudaSuccess) e = cudaMemsetAsync(flag, 0, sizeof(int), s);
            if (e == cudaSuccess)
            {
                ell_encode_kernel<T><<<grid, 256, 0, s>>>((const T *)A->val, A->col, A->rows, A->cols, A->ld, A->K, keys,
                                                          cos, A->code, A->delta, flag);
                count_launches(1);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) st = cuda_status(e, "ELL compaction (encode)");
            ok = st == HB2_OK && hflag == 0;
            A->ntable = (uint32_t)table.size();
        }
        else ok = false;
        if (! ok)
        {
            // not eligible (too many distinct values, offsets beyond 16 bits) or failed: stay plain
            cudaFree(A->table);
            cudaFree(A->code);
            cudaFree(A->delta);
            A->table = 0;
            A->code = 0;
            A->delta = 0;
            A->ntable = 0;
        }
        else A->compact_bytes = n * 3 + table.size() * sizeof(T);
        cudaFree(keys);
        cudaFree(flag);
        cudaFree(cos);
        return st;
    }

    // Autotuner: time y = A x and the defect with its fused norm on every layout
    // the matrix admits -- plain; compressed with 2, 4 or 8 rows per thread;
    // row patterns with 1, 2 or 4 rows per thread (and the Q1 gather form) --
    // and keep the fastest for each of the two kernel classes; then time the
    // winner's launch shape: blocks of 128, 256 or 512 threads where its kernel
    // takes them (plain, compressed, Q1 gather; the plain one with one thread per
    // row up to 256), and on the plain layout one or two threads per row.  The arrays of a layout neither class uses are
    // freed.  Runs once per matrix shape and process, at creation, on `stream`.
    //
    // The decision is kept per (device, element type, shape, slots, table size)
    // for the life of the process: matrices of one shape always run the same
    // launch shape, so a reduction over them sums in the same order whichever
    // matrix instance (or solver built on it) computes it.
    struct TuneKey
    {
        int device, dtype;
        uint64_t rows, cols;
        uint32_t K, ntable, npat;
        uint32_t kind;   // 0, or for the BF16 layout 1 + 2 * form + compensated
        bool operator<(const TuneKey & o) const
        {
            return std::tie(device, dtype, rows, cols, K, ntable, npat, kind) <
                   std::tie(o.device, o.dtype, o.rows, o.cols, o.K, o.ntable, o.npat, o.kind);
        }
    };
    struct Choice
    {
        int layout[2], rpt[2], bs[2], tpr[2];
    };
    static std::mutex g_tune_mutex;
    static std::map<TuneKey, Choice> g_tune;

    // HB2_TUNE_FILE=<path>: decisions are read from the file when it exists and
    // every new decision is appended to it, so a later process (a profiler
    // run, whose replays would distort the timings) makes the same choices.
    // Called with g_tune_mutex held.
    static void tune_file_load()
    {
        static bool loaded = false;
        if (loaded) return;
        loaded = true;
        const char * path = getenv("HB2_TUNE_FILE");
        if (! path || ! *path) return;
        FILE * f = fopen(path, "r");
        if (! f) return;
        TuneKey k;
        Choice c;
        unsigned long long rows, cols;
        while (fscanf(f, "%d %d %llu %llu %u %u %u %u %d %d %d %d %d %d %d %d", &k.device, &k.dtype, &rows, &cols,
                      &k.K, &k.ntable, &k.npat, &k.kind, &c.layout[0], &c.rpt[0], &c.layout[1], &c.rpt[1], &c.bs[0],
                      &c.tpr[0], &c.bs[1], &c.tpr[1]) == 16)
        {
            k.rows = rows;
            k.cols = cols;
            g_tune[k] = c;
        }
        fclose(f);
    }

    static void tune_file_append(const TuneKey & k, const Choice & c)
    {
        const char * path = getenv("HB2_TUNE_FILE");
        if (! path || ! *path) return;
        FILE * f = fopen(path, "a");
        if (! f) return;
        fprintf(f, "%d %d %llu %llu %u %u %u %u %d %d %d %d %d %d %d %d\n", k.device, k.dtype,
                (unsigned long long)k.rows, (unsigned long long)k.cols, k.K, k.ntable, k.npat, k.kind, c.layout[0],
                c.rpt[0], c.layout[1], c.rpt[1], c.bs[0], c.tpr[0], c.bs[1], c.tpr[1]);
        fclose(f);
    }

    // HB2_ELL_BLOCK=128|256|512 and HB2_ELL_TPR=1|2 override the tuned launch
    // shape (threads per row on the plain layout only; the plain kernel with one
    // thread per row runs 512 as 256); read at each matrix creation
    static int shape_pin(const char * name, int a, int b, int c)
    {
        const char * v = getenv(name);
        const int p = v && *v ? atoi(v) : 0;
        return (p == a || p == b || p == c) ? p : 0;
    }

    static void apply_shape_pins(hb2_ell_s * A)
    {
        const int bs = shape_pin("HB2_ELL_BLOCK", 128, 256, 512), tpr = shape_pin("HB2_ELL_TPR", 1, 2, 1);
        for (int cls = 0; cls < 2; ++cls)
        {
            if (bs) A->bs[cls] = bs;
            if (tpr && A->layout[cls] == kLayoutPlain) A->tpr[cls] = tpr;
            if (A->layout[cls] != kLayoutPlain) A->tpr[cls] = 1;
        }
    }

    static void apply_choice(hb2_ell_s * A, const Choice & c)
    {
        for (int cls = 0; cls < 2; ++cls)
        {
            A->layout[cls] = c.layout[cls];
            A->rpt[cls] = c.rpt[cls];
            A->bs[cls] = c.bs[cls];
            A->tpr[cls] = c.tpr[cls];
        }
        if (c.layout[0] == kLayoutCompact) A->compact_rpt = c.rpt[0];
        if (c.layout[1] == kLayoutCompact) A->compact_rpt_red = c.rpt[1];
        if (c.layout[0] != kLayoutCompact && c.layout[1] != kLayoutCompact)
        {
            ell_free_compact(A);
            A->compact_bytes = 0;
        }
        if (c.layout[0] != kLayoutPattern && c.layout[1] != kLayoutPattern) ell_free_pattern(A);
        apply_shape_pins(A);
    }

    static int autotune(hb2_ell_s * A, cudaStream_t s)
    {
        const TuneKey key = {A->device, A->dtype, A->rows, A->cols, A->K, A->ntable, A->npat,
                             A->bval ? 1u + 2u * (uint32_t)A->bform + (A->bdiag ? 1u : 0u) : 0u};
        {
            std::lock_guard<std::mutex> lock(g_tune_mutex);
            tune_file_load();
            auto it = g_tune.find(key);
            if (it != g_tune.end())
            {
                apply_choice(A, it->second);
                return HB2_OK;
            }
        }
        const size_t es = dtype_size(A->dtype);
        const bool square = A->rows == A->cols;
        Workspace * ws = 0;
        int st = square ? stream_workspace(s, &ws) : HB2_OK;
        if (st) return st;
        // One launch reads and writes a set of four vectors.  Where a set fills an
        // eighth of L2 or more, the bursts rotate over up to eight sets (more than L2 in
        // all) and the candidates are timed against DRAM; smaller sets are timed
        // L2-resident (one set).  Inside a V-cycle a level's passes alternate with the
        // other levels' ones: timed on one 17 MB set, the FP32 level-10 sweep took two
        // rows per thread, and the level-11 mixed solve ran 3.5 % slower than with one.
        void * buf = 0;
        const size_t vb = ((std::max(A->rows, A->cols) * es + 255) / 256) * 256;
        int l2 = 0;
        cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, A->device);
        const size_t set = 4 * vb, l2b = l2 > 0 ? (size_t)l2 : ((size_t)126 << 20);
        const int nsets = set >= l2b / 8 ? (int)std::min<size_t>(8, (2 * l2b + set - 1) / set) : 1;
        HB2_CUDA(cudaMalloc(&buf, nsets * set + 256));
        HB2_CUDA(cudaMemsetAsync(buf, 0, nsets * set + 256, s));
        double * nrm = (double *)((char *)buf + nsets * set);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        // a BF16 matrix runs on its BF16 arrays (1, 2, 4 or 8 rows per thread)
        std::vector<std::pair<int, int>> variants = {{A->bval ? (int)kLayoutBF16 : (int)kLayoutPlain, A->bval ? 1 : 0}};
        if (A->bval)
            for (int r : {2, 4, 8}) variants.push_back(std::make_pair((int)kLayoutBF16, r));
        if (A->code)
            for (int r : {2, 4, 8}) variants.push_back(std::make_pair((int)kLayoutCompact, r));
        if (A->pat)
            for (int r : {1, 2, 4}) variants.push_back(std::make_pair((int)kLayoutPattern, r));
        if (A->pat && A->pat_win_m)
            for (int r : {1, 2}) variants.push_back(std::make_pair((int)kLayoutPattern, r | kPatWin));
        // the Q1 stencil kernel's gather form (its bulk-copy, pair and strip forms
        // measured slower on every level and precision: they stay available as pins)
        if (A->pat && A->q1_full >= 0)
            for (int r : {1, 2, 4}) variants.push_back(std::make_pair((int)kLayoutPattern, r | kPatQ1G));
        // Each candidate is timed as a burst of back-to-back launches (the way the
        // solvers issue them, and long enough for the event clock's granularity),
        // the candidates interleaved over several rounds so that clock or
        // neighbour drift hits all of them; a candidate's time is its best round.
        constexpr int kRounds = 4, kBurst = 8;
        // the fastest candidate; with `incumbent` set, that one unless another beats it
        // by more than kMargin (launch shapes that differ by less than the timing's
        // scatter keep the default)
        constexpr float kMargin = 0.97f;
        auto fastest = [&](int cls, size_t count, const std::function<void(size_t)> & select,
                           long incumbent = -1) -> size_t {
            std::vector<float> best(count, 1e30f);
            for (int round = 0; round <= kRounds && ! st; ++round)   // round 0 warms up
                for (size_t vi = 0; vi < count && ! st; ++vi)
                {
                    select(vi);
                    // a fused reduction needs one partial per row block: shapes beyond
                    // the workspace are not candidates
                    if (cls == 1 && (uint64_t)ell_grid(A, true) > ws->max_blocks) continue;
                    cudaEventRecord(e0, s);
                    // class 0 of a square matrix is timed on the Jacobi sweep (the
                    // multigrid's eight passes per level and cycle), of a rectangular
                    // one on the product
                    for (int b = 0; b < kBurst && ! st; ++b)
                    {
                        char * v = (char *)buf + (b % nsets) * set;
                        void * xv = v, * yv = v + vb, * bv = v + 2 * vb, * pv = v + 3 * vb;
                        st = cls == 1 ? launch_ell(A, kDefect, xv, yv, bv, 0, 0, nrm, 0, ws, s)
                             : square ? launch_ell(A, kJacobi, xv, yv, bv, pv, 0, 0, 0, 0, s)
                                      : launch_ell(A, kPlain, xv, yv, 0, 0, 0, 0, 0, 0, s);
                    }
                    cudaEventRecord(e1, s);
                    if (st) break;
                    cudaEventSynchronize(e1);
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (round > 0 && ms < best[vi]) best[vi] = ms;
                }
            size_t w = 0;
            for (size_t vi = 1; vi < count; ++vi)
                if (best[vi] < best[w]) w = vi;
            if (incumbent >= 0 && best[incumbent] < 1e30f && best[w] > kMargin * best[incumbent])
                w = (size_t)incumbent;
            return w;
        };
        Choice c = {{kLayoutPlain, kLayoutPlain}, {2, 2}, {kEllThreads, kEllThreads}, {1, 1}};
        for (int cls = 0; cls < (square ? 2 : 1) && ! st; ++cls)
        {
            // stage 1: layout and rows per thread, 256 threads per block, one per row
            A->bs[cls] = kEllThreads;
            A->tpr[cls] = 1;
            auto select = [&](const std::pair<int, int> & v) {
                A->layout[cls] = v.first;
                A->rpt[cls] = v.second;
                if (v.first == kLayoutCompact) (cls ? A->compact_rpt_red : A->compact_rpt) = v.second;
            };
            const size_t w = variants.size() > 1 ? fastest(cls, variants.size(), [&](size_t i) { select(variants[i]); }) : 0;
            select(variants[w]);
            c.layout[cls] = variants[w].first;
            c.rpt[cls] = variants[w].second;
            // stage 2: the winner's launch shape
            if (st || ! ell_shape_tunable(A, cls)) continue;   // a kernel of fixed shape
            std::vector<std::pair<int, int>> shapes;
            long incumbent = -1;
            for (int bs : {128, 256, 512})
                for (int tpr : {1, 2})
                    if ((tpr == 1 || A->layout[cls] == kLayoutPlain) &&
                        ! (A->layout[cls] == kLayoutPlain && tpr == 1 && bs > kEllThreads))
                    {
                        if (bs == kEllThreads && tpr == 1) incumbent = (long)shapes.size();
                        shapes.push_back(std::make_pair(bs, tpr));
                    }
            const size_t sw = fastest(cls, shapes.size(), [&](size_t i) {
                A->bs[cls] = shapes[i].first;
                A->tpr[cls] = shapes[i].second;
            }, incumbent);
            c.bs[cls] = shapes[sw].first;
            c.tpr[cls] = shapes[sw].second;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaStreamSynchronize(s);
        cudaFree(buf);
        if (st) return st;
        if (! square)
        {
            c.layout[1] = c.layout[0];
            c.rpt[1] = c.rpt[0];
            c.bs[1] = c.bs[0];
            c.tpr[1] = c.tpr[0];
        }
        {
            std::lock_guard<std::mutex> lock(g_tune_mutex);
            g_tune[key] = c;
            tune_file_append(key, c);
        }
        apply_choice(A, c);
        HB2_LAUNCH_CHECK("ELL layout autotuning");
        return HB2_OK;
    }

    int ell_autotune(hb2_ell_s * A, cudaStream_t stream)
    {
        // HB2_ELL_COMPACT=bf16r1|bf16r2|bf16r4|bf16r8: a BF16 matrix with that many rows per
        // thread, no timing
        const char * v = getenv("HB2_ELL_COMPACT");
        if (A->bval && v && strncmp(v, "bf16r", 5) == 0)
        {
            const int r = atoi(v + 5);
            A->rpt[0] = A->rpt[1] = (r == 1 || r == 2 || r == 8) ? r : 4;
            apply_shape_pins(A);
            return HB2_OK;
        }
        if (A->rows < kShapeMinRows)
        {
            apply_shape_pins(A);
            return HB2_OK;
        }
        return autotune(A, stream);
    }

    int ell_build_compact(hb2_ell_s * A, cudaStream_t stream)
    {
        // HB2_ELL_COMPACT=0 and matrices below kShapeMinRows: the plain layout in its
        // default (or pinned) shape, no timing; below kCompactMinRows, or without a
        // compressed form: the plain layout's shape is timed
        if (! compact_enabled() || A->rows < kShapeMinRows)
        {
            apply_shape_pins(A);
            return HB2_OK;
        }
        if (A->rows < kCompactMinRows) return autotune(A, stream);
        int st = A->dtype == HB2_F64 ? build_compact_typed<double>(A, stream) : build_compact_typed<float>(A, stream);
        if (st) return st;
        if (! A->code) return autotune(A, stream);
        st = ell_build_pattern(A, stream);
        if (st) return st;
        const char * v = getenv("HB2_ELL_COMPACT");
        if (v && (strncmp(v, "force", 5) == 0 || strncmp(v, "pattern", 7) == 0 || strncmp(v, "q1stencil", 9) == 0 ||
                  strncmp(v, "q1gather", 8) == 0 || strncmp(v, "q1pair", 6) == 0 || strncmp(v, "q1strip", 7) == 0))
        {
            // HB2_ELL_COMPACT=force[2|4|8]: the compressed layout with that many
            // rows per thread; pattern[1|2|4]: the row-pattern layout (square
            // matrices that admit it; the others compressed, 2 rows per thread);
            // patternwin[1|2] its windowed kernel where the offsets allow;
            // q1stencil[2|4|8] the Q1 stencil kernel where the matrix holds the full
            // nine-point stencil, q1gather[1|2|4] its gather form, q1pair its pair
            // form, q1strip[2|4|8] its strip form; no autotuning (the default launch shape, or HB2_ELL_BLOCK / HB2_ELL_TPR)
            Choice c = {{kLayoutPlain, kLayoutPlain}, {2, 2}, {kEllThreads, kEllThreads}, {1, 1}};
            if (v[0] == 'p' && A->pat)
            {
                // patternwin[1|2]: the windowed kernel where the matrix admits it
                const bool win = strncmp(v, "patternwin", 10) == 0;
                const int r = atoi(v + (win ? 10 : 7));
                c.layout[0] = c.layout[1] = kLayoutPattern;
                c.rpt[0] = c.rpt[1] = (r == 2 || r == 4) ? r : 1;
                if (win && A->pat_win_m && c.rpt[0] <= 2) c.rpt[0] = c.rpt[1] = c.rpt[0] | kPatWin;
            }
            else if (strncmp(v, "q1stencil", 9) == 0 && A->pat)
            {
                // q1stencil[2|4|8]: the Q1 stencil kernel where the matrix holds the
                // full stencil, else the row-pattern kernel with as many rows per thread
                const int r = atoi(v + 9);
                c.layout[0] = c.layout[1] = kLayoutPattern;
                c.rpt[0] = c.rpt[1] = (r == 4 || r == 8) ? r : 2;
                if (A->q1_full >= 0) c.rpt[0] = c.rpt[1] = c.rpt[0] | kPatQ1;
            }
            else if (strncmp(v, "q1pair", 6) == 0 && A->pat)
            {
                // q1pair: the Q1 stencil kernel's pair form (two adjacent rows per thread)
                c.layout[0] = c.layout[1] = kLayoutPattern;
                c.rpt[0] = c.rpt[1] = 2 | (A->q1_full >= 0 ? kPatQ1P : 0);
            }
            else if (strncmp(v, "q1strip", 7) == 0 && A->pat)
            {
                // q1strip[2|4|8]: the Q1 stencil kernel's strip form (that many grid rows
                // per thread)
                const int r = atoi(v + 7);
                c.layout[0] = c.layout[1] = kLayoutPattern;
                c.rpt[0] = c.rpt[1] = (r == 2 || r == 8) ? r : 4;
                if (A->q1_full >= 0) c.rpt[0] = c.rpt[1] = c.rpt[0] | kPatQ1S;
            }
            else if (strncmp(v, "q1gather", 8) == 0 && A->pat)
            {
                // q1gather[1|2|4]: the Q1 stencil kernel's gather form
                const int r = atoi(v + 8);
                c.layout[0] = c.layout[1] = kLayoutPattern;
                c.rpt[0] = c.rpt[1] = (r == 2 || r == 4) ? r : 1;
                if (A->q1_full >= 0) c.rpt[0] = c.rpt[1] = c.rpt[0] | kPatQ1G;
            }
            else
            {
                const int r = v[0] == 'f' ? atoi(v + 5) : 2;
                c.layout[0] = c.layout[1] = kLayoutCompact;
                c.rpt[0] = c.rpt[1] = (r == 4 || r == 8) ? r : 2;
            }
            apply_choice(A, c);
            return HB2_OK;
        }
        return autotune(A, stream);
    }

    void ell_free_compact(hb2_ell_s * A)
    {
        cudaFree(A->table);
        cudaFree(A->code);
        cudaFree(A->delta);
        A->table = 0;
        A->code = 0;
        A->delta = 0;
    }
}
