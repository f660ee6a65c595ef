// Matrix-free grid transfer: Prolongation<Tag, NONE> (math/prolongation.hh:42-139)
// and Restriction<Tag, NONE> (math/restriction.hh:41-173), each followed by
// ApplyDirichletBoundaries (math/apply_dirichlet_boundaries.hh:29-84).
//
// The reference accumulates each node's value across several sequential
// sweeps over the grid.  Here one thread owns one output node and replays the
// contributions that reach that node in the reference's sweep order, with the
// same roundings, so the output is bit-identical and every node is written
// exactly once (no atomics, one pass over the input).
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <cstdlib>

namespace hb2
{
    struct Mask
    {
        unsigned char bit[8];
    };

    // ApplyDirichletBoundaries: mask entry 2 zeroes a corner or an edge
    // (0 bottom-left, 1 bottom-right, 2 top-right, 3 top-left, 4 bottom edge,
    // 5 right edge, 6 top edge, 7 left edge; edges exclude their corners).
    __device__ __forceinline__ bool dirichlet_zero(const Mask & mk, uint64_t r, uint64_t c, uint64_t M)
    {
        const bool bottom = r == 0, top = r == M - 1, left = c == 0, right = c == M - 1;
        if (bottom && left) return mk.bit[0];
        if (bottom && right) return mk.bit[1];
        if (top && right) return mk.bit[2];
        if (top && left) return mk.bit[3];
        if (bottom) return mk.bit[4];
        if (right) return mk.bit[5];
        if (top) return mk.bit[6];
        if (left) return mk.bit[7];
        return false;
    }

    // fine node (I, J): injection on even/even; 0 + a/2 + b/2 on edge midpoints
    // (left then right, below then above); 0 + BL/4 + BR/4 + TL/4 + TR/4 at
    // cell centres.
    template <typename T>
    __global__ void prolongation_kernel(T * __restrict__ fine, const T * __restrict__ coarse, uint64_t mf, Mask mk)
    {
        typedef Arith<T> M;
        const uint64_t f = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (f >= mf * mf) return;
        const uint64_t mc = (mf + 1) / 2, I = f / mf, J = f % mf;
        const T h = T(0.5), q = T(0.25);
        T v;
        if (I % 2 == 0 && J % 2 == 0) v = coarse[(I / 2) * mc + J / 2];
        else if (I % 2 == 0)
        {
            const uint64_t row = (I / 2) * mc;
            v = M::add(M::add(T(0), M::mul(coarse[row + (J - 1) / 2], h)), M::mul(coarse[row + (J + 1) / 2], h));
        }
        else if (J % 2 == 0)
        {
            v = M::add(M::add(T(0), M::mul(coarse[((I - 1) / 2) * mc + J / 2], h)),
                       M::mul(coarse[((I + 1) / 2) * mc + J / 2], h));
        }
        else
        {
            const uint64_t lo = ((I - 1) / 2) * mc, hi = ((I + 1) / 2) * mc, jl = (J - 1) / 2, jr = (J + 1) / 2;
            v = M::add(T(0), M::mul(coarse[lo + jl], q));
            v = M::add(v, M::mul(coarse[lo + jr], q));
            v = M::add(v, M::mul(coarse[hi + jl], q));
            v = M::add(v, M::mul(coarse[hi + jr], q));
        }
        if (dirichlet_zero(mk, I, J, mf)) v = T(0);
        fine[f] = v;
    }

    // coarse node (I, J): injection of fine (2I, 2J), then for every strip
    // index i = 1..mc-1 that touches the node (I, I+1, J, J+1), in ascending
    // order, the reference's eight per-strip updates in their order:
    //   a (i == I)    += 1/2 fine(2I-1, 2J)      b (i == I+1)  += 1/2 fine(2I+1, 2J)
    //   c (i == J+1)  += 1/2 fine(2I, 2J+1)      d (i == J)    += 1/2 fine(2I, 2J-1)
    //   e1 (i == I+1, J < mc-1) += 1/4 fine(2I+1, 2J+1)
    //   e2 (i == I+1, J > 0)    += 1/4 fine(2I+1, 2J-1)
    //   e3 (i == I,   J < mc-1) += 1/4 fine(2I-1, 2J+1)
    //   e4 (i == I,   J > 0)    += 1/4 fine(2I-1, 2J-1)
    template <typename T>
    __global__ void restriction_kernel(T * __restrict__ coarse, const T * __restrict__ fine, uint64_t mf, Mask mk)
    {
        typedef Arith<T> M;
        const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        const uint64_t mc = (mf + 1) / 2;
        if (c >= mc * mc) return;
        const int64_t I = (int64_t)(c / mc), J = (int64_t)(c % mc), last = (int64_t)mc - 1;
        const int64_t F = (int64_t)mf;
        const T h = T(0.5), q = T(0.25);
#define FINE(r, cc) fine[(r) * F + (cc)]
        T v = FINE(2 * I, 2 * J);
        int64_t cand[4] = {I, I + 1, J, J + 1};
        // ascending unique strip indices in [1, mc-1]
        for (int a = 1; a < 4; ++a)
            for (int b = a; b > 0 && cand[b - 1] > cand[b]; --b) { int64_t t = cand[b]; cand[b] = cand[b - 1]; cand[b - 1] = t; }
        int64_t prev = -1;
        for (int k = 0; k < 4; ++k)
        {
            const int64_t i = cand[k];
            if (i == prev || i < 1 || i > last) { prev = i; continue; }
            prev = i;
            if (i == I) v = M::add(v, M::mul(h, FINE(2 * I - 1, 2 * J)));
            if (i == I + 1) v = M::add(v, M::mul(h, FINE(2 * I + 1, 2 * J)));
            if (i == J + 1) v = M::add(v, M::mul(h, FINE(2 * I, 2 * J + 1)));
            if (i == J) v = M::add(v, M::mul(h, FINE(2 * I, 2 * J - 1)));
            if (i == I + 1 && J < last) v = M::add(v, M::mul(q, FINE(2 * I + 1, 2 * J + 1)));
            if (i == I + 1 && J > 0) v = M::add(v, M::mul(q, FINE(2 * I + 1, 2 * J - 1)));
            if (i == I && J < last) v = M::add(v, M::mul(q, FINE(2 * I - 1, 2 * J + 1)));
            if (i == I && J > 0) v = M::add(v, M::mul(q, FINE(2 * I - 1, 2 * J - 1)));
        }
#undef FINE
        if (dirichlet_zero(mk, (uint64_t)I, (uint64_t)J, mc)) v = T(0);
        coarse[c] = v;
    }

    static bool grid_side(uint64_t n, uint64_t * m)
    {
        uint64_t s = 1;
        while (s * s < n) ++s;
        *m = s;
        return s * s == n && s >= 3 && (s - 1) % 2 == 0;
    }

    static Mask make_mask(const uint64_t * mask)
    {
        Mask mk;
        for (int i = 0; i < 8; ++i) mk.bit[i] = mask ? (mask[i] == 2) : 1;
        return mk;
    }

    // ------------------------------------------------------------------
    // The ProlongationMatrix of the identity index maps (math/prolongation_matrix.hh:44-100)
    // and its Transposition, applied without reading them.  Fine node (i, j) of a grid
    // with mf points per line, coarse node (I, J) = (i / 2, j / 2): the prolongation row
    // holds, in ascending column order, (I, J) with weight 1 (i, j even), (I, J) and
    // (I, J + 1) or (I, J) and (I + 1, J) with 1/2 (one odd), and (I, J), (I, J + 1),
    // (I + 1, J), (I + 1, J + 1) with 1/4 (both odd); the restriction row of (I, J)
    // holds the fine nodes (2I + di, 2J + dj), di, dj in -1..1 inside the grid, in
    // ascending column order, with weight (1 or 1/2) x (1 or 1/2).  Each row is summed
    // as the ELL kernels sum it (0 + v0 x0 + v1 x1 ..., products and sums rounded
    // separately; q1_prolong_row / q1_restrict_row), so the results are bit-identical
    // to the matrix products.
    // R fine rows per thread, interleaved over the block (every access coalesced); the
    // rows' y loads (kAdd) issued before their coarse gathers
    template <typename T, int MODE, int R>
    __global__ void __launch_bounds__(256)
    q1_prolong_kernel(const T * __restrict__ c, T * __restrict__ y, uint32_t mf, uint32_t mc, uint64_t nf,
                      int64_t pf)
    {
        typedef Arith<T> M;
        pdl_entry();
        const uint64_t r0 = (uint64_t)blockIdx.x * blockDim.x * R + threadIdx.x;
        T yv[R];
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const uint64_t r = r0 + (uint64_t)k * blockDim.x;
            yv[k] = (MODE == kAdd && r < nf) ? y[r] : T(0);
            // the fine vector of a later wave of blocks into L2 (y += P c reads it)
            if (MODE == kAdd && pf && r + pf < nf) prefetch_l2(y + r + pf);
        }
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const uint64_t r = r0 + (uint64_t)k * blockDim.x;
            if (r >= nf) break;
            const T acc = q1_prolong_row<T, false>(r, c, mf, mc);
            y[r] = MODE == kAdd ? M::add(yv[k], acc) : acc;
        }
    }

    // rows per thread of the prolongation kernel: 2 for fine grids of 2^21 rows or more,
    // else 1 (graph-timed at level 11 with an L2 prefetch: FP64 19.8 / 18.1 / 21.3 us for
    // 1 / 2 / 4 rows, FP32 18.9 / 16.1 / 16.1 us; the first form, one row and y loaded
    // after the gathers, 26.2 / 23.9 us; inside the MG solves two rows helped at level 11
    // and cost 0.5 % at levels 9 and 10, where the grid of blocks is small);
    // HB2_Q1_PROLONG_R (1, 2 or 4) overrides
    static int prolong_rows(uint64_t nf)
    {
        const char * v = getenv("HB2_Q1_PROLONG_R");
        const int r = v && *v ? atoi(v) : (nf >= (1u << 21) ? 2 : 1);
        return (r == 2 || r == 4) ? r : 1;
    }

    template <typename T, int MODE>
    __global__ void __launch_bounds__(256)
    q1_restrict_kernel(const T * __restrict__ x, T * __restrict__ y, T * __restrict__ zero, uint32_t mf,
                       uint32_t mc, uint64_t nc, int64_t pf)
    {
        pdl_entry();
        const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (r >= nc) return;
        if (pf && r + pf < nc)
        {
            // the three fine grid rows a later wave's coarse row reads, into L2
            const uint64_t rr = r + pf, I = rr / mc, J = rr - I * mc, f = 2 * I * mf + 2 * J, nf = (uint64_t)mf * mf;
            if (f >= mf) prefetch_l2(x + f - mf);
            prefetch_l2(x + f);
            if (f + mf < nf) prefetch_l2(x + f + mf);
        }
        y[r] = q1_restrict_row<T, false>(r, x, mf, mc);
        if (MODE == kRestrict) zero[r] = T(0);
    }

    template <typename T>
    static int q1_transfer_typed(const hb2_ell_s * A, int mode, const void * x, void * y, void * zero,
                                 cudaStream_t s)
    {
        const int L = A->q1_transfer > 0 ? A->q1_transfer : -A->q1_transfer;
        const uint32_t mf = (1u << L) + 1, mc = (1u << (L - 1)) + 1;
        const T * xp = (const T *)x;
        T * yp = (T *)y;
        const dim3 grid(ceil_div(A->rows, 256));
        const int64_t pf = l2_prefetch_rows(sizeof(T));
        if (A->q1_transfer > 0)
        {
            const int R = prolong_rows(A->rows);
            const dim3 pgrid(ceil_div(A->rows, 256 * R));
#define HB2_PROL(R_)                                                                                                   \
            if (mode == kAdd) launch_pdl(q1_prolong_kernel<T, kAdd, R_>, pgrid, dim3(256), 0, s, xp, yp, mf, mc, A->rows, pf); \
            else launch_pdl(q1_prolong_kernel<T, kPlain, R_>, pgrid, dim3(256), 0, s, xp, yp, mf, mc, A->rows, pf)
            if (R == 4) { HB2_PROL(4); }
            else if (R == 2) { HB2_PROL(2); }
            else { HB2_PROL(1); }
#undef HB2_PROL
        }
        else
        {
            if (mode == kRestrict)
                launch_pdl(q1_restrict_kernel<T, kRestrict>, grid, dim3(256), 0, s, xp, yp, (T *)zero, mf, mc, A->rows,
                           pf);
            else launch_pdl(q1_restrict_kernel<T, kPlain>, grid, dim3(256), 0, s, xp, yp, (T *)zero, mf, mc, A->rows,
                            pf);
        }
        return HB2_OK;
    }

    int launch_q1_transfer(const hb2_ell_s * A, int mode, const void * x, void * y, void * zero, cudaStream_t stream)
    {
        // a prolongation computes kPlain / kAdd rows, a restriction kPlain / kRestrict rows
        if ((A->q1_transfer > 0 && mode == kRestrict) || (A->q1_transfer < 0 && mode == kAdd))
            return fail(HB2_ERR_UNSUPPORTED, "Q1 transfer kernel: mode");
        const int st = A->dtype == HB2_F64 ? q1_transfer_typed<double>(A, mode, x, y, zero, stream)
                                           : q1_transfer_typed<float>(A, mode, x, y, zero, stream);
        count_launches(1);
        HB2_LAUNCH_CHECK("Q1 transfer kernel launch");
        return st;
    }
}

using namespace hb2;

extern "C" int hb2_prolongation(hb2_dtype dt, void * fine, uint64_t n_fine, const void * coarse, uint64_t n_coarse,
                                const uint64_t * mask, cudaStream_t stream)
{
    uint64_t mf = 0;
    if (! fine || ! coarse) return fail(HB2_ERR_ARG, "hb2_prolongation: null vector");
    if (! grid_side(n_fine, &mf) || ((mf + 1) / 2) * ((mf + 1) / 2) != n_coarse)
        return fail(HB2_ERR_SIZE, "hb2_prolongation: sizes are not (2m-1)^2 / m^2 grids");
    unsigned grid = ceil_div(n_fine, 256);
    Mask mk = make_mask(mask);
    if (dt == HB2_F64) prolongation_kernel<double><<<grid, 256, 0, stream>>>((double *)fine, (const double *)coarse, mf, mk);
    else prolongation_kernel<float><<<grid, 256, 0, stream>>>((float *)fine, (const float *)coarse, mf, mk);
    count_launches(1);
    HB2_LAUNCH_CHECK("hb2_prolongation");
    return HB2_OK;
}

extern "C" int hb2_restriction(hb2_dtype dt, void * coarse, uint64_t n_coarse, const void * fine, uint64_t n_fine,
                               const uint64_t * mask, cudaStream_t stream)
{
    uint64_t mf = 0;
    if (! fine || ! coarse) return fail(HB2_ERR_ARG, "hb2_restriction: null vector");
    if (! grid_side(n_fine, &mf) || ((mf + 1) / 2) * ((mf + 1) / 2) != n_coarse)
        return fail(HB2_ERR_SIZE, "hb2_restriction: sizes are not (2m-1)^2 / m^2 grids");
    unsigned grid = ceil_div(n_coarse, 256);
    Mask mk = make_mask(mask);
    if (dt == HB2_F64) restriction_kernel<double><<<grid, 256, 0, stream>>>((double *)coarse, (const double *)fine, mf, mk);
    else restriction_kernel<float><<<grid, 256, 0, stream>>>((float *)coarse, (const float *)fine, mf, mk);
    count_launches(1);
    HB2_LAUNCH_CHECK("hb2_restriction");
    return HB2_OK;
}
