/*
 * CPU oracle for the HONEI sparse Poisson solver path -- TEST INFRASTRUCTURE ONLY.
 * See honei_oracle.h for the contract.  Every routine restates the reference
 * algorithm named in its comment; none of it is product code.
 *
 * Build: gcc -std=c99 -O2 -ffp-contract=off -fPIC -shared: every a*b+c is
 * rounded twice, as in the reference's compiled tags::CPU loops.
 */
#include "honei_oracle.h"

#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* seeded inputs                                                             */
/* ------------------------------------------------------------------------ */
static uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double hbo_uniform(uint64_t seed, uint64_t i, double lo, double hi)
{
    uint64_t z = mix64(seed + (i + 1) * 0x9E3779B97F4A7C15ULL);
    double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    return lo + (hi - lo) * u;
}

void hbo_uniform_fill_f64(double *out, uint64_t n, uint64_t seed, double lo, double hi)
{
    for (uint64_t i = 0; i < n; ++i) out[i] = hbo_uniform(seed, i, lo, hi);
}

void hbo_uniform_fill_f32(float *out, uint64_t n, uint64_t seed, double lo, double hi)
{
    for (uint64_t i = 0; i < n; ++i) out[i] = (float)hbo_uniform(seed, i, lo, hi);
}

/* ------------------------------------------------------------------------ */
/* Q1 operator and ELL assembly                                              */
/* ------------------------------------------------------------------------ */
uint64_t hbo_q1_m(unsigned L) { return (1ULL << L) + 1; }
uint64_t hbo_q1_n(unsigned L) { uint64_t m = hbo_q1_m(L); return m * m; }

enum { LL, LD, LU, DL, DD, DU, UL, UD, UU };

/* a*b + c with two roundings: the reference's compiled CPU loops do not contract
 * to fma (checked bit-for-bit against its tags::CPU outputs), and this file is
 * built with -ffp-contract=off so the compiler cannot contract it either. */
#define MULADD(a, b, c) ((a) * (b) + (c))

/* math/fill_matrix.hh:37-79.  1-based row i is a Dirichlet unit row when
 * i <= M, i > N-M, i%M == 1 or i%M == 0; otherwise diag 8/3, neighbours -1/3. */
#define DEFINE_Q1_BANDS(T, SFX)                                                     \
void hbo_q1_bands_##SFX(unsigned L, double aniso, T *bands)                         \
{                                                                                   \
    uint64_t M = hbo_q1_m(L), N = M * M;                                            \
    for (uint64_t i = 1; i <= N; ++i) {                                             \
        int dirichlet = (i <= M || i > N - M || (i % M) == 1 || (i % M) == 0);     \
        for (int b = 0; b < 9; ++b) bands[b * N + i - 1] = (T)0.0;                  \
        if (dirichlet) {                                                            \
            bands[DD * N + i - 1] = (T)1.0;                                         \
        } else {                                                                    \
            for (int b = 0; b < 9; ++b) bands[b * N + i - 1] = (T)(-1.0 / 3.0);     \
            if (aniso == 1.0) {                                                     \
                bands[DD * N + i - 1] = (T)(8.0 / 3.0);                             \
            } else {                                                                \
                bands[DL * N + i - 1] = (T)(-aniso / 3.0);                          \
                bands[DU * N + i - 1] = (T)(-aniso / 3.0);                          \
                bands[DD * N + i - 1] = (T)((6.0 + 2.0 * aniso) / 3.0);             \
            }                                                                       \
        }                                                                           \
    }                                                                               \
}
DEFINE_Q1_BANDS(double, f64)
DEFINE_Q1_BANDS(float, f32)

/* la/sparse_matrix.hh:221-300: each band contributes (row, row+offset) for the
 * rows where that column exists and the entry is nonzero; SparseVector keeps
 * each row sorted by column, so the CSR rows come out in band-offset order. */
#define DEFINE_Q1_CSR(T, SFX)                                                       \
uint64_t hbo_q1_csr_##SFX(unsigned L, const T *bands, uint64_t *rowptr,             \
                          uint64_t *colidx, T *vals)                                \
{                                                                                   \
    int64_t m = (int64_t)hbo_q1_m(L), n = m * m;                                    \
    const int64_t off[9] = {-m - 1, -m, -m + 1, -1, 0, 1, m - 1, m, m + 1};         \
    uint64_t nnz = 0;                                                               \
    for (int64_t r = 0; r < n; ++r) {                                               \
        rowptr[r] = nnz;                                                            \
        for (int b = 0; b < 9; ++b) {                                               \
            int64_t c = r + off[b];                                                 \
            if (c < 0 || c >= n) continue;                                          \
            T v = bands[b * n + r];                                                 \
            if (v == (T)0) continue;                                                \
            colidx[nnz] = (uint64_t)c; vals[nnz] = v; ++nnz;                        \
        }                                                                           \
    }                                                                               \
    rowptr[n] = nnz;                                                                \
    return nnz;                                                                     \
}
DEFINE_Q1_CSR(double, f64)
DEFINE_Q1_CSR(float, f32)

/* la/sparse_matrix_ell-impl.hh:75-99 */
void hbo_ell_dims(uint64_t rows, const uint64_t *rowptr, uint64_t T,
                  uint64_t *stride, uint64_t *K)
{
    uint64_t maxnz = 1;
    for (uint64_t r = 0; r < rows; ++r) {
        uint64_t u = rowptr[r + 1] - rowptr[r];
        if (u > maxnz) maxnz = u;
    }
    *K = (maxnz + T - 1) / T;
    *stride = 32 * ((rows * T + 31) / 32);
}

/* la/sparse_matrix_ell-impl.hh:84-118: zero values are skipped in placement but
 * still counted in Arl (ceil(used/T)). */
#define DEFINE_ELL_FROM_CSR(T_, SFX)                                                \
void hbo_ell_from_csr_##SFX(uint64_t rows, const uint64_t *rowptr,                  \
                            const uint64_t *colidx, const T_ *vals, uint64_t T,     \
                            uint64_t stride, uint64_t K, uint64_t *Aj, T_ *Ax,      \
                            uint64_t *Arl)                                          \
{                                                                                   \
    memset(Aj, 0, sizeof(uint64_t) * K * stride);                                   \
    memset(Ax, 0, sizeof(T_) * K * stride);                                         \
    for (uint64_t r = 0; r < rows; ++r) {                                           \
        uint64_t used = rowptr[r + 1] - rowptr[r], t = 0;                           \
        Arl[r] = (used + T - 1) / T;                                                \
        for (uint64_t e = rowptr[r]; e < rowptr[r + 1]; ++e) {                      \
            if (vals[e] == (T_)0) continue;                                         \
            uint64_t pos = (t % T) + r * T + (t / T) * stride;                      \
            Aj[pos] = colidx[e]; Ax[pos] = vals[e]; ++t;                            \
        }                                                                           \
    }                                                                               \
}
DEFINE_ELL_FROM_CSR(double, f64)
DEFINE_ELL_FROM_CSR(float, f32)

/* la/sparse_matrix_ell-impl.hh:186-208 */
void hbo_ell_row_length_f64(uint64_t rows, uint64_t stride, uint64_t K, uint64_t T,
                            const double *Ax, uint64_t *Arl)
{
    uint64_t size = K * stride;
    for (uint64_t r = 0; r < rows; ++r) {
        uint64_t count = 0;
        for (uint64_t i = r * T; i < size; i += stride) {
            int stop = 0;
            for (uint64_t t = 0; t < T; ++t) {
                if (Ax[i + t] == 0.0) { stop = 1; break; }
                if (t == 0) ++count;
            }
            if (stop) break;
        }
        Arl[r] = count;
    }
}

/* math/prolongation_matrix.hh:36-39 */
static uint64_t coarse_index(uint64_t fine_index, uint64_t fine_grid_row, uint64_t offset)
{
    return (fine_index / 2) - ((fine_grid_row / 2) * ((offset - 1) / 2));
}

static void sort_row(uint64_t *c, double *v, uint64_t k)
{
    for (uint64_t a = 1; a < k; ++a)
        for (uint64_t b = a; b > 0 && c[b - 1] > c[b]; --b) {
            uint64_t tc = c[b]; c[b] = c[b - 1]; c[b - 1] = tc;
            double tv = v[b]; v[b] = v[b - 1]; v[b - 1] = tv;
        }
}

/* math/prolongation_matrix.hh:44-100 with identity index arrays */
uint64_t hbo_prolmat_csr_f64(unsigned Lf, uint64_t *rowptr, uint64_t *colidx, double *vals)
{
    uint64_t d = hbo_q1_m(Lf), nnz = 0;
    for (uint64_t i = 0; i < d; ++i)
        for (uint64_t j = 0; j < d; ++j) {
            uint64_t f = i * d + j, k = 0;
            uint64_t *c = colidx + nnz;
            double *v = vals + nnz;
            rowptr[f] = nnz;
            if (i % 2 == 0) {
                if (j % 2 == 0) {
                    c[k] = coarse_index(f, i, d); v[k++] = 1.0;
                } else {
                    c[k] = coarse_index(f - 1, i, d); v[k++] = 0.5;
                    c[k] = coarse_index(f + 1, i, d); v[k++] = 0.5;
                }
            } else if (j % 2 == 0) {
                c[k] = coarse_index(f + d, i + 1, d); v[k++] = 0.5;
                c[k] = coarse_index(f - d, i - 1, d); v[k++] = 0.5;
            } else {
                c[k] = coarse_index(f + d + 1, i + 1, d); v[k++] = 0.25;
                c[k] = coarse_index(f + d - 1, i + 1, d); v[k++] = 0.25;
                c[k] = coarse_index(f - d + 1, i - 1, d); v[k++] = 0.25;
                c[k] = coarse_index(f - d - 1, i - 1, d); v[k++] = 0.25;
            }
            sort_row(c, v, k);
            nnz += k;
        }
    rowptr[d * d] = nnz;
    return nnz;
}

/* math/transposition.hh:36-50 */
void hbo_csr_transpose_f64(uint64_t rows, uint64_t cols, const uint64_t *rowptr,
                           const uint64_t *colidx, const double *vals,
                           uint64_t *rowptr_t, uint64_t *colidx_t, double *vals_t)
{
    uint64_t nnz = rowptr[rows];
    memset(rowptr_t, 0, sizeof(uint64_t) * (cols + 1));
    for (uint64_t e = 0; e < nnz; ++e) rowptr_t[colidx[e] + 1]++;
    for (uint64_t c = 0; c < cols; ++c) rowptr_t[c + 1] += rowptr_t[c];
    uint64_t *fill = (uint64_t *)malloc(sizeof(uint64_t) * (cols + 1));
    memcpy(fill, rowptr_t, sizeof(uint64_t) * (cols + 1));
    /* rows visited in ascending order -> every transposed row is column-sorted */
    for (uint64_t r = 0; r < rows; ++r)
        for (uint64_t e = rowptr[r]; e < rowptr[r + 1]; ++e) {
            uint64_t p = fill[colidx[e]]++;
            colidx_t[p] = r; vals_t[p] = vals[e];
        }
    free(fill);
}

/* ------------------------------------------------------------------------ */
/* operators                                                                 */
/* ------------------------------------------------------------------------ */
/* la/product.hh:148-206 (sum over Arl[row] slot groups of T entries) */
#define DEFINE_ELL_SPMV(T_, SFX, FMA)                                               \
void hbo_ell_spmv_##SFX(uint64_t rows, uint64_t stride, uint64_t T,                 \
                        const uint64_t *Aj, const T_ *Ax, const uint64_t *Arl,      \
                        const T_ *x, T_ *y)                                         \
{                                                                                   \
    for (uint64_t r = 0; r < rows; ++r) {                                           \
        T_ sum = 0;                                                                 \
        for (uint64_t col = 0, j = r * T; col < Arl[r]; ++col, j += stride)        \
            for (uint64_t t = 0; t < T; ++t)                                        \
                sum = FMA(Ax[j + t], x[Aj[j + t]], sum);                            \
        y[r] = sum;                                                                 \
    }                                                                               \
}                                                                                   \
void hbo_ell_defect_##SFX(uint64_t rows, uint64_t stride, uint64_t T,               \
                          const uint64_t *Aj, const T_ *Ax, const uint64_t *Arl,    \
                          const T_ *rhs, const T_ *x, T_ *r)                        \
{                                                                                   \
    for (uint64_t i = 0; i < rows; ++i) {                                           \
        T_ sum = 0;                                                                 \
        for (uint64_t col = 0, j = i * T; col < Arl[i]; ++col, j += stride)        \
            for (uint64_t t = 0; t < T; ++t)                                        \
                sum = FMA(Ax[j + t], x[Aj[j + t]], sum);                            \
        r[i] = rhs[i] - sum;                                                        \
    }                                                                               \
}
DEFINE_ELL_SPMV(double, f64, MULADD)
DEFINE_ELL_SPMV(float, f32, MULADD)

/* la/product.hh:208-244, math/defect.hh:385-420: SparseMatrixCSR with csr::blocksize
 * bs -- Ar[row]..Ar[row+1] blocks, block i starting at column Aj[i] with bs values
 * Ax[i*bs ..]; a block value whose column is >= the vector size is skipped */
#define DEFINE_CSR_SPMV(T_, SFX, FMA)                                               \
static T_ csr_row_##SFX(uint64_t row, uint64_t bs, uint64_t ncols, const uint64_t *Ar, \
                        const uint64_t *Aj, const T_ *Ax, const T_ *x)              \
{                                                                                   \
    T_ sum = 0;                                                                     \
    for (uint64_t i = Ar[row]; i < Ar[row + 1]; ++i)                                \
        for (uint64_t b = 0; b < bs; ++b)                                           \
            if (Aj[i] + b < ncols) sum = FMA(Ax[i * bs + b], x[Aj[i] + b], sum);    \
    return sum;                                                                     \
}                                                                                   \
void hbo_csr_spmv_##SFX(uint64_t rows, uint64_t bs, uint64_t ncols, const uint64_t *Ar, \
                        const uint64_t *Aj, const T_ *Ax, const T_ *x, T_ *y)       \
{                                                                                   \
    for (uint64_t r = 0; r < rows; ++r) y[r] = csr_row_##SFX(r, bs, ncols, Ar, Aj, Ax, x); \
}                                                                                   \
void hbo_csr_defect_##SFX(uint64_t rows, uint64_t bs, uint64_t ncols, const uint64_t *Ar, \
                          const uint64_t *Aj, const T_ *Ax, const T_ *rhs, const T_ *x, \
                          T_ *res)                                                  \
{                                                                                   \
    for (uint64_t r = 0; r < rows; ++r)                                             \
        res[r] = rhs[r] - csr_row_##SFX(r, bs, ncols, Ar, Aj, Ax, x);               \
}
DEFINE_CSR_SPMV(double, f64, fma)
DEFINE_CSR_SPMV(float, f32, fmaf)

/* la/product.hh:370-403 */
#define DEFINE_Q1_SPMV(T_, SFX, FMA)                                                \
void hbo_q1_spmv_##SFX(uint64_t n, uint64_t m, const T_ *bands, const T_ *x, T_ *y)\
{                                                                                   \
    int64_t N = (int64_t)n, root = (int64_t)m;                                      \
    const int64_t off[9] = {-root - 1, -root, -root + 1, -1, 0, 1, root - 1, root, root + 1}; \
    for (int64_t i = 0; i < N; ++i) {                                               \
        T_ s = bands[DD * N + i] * x[i];                                            \
        for (int b = 0; b < 9; ++b) {                                               \
            if (b == DD) continue;                                                  \
            int64_t c = i + off[b];                                                 \
            if (c >= 0 && c < N) s = FMA(bands[b * N + i], x[c], s);                \
        }                                                                           \
        y[i] = s;                                                                   \
    }                                                                               \
}                                                                                   \
void hbo_q1_defect_##SFX(uint64_t n, uint64_t m, const T_ *bands, const T_ *rhs,   \
                         const T_ *x, T_ *r)                                        \
{                                                                                   \
    hbo_q1_spmv_##SFX(n, m, bands, x, r);                                           \
    for (uint64_t i = 0; i < n; ++i) r[i] = rhs[i] - r[i];                          \
}
DEFINE_Q1_SPMV(double, f64, MULADD)
DEFINE_Q1_SPMV(float, f32, MULADD)

/* la/dot_product.hh:72-89: sequential in index order.  Unlike the ELL product,
 * the reference's compiled dot product contracts to fma (checked bit-for-bit). */
double hbo_dot_f64(uint64_t n, const double *x, const double *y)
{
    double s = 0;
    for (uint64_t i = 0; i < n; ++i) s = fma(x[i], y[i], s);
    return s;
}

float hbo_dot_f32(uint64_t n, const float *x, const float *y)
{
    float s = 0;
    for (uint64_t i = 0; i < n; ++i) s = fmaf(x[i], y[i], s);
    return s;
}

/* math/apply_dirichlet_boundaries.hh:29-84 */
#define DEFINE_DIRICHLET(T_, SFX)                                                   \
static void dirichlet_##SFX(T_ *g, uint64_t N, const uint64_t *mask)                \
{                                                                                   \
    uint64_t M = (uint64_t)sqrt((double)N);                                         \
    if (mask[0] == 2) g[0] = 0;                                                     \
    if (mask[1] == 2) g[M - 1] = 0;                                                 \
    if (mask[2] == 2) g[N - 1] = 0;                                                 \
    if (mask[3] == 2) g[N - M] = 0;                                                 \
    if (mask[4] == 2) for (uint64_t i = 1; i < M - 1; ++i) g[i] = 0;                \
    if (mask[5] == 2) for (uint64_t i = 2 * M - 1; i < N - M; i += M) g[i] = 0;     \
    if (mask[6] == 2) for (uint64_t i = N - M + 1; i < N - 1; ++i) g[i] = 0;        \
    if (mask[7] == 2) for (uint64_t i = M; i < N - M; i += M) g[i] = 0;             \
}
DEFINE_DIRICHLET(double, f64)
DEFINE_DIRICHLET(float, f32)

/* math/prolongation.hh:42-139: inject coarse nodes, then edge midpoints as
 * 0.5*(a+b) accumulated a then b, then cell centres as 0.25 * (BL, BR, TL, TR)
 * accumulated in that order; finally zero the Dirichlet boundary. */
#define DEFINE_PROLONGATION(T_, SFX)                                                \
void hbo_prolongation_##SFX(uint64_t n_fine, T_ *fine, uint64_t n_coarse,           \
                            const T_ *coarse, const uint64_t *mask)                 \
{                                                                                   \
    uint64_t mf = (uint64_t)sqrt((double)n_fine), mc = (mf + 1) / 2;                \
    (void)n_coarse;                                                                 \
    for (uint64_t i = 0; i < n_fine; ++i) fine[i] = 0;                              \
    for (uint64_t i = 0; i < mc; ++i)                                               \
        for (uint64_t j = 0; j < mc; ++j)                                           \
            fine[2 * i * mf + 2 * j] = coarse[i * mc + j];                          \
    for (uint64_t i = 1; i < mc; ++i) {                                             \
        for (uint64_t j = 0; j < mc; ++j) {                                         \
            T_ *f = &fine[2 * j * mf + 2 * i - 1];                                  \
            *f += coarse[j * mc + i - 1] * (T_)0.5;                                 \
            *f += coarse[j * mc + i] * (T_)0.5;                                     \
        }                                                                           \
        for (uint64_t j = 0; j < mc; ++j) {                                         \
            uint64_t k = (2 * i - 1) * mf + 2 * j;                                  \
            fine[k] += fine[k - mf] * (T_)0.5;                                      \
            fine[k] += fine[k + mf] * (T_)0.5;                                      \
        }                                                                           \
    }                                                                               \
    for (uint64_t i = 1; i < mc; ++i)                                               \
        for (uint64_t j = 0; j + 1 < mc; ++j) {                                     \
            uint64_t k = (2 * i - 1) * mf + 2 * j + 1;                              \
            fine[k] += fine[k - mf - 1] * (T_)0.25;                                 \
            fine[k] += fine[k - mf + 1] * (T_)0.25;                                 \
            fine[k] += fine[k + mf - 1] * (T_)0.25;                                 \
            fine[k] += fine[k + mf + 1] * (T_)0.25;                                 \
        }                                                                           \
    dirichlet_##SFX(fine, n_fine, mask);                                            \
}
DEFINE_PROLONGATION(double, f64)
DEFINE_PROLONGATION(float, f32)

/* math/restriction.hh:41-173: inject, then for every coarse column/row strip i
 * the four half-weight edge contributions and the four quarter-weight centre
 * contributions, in the reference's loop order; then the Dirichlet boundary. */
#define DEFINE_RESTRICTION(T_, SFX)                                                 \
void hbo_restriction_##SFX(uint64_t n_coarse, T_ *coarse, uint64_t n_fine,          \
                           const T_ *fine, const uint64_t *mask)                    \
{                                                                                   \
    uint64_t mf = (uint64_t)sqrt((double)n_fine), mc = (mf + 1) / 2;                \
    for (uint64_t i = 0; i < mc; ++i)                                               \
        for (uint64_t j = 0; j < mc; ++j)                                           \
            coarse[i * mc + j] = fine[2 * i * mf + 2 * j];                          \
    for (uint64_t i = 1; i < mc; ++i) {                                             \
        for (uint64_t j = 0; j < mc; ++j)                                           \
            coarse[i * mc + j] += (T_)0.5 * fine[(2 * i - 1) * mf + 2 * j];         \
        for (uint64_t j = 0; j < mc; ++j)                                           \
            coarse[(i - 1) * mc + j] += (T_)0.5 * fine[(2 * i - 1) * mf + 2 * j];   \
        for (uint64_t j = 0; j < mc; ++j)                                           \
            coarse[j * mc + i - 1] += (T_)0.5 * fine[2 * j * mf + 2 * i - 1];       \
        for (uint64_t j = 0; j < mc; ++j)                                           \
            coarse[j * mc + i] += (T_)0.5 * fine[2 * j * mf + 2 * i - 1];           \
        for (uint64_t j = 0; j + 1 < mc; ++j)                                       \
            coarse[(i - 1) * mc + j] += (T_)0.25 * fine[(2 * i - 1) * mf + 2 * j + 1]; \
        for (uint64_t j = 0; j + 1 < mc; ++j)                                       \
            coarse[(i - 1) * mc + j + 1] += (T_)0.25 * fine[(2 * i - 1) * mf + 2 * j + 1]; \
        for (uint64_t j = 0; j + 1 < mc; ++j)                                       \
            coarse[i * mc + j] += (T_)0.25 * fine[(2 * i - 1) * mf + 2 * j + 1];    \
        for (uint64_t j = 0; j + 1 < mc; ++j)                                       \
            coarse[i * mc + j + 1] += (T_)0.25 * fine[(2 * i - 1) * mf + 2 * j + 1]; \
    }                                                                               \
    dirichlet_##SFX(coarse, n_coarse, mask);                                        \
}
DEFINE_RESTRICTION(double, f64)
DEFINE_RESTRICTION(float, f32)

/* ------------------------------------------------------------------------ */
/* solvers                                                                   */
/* ------------------------------------------------------------------------ */
#define DEFINE_SOLVERS(T_, SFX, EPS_MACH, FMA)                                           \
typedef struct {                                                                    \
    uint64_t rows, cols, stride, K;                                                 \
    uint64_t *Aj, *Arl;                                                             \
    T_ *Ax;                                                                         \
} ell_##SFX;                                                                        \
                                                                                    \
static void ell_free_##SFX(ell_##SFX *e)                                            \
{ free(e->Aj); free(e->Arl); free(e->Ax); }                                         \
                                                                                    \
static void ell_from_csr_##SFX(ell_##SFX *e, uint64_t rows, uint64_t cols,          \
                               const uint64_t *rp, const uint64_t *ci, const T_ *v) \
{                                                                                   \
    e->rows = rows; e->cols = cols;                                                 \
    hbo_ell_dims(rows, rp, 1, &e->stride, &e->K);                                   \
    e->Aj = (uint64_t *)malloc(sizeof(uint64_t) * e->K * e->stride);                \
    e->Ax = (T_ *)malloc(sizeof(T_) * e->K * e->stride);                            \
    e->Arl = (uint64_t *)malloc(sizeof(uint64_t) * rows);                           \
    hbo_ell_from_csr_##SFX(rows, rp, ci, v, 1, e->stride, e->K, e->Aj, e->Ax, e->Arl); \
}                                                                                   \
                                                                                    \
static void q1_ell_##SFX(ell_##SFX *e, unsigned L, double aniso)                    \
{                                                                                   \
    uint64_t n = hbo_q1_n(L);                                                       \
    T_ *bands = (T_ *)malloc(sizeof(T_) * 9 * n);                                   \
    uint64_t *rp = (uint64_t *)malloc(sizeof(uint64_t) * (n + 1));                  \
    uint64_t *ci = (uint64_t *)malloc(sizeof(uint64_t) * 9 * n);                    \
    T_ *v = (T_ *)malloc(sizeof(T_) * 9 * n);                                       \
    hbo_q1_bands_##SFX(L, aniso, bands);                                            \
    hbo_q1_csr_##SFX(L, bands, rp, ci, v);                                          \
    ell_from_csr_##SFX(e, n, n, rp, ci, v);                                         \
    free(bands); free(rp); free(ci); free(v);                                       \
}                                                                                   \
                                                                                    \
/* prolongation P(Lf <- Lf-1) and restriction R = P^T as ELL (T=1) */              \
static void transfer_ell_##SFX(ell_##SFX *P, ell_##SFX *R, unsigned Lf)             \
{                                                                                   \
    uint64_t nf = hbo_q1_n(Lf), nc = hbo_q1_n(Lf - 1);                              \
    uint64_t *rp = (uint64_t *)malloc(sizeof(uint64_t) * (nf + 1));                 \
    uint64_t *ci = (uint64_t *)malloc(sizeof(uint64_t) * 4 * nf);                   \
    double *v = (double *)malloc(sizeof(double) * 4 * nf);                          \
    uint64_t nnz = hbo_prolmat_csr_f64(Lf, rp, ci, v);                              \
    uint64_t *rpt = (uint64_t *)malloc(sizeof(uint64_t) * (nc + 1));                \
    uint64_t *cit = (uint64_t *)malloc(sizeof(uint64_t) * nnz);                     \
    double *vt = (double *)malloc(sizeof(double) * nnz);                            \
    hbo_csr_transpose_f64(nf, nc, rp, ci, v, rpt, cit, vt);                         \
    T_ *tv = (T_ *)malloc(sizeof(T_) * nnz);                                        \
    for (uint64_t e = 0; e < nnz; ++e) tv[e] = (T_)v[e];                            \
    ell_from_csr_##SFX(P, nf, nc, rp, ci, tv);                                      \
    for (uint64_t e = 0; e < nnz; ++e) tv[e] = (T_)vt[e];                           \
    ell_from_csr_##SFX(R, nc, nf, rpt, cit, tv);                                    \
    free(rp); free(ci); free(v); free(rpt); free(cit); free(vt); free(tv);          \
}                                                                                   \
                                                                                    \
static void spmv_##SFX(const ell_##SFX *A, const T_ *x, T_ *y)                      \
{ hbo_ell_spmv_##SFX(A->rows, A->stride, 1, A->Aj, A->Ax, A->Arl, x, y); }         \
static void defect_##SFX(const ell_##SFX *A, const T_ *b, const T_ *x, T_ *r)       \
{ hbo_ell_defect_##SFX(A->rows, A->stride, 1, A->Aj, A->Ax, A->Arl, b, x, r); }    \
                                                                                    \
/* diagonal entry A(j,j) as the reference's element access finds it */              \
static T_ ell_diag_##SFX(const ell_##SFX *A, uint64_t r)                            \
{                                                                                   \
    for (uint64_t k = 0; k < A->Arl[r]; ++k)                                        \
        if (A->Aj[r + k * A->stride] == r) return A->Ax[r + k * A->stride];         \
    return (T_)0;                                                                   \
}                                                                                   \
                                                                                    \
/* math/cg.hh:64-135 */                                                             \
static uint64_t cg_##SFX(const ell_##SFX *A, const T_ *b, T_ *x, uint64_t max_iters,\
                         T_ eps)                                                    \
{                                                                                   \
    uint64_t n = A->rows, it = 0, used = 0;                                         \
    T_ *p = (T_ *)malloc(sizeof(T_) * n), *r = (T_ *)malloc(sizeof(T_) * n);        \
    T_ *v = (T_ *)malloc(sizeof(T_) * n);                                           \
    defect_##SFX(A, b, x, r);                                                       \
    memcpy(p, r, sizeof(T_) * n);                                                   \
    T_ alpha = hbo_dot_##SFX(n, r, r), alpha_old, lambda, temp;                     \
    T_ initial = (T_)sqrt(alpha);                                                   \
    while (it < max_iters) {                                                        \
        spmv_##SFX(A, p, v);                                                        \
        temp = hbo_dot_##SFX(n, v, p);                                              \
        lambda = alpha / (fabs(temp) > EPS_MACH ? temp : EPS_MACH);                 \
        /* ScaledSum x += b*y (la/scaled_sum.hh:73-88) */                          \
        for (uint64_t i = 0; i < n; ++i) x[i] = FMA(lambda, p[i], x[i]);            \
        for (uint64_t i = 0; i < n; ++i) r[i] = FMA(-lambda, v[i], r[i]);           \
        alpha_old = alpha;                                                          \
        alpha = hbo_dot_##SFX(n, r, r);                                             \
        T_ talpha = alpha / (fabs(alpha_old) > EPS_MACH ? alpha_old : EPS_MACH);    \
        /* Scale then Sum: two separately rounded steps */                         \
        for (uint64_t i = 0; i < n; ++i) { p[i] = p[i] * talpha; p[i] = p[i] + r[i]; } \
        ++it;                                                                       \
        T_ cur = (T_)sqrt(alpha);                                                   \
        if (cur < eps * initial || cur < eps) { used = it; break; }                 \
        if (it == max_iters) used = it;                                             \
    }                                                                               \
    free(p); free(r); free(v);                                                      \
    return used;                                                                    \
}                                                                                   \
                                                                                    \
typedef struct {                                                                    \
    unsigned min_level, max_level;                                                  \
    ell_##SFX A[32], P[32], R[32];  /* indexed by level; P/R[l]: l <-> l-1 */       \
    T_ *jac[32], *b[32], *x[32], *d[32], *c[32], *store[32], *t0[32], *t1[32];     \
    uint64_t n_pre, n_post, max_iters_coarse, coarse_used;                          \
    T_ coarse_eps;                                                                  \
    int cycle;                      /* 0 V::STATIC, 1 W::STATIC */                  \
} mg_##SFX;                                                                         \
                                                                                    \
/* per-level vectors and the "jac" preconditioner of level l (A[l] set) */         \
static void mg_level_vectors_##SFX(mg_##SFX *h, unsigned l, double omega)           \
{                                                                                   \
    uint64_t n = h->A[l].rows;                                                      \
    h->jac[l] = (T_ *)malloc(sizeof(T_) * n);                                       \
    /* PreconFill "jac" (math/mg.hh:266-273): P[j] = omega, then /= A(j,j) */       \
    for (uint64_t j = 0; j < n; ++j) {                                              \
        T_ pj = (T_)omega; pj /= ell_diag_##SFX(&h->A[l], j); h->jac[l][j] = pj;    \
    }                                                                               \
    h->b[l] = (T_ *)calloc(n, sizeof(T_)); h->x[l] = (T_ *)calloc(n, sizeof(T_));   \
    h->d[l] = (T_ *)calloc(n, sizeof(T_)); h->c[l] = (T_ *)calloc(n, sizeof(T_));   \
    h->store[l] = (T_ *)calloc(n, sizeof(T_));                                      \
    h->t0[l] = (T_ *)calloc(n, sizeof(T_)); h->t1[l] = (T_ *)calloc(n, sizeof(T_)); \
}                                                                                   \
                                                                                    \
static void mg_setup_##SFX(mg_##SFX *h, unsigned lmin, unsigned lmax, double aniso, \
                           double omega)                                            \
{                                                                                   \
    memset(h, 0, sizeof(*h));                                                       \
    h->min_level = lmin; h->max_level = lmax;                                       \
    for (unsigned l = lmin; l <= lmax; ++l) {                                       \
        q1_ell_##SFX(&h->A[l], l, aniso);                                           \
        if (l > lmin) transfer_ell_##SFX(&h->P[l], &h->R[l], l);                    \
        mg_level_vectors_##SFX(h, l, omega);                                        \
    }                                                                               \
}                                                                                   \
                                                                                    \
static void mg_free_##SFX(mg_##SFX *h)                                              \
{                                                                                   \
    for (unsigned l = h->min_level; l <= h->max_level; ++l) {                       \
        ell_free_##SFX(&h->A[l]);                                                   \
        if (l > h->min_level) { ell_free_##SFX(&h->P[l]); ell_free_##SFX(&h->R[l]); }\
        free(h->jac[l]); free(h->b[l]); free(h->x[l]); free(h->d[l]); free(h->c[l]);\
        free(h->store[l]); free(h->t0[l]); free(h->t1[l]);                          \
    }                                                                               \
}                                                                                   \
                                                                                    \
/* math/ri.hh:110-133: t0 = b - A x; t1 = P (.) t0; x += t1 */                     \
static void smooth_##SFX(mg_##SFX *h, unsigned l, T_ *b, T_ *x, uint64_t sweeps)    \
{                                                                                   \
    uint64_t n = h->A[l].rows;                                                      \
    for (uint64_t s = 0; s < sweeps; ++s) {                                         \
        defect_##SFX(&h->A[l], b, x, h->t0[l]);                                     \
        for (uint64_t i = 0; i < n; ++i) h->t1[l][i] = h->jac[l][i] * h->t0[l][i];  \
        for (uint64_t i = 0; i < n; ++i) x[i] += h->t1[l][i];                       \
    }                                                                               \
}                                                                                   \
                                                                                    \
/* math/mg.hh:577-640 (V), 673-742 (W), executed directly, not as an OperatorList */     \
static void vcycle_##SFX(mg_##SFX *h, unsigned l, T_ *x, T_ *b)                     \
{                                                                                   \
    if (l == h->min_level) {                                                        \
        h->coarse_used = cg_##SFX(&h->A[l], b, x, h->max_iters_coarse, h->coarse_eps);\
        return;                                                                     \
    }                                                                               \
    uint64_t n = h->A[l].rows;                                                      \
    smooth_##SFX(h, l, b, x, h->n_pre);                                             \
    defect_##SFX(&h->A[l], b, x, h->store[l]);                                      \
    spmv_##SFX(&h->R[l], h->store[l], h->d[l - 1]);                                 \
    memset(h->c[l - 1], 0, sizeof(T_) * h->A[l - 1].rows);                          \
    vcycle_##SFX(h, l - 1, h->c[l - 1], h->d[l - 1]);                               \
    /* W::STATIC (math/mg.hh:719-721): the coarser cycle twice, except directly   \
       above the coarsest level */                                                  \
    if (h->cycle == 1 && l - 1 != h->min_level)                                     \
        vcycle_##SFX(h, l - 1, h->c[l - 1], h->d[l - 1]);                           \
    spmv_##SFX(&h->P[l], h->c[l - 1], h->store[l]);                                 \
    for (uint64_t i = 0; i < n; ++i) x[i] += h->store[l][i];                        \
    smooth_##SFX(h, l, b, x, h->n_post);                                            \
}                                                                                   \
                                                                                    \
/* math/mg.hh:1094-1127 with Norm<l2, true> */                                      \
static uint64_t mg_solve_##SFX(mg_##SFX *h, uint64_t max_iters, T_ eps, double *stats)\
{                                                                                   \
    unsigned L = h->max_level;                                                      \
    uint64_t n = h->A[L].rows, used = 0;                                            \
    T_ *r = (T_ *)malloc(sizeof(T_) * n);                                           \
    defect_##SFX(&h->A[L], h->b[L], h->x[L], r);                                    \
    T_ r0 = (T_)sqrt(hbo_dot_##SFX(n, r, r)), rc = (T_)1e16;                        \
    for (uint64_t i = 0; i < max_iters; ++i) {                                      \
        vcycle_##SFX(h, L, h->x[L], h->b[L]);                                       \
        defect_##SFX(&h->A[L], h->b[L], h->x[L], r);                                \
        rc = (T_)sqrt(hbo_dot_##SFX(n, r, r));                                      \
        used = i + 1;                                                               \
        if (rc < eps * r0) break;                                                   \
    }                                                                               \
    if (stats) { stats[0] = (double)used; stats[1] = r0; stats[2] = rc;             \
                 stats[3] = (double)h->coarse_used; }                               \
    free(r);                                                                        \
    return used;                                                                    \
}                                                                                   \
                                                                                    \
uint64_t hbo_mg_q1_##SFX(unsigned min_level, unsigned max_level, double aniso,      \
                         double omega, uint64_t n_pre, uint64_t n_post,             \
                         uint64_t max_iters, uint64_t max_iters_coarse, double eps, \
                         double coarse_eps, const T_ *b, T_ *x, double *stats)      \
{                                                                                   \
    return hbo_mg_q1_cycle_##SFX(0, min_level, max_level, aniso, omega, n_pre,      \
                                 n_post, max_iters, max_iters_coarse, eps,          \
                                 coarse_eps, b, x, stats);                          \
}                                                                                   \
                                                                                    \
uint64_t hbo_mg_q1_cycle_##SFX(int cycle, unsigned min_level, unsigned max_level,  \
                               double aniso, double omega, uint64_t n_pre,         \
                               uint64_t n_post, uint64_t max_iters,                \
                               uint64_t max_iters_coarse, double eps,              \
                               double coarse_eps, const T_ *b, T_ *x,              \
                               double *stats)                                      \
{                                                                                   \
    mg_##SFX h;                                                                     \
    mg_setup_##SFX(&h, min_level, max_level, aniso, omega);                         \
    h.cycle = cycle;                                                                \
    h.n_pre = n_pre; h.n_post = n_post; h.max_iters_coarse = max_iters_coarse;      \
    h.coarse_eps = (T_)coarse_eps;                                                  \
    uint64_t n = hbo_q1_n(max_level);                                               \
    memcpy(h.b[max_level], b, sizeof(T_) * n);                                      \
    memcpy(h.x[max_level], x, sizeof(T_) * n);                                      \
    uint64_t used = mg_solve_##SFX(&h, max_iters, (T_)eps, stats);                  \
    memcpy(x, h.x[max_level], sizeof(T_) * n);                                      \
    mg_free_##SFX(&h);                                                              \
    return used;                                                                    \
}

DEFINE_SOLVERS(double, f64, DBL_EPSILON, MULADD)
DEFINE_SOLVERS(float, f32, FLT_EPSILON, MULADD)

static void ell_copy_f64(ell_f64 *e, const hbo_ell_view *v)
{
    const uint64_t size = v->K * v->stride;
    e->rows = v->rows; e->cols = v->cols; e->stride = v->stride; e->K = v->K;
    e->Aj = (uint64_t *)malloc(sizeof(uint64_t) * size);
    e->Ax = (double *)malloc(sizeof(double) * size);
    e->Arl = (uint64_t *)malloc(sizeof(uint64_t) * (v->rows ? v->rows : 1));
    memcpy(e->Aj, v->Aj, sizeof(uint64_t) * size);
    memcpy(e->Ax, v->Ax, sizeof(double) * size);
    memcpy(e->Arl, v->Arl, sizeof(uint64_t) * v->rows);
}

/* MGUtil::load_data (math/mg.hh:442-545) on given matrices: level l = 1..nlev holds
 * A[l-1]; prol[l-2] / res[l-2] connect level l and l-1; P = omega / diag(A). */
uint64_t hbo_mg_ell_f64(int cycle, unsigned nlev, const hbo_ell_view *A, const hbo_ell_view *prol,
                        const hbo_ell_view *res, double omega, uint64_t n_pre, uint64_t n_post,
                        uint64_t max_iters, uint64_t max_iters_coarse, double eps, double coarse_eps,
                        const double *b, double *x, double *stats)
{
    mg_f64 h;
    if (nlev < 1 || nlev > 31) return 0;
    memset(&h, 0, sizeof(h));
    h.min_level = 1; h.max_level = nlev; h.cycle = cycle;
    for (unsigned l = 1; l <= nlev; ++l) {
        ell_copy_f64(&h.A[l], &A[l - 1]);
        if (l > 1) { ell_copy_f64(&h.P[l], &prol[l - 2]); ell_copy_f64(&h.R[l], &res[l - 2]); }
        mg_level_vectors_f64(&h, l, omega);
    }
    h.n_pre = n_pre; h.n_post = n_post; h.max_iters_coarse = max_iters_coarse;
    h.coarse_eps = coarse_eps;
    const uint64_t n = h.A[nlev].rows;
    memcpy(h.b[nlev], b, sizeof(double) * n);
    memcpy(h.x[nlev], x, sizeof(double) * n);
    uint64_t used = mg_solve_f64(&h, max_iters, eps, stats);
    memcpy(x, h.x[nlev], sizeof(double) * n);
    mg_free_f64(&h);
    return used;
}

uint64_t hbo_cg_q1_f64(unsigned L, double aniso, const double *b, double *x,
                       uint64_t max_iters, double eps)
{
    ell_f64 A;
    q1_ell_f64(&A, L, aniso);
    uint64_t used = cg_f64(&A, b, x, max_iters, eps);
    ell_free_f64(&A);
    return used;
}

void hbo_jacobi_q1_f64(unsigned L, double aniso, double omega, const double *b, double *x,
                       uint64_t sweeps)
{
    mg_f64 h;
    mg_setup_f64(&h, L, L, aniso, omega);
    smooth_f64(&h, L, (double *)b, x, sweeps);
    mg_free_f64(&h);
}

/* math/ir.hh:31-80: outer FP64 defect / norm / update, inner FP32 MG on the
 * converted defect.  The inner solution vector is the finest-level x of the
 * inner hierarchy; the reference never resets it (reset_inner = 0). */
uint64_t hbo_ir_q1(unsigned min_level, unsigned max_level, double aniso, double omega,
                   uint64_t n_pre, uint64_t n_post, uint64_t max_inner, uint64_t max_iters_coarse,
                   double inner_eps, double coarse_eps, uint64_t max_outer, double eps,
                   int reset_inner, const double *b, double *x, double *stats)
{
    ell_f64 A;
    q1_ell_f64(&A, max_level, aniso);
    mg_f32 h;
    mg_setup_f32(&h, min_level, max_level, aniso, omega);
    h.n_pre = n_pre; h.n_post = n_post; h.max_iters_coarse = max_iters_coarse;
    h.coarse_eps = (float)coarse_eps;
    uint64_t n = A.rows, used = 0, inner_total = 0;
    double *r = (double *)malloc(sizeof(double) * n);
    double r0 = 1e16, rc = 1e16;
    for (uint64_t i = 0; i < max_outer; ++i) {
        defect_f64(&A, b, x, r);
        if (i == 0) {
            r0 = sqrt(hbo_dot_f64(n, r, r));
        } else {
            rc = sqrt(hbo_dot_f64(n, r, r));
            used = i;
            if (rc < eps * r0) break;
        }
        for (uint64_t k = 0; k < n; ++k) h.b[max_level][k] = (float)r[k];
        if (reset_inner) memset(h.x[max_level], 0, sizeof(float) * n);
        double st[4];
        mg_solve_f32(&h, max_inner, (float)inner_eps, st);
        inner_total += (uint64_t)st[0];
        for (uint64_t k = 0; k < n; ++k) x[k] += (double)h.x[max_level][k];
    }
    if (stats) { stats[0] = (double)used; stats[1] = r0; stats[2] = rc; stats[3] = (double)inner_total; }
    free(r);
    ell_free_f64(&A);
    mg_free_f32(&h);
    return used;
}


/* ---- Krylov solvers with a variable preconditioner ------------------------ */
/* P: a vector (Product of two DenseVectors = ElementProduct, la/product.hh:1198-1204)
 * when pdiag != NULL, else an ELL matrix (Product ELL, la/product.hh:148-206) */
static void pc_apply_f64(const double *pdiag, const ell_f64 *P, uint64_t n, const double *r, double *z)
{
    if (pdiag) for (uint64_t i = 0; i < n; ++i) z[i] = pdiag[i] * r[i];
    else spmv_f64(P, r, z);
}

/* the reference's guard against division by a tiny number */
static double eps_guard(double t)
{
    return fabs(t) > DBL_EPSILON ? t : DBL_EPSILON * (t / fabs(t));
}

/* ScaledSum<Tag>::value(x, y, b) x += b*y and value(r, x, y, b) r = b*y + x
 * (la/scaled_sum.hh:73-108), each product and sum rounded */
static void axpy(uint64_t n, double *x, const double *y, double b)
{ for (uint64_t i = 0; i < n; ++i) x[i] = MULADD(b, y[i], x[i]); }
static void axpy3(uint64_t n, double *r, const double *x, const double *y, double b)
{ for (uint64_t i = 0; i < n; ++i) r[i] = MULADD(b, y[i], x[i]); }

uint64_t hbo_cgvar_f64(const hbo_ell_view *Av, const double *pdiag, const hbo_ell_view *Pv, const double *b,
                       double *x, uint64_t max_iters, double eps, int smoother)
{
    ell_f64 A, P;
    ell_copy_f64(&A, Av);
    if (! pdiag) ell_copy_f64(&P, Pv);
    const uint64_t n = A.rows;
    double *p = (double *)malloc(sizeof(double) * n), *r = (double *)malloc(sizeof(double) * n);
    double *v = (double *)malloc(sizeof(double) * n), *z = (double *)malloc(sizeof(double) * n);
    uint64_t it = 0, used = 0;
    /* math/cg.hh:161-210 (CGSolver VAR); CGSmoother (math/cg.hh:230-288) has no
       convergence test and stops after max_iters */
    defect_f64(&A, b, x, r);
    pc_apply_f64(pdiag, &P, n, r, p);
    const double initial = sqrt(hbo_dot_f64(n, r, r));
    double alpha_new = hbo_dot_f64(n, r, p), alpha, lambda, temp;
    while (it < max_iters) {
        spmv_f64(&A, p, v);
        temp = hbo_dot_f64(n, v, p);
        lambda = alpha_new / eps_guard(temp);
        ++it;
        axpy(n, x, p, lambda);
        axpy(n, r, v, -lambda);
        if (smoother) {
            if (it == max_iters) break;
        } else {
            const double cur = sqrt(hbo_dot_f64(n, r, r));
            if (cur < eps * initial) { used = it; break; }
            if (cur < eps) { used = it; break; }
            if (it == max_iters) { used = it; break; }
        }
        pc_apply_f64(pdiag, &P, n, r, z);
        alpha = alpha_new;
        alpha_new = hbo_dot_f64(n, r, z);
        const double talpha = alpha_new / eps_guard(alpha);
        for (uint64_t i = 0; i < n; ++i) { p[i] = p[i] * talpha; p[i] = p[i] + z[i]; }
    }
    free(p); free(r); free(v); free(z);
    ell_free_f64(&A);
    if (! pdiag) ell_free_f64(&P);
    return smoother ? it : used;
}

/* BiCGStabSolver<Tag, methods::VAR> (math/bicgstab.hh:71-210); the norms are
 * Norm<vnt_l_two, false> (squared), compared with eps times the squared initial
 * defect; returns the reference's used_iters (iterations + 1) */
uint64_t hbo_bicgstab_f64(const hbo_ell_view *Av, const double *pdiag, const hbo_ell_view *Pv, const double *b,
                          double *x, uint64_t max_iters, double eps)
{
    ell_f64 A, P;
    ell_copy_f64(&A, Av);
    if (! pdiag) ell_copy_f64(&P, Pv);
    const uint64_t n = A.rows;
    double *vec[10];
    for (int i = 0; i < 10; ++i) vec[i] = (double *)malloc(sizeof(double) * (n ? n : 1));
    double *r = vec[0], *rt = vec[1], *rt0 = vec[2], *pt = vec[3], *v = vec[4], *vt = vec[5], *s = vec[6],
           *st = vec[7], *t = vec[8], *tt = vec[9];
    double defnorm, defnorm_0, defnorm_00 = 1e14, rho, rho_old, alpha, omega, beta, gamma;
    uint64_t iter = 0;
    int restarted = 0, converged = 0;
    do {
        defect_f64(&A, b, x, r);
        defnorm_0 = hbo_dot_f64(n, r, r);
        defnorm = defnorm_0;
        pc_apply_f64(pdiag, &P, n, r, rt0);
        if (! restarted) defnorm_00 = defnorm_0;
        memcpy(rt, rt0, sizeof(double) * n);
        memcpy(pt, rt0, sizeof(double) * n);
        rho = hbo_dot_f64(n, rt0, rt0);
        do {
            iter = iter + 1;
            spmv_f64(&A, pt, v);
            pc_apply_f64(pdiag, &P, n, v, vt);
            gamma = hbo_dot_f64(n, vt, rt0);
            if (fabs(gamma) < fabs(rho) * 1e-14) { restarted = 1; break; }
            alpha = rho / gamma;
            /* the reference also sets `restarted` (without leaving the loop) when
               |alpha| ||vt||^2 / defnorm < 1e-5; the flag is read only before the
               first pass, so it changes nothing and is not computed here */
            axpy3(n, s, r, v, -alpha);
            defnorm = hbo_dot_f64(n, s, s);
            if (defnorm < eps * defnorm_00) {
                axpy(n, x, pt, alpha);
                converged = 1;
                break;
            }
            axpy3(n, st, rt, vt, -alpha);
            spmv_f64(&A, st, t);
            pc_apply_f64(pdiag, &P, n, t, tt);
            gamma = hbo_dot_f64(n, tt, tt);
            omega = hbo_dot_f64(n, tt, st);
            if (fabs(gamma) < fabs(omega) * 1e-14) { restarted = 1; break; }
            omega = omega / gamma;
            axpy(n, x, st, omega);
            axpy(n, x, pt, alpha);
            axpy3(n, r, s, t, -omega);
            defnorm = hbo_dot_f64(n, r, r);
            if (defnorm < eps * defnorm_00) { converged = 1; break; }
            axpy3(n, rt, st, tt, -omega);
            rho_old = rho;
            rho = hbo_dot_f64(n, rt, rt0);
            beta = (alpha / omega) * (rho / rho_old);
            axpy(n, pt, vt, -omega);
            for (uint64_t i = 0; i < n; ++i) pt[i] = pt[i] * beta;
            for (uint64_t i = 0; i < n; ++i) pt[i] = pt[i] + rt[i];
        } while (iter <= max_iters);
    } while (converged == 0 && iter < max_iters);
    (void)defnorm;
    for (int i = 0; i < 10; ++i) free(vec[i]);
    ell_free_f64(&A);
    if (! pdiag) ell_free_f64(&P);
    return iter + 1;
}

/* ---- legacy Multigrid<Tag, OuterTag, NONE, JAC, CYCLE::V, FIXED> on BandedMatrixQx ---- */
/* math/conjugate_gradients.hh:491-560 with the banded cg_kernel (:108-151): x = 0,
 * g = A x - b, u = -g; while ||x||^2 grows by more than konv_rad: one CG step with
 * the gradient recomputed as A x - b.  Norm<l2, false> = the fma dot of x with itself.
 * A cap of 100000 steps guards the loop (the reference has none). */
#define DEFINE_LMG(T_, SFX, EPS_MACH)                                               \
static uint64_t lmg_cg_##SFX(uint64_t n, uint64_t m, const T_ *bands, const T_ *rhs, \
                             T_ *x, double konv_rad)                                \
{                                                                                   \
    T_ *ng = (T_ *)malloc(sizeof(T_) * n), *g = (T_ *)malloc(sizeof(T_) * n);       \
    T_ *u = (T_ *)malloc(sizeof(T_) * n), *e = (T_ *)malloc(sizeof(T_) * n);        \
    for (uint64_t i = 0; i < n; ++i) x[i] = 0;                                      \
    hbo_q1_spmv_##SFX(n, m, bands, x, g);                                           \
    for (uint64_t i = 0; i < n; ++i) g[i] = g[i] - rhs[i];                          \
    for (uint64_t i = 0; i < n; ++i) u[i] = g[i] * (T_)-1;                          \
    T_ norm_x = hbo_dot_##SFX(n, x, x), norm_x_last = (T_)(norm_x - 1);             \
    uint64_t it = 0;                                                                \
    while (norm_x - norm_x_last > konv_rad && it < 100000) {                        \
        T_ upper = hbo_dot_##SFX(n, g, g);                                          \
        hbo_q1_spmv_##SFX(n, m, bands, u, e);                                       \
        T_ lower = hbo_dot_##SFX(n, e, u);                                          \
        T_ f = fabs(lower) >= EPS_MACH ? upper / lower : upper / EPS_MACH;          \
        for (uint64_t i = 0; i < n; ++i) { e[i] = u[i] * f; e[i] = e[i] + x[i]; }   \
        lower = upper;                                                              \
        hbo_q1_spmv_##SFX(n, m, bands, e, ng);                                      \
        for (uint64_t i = 0; i < n; ++i) ng[i] = ng[i] - rhs[i];                    \
        upper = hbo_dot_##SFX(n, ng, ng);                                           \
        f = fabs(lower) >= EPS_MACH ? upper / lower : upper / EPS_MACH;             \
        for (uint64_t i = 0; i < n; ++i) { u[i] = u[i] * f; u[i] = u[i] - ng[i]; }  \
        memcpy(g, ng, sizeof(T_) * n);                                              \
        memcpy(x, e, sizeof(T_) * n);                                               \
        norm_x_last = norm_x;                                                       \
        norm_x = hbo_dot_##SFX(n, x, x);                                            \
        ++it;                                                                       \
    }                                                                               \
    free(ng); free(g); free(u); free(e);                                            \
    return it;                                                                      \
}                                                                                   \
                                                                                    \
/* math/jacobi.hh (the MG variants): x = d^-1 (.) b, then sweeps of                \
 * t = b - A x; x += t (.) d^-1 (in place, t computed from the whole old x) */      \
static void lmg_sweeps_##SFX(uint64_t n, uint64_t m, const T_ *bands, const T_ *b,  \
                             T_ *x, const T_ *dinv, uint64_t sweeps, T_ *t)         \
{                                                                                   \
    for (uint64_t s = 0; s < sweeps; ++s) {                                         \
        hbo_q1_defect_##SFX(n, m, bands, b, x, t);                                  \
        for (uint64_t i = 0; i < n; ++i) x[i] = x[i] + t[i] * dinv[i];              \
    }                                                                               \
}                                                                                   \
                                                                                    \
typedef struct {                                                                    \
    unsigned lmin, lmax;                                                            \
    uint64_t N[32], M[32];                                                          \
    const T_ *bands[32], *dinv[32];                                                 \
    T_ *x[32], *c[32], *d[32], *rhs[32], *t[32];                                    \
} lmg_##SFX;                                                                        \
                                                                                    \
static void lmg_alloc_##SFX(lmg_##SFX *h, unsigned lmin, unsigned lmax,             \
                            const T_ *const *bands, const T_ *const *dinv)          \
{                                                                                   \
    h->lmin = lmin; h->lmax = lmax;                                                 \
    for (unsigned l = lmin; l <= lmax; ++l) {                                       \
        h->M[l] = ((uint64_t)1 << l) + 1; h->N[l] = h->M[l] * h->M[l];              \
        h->bands[l] = bands[l]; h->dinv[l] = dinv[l];                               \
        h->x[l] = (T_ *)calloc(h->N[l], sizeof(T_)); h->c[l] = (T_ *)calloc(h->N[l], sizeof(T_)); \
        h->d[l] = (T_ *)calloc(h->N[l], sizeof(T_)); h->rhs[l] = (T_ *)calloc(h->N[l], sizeof(T_)); \
        h->t[l] = (T_ *)calloc(h->N[l], sizeof(T_));                                \
    }                                                                               \
}                                                                                   \
static void lmg_release_##SFX(lmg_##SFX *h)                                         \
{                                                                                   \
    for (unsigned l = h->lmin; l <= h->lmax; ++l) {                                 \
        free(h->x[l]); free(h->c[l]); free(h->d[l]); free(h->rhs[l]); free(h->t[l]); \
    }                                                                               \
}                                                                                   \
                                                                                    \
/* _multigrid_kernel (math/multigrid.hh:159-466 FIXED, 1619-1934 MIXED) on the      \
 * state's finest x (iterate) and rhs.  mixed: the MIXED class's kernel, whose      \
 * coarse-grid correction factor 0 means alpha = <d, c> / <A c, c>.  Returns the    \
 * cycles run. */                                                                   \
static uint64_t lmg_kernel_##SFX(lmg_##SFX *h, uint64_t n_max_iter, int initial_zero, \
                                 int convergence_check, int is_smoother,            \
                                 double tolerance, uint64_t n_pre, double adapt,    \
                                 const uint64_t *mask, int mixed)                   \
{                                                                                   \
    const unsigned L = h->lmax, lmin = h->lmin;                                     \
    const uint64_t n = h->N[L];                                                     \
    T_ **x = h->x, **c = h->c, **d = h->d, **rhs = h->rhs, **t = h->t;              \
    if (initial_zero) memcpy(d[L], rhs[L], sizeof(T_) * n);                         \
    else hbo_q1_defect_##SFX(n, h->M[L], h->bands[L], rhs[L], x[L], d[L]);          \
    T_ defect, initial;                                                             \
    if (! is_smoother) { defect = (T_)sqrt(hbo_dot_##SFX(n, d[L], d[L])); initial = defect; } \
    else { defect = (T_)1e8; initial = defect; }                                    \
    uint64_t cycles = 0;                                                            \
    if (convergence_check && defect <= (T_)tolerance) return 0;                     \
    for (uint64_t iter = 1; iter <= n_max_iter; ++iter) {                           \
        unsigned l = L;                                                             \
        int started = 1;                                                            \
        cycles = iter;                                                              \
        while (lmin != L) {                                                         \
            const uint64_t Nl = h->N[l], Ml = h->M[l];                              \
            if (started) {                                                          \
                for (uint64_t i = 0; i < Nl; ++i) c[l][i] = h->dinv[l][i] * d[l][i]; \
                lmg_sweeps_##SFX(Nl, Ml, h->bands[l], d[l], c[l], h->dinv[l], n_pre - 1, t[l]); \
                for (uint64_t i = 0; i < Nl; ++i) x[l][i] = x[l][i] + c[l][i];      \
            } else {                                                                \
                for (uint64_t i = 0; i < Nl; ++i) x[l][i] = h->dinv[l][i] * d[l][i]; \
                lmg_sweeps_##SFX(Nl, Ml, h->bands[l], d[l], x[l], h->dinv[l], n_pre - 1, t[l]); \
            }                                                                       \
            hbo_q1_defect_##SFX(Nl, Ml, h->bands[l], rhs[l], x[l], d[l]);           \
            --l;                                                                    \
            hbo_restriction_##SFX(h->N[l], d[l], h->N[l + 1], d[l + 1], mask);      \
            memcpy(rhs[l], d[l], sizeof(T_) * h->N[l]);                             \
            if (l == lmin) break;                                                   \
            started = 0;                                                            \
        }                                                                           \
        lmg_cg_##SFX(h->N[l], h->M[l], h->bands[l], d[l], x[l], (double)EPS_MACH);  \
        if (lmin == L) {                                                            \
            hbo_q1_defect_##SFX(h->N[l], h->M[l], h->bands[l], rhs[l], x[l], d[l]); \
            break;                                                                  \
        }                                                                           \
        while (1) {                                                                 \
            ++l;                                                                    \
            const uint64_t Nl = h->N[l], Ml = h->M[l];                              \
            hbo_prolongation_##SFX(Nl, c[l], h->N[l - 1], x[l - 1], mask);          \
            T_ alpha = (T_)adapt;                                                   \
            if (mixed && adapt == 0.0) {                                            \
                const T_ d1 = hbo_dot_##SFX(Nl, d[l], c[l]);                        \
                hbo_q1_spmv_##SFX(Nl, Ml, h->bands[l], c[l], t[l]);                 \
                const T_ d2 = hbo_dot_##SFX(Nl, t[l], c[l]);                        \
                alpha = (T_)(d1 / d2);                                              \
            }                                                                       \
            for (uint64_t i = 0; i < Nl; ++i) x[l][i] = x[l][i] + alpha * c[l][i];  \
            lmg_sweeps_##SFX(Nl, Ml, h->bands[l], rhs[l], x[l], h->dinv[l], n_pre, t[l]); \
            hbo_q1_defect_##SFX(Nl, Ml, h->bands[l], rhs[l], x[l], d[l]);           \
            if (l == L) break;                                                      \
        }                                                                           \
        if (! is_smoother) {                                                        \
            defect = (T_)sqrt(hbo_dot_##SFX(n, d[L], d[L]));                        \
            if (defect <= initial * (T_)tolerance) break;                           \
        }                                                                           \
    }                                                                               \
    return cycles;                                                                  \
}                                                                                   \
                                                                                    \
/* Multigrid<..., JAC, CYCLE::V, FIXED>::value (math/multigrid.hh:781-825) */       \
uint64_t hbo_lmg_##SFX(unsigned lmin, unsigned lmax, const T_ *const *bands,        \
                       const T_ *const *dinv, const T_ *rhs_in, T_ *x_io,           \
                       uint64_t n_max_iter, int initial_zero, int convergence_check, \
                       int is_smoother, double tolerance, uint64_t n_pre,           \
                       double adapt, const uint64_t *mask)                          \
{                                                                                   \
    lmg_##SFX h;                                                                    \
    lmg_alloc_##SFX(&h, lmin, lmax, bands, dinv);                                   \
    const unsigned L = lmax;                                                        \
    const uint64_t n = h.N[L], sq = h.M[L];                                         \
    memcpy(h.rhs[L], rhs_in, sizeof(T_) * n);                                       \
    /* the initial guess with b's values on the first row, the last row and the first column */ \
    memcpy(h.x[L], x_io, sizeof(T_) * n);                                           \
    for (uint64_t i = 0; i < sq; ++i) h.x[L][i] = rhs_in[i];                        \
    for (uint64_t i = n - sq; i < n; ++i) h.x[L][i] = rhs_in[i];                    \
    for (uint64_t i = 0; i < n; i += sq) h.x[L][i] = rhs_in[i];                     \
    const uint64_t cycles = lmg_kernel_##SFX(&h, n_max_iter, initial_zero, convergence_check, \
                                             is_smoother, tolerance, n_pre, adapt, mask, 0); \
    memcpy(x_io, h.x[L], sizeof(T_) * n);                                           \
    lmg_release_##SFX(&h);                                                          \
    return cycles;                                                                  \
}
DEFINE_LMG(double, f64, DBL_EPSILON)
DEFINE_LMG(float, f32, FLT_EPSILON)


/* Multigrid<Tag, OuterTag, NONE, JAC, CYCLE::V, MIXED>::value on BandedMatrixQx
 * (math/multigrid.hh:2252-2394): the FP64 defect of the initial guess (b's Dirichlet
 * values on the first row, the last row and the first column) scaled into the FP32
 * inner right-hand side, the inner kernel on its persistent iterate, result (starting
 * at 0) += scale x_inner, the FP64 defect, its norm, stop below tolerance (the inner
 * MGInfo's float, widened) times the initial norm, else scale by 1 / norm.  At most
 * max_outer outer steps (the reference has no cap).  Returns the outer steps;
 * *inner_total: the inner cycles. */
uint64_t hbo_lmg_mixed(unsigned lmin, unsigned lmax, const float *const *bands, const float *const *dinv,
                       const double *bands64, const double *b, double *x, uint64_t n_max_iter, int initial_zero,
                       double tolerance, uint64_t n_pre, double adapt, const uint64_t *mask, uint64_t max_outer,
                       uint64_t *inner_total)
{
    lmg_f32 h;
    lmg_alloc_f32(&h, lmin, lmax, bands, dinv);
    const unsigned L = lmax;
    const uint64_t n = h.N[L], sq = h.M[L];
    double *ig = (double *)malloc(sizeof(double) * n), *od = (double *)malloc(sizeof(double) * n);
    double *res = (double *)calloc(n, sizeof(double));
    memcpy(ig, x, sizeof(double) * n);
    for (uint64_t i = 0; i < sq; ++i) ig[i] = b[i];
    for (uint64_t i = n - sq; i < n; ++i) ig[i] = b[i];
    for (uint64_t i = 0; i < n; i += sq) ig[i] = b[i];
    for (uint64_t i = 0; i < n; ++i) h.x[L][i] = (float)ig[i];
    hbo_q1_defect_f64(n, sq, bands64, b, ig, od);
    const double initial = sqrt(hbo_dot_f64(n, od, od));
    const double outer_eps = (double)(float)tolerance;
    double scale = 1.0;
    uint64_t outer = 0, inner = 0;
    while (outer < max_outer) {
        for (uint64_t i = 0; i < n; ++i) h.rhs[L][i] = (float)od[i];
        inner += lmg_kernel_f32(&h, n_max_iter, initial_zero, 0, 0, (double)(float)tolerance, n_pre, adapt, mask, 1);
        ++outer;
        for (uint64_t i = 0; i < n; ++i) res[i] = res[i] + scale * (double)h.x[L][i];
        hbo_q1_defect_f64(n, sq, bands64, b, res, od);
        const double def = sqrt(hbo_dot_f64(n, od, od));
        if (def < outer_eps * initial) break;
        scale = def;
        const double inv = 1.0 / scale;
        for (uint64_t i = 0; i < n; ++i) od[i] = od[i] * inv;
    }
    memcpy(x, res, sizeof(double) * n);
    free(ig); free(od); free(res);
    lmg_release_f32(&h);
    if (inner_total) *inner_total = inner;
    return outer;
}

/* ------------------------------------------------------------------------ */
/* BF16-stored matrix of the FP32 inner solve (no counterpart in the         */
/* reference): the storage and product of hb2_ell_create_bf16 restated       */
/* ------------------------------------------------------------------------ */
/* to nearest BF16 (8 significant bits, exponent range of float), ties to even:
 * scale the magnitude so that the BF16 spacing of its binade is 1, round to an
 * integer in the current (nearest-even) mode, scale back */
double hbo_bf16_round(double t)
{
    if (t != t || t == 0.0 || isinf(t)) return t;
    const double a = fabs(t);
    int e;
    frexp(a, &e);                          /* a = m 2^e, 1/2 <= m < 1 */
    int q = e - 8;                         /* spacing of the binade [2^(e-1), 2^e) */
    if (q < -133) q = -133;                /* the subnormal spacing */
    double v = ldexp(nearbyint(ldexp(a, -q)), q);
    if (v >= 0x1p128) v = INFINITY;
    return t < 0 ? -v : v;
}

void hbo_bf16_round_array(uint64_t n, const double *t, double *out)
{
    for (uint64_t i = 0; i < n; ++i) out[i] = hbo_bf16_round(t[i]);
}

/* row r's diagonal slot in visiting order (the first with Aj == r), or -1 */
static int64_t bf16_diag(uint64_t r, uint64_t stride, uint64_t T, const uint64_t *Aj, const uint64_t *Arl)
{
    for (uint64_t col = 0, j = r * T; col < Arl[r]; ++col, j += stride)
        for (uint64_t t = 0; t < T; ++t)
            if (Aj[j + t] == r) return (int64_t)(j + t);
    return -1;
}

#define DEFINE_ELL_BF16(T_, SFX)                                                             \
void hbo_ell_bf16_scale_##SFX(uint64_t rows, uint64_t stride, uint64_t T, const uint64_t *Aj,   \
                              const T_ *Ax, const uint64_t *Arl, int compensate, double *err)   \
{                                                                                            \
    for (int c = 0; c < 8; ++c) err[c] = 0.0;                                                \
    for (uint64_t r = 0; r < rows; ++r) {                                                    \
        const int64_t dj = compensate ? bf16_diag(r, stride, T, Aj, Arl) : -1;               \
        for (uint64_t col = 0, j = r * T; col < Arl[r]; ++col, j += stride)                  \
            for (uint64_t t = 0; t < T; ++t) {                                               \
                const double a = (double)Ax[j + t];                                          \
                if ((int64_t)(j + t) == dj || a == 0.0) continue;                            \
                for (int c = 0; c < 8; ++c) {                                                \
                    const double v = a * (double)(2 * c + 1);                                \
                    const double e = fabs(hbo_bf16_round(v) - v) / fabs(v);                  \
                    if (e > err[c]) err[c] = e;                                              \
                }                                                                            \
            }                                                                                \
    }                                                                                        \
}                                                                                            \
/* d of row r (compensated form) */                                                          \
static float bf16_d_##SFX(uint64_t r, uint64_t stride, uint64_t T, const uint64_t *Aj,       \
                          const T_ *Ax, const uint64_t *Arl, double s, int64_t dj)           \
{                                                                                            \
    double comp = 0.0;                                                                       \
    for (uint64_t col = 0, j = r * T; col < Arl[r]; ++col, j += stride)                      \
        for (uint64_t t = 0; t < T; ++t) {                                                   \
            if ((int64_t)(j + t) == dj) continue;                                            \
            const double v = (double)Ax[j + t] * s;                                          \
            comp += v - hbo_bf16_round(v);                                                   \
        }                                                                                    \
    return (float)((double)Ax[dj] * s + comp);                                               \
}                                                                                            \
void hbo_ell_bf16_spmv_##SFX(uint64_t rows, uint64_t stride, uint64_t T, const uint64_t *Aj,    \
                             const T_ *Ax, const uint64_t *Arl, double s, int compensate,    \
                             const float *x, float *y)                                       \
{                                                                                            \
    const float inv = (float)(1.0 / s);                                                      \
    for (uint64_t r = 0; r < rows; ++r) {                                                    \
        const int64_t dj = compensate ? bf16_diag(r, stride, T, Aj, Arl) : -1;               \
        const float d = dj >= 0 ? bf16_d_##SFX(r, stride, T, Aj, Ax, Arl, s, dj) : 0.f;      \
        const float h = (float)hbo_bf16_round((double)d), l = d - h;                         \
        float acc = 0.f;                                                                     \
        for (uint64_t col = 0, j = r * T; col < Arl[r]; ++col, j += stride)                  \
            for (uint64_t t = 0; t < T; ++t) {                                               \
                const float v = (int64_t)(j + t) == dj ? h                                   \
                                : (float)hbo_bf16_round((double)Ax[j + t] * s);              \
                acc = fmaf(v, x[Aj[j + t]], acc);                                            \
            }                                                                                \
        if (dj >= 0) acc = fmaf(l, x[r], acc);                                               \
        y[r] = s == 1.0 ? acc : acc * inv;                                                   \
    }                                                                                        \
}                                                                                            \
void hbo_ell_bf16_values_##SFX(uint64_t rows, uint64_t stride, uint64_t T, uint64_t K,       \
                               const uint64_t *Aj, const T_ *Ax, const uint64_t *Arl,        \
                               double s, int compensate, float *val32)                       \
{                                                                                            \
    memset(val32, 0, K * stride * sizeof(float));                                            \
    for (uint64_t r = 0; r < rows; ++r) {                                                    \
        const int64_t dj = compensate ? bf16_diag(r, stride, T, Aj, Arl) : -1;               \
        for (uint64_t col = 0, j = r * T; col < Arl[r]; ++col, j += stride)                  \
            for (uint64_t t = 0; t < T; ++t) {                                               \
                const double q = (int64_t)(j + t) == dj                                      \
                    ? (double)bf16_d_##SFX(r, stride, T, Aj, Ax, Arl, s, dj)                 \
                    : hbo_bf16_round((double)Ax[j + t] * s);                                 \
                val32[j + t] = (float)(q / s);                                               \
            }                                                                                \
    }                                                                                        \
}
DEFINE_ELL_BF16(double, f64)
DEFINE_ELL_BF16(float, f32)
