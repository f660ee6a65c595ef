// Helpers shared by the reference drivers in oracle/ (test infrastructure only).
// They build the reference's own containers through its public constructors.
#pragma once

#include <honei/la/banded_matrix_qx.hh>
#include <honei/la/dense_vector.hh>
#include <honei/la/sparse_matrix.hh>
#include <honei/la/sparse_matrix_ell.hh>
#include <honei/math/fill_matrix.hh>
#include <honei/math/prolongation_matrix.hh>
#include <honei/math/transposition.hh>

extern "C" {
#include "honei_oracle.h"
}

#include <cstdio>
#include <string>
#include <sys/time.h>
#include <vector>

namespace hbref
{
    using namespace honei;

    inline double now()
    {
        timeval tv;
        gettimeofday(&tv, 0);
        return tv.tv_sec + tv.tv_usec * 1e-6;
    }

    // The reference's slow assembly path: BandedMatrixQx -> FillMatrix ->
    // SparseMatrix -> SparseMatrixELL (math/fill_matrix.hh:37-79,
    // la/sparse_matrix.hh:221, la/sparse_matrix_ell-impl.hh:75-122).
    template <typename DT_>
    SparseMatrixELL<DT_> q1_ell_assembled(unsigned L)
    {
        unsigned long n(hbo_q1_n(L));
        DenseVector<DT_> b0(n, DT_(0)), b1(n, DT_(0)), b2(n, DT_(0)), b3(n, DT_(0)), b4(n, DT_(0)),
            b5(n, DT_(0)), b6(n, DT_(0)), b7(n, DT_(0)), b8(n, DT_(0));
        BandedMatrixQx<Q1Type, DT_> A(n, b0, b1, b2, b3, b4, b5, b6, b7, b8);
        FillMatrix<tags::CPU, applications::POISSON, boundary_types::DIRICHLET::DIRICHLET_0>::value(A);
        SparseMatrix<DT_> S(A);
        SparseMatrixELL<DT_> E(S);
        return E;
    }

    template <typename DT_>
    BandedMatrixQx<Q1Type, DT_> q1_banded(unsigned L)
    {
        unsigned long n(hbo_q1_n(L));
        DenseVector<DT_> b0(n, DT_(0)), b1(n, DT_(0)), b2(n, DT_(0)), b3(n, DT_(0)), b4(n, DT_(0)),
            b5(n, DT_(0)), b6(n, DT_(0)), b7(n, DT_(0)), b8(n, DT_(0));
        BandedMatrixQx<Q1Type, DT_> A(n, b0, b1, b2, b3, b4, b5, b6, b7, b8);
        FillMatrix<tags::CPU, applications::POISSON, boundary_types::DIRICHLET::DIRICHLET_0>::value(A);
        return A;
    }

    // ProlongationMatrix + Transposition with identity index maps
    // (math/prolongation_matrix.hh:44-100, math/transposition.hh:36-50).
    template <typename DT_>
    void transfer_assembled(unsigned Lf, SparseMatrixELL<DT_> *& P, SparseMatrixELL<DT_> *& R)
    {
        unsigned long nf(hbo_q1_n(Lf)), nc(hbo_q1_n(Lf - 1));
        SparseMatrix<DT_> Ps(nf, nc);
        DenseVector<unsigned long> idf(nf), idc(nc);
        for (unsigned long i(0); i < nf; ++i) idf[i] = i;
        for (unsigned long i(0); i < nc; ++i) idc[i] = i;
        ProlongationMatrix<tags::CPU>::value(Ps, idf, idc);
        P = new SparseMatrixELL<DT_>(Ps);
        R = new SparseMatrixELL<DT_>(Transposition<tags::CPU>::value(*P));
    }

    // Fast path used for timing at large levels: the same ELL arrays produced by
    // the oracle's restatement (pinned bit-exact against q1_ell_assembled at
    // small levels) handed to the reference's raw-array constructor
    // (la/sparse_matrix_ell-impl.hh:58-72), which recomputes Arl itself.
    template <typename DT_> struct OracleFill;
    template <> struct OracleFill<double>
    {
        static void bands(unsigned L, double a, double * o) { hbo_q1_bands_f64(L, a, o); }
        static unsigned long csr(unsigned L, const double * b, unsigned long * rp, unsigned long * ci, double * v)
        { return hbo_q1_csr_f64(L, b, (uint64_t *)rp, (uint64_t *)ci, v); }
    };
    template <> struct OracleFill<float>
    {
        static void bands(unsigned L, double a, float * o) { hbo_q1_bands_f32(L, a, o); }
        static unsigned long csr(unsigned L, const float * b, unsigned long * rp, unsigned long * ci, float * v)
        { return hbo_q1_csr_f32(L, b, (uint64_t *)rp, (uint64_t *)ci, v); }
    };

    template <typename DT_>
    SparseMatrixELL<DT_> ell_from_csr(unsigned long rows, unsigned long cols, const std::vector<unsigned long> & rp,
            const std::vector<unsigned long> & ci, const std::vector<DT_> & v)
    {
        uint64_t stride, K;
        hbo_ell_dims(rows, (const uint64_t *)&rp[0], 1, &stride, &K);
        DenseVector<unsigned long> Aj(K * stride, 0ul);
        DenseVector<DT_> Ax(K * stride, DT_(0));
        for (unsigned long r(0); r < rows; ++r)
        {
            unsigned long t(0);
            for (unsigned long e(rp[r]); e < rp[r + 1]; ++e)
            {
                if (v[e] == DT_(0)) continue;
                Aj[r + t * stride] = ci[e];
                Ax[r + t * stride] = v[e];
                ++t;
            }
        }
        return SparseMatrixELL<DT_>(rows, cols, stride, K, Aj, Ax, 1);
    }

    template <typename DT_>
    SparseMatrixELL<DT_> q1_ell_fast(unsigned L, double aniso = 1.0)
    {
        unsigned long n(hbo_q1_n(L));
        std::vector<DT_> bands(9 * n), v(9 * n);
        std::vector<unsigned long> rp(n + 1), ci(9 * n);
        OracleFill<DT_>::bands(L, aniso, &bands[0]);
        OracleFill<DT_>::csr(L, &bands[0], &rp[0], &ci[0], &v[0]);
        return ell_from_csr<DT_>(n, n, rp, ci, v);
    }

    template <typename DT_>
    void transfer_fast(unsigned Lf, SparseMatrixELL<DT_> *& P, SparseMatrixELL<DT_> *& R)
    {
        unsigned long nf(hbo_q1_n(Lf)), nc(hbo_q1_n(Lf - 1));
        std::vector<unsigned long> rp(nf + 1), ci(4 * nf), rpt(nc + 1), cit(4 * nf);
        std::vector<double> v(4 * nf), vt(4 * nf);
        unsigned long nnz = hbo_prolmat_csr_f64(Lf, (uint64_t *)&rp[0], (uint64_t *)&ci[0], &v[0]);
        hbo_csr_transpose_f64(nf, nc, (uint64_t *)&rp[0], (uint64_t *)&ci[0], &v[0],
                (uint64_t *)&rpt[0], (uint64_t *)&cit[0], &vt[0]);
        std::vector<DT_> tv(nnz), tvt(nnz);
        for (unsigned long e(0); e < nnz; ++e) { tv[e] = DT_(v[e]); tvt[e] = DT_(vt[e]); }
        P = new SparseMatrixELL<DT_>(ell_from_csr<DT_>(nf, nc, rp, ci, tv));
        R = new SparseMatrixELL<DT_>(ell_from_csr<DT_>(nc, nf, rpt, cit, tvt));
    }

    template <typename DT_>
    DenseVector<DT_> uniform(unsigned long n, unsigned long seed)
    {
        DenseVector<DT_> v(n);
        for (unsigned long i(0); i < n; ++i) v[i] = DT_(hbo_uniform(seed, i, -1.0, 1.0));
        return v;
    }

    template <typename DT_>
    void write_raw(const std::string & path, const DT_ * p, unsigned long count)
    {
        FILE * f = fopen(path.c_str(), "wb");
        if (! f) { perror(path.c_str()); return; }
        fwrite(p, sizeof(DT_), count, f);
        fclose(f);
    }
}
