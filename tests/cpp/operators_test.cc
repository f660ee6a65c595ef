// Parity tests of the C++ operator and solver templates of the B200 tag
// (include/honei_b200.hh) against the oracle's CPU restatement of the reference
// (oracle/honei_oracle.h), one test per template as the reference's *_TEST.cc
// files have them (la/product_TEST.cc, math/defect_TEST.cc, math/cg_TEST.cc,
// math/mg_TEST.cc, math/ir_TEST.cc).  Products, defects and the MG iterates are
// compared bit for bit; dots, norms and solver iterates where the summation order
// of a GPU reduction differs from the reference's within stated tolerances.
//
// Built and run by tests/test_cpp_api.py; compile with -ffp-contract=off so the
// host-side expectations round like the reference's CPU code.
#include "honei_b200.hh"
#include "honei_oracle.h"

#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

using namespace honei_b200;

namespace
{
    struct Failure
    {
        std::string what;
    };

#define TEST_CHECK(cond)                                                                                  \
    do                                                                                                    \
    {                                                                                                     \
        if (! (cond)) throw Failure{std::string(__FILE__) + ":" + std::to_string(__LINE__) + ": " #cond}; \
    } while (0)

    template <typename DT_>
    bool same_bits(const std::vector<DT_> & a, const std::vector<DT_> & b)
    {
        return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(DT_)) == 0);
    }

    double rel_diff(const std::vector<double> & a, const std::vector<double> & b)
    {
        double d = 0.0, n = 0.0;
        for (size_t i = 0; i < a.size(); ++i)
        {
            d += (a[i] - b[i]) * (a[i] - b[i]);
            n += b[i] * b[i];
        }
        return std::sqrt(d / n);
    }

    std::vector<double> uniform(uint64_t n, uint64_t seed)
    {
        std::vector<double> v(n);
        hbo_uniform_fill_f64(v.data(), n, seed, -1.0, 1.0);
        return v;
    }

    /* the level-L Q1 Poisson operator in the reference's ELL arrays (T = 1) */
    struct RefEll
    {
        uint64_t rows, stride, K;
        std::vector<uint64_t> Aj, Arl;
        std::vector<double> Ax;
        std::vector<double> bands;
    };

    RefEll q1_ell(unsigned L)
    {
        RefEll e;
        e.rows = hbo_q1_n(L);
        e.bands.resize(9 * e.rows);
        hbo_q1_bands_f64(L, 1.0, e.bands.data());
        std::vector<uint64_t> rowptr(e.rows + 1), col(9 * e.rows);
        std::vector<double> val(9 * e.rows);
        hbo_q1_csr_f64(L, e.bands.data(), rowptr.data(), col.data(), val.data());
        hbo_ell_dims(e.rows, rowptr.data(), 1, &e.stride, &e.K);
        e.Aj.assign(e.K * e.stride, 0);
        e.Ax.assign(e.K * e.stride, 0.0);
        e.Arl.assign(e.rows, 0);
        hbo_ell_from_csr_f64(e.rows, rowptr.data(), col.data(), val.data(), 1, e.stride, e.K, e.Aj.data(),
                             e.Ax.data(), e.Arl.data());
        return e;
    }

    std::vector<double> ref_spmv(const RefEll & e, const std::vector<double> & x)
    {
        std::vector<double> y(e.rows);
        hbo_ell_spmv_f64(e.rows, e.stride, 1, e.Aj.data(), e.Ax.data(), e.Arl.data(), x.data(), y.data());
        return y;
    }

    // ---------------------------------------------------------------- tests
    void product_ell_test()
    {
        for (unsigned L : {2u, 5u, 8u})
        {
            const RefEll e = q1_ell(L);
            SparseMatrixELL<double> A(e.rows, e.rows, e.stride, e.K, e.Aj, e.Ax, e.Arl);
            TEST_CHECK(A.rows() == e.rows && A.columns() == e.rows && A.stride() == e.stride &&
                       A.num_cols_per_row() == e.K && A.threads() == 1);
            const std::vector<double> xh = uniform(e.rows, 7);
            DenseVector<double> x(xh), y(e.rows);
            Product<tags::B200>::value(y, A, x);
            TEST_CHECK(same_bits(y.to_host(), ref_spmv(e, xh)));
            // the device-assembled operator has the reference's arrays and products
            SparseMatrixELL<double> Q = SparseMatrixELL<double>::poisson_q1(L);
            std::vector<uint64_t> Aj, Arl;
            std::vector<double> Ax;
            Q.export_arrays(Aj, Ax, Arl);
            TEST_CHECK(same_bits(Aj, e.Aj) && same_bits(Ax, e.Ax) && same_bits(Arl, e.Arl));
            DenseVector<double> y2(e.rows);
            Product<tags::B200>::value(y2, Q, x);
            TEST_CHECK(same_bits(y2.to_host(), y.to_host()));
        }
    }

    void defect_ell_test()
    {
        const unsigned L = 7;
        const RefEll e = q1_ell(L);
        SparseMatrixELL<double> A(e.rows, e.rows, e.stride, e.K, e.Aj, e.Ax, e.Arl);
        const std::vector<double> xh = uniform(e.rows, 3), bh = uniform(e.rows, 4);
        DenseVector<double> x(xh), b(bh), r(e.rows);
        Defect<tags::B200>::value(r, b, A, x);
        std::vector<double> want(e.rows);
        hbo_ell_defect_f64(e.rows, e.stride, 1, e.Aj.data(), e.Ax.data(), e.Arl.data(), bh.data(), xh.data(),
                           want.data());
        TEST_CHECK(same_bits(r.to_host(), want));
    }

    void banded_q1_test()
    {
        const unsigned L = 7;
        const RefEll e = q1_ell(L);
        const uint64_t n = e.rows, m = hbo_q1_m(L);
        BandedMatrixQx<double> Q(n, e.bands);
        const std::vector<double> xh = uniform(n, 11), bh = uniform(n, 12);
        DenseVector<double> x(xh), b(bh), y(n), r(n);
        Product<tags::B200>::value(y, Q, x);
        std::vector<double> want(n);
        hbo_q1_spmv_f64(n, m, e.bands.data(), xh.data(), want.data());
        TEST_CHECK(same_bits(y.to_host(), want));
        Defect<tags::B200>::value(r, b, Q, x);
        hbo_q1_defect_f64(n, m, e.bands.data(), bh.data(), xh.data(), want.data());
        TEST_CHECK(same_bits(r.to_host(), want));
        BandedMatrixQx<double> Qd = BandedMatrixQx<double>::poisson_q1(L);
        Product<tags::B200>::value(y, Qd, x);
        hbo_q1_spmv_f64(n, m, e.bands.data(), xh.data(), want.data());
        TEST_CHECK(same_bits(y.to_host(), want));
    }

    void blas1_test()
    {
        const uint64_t n = 100003;
        const std::vector<double> xh = uniform(n, 21), yh = uniform(n, 22);
        const double b = 0.3;
        // ScaledSum x += b y: the product and the sum rounded separately
        DenseVector<double> x(xh), y(yh);
        ScaledSum<tags::B200>::value(x, y, b);
        std::vector<double> want(n);
        for (uint64_t i = 0; i < n; ++i)
        {
            const volatile double p = b * yh[i];
            want[i] = xh[i] + p;
        }
        TEST_CHECK(same_bits(x.to_host(), want));
        // ScaledSum r = b y + x into a third vector; the shallow copy shares the array
        DenseVector<double> r(n), x0(xh);
        DenseVector<double> alias = r;
        ScaledSum<tags::B200>::value(r, x0, y, b);
        TEST_CHECK(same_bits(alias.to_host(), want));
        // Sum, Difference, Scale, ElementProduct
        DenseVector<double> s = x0.clone();
        Sum<tags::B200>::value(s, y);
        Difference<tags::B200>::value(s, y);
        Scale<tags::B200>::value(s, 2.0);
        std::vector<double> sh = s.to_host();
        bool ok = true;
        for (uint64_t i = 0; i < n; ++i)
        {
            const volatile double t = xh[i] + yh[i];
            const volatile double u = t - yh[i];
            ok = ok && sh[i] == 2.0 * u;
        }
        TEST_CHECK(ok);
        DenseVector<double> e(n);
        ElementProduct<tags::B200>::value(e, x0, y);
        std::vector<double> eh = e.to_host();
        for (uint64_t i = 0; i < n; ++i) ok = ok && eh[i] == xh[i] * yh[i];
        TEST_CHECK(ok);
        // DotProduct / Norm: a tree-ordered sum against the reference's sequential one
        const double d = DotProduct<tags::B200>::value(x0, y), dref = hbo_dot_f64(n, xh.data(), yh.data());
        TEST_CHECK(std::fabs(d - dref) <= 1e-12 * std::fabs(dref) + 1e-12);
        const double n2 = Norm<vnt_l_two, false, tags::B200>::value(x0), n2ref = hbo_dot_f64(n, xh.data(), xh.data());
        TEST_CHECK(std::fabs(n2 - n2ref) <= 1e-12 * n2ref);
        const double n1 = Norm<vnt_l_two, true, tags::B200>::value(x0);
        TEST_CHECK(std::fabs(n1 - std::sqrt(n2ref)) <= 1e-12 * std::sqrt(n2ref));
    }

    void ri_smoother_test()
    {
        const unsigned L = 6;
        const uint64_t n = hbo_q1_n(L);
        SparseMatrixELL<double> A = SparseMatrixELL<double>::poisson_q1(L);
        const std::vector<double> bh = uniform(n, 31);
        DenseVector<double> b(bh), x(n);
        DenseVector<double> P = RISmoother<tags::B200>::jacobi_precon(A, 0.7);
        std::vector<DenseVector<double>> temps;
        RISmoother<tags::B200>::value(A, P, b, x, temps, 5);
        std::vector<double> want(n, 0.0);
        hbo_jacobi_q1_f64(L, 1.0, 0.7, bh.data(), want.data(), 5);
        TEST_CHECK(same_bits(x.to_host(), want));
    }

    void cg_solver_test()
    {
        const unsigned L = 5;
        const RefEll e = q1_ell(L);
        SparseMatrixELL<double> A(e.rows, e.rows, e.stride, e.K, e.Aj, e.Ax, e.Arl);
        const std::vector<double> bh = ref_spmv(e, uniform(e.rows, 42));
        DenseVector<double> b(bh), x(e.rows);
        uint64_t used = 0;
        CGSolver<tags::B200, methods::NONE>::value(A, A, b, x, 2000, used, 1e-8);
        std::vector<double> xr(e.rows, 0.0);
        const uint64_t ref_used = hbo_cg_q1_f64(L, 1.0, bh.data(), xr.data(), 2000, 1e-8);
        TEST_CHECK(used + 1 >= ref_used && used <= ref_used + 1);
        std::vector<double> xs = x.to_host(), res = ref_spmv(e, xs);
        double rn = 0.0, bn = 0.0;
        for (uint64_t i = 0; i < e.rows; ++i)
        {
            rn += (bh[i] - res[i]) * (bh[i] - res[i]);
            bn += bh[i] * bh[i];
        }
        TEST_CHECK(std::sqrt(rn / bn) < 1.5e-8);
    }

    void mg_solver_test()
    {
        // MG V(4,4) with the reference-order coarse CG: the reference's iterates bit
        // for bit (coarse cap 1000, math/mg_TEST.cc)
        for (unsigned L : {5u, 6u})
        {
            const RefEll e = q1_ell(L);
            const std::vector<double> bh = ref_spmv(e, uniform(e.rows, 42));
            MGData<double> data = MGData<double>::poisson_q1(3, L, mg_params(1e-10, 100, 1000));
            DenseVector<double> b(bh), x(e.rows);
            MGSolver<tags::B200, Norm<vnt_l_two, true, tags::B200>>::value(data, b, x);
            std::vector<double> xr(e.rows, 0.0);
            double stats[4];
            const uint64_t it = hbo_mg_q1_f64(3, L, 1.0, 0.7, 4, 4, 100, 1000, 1e-10, 1e-10, bh.data(), xr.data(),
                                              stats);
            TEST_CHECK(data.used_iters == it);
            TEST_CHECK(same_bits(x.to_host(), xr));
        }
    }

    void ir_solver_test()
    {
        const unsigned L = 6;
        const RefEll e = q1_ell(L);
        const std::vector<double> bh = ref_spmv(e, uniform(e.rows, 42));
        SparseMatrixELL<double> A = SparseMatrixELL<double>::poisson_q1(L);
        MGData<float> inner = MGData<float>::poisson_q1(3, L, mg_params(1e-3, 100, 1000));
        DenseVector<double> b(bh), x(e.rows);
        uint64_t used = 0;
        IRSolver<tags::B200, tags::B200, Norm<vnt_l_two, true, tags::B200>>::value(A, b, x, inner, 1e-10, 100, used);
        std::vector<double> xr(e.rows, 0.0);
        double stats[4];
        const uint64_t ref_used = hbo_ir_q1(3, L, 1.0, 0.7, 4, 4, 100, 1000, 1e-3, 1e-3, 100, 1e-10, 0, bh.data(),
                                            xr.data(), stats);
        TEST_CHECK(used + 1 >= ref_used && used <= ref_used + 1);
        TEST_CHECK(rel_diff(x.to_host(), xr) < 1e-9);
    }

    void transfer_test()
    {
        const unsigned L = 6;
        const uint64_t nf = hbo_q1_n(L), nc = hbo_q1_n(L - 1);
        const std::vector<uint64_t> mask = all_dirichlet();
        const std::vector<double> ch = uniform(nc, 51), fh = uniform(nf, 52);
        DenseVector<double> c(ch), f(fh), fine(nf), coarse(nc);
        std::pair<SparseMatrixELL<double>, SparseMatrixELL<double>> PR = q1_transfer<double>(L);
        Prolongation<tags::B200, methods::NONE>::value(fine, c, mask, PR.first);
        std::vector<double> want(nf);
        hbo_prolongation_f64(nf, want.data(), nc, ch.data(), mask.data());
        TEST_CHECK(same_bits(fine.to_host(), want));
        Restriction<tags::B200, methods::NONE>::value(coarse, f, mask, PR.second);
        std::vector<double> wantc(nc);
        hbo_restriction_f64(nc, wantc.data(), nf, fh.data(), mask.data());
        TEST_CHECK(same_bits(coarse.to_host(), wantc));
        // PROLMAT: the ProlongationMatrix of the oracle, as ELL, applied on the host
        std::vector<uint64_t> rowptr(nf + 1), col(4 * nf);
        std::vector<double> val(4 * nf);
        hbo_prolmat_csr_f64(L, rowptr.data(), col.data(), val.data());
        uint64_t stride = 0, K = 0;
        hbo_ell_dims(nf, rowptr.data(), 1, &stride, &K);
        std::vector<uint64_t> Aj(K * stride, 0), Arl(nf, 0);
        std::vector<double> Ax(K * stride, 0.0);
        hbo_ell_from_csr_f64(nf, rowptr.data(), col.data(), val.data(), 1, stride, K, Aj.data(), Ax.data(), Arl.data());
        std::vector<uint64_t> dAj, dArl;
        std::vector<double> dAx;
        PR.first.export_arrays(dAj, dAx, dArl);
        TEST_CHECK(same_bits(dAj, Aj) && same_bits(dAx, Ax) && same_bits(dArl, Arl));
        Prolongation<tags::B200, methods::PROLMAT>::value(fine, c, mask, PR.first);
        hbo_ell_spmv_f64(nf, stride, 1, Aj.data(), Ax.data(), Arl.data(), ch.data(), want.data());
        TEST_CHECK(same_bits(fine.to_host(), want));
        // the restriction matrix is the Transposition of the prolongation matrix
        SparseMatrixELL<double> Rt = Transposition<tags::B200>::value(PR.first);
        std::vector<uint64_t> rAj, rArl, tAj, tArl;
        std::vector<double> rAx, tAx;
        PR.second.export_arrays(rAj, rAx, rArl);
        Rt.export_arrays(tAj, tAx, tArl);
        TEST_CHECK(same_bits(rAj, tAj) && same_bits(rAx, tAx) && same_bits(rArl, tArl));
        Restriction<tags::B200, methods::PROLMAT>::value(coarse, f, mask, Rt);
        DenseVector<double> coarse2(nc);
        Product<tags::B200>::value(coarse2, PR.second, f);
        TEST_CHECK(same_bits(coarse.to_host(), coarse2.to_host()));
    }

    void matrix_io_test()
    {
        SparseMatrixELL<double> A = SparseMatrixELL<double>::poisson_q1(5);
        char path[] = "/tmp/hb2_matrix_io_XXXXXX";
        const int fd = mkstemp(path);
        TEST_CHECK(fd >= 0);
        close(fd);
        MatrixIO<io_formats::ELL>::write_matrix(path, A);
        SparseMatrixELL<double> B = MatrixIO<io_formats::ELL>::read_matrix(path, double(0));
        std::remove(path);
        std::vector<uint64_t> aj, arl, bj, brl;
        std::vector<double> ax, bx;
        A.export_arrays(aj, ax, arl);
        B.export_arrays(bj, bx, brl);
        TEST_CHECK(same_bits(aj, bj) && same_bits(ax, bx) && same_bits(arl, brl));
        bool thrown = false;
        try
        {
            MatrixIO<io_formats::ELL>::read_matrix("/nonexistent/file.ell", double(0));
        }
        catch (const InternalError &)
        {
            thrown = true;
        }
        TEST_CHECK(thrown);
    }

    void csr_test()
    {
        const unsigned L = 7;
        SparseMatrixELL<double> A = SparseMatrixELL<double>::poisson_q1(L);
        for (uint64_t bs : {1ull, 2ull})
        {
            SparseMatrixCSR<double> C = SparseMatrixCSR<double>::from_ell(A, bs);
            TEST_CHECK(C.rows() == A.rows() && C.columns() == A.columns() && C.blocksize() == bs);
            std::vector<uint64_t> Ar, Aj;
            std::vector<double> Ax;
            C.export_arrays(Ar, Aj, Ax);
            SparseMatrixCSR<double> C2(C.rows(), C.columns(), bs, Ar, Aj, Ax);
            const uint64_t n = A.rows();
            const std::vector<double> xh = uniform(n, 61), bh = uniform(n, 62);
            DenseVector<double> x(xh), b(bh), y(n), r(n);
            Product<tags::B200>::value(y, C2, x);
            std::vector<double> want(n);
            hbo_csr_spmv_f64(n, bs, n, Ar.data(), Aj.data(), Ax.data(), xh.data(), want.data());
            TEST_CHECK(same_bits(y.to_host(), want));
            Defect<tags::B200>::value(r, b, C, x);
            hbo_csr_defect_f64(n, bs, n, Ar.data(), Aj.data(), Ax.data(), bh.data(), xh.data(), want.data());
            TEST_CHECK(same_bits(r.to_host(), want));
        }
    }

    void krylov_test()
    {
        const unsigned L = 5;
        const RefEll e = q1_ell(L);
        SparseMatrixELL<double> A(e.rows, e.rows, e.stride, e.K, e.Aj, e.Ax, e.Arl);
        const std::vector<double> bh = ref_spmv(e, uniform(e.rows, 42));
        DenseVector<double> P = RISmoother<tags::B200>::jacobi_precon(A, 1.0);   // 1 / diag
        const std::vector<double> ph = P.to_host();
        hbo_ell_view v{e.rows, e.rows, e.stride, e.K, e.Aj.data(), e.Ax.data(), e.Arl.data()};
        DenseVector<double> b(bh);
        {
            DenseVector<double> x(e.rows);
            uint64_t used = 0;
            CGSolver<tags::B200, methods::VAR>::value(A, P, b, x, 1000, used, 1e-8);
            std::vector<double> xr(e.rows, 0.0);
            const uint64_t ref = hbo_cgvar_f64(&v, ph.data(), nullptr, bh.data(), xr.data(), 1000, 1e-8, 0);
            TEST_CHECK(used + 1 >= ref && used <= ref + 1);
            TEST_CHECK(rel_diff(x.to_host(), xr) < 1e-6);
        }
        {
            DenseVector<double> x(e.rows);
            uint64_t used = 0;
            BiCGStabSolver<tags::B200, methods::VAR>::value(A, P, b, x, 1000, used, 1e-8);
            std::vector<double> xr(e.rows, 0.0);
            const uint64_t ref = hbo_bicgstab_f64(&v, ph.data(), nullptr, bh.data(), xr.data(), 1000, 1e-8);
            TEST_CHECK(used + 1 >= ref && used <= ref + 1);
            TEST_CHECK(rel_diff(x.to_host(), xr) < 1e-3);
        }
        {
            DenseVector<double> x(e.rows);
            std::vector<DenseVector<double>> temps;
            CGSmoother<tags::B200>::value(A, P, b, x, temps, 5);
            std::vector<double> xr(e.rows, 0.0);
            hbo_cgvar_f64(&v, ph.data(), nullptr, bh.data(), xr.data(), 5, 0.0, 1);
            TEST_CHECK(rel_diff(x.to_host(), xr) < 1e-10);
        }
    }

    void legacy_multigrid_test()
    {
        // FIXED on an assembled hierarchy, levels 1..8: the oracle's cycles and iterates
        const unsigned lmin = 1, L = 8;
        std::vector<std::vector<double>> bands(L + 1), dinv(L + 1);
        std::vector<BandedMatrixQx<double>> levels;
        const double * bp[32] = {nullptr};
        const double * dp[32] = {nullptr};
        for (unsigned l = lmin; l <= L; ++l)
        {
            const uint64_t n = hbo_q1_n(l);
            bands[l].resize(9 * n);
            hbo_q1_bands_f64(l, 1.0, bands[l].data());
            dinv[l].resize(n);
            for (uint64_t i = 0; i < n; ++i)
            {
                const double dd = bands[l][4 * n + i];
                const double inv = dd == 0.0 ? 0.0 : 1.0 / dd;
                dinv[l][i] = inv * 0.7;
            }
            bp[l] = bands[l].data();
            dp[l] = dinv[l].data();
            levels.push_back(BandedMatrixQx<double>::poisson_q1(l));
        }
        const uint64_t n = hbo_q1_n(L), m = hbo_q1_m(L);
        std::vector<double> bh(n), x0 = uniform(n, 4);
        const std::vector<double> u = uniform(n, 3);
        hbo_q1_spmv_f64(n, m, bands[L].data(), u.data(), bh.data());
        for (double & v : x0) v *= 0.01;
        MGInfo<double> info(lmin, levels, mg_info_params(40, true, 1e-10, 2));
        DenseVector<double> b(bh), x(x0);
        Multigrid<tags::B200, tags::B200, methods::NONE, methods::JAC, methods::CYCLE::V, methods::FIXED>::value(
            levels.back(), b, x, L, 0.0, info);
        std::vector<double> xr = x0;
        const uint64_t mask[8] = {2, 2, 2, 2, 2, 2, 2, 2};
        const uint64_t cycles = hbo_lmg_f64(lmin, L, bp, dp, bh.data(), xr.data(), 40, 1, 0, 0, 1e-10, 2, 1.0, mask);
        TEST_CHECK(info.cycles == cycles);
        TEST_CHECK(same_bits(x.to_host(), xr));
    }

    void size_error_test()
    {
        SparseMatrixELL<double> A = SparseMatrixELL<double>::poisson_q1(4);
        DenseVector<double> x(A.columns()), y(A.rows() + 1), b(A.rows() + 2);
        bool thrown = false;
        try
        {
            Product<tags::B200>::value(y, A, x);
        }
        catch (const VectorSizeDoesNotMatch &)
        {
            thrown = true;
        }
        TEST_CHECK(thrown);
        DenseVector<double> r(A.rows());
        thrown = false;
        try
        {
            Defect<tags::B200>::value(r, b, A, x);
        }
        catch (const MatrixRowsDoNotMatch &)
        {
            thrown = true;
        }
        TEST_CHECK(thrown);
        thrown = false;
        try
        {
            MGData<double> data = MGData<double>::poisson_q1(5, 4, mg_params());   // min above max
        }
        catch (const InternalError &)
        {
            thrown = true;
        }
        TEST_CHECK(thrown);
    }
}

int main()
{
    const std::vector<std::pair<const char *, std::function<void()>>> tests = {
        {"product_ell_test", product_ell_test}, {"defect_ell_test", defect_ell_test},
        {"banded_q1_test", banded_q1_test},     {"blas1_test", blas1_test},
        {"ri_smoother_test", ri_smoother_test}, {"cg_solver_test", cg_solver_test},
        {"mg_solver_test", mg_solver_test},     {"ir_solver_test", ir_solver_test},
        {"transfer_test", transfer_test},       {"matrix_io_test", matrix_io_test},
        {"csr_test", csr_test},                 {"krylov_test", krylov_test},
        {"legacy_multigrid_test", legacy_multigrid_test},
        {"size_error_test", size_error_test}};
    int failed = 0;
    for (const auto & t : tests)
    {
        try
        {
            t.second();
            std::printf("PASSED %s\n", t.first);
        }
        catch (const Failure & f)
        {
            std::printf("FAILED %s: %s\n", t.first, f.what.c_str());
            ++failed;
        }
        catch (const std::exception & ex)
        {
            std::printf("FAILED %s: exception %s\n", t.first, ex.what());
            ++failed;
        }
    }
    std::printf("%zu tests, %d failed\n", tests.size(), failed);
    return failed ? 1 : 0;
}
