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
