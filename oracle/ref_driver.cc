// Driver around the reference implementation's own CPU path (test infrastructure
// only; compiled with the reference sources by oracle/ref.mk into oracle/_ref/).
//
//   honei_ref golden <outdir>
//       writes golden fixtures computed by the reference's tags::CPU code
//       (raw little-endian arrays + scalars.txt); tests/golden/make_golden.py
//       packs them into the committed fixtures.
//   honei_ref mglegacy <testdata dir> <outdir>
//       Multigrid<..., JAC, CYCLE::V, FIXED> on the banded Q1 test data
//   honei_ref krylov <outdir>
//       CGSolver VAR, BiCGStabSolver VAR and CGSmoother on the Q1 operator
//   honei_ref csr <outdir>
//       SparseMatrixCSR arrays (csr::blocksize 1..4) and their Product / Defect
//   honei_ref mgquad <datadir> <outdir>
//       the reference's MGSolverTestQuad on its FEAST test data (W-cycle); writes
//       the solution (raw doubles), the iteration counts and the restriction
//       matrices (res_<level>.ell, reference ELL files)
//   honei_ref bench <cg|mg|ir|spmv> <cpu|generic|sse|mc> <level> <reps> [warmup]
//       times the solve phase (operator setup excluded; `warmup` untimed solves
//       first) and prints one "RESULT {json}" line.  The thread count of the MultiCore tag comes from
//       the honeirc named by $HONEI_CONFIG (mc::num_threads).
#include "ref_common.hh"

#include <honei/la/dot_product.hh>
#include <honei/la/sparse_matrix_csr.hh>
#include <honei/la/norm.hh>
#include <honei/la/product.hh>
#include <honei/la/scaled_sum.hh>
#include <honei/la/sum.hh>
#include <honei/math/bicgstab.hh>
#include <honei/math/cg.hh>
#include <honei/math/defect.hh>
#include <honei/math/ir.hh>
#include <honei/math/matrix_io.hh>
#include <honei/math/mg.hh>
#include <honei/math/multigrid.hh>
#include <honei/math/vector_io.hh>
#include <honei/math/prolongation.hh>
#include <honei/math/restriction.hh>
#include <honei/math/ri.hh>
#include <honei/util/configuration.hh>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <algorithm>

using namespace honei;
using namespace hbref;

namespace
{
    std::ofstream scalars;
    std::string outdir;
    // coarse CG iteration cap of the timed MG solves: the value the reference's
    // own MG tests use (math/mg_TEST.cc:421); overridable with $HONEI_COARSE_CAP
    unsigned long coarse_cap = 100;

    template <typename DT_>
    void put_vec(const std::string & name, const DenseVector<DT_> & v)
    {
        write_raw(outdir + "/" + name, v.elements(), v.size());
    }

    template <typename DT_>
    void put_ell(const std::string & name, const SparseMatrixELL<DT_> & A)
    {
        put_vec(name + ".Aj", A.Aj());
        put_vec(name + ".Ax", A.Ax());
        put_vec(name + ".Arl", A.Arl());
        scalars << name << ".rows " << A.rows() << "\n" << name << ".cols " << A.columns() << "\n"
                << name << ".stride " << A.stride() << "\n" << name << ".K " << A.num_cols_per_row() << "\n"
                << name << ".T " << A.threads() << "\n";
    }

    std::string key(const char * fmt, unsigned a, const char * b = "")
    {
        char buf[128];
        snprintf(buf, sizeof buf, fmt, a, b);
        return buf;
    }

    // MGData over levels 1..L (internal index = level - 1), V(n_pre, n_post),
    // Jacobi preconditioner "jac" (math/mg.hh:255-288), PROLMAT transfers.
    template <typename DT_>
    struct Hierarchy
    {
        std::vector<SparseMatrixELL<DT_> > A, Res, Prol;
        std::vector<DenseVector<DT_> > P, b, x, d, c, store;
        std::vector<std::vector<DenseVector<DT_> > > temps;

        Hierarchy(unsigned L, double omega, bool assembled, double aniso = 1.0)
        {
            for (unsigned l(1); l <= L; ++l)
            {
                SparseMatrixELL<DT_> Al(assembled ? q1_ell_assembled<DT_>(l) : q1_ell_fast<DT_>(l, aniso));
                A.push_back(Al);
                DenseVector<DT_> Pl(Al.rows(), DT_(omega));
                for (unsigned long j(0); j < Pl.size(); ++j)
                    Pl[j] /= Al(j, j);
                P.push_back(Pl);
                if (l >= 2)
                {
                    SparseMatrixELL<DT_> * p, * r;
                    if (assembled) transfer_assembled<DT_>(l, p, r); else transfer_fast<DT_>(l, p, r);
                    Prol.push_back(*p);
                    Res.push_back(*r);
                    delete p;
                    delete r;
                }
                DenseVector<DT_> z(Al.rows(), DT_(0));
                b.push_back(z.copy());
                x.push_back(z.copy());
                d.push_back(z.copy());
                c.push_back(z.copy());
                store.push_back(z.copy());
                temps.push_back(std::vector<DenseVector<DT_> >());
            }
        }

        MGData<SparseMatrixELL<DT_>, DenseVector<DT_>, SparseMatrixELL<DT_>, DenseVector<DT_>, DT_>
        data(unsigned long max_iters, unsigned long max_iters_coarse, unsigned long n_pre, unsigned long n_post,
             unsigned long min_level, DT_ eps)
        {
            return MGData<SparseMatrixELL<DT_>, DenseVector<DT_>, SparseMatrixELL<DT_>, DenseVector<DT_>, DT_>(
                    A, Res, Prol, P, b, x, d, c, store, temps, max_iters, max_iters_coarse, n_pre, n_post,
                    min_level, eps);
        }
    };

    template <typename Tag_, typename DT_>
    OperatorList v_cycle(MGData<SparseMatrixELL<DT_>, DenseVector<DT_>, SparseMatrixELL<DT_>, DenseVector<DT_>, DT_> & data)
    {
        return MGCycleCreation<Tag_, methods::CYCLE::V::STATIC, CGSolver<Tag_, methods::NONE>, RISmoother<Tag_>,
               Restriction<Tag_, methods::PROLMAT>, Prolongation<Tag_, methods::PROLMAT>, DT_>::value(data);
    }

    double rel_residual(const SparseMatrixELL<double> & A, const DenseVector<double> & b, const DenseVector<double> & x)
    {
        DenseVector<double> r(b.size());
        Defect<tags::CPU>::value(r, b, A, x);
        return Norm<vnt_l_two, true, tags::CPU>::value(r) / Norm<vnt_l_two, true, tags::CPU>::value(b);
    }

    // ---------------------------------------------------------------- golden
    int golden()
    {
        scalars.open((outdir + "/scalars.txt").c_str());
        scalars.precision(17);

        // ELL assembly, T = 1 (and T = 2, 3 through the ell::threads key)
        for (unsigned L(1); L <= 8; ++L)
        {
            put_ell(key("ell_L%u_T1_f64", L), q1_ell_assembled<double>(L));
            if (L <= 6) put_ell(key("ell_L%u_T1_f32", L), q1_ell_assembled<float>(L));
        }
        for (unsigned T(2); T <= 3; ++T)
        {
            Configuration::instance()->set_value("ell::threads", int(T));
            for (unsigned L(2); L <= 4; ++L)
            {
                char nm[64];
                snprintf(nm, sizeof nm, "ell_L%u_T%u_f64", L, T);
                SparseMatrixELL<double> A(q1_ell_assembled<double>(L));
                put_ell(nm, A);
                DenseVector<double> xv(uniform<double>(A.columns(), 7)), yv(A.rows());
                Product<tags::CPU>::value(yv, A, xv);
                snprintf(nm, sizeof nm, "spmv_L%u_T%u_f64", L, T);
                put_vec(nm, yv);
            }
        }
        Configuration::instance()->set_value("ell::threads", 1);

        // grid transfer matrices
        for (unsigned L(2); L <= 8; ++L)
        {
            SparseMatrixELL<double> * P, * R;
            transfer_assembled<double>(L, P, R);
            put_ell(key("prol_L%u_f64", L), *P);
            put_ell(key("res_L%u_f64", L), *R);
            delete P;
            delete R;
        }

        // SpMV / defect on ELL and on the banded Q1 matrix
        for (unsigned L(1); L <= 7; ++L)
        {
            SparseMatrixELL<double> A(q1_ell_assembled<double>(L));
            DenseVector<double> xv(uniform<double>(A.columns(), 7)), rhs(uniform<double>(A.rows(), 11));
            DenseVector<double> y(A.rows()), r(A.rows());
            Product<tags::CPU>::value(y, A, xv);
            Defect<tags::CPU>::value(r, rhs, A, xv);
            put_vec(key("spmv_L%u_f64", L), y);
            put_vec(key("defect_L%u_f64", L), r);

            SparseMatrixELL<float> Af(q1_ell_assembled<float>(L));
            DenseVector<float> xf(uniform<float>(A.columns(), 7)), rf(uniform<float>(A.rows(), 11));
            DenseVector<float> yf(A.rows()), df(A.rows());
            Product<tags::CPU>::value(yf, Af, xf);
            Defect<tags::CPU>::value(df, rf, Af, xf);
            put_vec(key("spmv_L%u_f32", L), yf);
            put_vec(key("defect_L%u_f32", L), df);

            BandedMatrixQx<Q1Type, double> Q(q1_banded<double>(L));
            DenseVector<double> yq(A.rows()), rq(A.rows());
            Product<tags::CPU>::value(yq, Q, xv);
            Defect<tags::CPU>::value(rq, rhs, Q, xv);
            put_vec(key("q1spmv_L%u_f64", L), yq);
            put_vec(key("q1defect_L%u_f64", L), rq);
        }

        // BLAS-1 on seeded vectors (n = 1000)
        {
            DenseVector<double> a(uniform<double>(1000, 21)), b(uniform<double>(1000, 22));
            scalars << "dot_1000_f64 " << DotProduct<tags::CPU>::value(a, b) << "\n";
            scalars << "norm2sq_1000_f64 " << Norm<vnt_l_two, false, tags::CPU>::value(a) << "\n";
            scalars << "norm2_1000_f64 " << Norm<vnt_l_two, true, tags::CPU>::value(a) << "\n";
            DenseVector<double> s1(a.copy());
            ScaledSum<tags::CPU>::value(s1, b, 0.375);
            put_vec("scaledsum2_1000_f64", s1);
            DenseVector<double> s2(1000);
            ScaledSum<tags::CPU>::value(s2, a, b, -1.25);
            put_vec("scaledsum3_1000_f64", s2);
        }

        // matrix-free and PROLMAT grid transfer outputs (mask: all Dirichlet)
        for (unsigned L(2); L <= 7; ++L)
        {
            unsigned long nf(hbo_q1_n(L)), nc(hbo_q1_n(L - 1));
            DenseVector<unsigned long> mask(8, 2ul);
            DenseVector<double> coarse(uniform<double>(nc, 31)), fine(uniform<double>(nf, 32));
            DenseVector<double> pf(nf), rc(nc), pfm(nf), rcm(nc);
            SparseMatrixELL<double> * P, * R;
            transfer_assembled<double>(L, P, R);
            Prolongation<tags::CPU, methods::NONE>::value(pf, coarse, mask, *P);
            Restriction<tags::CPU, methods::NONE>::value(rc, fine, mask, *R);
            Prolongation<tags::CPU, methods::PROLMAT>::value(pfm, coarse, mask, *P);
            Restriction<tags::CPU, methods::PROLMAT>::value(rcm, fine, mask, *R);
            put_vec(key("prolong_L%u_f64", L), pf);
            put_vec(key("restrict_L%u_f64", L), rc);
            put_vec(key("prolmat_L%u_f64", L), pfm);
            put_vec(key("resmat_L%u_f64", L), rcm);
            delete P;
            delete R;
        }

        // CG, FP64, b = A u*, x0 = 0, rel. tol 1e-8 (the CPU-sized CG workload at L = 5, 7)
        for (unsigned L(5); L <= 7; L += 2)
        {
            SparseMatrixELL<double> A(q1_ell_assembled<double>(L));
            DenseVector<double> u(uniform<double>(A.rows(), 42)), b(A.rows()), x(A.rows(), 0.0);
            Product<tags::CPU>::value(b, A, u);
            unsigned long used(0);
            DenseVector<double> dummy(1);
            CGSolver<tags::CPU, methods::NONE>::value(A, dummy, b, x, 2000ul, used, 1e-8);
            scalars << key("cg_L%u.iters", L) << " " << used << "\n";
            scalars << key("cg_L%u.relres", L) << " " << rel_residual(A, b, x) << "\n";
            put_vec(key("cg_L%u.x", L), x);
            put_vec(key("cg_L%u.b", L), b);
        }

        // Jacobi smoothing: 4 sweeps, omega 0.7, from x = 0
        for (unsigned L(3); L <= 6; ++L)
        {
            SparseMatrixELL<double> A(q1_ell_assembled<double>(L));
            DenseVector<double> P(A.rows(), 0.7);
            for (unsigned long j(0); j < P.size(); ++j) P[j] /= A(j, j);
            DenseVector<double> b(uniform<double>(A.rows(), 5)), x(A.rows(), 0.0);
            std::vector<DenseVector<double> > temps;
            temps.push_back(DenseVector<double>(A.rows()));
            temps.push_back(DenseVector<double>(A.rows()));
            RISmoother<tags::CPU>::value(A, P, b, x, temps, 4);
            put_vec(key("jacobi_L%u_f64", L), x);
        }

        // MG V(4,4), omega 0.7, coarse CG on level 3, eps 1e-10 shared with the coarse CG
        for (unsigned L(5); L <= 7; ++L)
        {
            Hierarchy<double> h(L, 0.7, true);
            DenseVector<double> u(uniform<double>(h.A.back().rows(), 42));
            Product<tags::CPU>::value(h.b.back(), h.A.back(), u);
            MGData<SparseMatrixELL<double>, DenseVector<double>, SparseMatrixELL<double>, DenseVector<double>, double>
                data(h.data(100, 1000, 4, 4, 3, 1e-10));
            OperatorList cycle(v_cycle<tags::CPU, double>(data));
            MGSolver<tags::CPU, Norm<vnt_l_two, true, tags::CPU> >::value(data, cycle);
            scalars << key("mg_L%u.iters", L) << " " << data.used_iters << "\n";
            scalars << key("mg_L%u.coarse_iters", L) << " " << data.used_iters_coarse << "\n";
            scalars << key("mg_L%u.relres", L) << " " << rel_residual(h.A.back(), h.b.back(), data.x.back()) << "\n";
            put_vec(key("mg_L%u.x", L), data.x.back());
        }

        // MG FP32 at level 6, eps 1e-5
        {
            Hierarchy<float> h(6, 0.7, true);
            DenseVector<float> u(uniform<float>(h.A.back().rows(), 42));
            Product<tags::CPU>::value(h.b.back(), h.A.back(), u);
            MGData<SparseMatrixELL<float>, DenseVector<float>, SparseMatrixELL<float>, DenseVector<float>, float>
                data(h.data(100, 1000, 4, 4, 3, 1e-5f));
            OperatorList cycle(v_cycle<tags::CPU, float>(data));
            MGSolver<tags::CPU, Norm<vnt_l_two, true, tags::CPU> >::value(data, cycle);
            scalars << "mg32_L6.iters " << data.used_iters << "\n";
            put_vec("mg32_L6.x", data.x.back());
        }

        // IR: FP64 outer (eps 1e-10), FP32 inner MG V(4,4) with eps 1e-3 (shared with the coarse CG)
        for (unsigned L(5); L <= 6; ++L)
        {
            SparseMatrixELL<double> A(q1_ell_assembled<double>(L));
            DenseVector<double> u(uniform<double>(A.rows(), 42)), b(A.rows()), x(A.rows(), 0.0);
            Product<tags::CPU>::value(b, A, u);
            Hierarchy<float> h(L, 0.7, true);
            MGData<SparseMatrixELL<float>, DenseVector<float>, SparseMatrixELL<float>, DenseVector<float>, float>
                data(h.data(100, 1000, 4, 4, 3, 1e-3f));
            OperatorList cycle(v_cycle<tags::CPU, float>(data));
            unsigned long used(0);
            IRSolver<tags::CPU, tags::CPU, Norm<vnt_l_two, true, tags::CPU> >::value(A, b, x, data, cycle, 1e-10, 100ul, used);
            scalars << key("ir_L%u.iters", L) << " " << used << "\n";
            scalars << key("ir_L%u.relres", L) << " " << rel_residual(A, b, x) << "\n";
            put_vec(key("ir_L%u.x", L), x);
        }
        scalars.close();
        return 0;
    }

    // ---------------------------------------------------------------- bench
    template <typename Tag_>
    int bench(const std::string & which, unsigned L, unsigned reps, unsigned warmup, const char * tagname)
    {
        std::vector<double> times;
        double t_setup0(now());
        double secs(0), relres(0);
        unsigned long iters(0);
        if (which == "cg")
        {
            SparseMatrixELL<double> A(q1_ell_fast<double>(L));
            DenseVector<double> u(uniform<double>(A.rows(), 42)), b(A.rows());
            Product<tags::CPU>::value(b, A, u);
            DenseVector<double> dummy(1);
            double setup(now() - t_setup0);
            for (unsigned r(0); r < reps; ++r)
            {
                DenseVector<double> x(A.rows(), 0.0);
                double t0(now());
                CGSolver<Tag_, methods::NONE>::value(A, dummy, b, x, 2000ul, iters, 1e-8);
                secs += now() - t0;
                relres = rel_residual(A, b, x);
            }
            printf("RESULT {\"which\": \"cg\", \"tag\": \"%s\", \"level\": %u, \"reps\": %u, \"seconds_per_solve\": %.6g, "
                   "\"iters\": %lu, \"relres\": %.6g, \"setup_s\": %.3g}\n", tagname, L, reps, secs / reps, iters, relres, setup);
        }
        else if (which == "mg")
        {
            Hierarchy<double> h(L, 0.7, false);
            DenseVector<double> u(uniform<double>(h.A.back().rows(), 42));
            Product<tags::CPU>::value(h.b.back(), h.A.back(), u);
            double setup(now() - t_setup0);
            for (unsigned r(0); r < reps + warmup; ++r)
            {
                for (unsigned long i(0); i < h.x.back().size(); ++i) h.x.back()[i] = 0.0;
                MGData<SparseMatrixELL<double>, DenseVector<double>, SparseMatrixELL<double>, DenseVector<double>, double>
                    data(h.data(100, coarse_cap, 4, 4, 3, 1e-10));
                OperatorList cycle(v_cycle<Tag_, double>(data));
                double t0(now());
                MGSolver<Tag_, Norm<vnt_l_two, true, Tag_> >::value(data, cycle);
                if (r >= warmup) { secs += now() - t0; times.push_back(now() - t0); }
                iters = data.used_iters;
                relres = rel_residual(h.A.back(), h.b.back(), data.x.back());
            }
            std::sort(times.begin(), times.end());
            // HONEI_DUMP_X=<file>: the solution, raw doubles (the checker of other solvers' results)
            if (const char * dump = getenv("HONEI_DUMP_X"))
                if (FILE * f = fopen(dump, "wb"))
                {
                    const DenseVector<double> & xs(h.x.back());   // shared with the solver's MGData
                    for (unsigned long i(0); i < xs.size(); ++i)
                    {
                        const double v(xs[i]);
                        fwrite(&v, sizeof(double), 1, f);
                    }
                    fclose(f);
                }
            printf("RESULT {\"which\": \"mg\", \"tag\": \"%s\", \"level\": %u, \"reps\": %u, \"seconds_per_solve\": %.6g, "
                   "\"min_s\": %.6g, \"max_s\": %.6g, \"iters\": %lu, \"relres\": %.6g, \"setup_s\": %.3g, "
                   "\"coarse_cap\": %lu}\n", tagname, L, reps, secs / reps, times.front(), times.back(), iters, relres,
                   setup, coarse_cap);
        }
        else if (which == "ir")
        {
            SparseMatrixELL<double> A(q1_ell_fast<double>(L));
            DenseVector<double> u(uniform<double>(A.rows(), 42)), b(A.rows());
            Product<tags::CPU>::value(b, A, u);
            Hierarchy<float> h(L, 0.7, false);
            double setup(now() - t_setup0);
            for (unsigned r(0); r < reps; ++r)
            {
                for (unsigned long i(0); i < h.x.back().size(); ++i) h.x.back()[i] = 0.f;
                DenseVector<double> x(A.rows(), 0.0);
                MGData<SparseMatrixELL<float>, DenseVector<float>, SparseMatrixELL<float>, DenseVector<float>, float>
                    data(h.data(100, 1000, 4, 4, 3, 1e-3f));
                OperatorList cycle(v_cycle<Tag_, float>(data));
                double t0(now());
                IRSolver<Tag_, Tag_, Norm<vnt_l_two, true, Tag_> >::value(A, b, x, data, cycle, 1e-10, 100ul, iters);
                secs += now() - t0;
                relres = rel_residual(A, b, x);
            }
            printf("RESULT {\"which\": \"ir\", \"tag\": \"%s\", \"level\": %u, \"reps\": %u, \"seconds_per_solve\": %.6g, "
                   "\"iters\": %lu, \"relres\": %.6g, \"setup_s\": %.3g}\n", tagname, L, reps, secs / reps, iters, relres, setup);
        }
        else if (which == "spmv")
        {
            SparseMatrixELL<double> A(q1_ell_fast<double>(L));
            DenseVector<double> x(uniform<double>(A.rows(), 7)), y(A.rows());
            double setup(now() - t_setup0);
            Product<Tag_>::value(y, A, x);
            double t0(now());
            for (unsigned r(0); r < reps; ++r)
                Product<Tag_>::value(y, A, x);
            secs = now() - t0;
            printf("RESULT {\"which\": \"spmv\", \"tag\": \"%s\", \"level\": %u, \"reps\": %u, \"seconds_per_spmv\": %.6g, "
                   "\"setup_s\": %.3g}\n", tagname, L, reps, secs / reps, setup);
        }
        else
        {
            fprintf(stderr, "unknown benchmark '%s'\n", which.c_str());
            return 2;
        }
        fflush(stdout);
        return 0;
    }
}

namespace
{
    // The reference's own MGSolverTestQuad flow (math/mg_TEST.cc:398-463): FEAST
    // matrices A_1..A_6 and prol_2..prol_6 read by MatrixIO<ELL>, rhs_6 / init_6
    // by VectorIO<EXP>, Jacobi 0.7, W-cycle, V(4,4), coarse CG on level 1, eps 1e-8.
    int mgquad(const std::string & dir, const std::string & out)
    {
        typedef MGUtil<tags::CPU, SparseMatrixELL<double>, DenseVector<double>, SparseMatrixELL<double>,
                       DenseVector<double>, MatrixIO<io_formats::ELL>, VectorIO<io_formats::EXP>, double> Util;
        const unsigned long max_level(6), min_level(1);
        MGData<SparseMatrixELL<double>, DenseVector<double>, SparseMatrixELL<double>, DenseVector<double>, double>
            data(Util::load_data(dir, max_level, double(0.7), "jac"));
        Util::configure(data, 100, 100, 4, 4, min_level, double(1e-8));
        OperatorList ol(MGCycleCreation<tags::CPU, methods::CYCLE::W::STATIC, CGSolver<tags::CPU, methods::NONE>,
                        RISmoother<tags::CPU>, Restriction<tags::CPU, methods::PROLMAT>,
                        Prolongation<tags::CPU, methods::PROLMAT>, double>::value(data));
        MGSolver<tags::CPU, Norm<vnt_l_two, true, tags::CPU> >::value(data, ol);
        DenseVector<double> & x(data.x.at(MGDataIndex::internal_index_A(max_level)));
        write_raw(out + "/mgquad_x", x.elements(), x.size());
        // the restriction matrices load_data built (Transposition of each prol file),
        // written by the reference's own ELL writer
        for (unsigned long i(0); i < data.resmat.size(); ++i)
        {
            std::string name(out + "/res_" + stringify(i + 2) + ".ell");
            MatrixIO<io_formats::ELL>::write_matrix(name, data.resmat.at(i));
        }
        std::ofstream sc((out + "/mgquad_scalars.txt").c_str());
        sc.precision(17);
        sc << "used_iters " << data.used_iters << "\n" << "used_iters_coarse " << data.used_iters_coarse << "\n";
        return 0;
    }
}

namespace
{
    template <typename DT_>
    void put_csr_case(const std::string & name, const SparseMatrixCSR<DT_> & A)
    {
        put_vec(name + ".Ar", A.Ar());
        put_vec(name + ".Aj", A.Aj());
        put_vec(name + ".Ax", A.Ax());
        scalars << name << ".rows " << A.rows() << "\n" << name << ".cols " << A.columns() << "\n"
                << name << ".bs " << A.blocksize() << "\n" << name << ".used " << A.used_elements() << "\n";
        DenseVector<DT_> x(uniform<DT_>(A.columns(), 7)), rhs(uniform<DT_>(A.rows(), 11));
        DenseVector<DT_> y(A.rows()), r(A.rows());
        Product<tags::CPU>::value(y, A, x);
        Defect<tags::CPU>::value(r, rhs, A, x);
        put_vec(name + ".spmv", y);
        put_vec(name + ".defect", r);
    }

    // rows of very different lengths: empty rows, short rows, rows of a few
    // thousand entries and one full row; a column count that is not a multiple
    // of the block sizes tested
    SparseMatrix<double> skewed(unsigned long n, unsigned long m)
    {
        SparseMatrix<double> S(n, m);
        for (unsigned long r(0); r < n; ++r)
        {
            if (r % 11 == 3) continue;
            if (r == n / 2 + 1)
            {
                for (unsigned long c(0); c < m; ++c) S(r, c, hbo_uniform(99, r * 10007 + c, 0.25, 1.0));
                continue;
            }
            if (r % 500 == 7)
            {
                for (unsigned long c(0); c < m; ++c)
                    if ((c + r) % 3 != 2) S(r, c, hbo_uniform(99, r * 10007 + c, -1.0, -0.25));
                continue;
            }
            const unsigned long k(1 + (r * 7) % 17);
            for (unsigned long j(0); j < k; ++j)
            {
                const unsigned long c((r + j * j * 31 + j) % m);
                S(r, c, hbo_uniform(99, r * 10007 + c, 0.25, 1.0) * ((r + j) % 2 ? 1.0 : -1.0));
            }
        }
        return S;
    }

    // SparseMatrixCSR (la/sparse_matrix_csr-impl.hh:73-135) with csr::blocksize
    // 1, 2, 4 on the Q1 operator and 1, 3 on the skewed matrix; Product and Defect
    // (la/product.hh:208-244, math/defect.hh:385-420) on seeded vectors
    int csr()
    {
        scalars.open((outdir + "/scalars.txt").c_str());
        scalars.precision(17);
        const unsigned long bss[] = {1, 2, 4};
        for (unsigned L(4); L <= 6; L += 2)
            for (unsigned i(0); i < 3; ++i)
            {
                Configuration::instance()->set_value("csr::blocksize", int(bss[i]));
                SparseMatrixCSR<double> A(q1_ell_assembled<double>(L));
                char nm[64];
                snprintf(nm, sizeof nm, "q1_L%u_bs%lu_f64", L, bss[i]);
                put_csr_case(nm, A);
            }
        Configuration::instance()->set_value("csr::blocksize", 1);
        {
            SparseMatrixCSR<float> Af(q1_ell_assembled<float>(6));
            put_csr_case("q1_L6_bs1_f32", Af);
        }
        SparseMatrix<double> S(skewed(5000, 4700));
        for (unsigned long bs(1); bs <= 3; bs += 2)
        {
            Configuration::instance()->set_value("csr::blocksize", int(bs));
            SparseMatrixCSR<double> A(S);
            put_csr_case(bs == 1 ? "skew_bs1_f64" : "skew_bs3_f64", A);
        }
        Configuration::instance()->set_value("csr::blocksize", 1);
        return 0;
    }
}

namespace
{
    // P = 2 D^-1 - D^-1 A D^-1 (two terms of the Neumann series of A^-1 around
    // its diagonal D), on A's pattern
    SparseMatrixELL<double> neumann2(const SparseMatrixELL<double> & A)
    {
        SparseMatrix<double> S(A);
        SparseMatrix<double> P(A.rows(), A.columns());
        for (unsigned long r(0); r < A.rows(); ++r)
            for (typename SparseVector<double>::NonZeroConstElementIterator i(S[r].begin_non_zero_elements()),
                     i_end(S[r].end_non_zero_elements()); i != i_end; ++i)
            {
                const unsigned long c(i.index());
                double v = -(*i) / (S(r, r) * S(c, c));
                if (c == r) v += 2.0 / S(r, r);
                if (v != 0.0) P(r, c, v);
            }
        return SparseMatrixELL<double>(P);
    }

    template <typename Solver_, typename PT_>
    void krylov_case(const std::string & name, SparseMatrixELL<double> & A, PT_ & P, DenseVector<double> & b)
    {
        DenseVector<double> x(A.rows(), 0.0);
        unsigned long used(0);
        Solver_::value(A, P, b, x, 1000ul, used, 1e-8);
        put_vec(name + ".x", x);
        scalars << name << ".iters " << used << "\n" << name << ".relres " << rel_residual(A, b, x) << "\n";
    }

    // CGSolver<tags::CPU, methods::VAR> (math/cg.hh:142-210), BiCGStabSolver<tags::CPU,
    // methods::VAR> (math/bicgstab.hh:60-210) and CGSmoother (math/cg.hh:217-290) on the
    // Q1 operator, b = A u, x0 = 0, eps 1e-8, 1000 iterations at most; P the Jacobi
    // vector 1 / diag(A) or the ELL matrix neumann2(A)
    int krylov()
    {
        scalars.open((outdir + "/scalars.txt").c_str());
        scalars.precision(17);
        for (unsigned L(5); L <= 6; ++L)
        {
            SparseMatrixELL<double> A(q1_ell_assembled<double>(L));
            DenseVector<double> u(uniform<double>(A.rows(), 42)), b(A.rows());
            Product<tags::CPU>::value(b, A, u);
            put_vec(key("kr_L%u.b", L), b);
            DenseVector<double> Pj(A.rows(), 1.0);
            for (unsigned long j(0); j < Pj.size(); ++j) Pj[j] /= A(j, j);
            SparseMatrixELL<double> Pn(neumann2(A));
            put_ell(key("kr_L%u.Pn", L), Pn);
            krylov_case<CGSolver<tags::CPU, methods::VAR> >(key("kr_L%u.cgvar_jac", L), A, Pj, b);
            krylov_case<CGSolver<tags::CPU, methods::VAR> >(key("kr_L%u.cgvar_neu", L), A, Pn, b);
            krylov_case<BiCGStabSolver<tags::CPU, methods::VAR> >(key("kr_L%u.bicg_jac", L), A, Pj, b);
            krylov_case<BiCGStabSolver<tags::CPU, methods::VAR> >(key("kr_L%u.bicg_neu", L), A, Pn, b);
            // CGSmoother: 5 iterations from x0 = 0
            std::vector<DenseVector<double> > tmp;
            for (int i(0); i < 4; ++i) tmp.push_back(DenseVector<double>(A.rows(), 0.0));
            DenseVector<double> xs(A.rows(), 0.0);
            CGSmoother<tags::CPU>::value(A, Pj, b, xs, tmp, 5ul);
            put_vec(key("kr_L%u.cgsmooth_jac.x", L), xs);
        }
        return 0;
    }
}

namespace
{
    // one level of the reference's FEAST banded Q1 test data (math/testdata/<n>.bin:
    // int32 n, then n doubles each of DD LL LD LU DL DU UL UD UU, b, the analytic
    // and the reference solution)
    template <typename DT_>
    void read_bin(const std::string & dir, unsigned long n, BandedMatrixQx<Q1Type, DT_> *& A, DenseVector<DT_> & b)
    {
        std::string path(dir + "/" + stringify(n) + ".bin");
        FILE * f(fopen(path.c_str(), "rb"));
        if (! f) throw InternalError("cannot open " + path);
        int k(0);
        if (1 != fread(&k, sizeof(int), 1, f) || (unsigned long)k != n) throw InternalError("bad header in " + path);
        std::vector<double> v(10 * n);
        if (10 * n != fread(&v[0], sizeof(double), 10 * n, f)) throw InternalError("short file " + path);
        fclose(f);
        // file order DD LL LD LU DL DU UL UD UU; BandedMatrixQx takes LL LD LU DL DD DU UL UD UU
        const unsigned long order[9] = {1, 2, 3, 4, 0, 5, 6, 7, 8};
        DenseVector<DT_> band[9] = {DenseVector<DT_>(n), DenseVector<DT_>(n), DenseVector<DT_>(n), DenseVector<DT_>(n),
                                    DenseVector<DT_>(n), DenseVector<DT_>(n), DenseVector<DT_>(n), DenseVector<DT_>(n),
                                    DenseVector<DT_>(n)};
        for (unsigned long q(0); q < 9; ++q)
            for (unsigned long i(0); i < n; ++i) band[q][i] = DT_(v[order[q] * n + i]);
        for (unsigned long i(0); i < n; ++i) b[i] = DT_(v[9 * n + i]);
        A = new BandedMatrixQx<Q1Type, DT_>(n, band[0], band[1], band[2], band[3], band[4], band[5], band[6], band[7],
                                            band[8]);
    }

    // The setup of math/poisson_mg_double_banded_TEST.cc / poisson_mg_mixed_banded_TEST.cc:
    // MGInfo levels 0..L, the matrices and right-hand sides of levels 1..L from the
    // test data, diags_inverted = ElementInverse(DD) scaled by 0.7 (a double, as the
    // tests pass it), zero x below the finest level.
    template <typename DT_>
    void fill_info(MGInfo<DT_, BandedMatrixQx<Q1Type, DT_> > & info, std::vector<BandedMatrixQx<Q1Type, DT_> *> & keep,
                   const std::string & dir, unsigned long L, unsigned long iters, bool initial_zero,
                   bool convergence_check, bool is_smoother, double tolerance, unsigned long n_pre, double adapt,
                   const unsigned long * mask)
    {
        info.is_smoother = is_smoother;
        for (int i(0); i < 8; ++i) info.macro_border_mask[i] = mask[i];
        info.min_level = 1;
        info.max_level = L;
        info.n_max_iter = iters;
        info.initial_zero = initial_zero;
        info.tolerance = tolerance;
        info.convergence_check = convergence_check;
        info.n_pre_smooth = n_pre;
        info.n_post_smooth = n_pre;
        info.n_max_iter_coarse = 0;
        info.tolerance_coarse = 1e-2;
        info.adapt_correction_factor = adapt;
        for (unsigned long i(0); i <= L; ++i)
        {
            unsigned long size(((1ul << i) + 1) * ((1ul << i) + 1));
            if (i == 0) size = 9;
            DenseVector<DT_> zero(size, DT_(0));
            info.c.push_back(zero.copy());
            info.d.push_back(zero.copy());
            info.x.push_back(zero.copy());
            info.diags_inverted.push_back(zero.copy());
            if (i < info.min_level)
            {
                BandedMatrixQx<Q1Type, DT_> ac(size, zero.copy(), zero.copy(), zero.copy(), zero.copy(), zero.copy(),
                                               zero.copy(), zero.copy(), zero.copy(), zero.copy());
                info.a.push_back(ac);
                info.rhs.push_back(zero.copy());
            }
            else
            {
                BandedMatrixQx<Q1Type, DT_> * A(0);
                DenseVector<DT_> b(size);
                read_bin<DT_>(dir, size, A, b);
                keep.push_back(A);
                info.a.push_back(*A);
                info.rhs.push_back(b);
            }
        }
        for (unsigned long i(0); i <= L; ++i)
        {
            DenseVector<DT_> sdi(info.a[i].band(DD).copy());
            ElementInverse<tags::CPU>::value(sdi);
            Scale<tags::CPU>::value(sdi, 0.7);
            info.diags_inverted[i] = sdi.copy();
        }
    }

    // Multigrid<tags::CPU, tags::CPU, methods::NONE, methods::JAC, methods::CYCLE::V, methods::FIXED>
    template <typename DT_>
    DenseVector<DT_> legacy_mg(const std::string & dir, unsigned long L, unsigned long iters, bool initial_zero,
                               bool convergence_check, bool is_smoother, double tolerance, unsigned long n_pre,
                               double adapt, const unsigned long * mask, const DenseVector<DT_> & x0)
    {
        MGInfo<DT_, BandedMatrixQx<Q1Type, DT_> > info;
        std::vector<BandedMatrixQx<Q1Type, DT_> *> keep;
        fill_info<DT_>(info, keep, dir, L, iters, initial_zero, convergence_check, is_smoother, tolerance, n_pre, adapt,
                       mask);
        DenseVector<DT_> b(info.rhs[L].copy());
        DenseVector<DT_> result(x0.copy());
        Multigrid<tags::CPU, tags::CPU, methods::NONE, methods::JAC, methods::CYCLE::V, methods::FIXED>::value(
            info.a[L], b, result, (unsigned long)11, std::numeric_limits<DT_>::epsilon(), info);
        for (size_t i(0); i < keep.size(); ++i) delete keep[i];
        return result;
    }

    // Multigrid<tags::CPU, tags::CPU, methods::NONE, methods::JAC, methods::CYCLE::V, methods::MIXED>:
    // an FP32 MGInfo under FP64 defect correction with the FP64 finest matrix and b
    DenseVector<double> legacy_mg_mixed(const std::string & dir, unsigned long L, unsigned long iters,
                                        double adapt, const unsigned long * mask, const DenseVector<double> & x0)
    {
        MGInfo<float, BandedMatrixQx<Q1Type, float> > info;
        std::vector<BandedMatrixQx<Q1Type, float> *> keep;
        fill_info<float>(info, keep, dir, L, iters, true, false, false, 1e-8, 2, adapt, mask);
        const unsigned long n(((1ul << L) + 1) * ((1ul << L) + 1));
        BandedMatrixQx<Q1Type, double> * A(0);
        DenseVector<double> b(n);
        read_bin<double>(dir, n, A, b);
        DenseVector<double> result(x0.copy());
        Multigrid<tags::CPU, tags::CPU, methods::NONE, methods::JAC, methods::CYCLE::V, methods::MIXED>::value(
            *A, b, result, (unsigned long)11, std::numeric_limits<double>::epsilon(), info);
        delete A;
        for (size_t i(0); i < keep.size(); ++i) delete keep[i];
        return result;
    }

    int mglegacy(const std::string & dir)
    {
        scalars.open((outdir + "/scalars.txt").c_str());
        scalars.precision(17);
        const unsigned long dirichlet[8] = {2, 2, 2, 2, 2, 2, 2, 2};
        const unsigned long mixed[8] = {2, 1, 2, 1, 2, 2, 1, 2};
        const unsigned long n5(1089);
        // A: the reference test's configuration
        put_vec("lmg_A.x", legacy_mg<double>(dir, 5, 16, true, false, false, 1e-8, 2, 1.0, dirichlet,
                                             DenseVector<double>(n5, 0.0)));
        // B: a nonzero start, V(3,3), damped correction, Neumann edges, the tolerance stop
        put_vec("lmg_B.x", legacy_mg<double>(dir, 5, 30, false, true, false, 1e-6, 3, 0.8, mixed,
                                             uniform<double>(n5, 5)));
        // C: smoother mode, 3 cycles, level 4
        put_vec("lmg_C.x", legacy_mg<double>(dir, 4, 3, true, false, true, 1e-8, 2, 1.0, dirichlet,
                                             DenseVector<double>(289, 0.0)));
        // D: configuration A in single precision
        put_vec("lmg_D.x", legacy_mg<float>(dir, 5, 16, true, false, false, 1e-8, 2, 1.0, dirichlet,
                                            DenseVector<float>(n5, 0.0f)));
        // E: the mixed-precision test's configuration (math/poisson_mg_mixed_banded_TEST.cc)
        put_vec("lmg_E.x", legacy_mg_mixed(dir, 5, 2, 1.0, dirichlet, DenseVector<double>(n5, 0.0)));
        // F: E with the adaptive coarse-grid correction (factor 0) and a nonzero start
        put_vec("lmg_F.x", legacy_mg_mixed(dir, 5, 2, 0.0, dirichlet, uniform<double>(n5, 6)));
        return 0;
    }
}

int main(int argc, char ** argv)
{
    if (argc >= 4 && std::string(argv[1]) == "mglegacy")
    {
        outdir = argv[3];
        return mglegacy(argv[2]);
    }
    if (argc >= 3 && std::string(argv[1]) == "krylov")
    {
        outdir = argv[2];
        return krylov();
    }
    if (argc >= 4 && std::string(argv[1]) == "mgquad") return mgquad(argv[2], argv[3]);
    if (argc >= 3 && std::string(argv[1]) == "csr")
    {
        outdir = argv[2];
        return csr();
    }
    if (argc >= 3 && std::string(argv[1]) == "golden")
    {
        outdir = argv[2];
        return golden();
    }
    if (argc >= 6 && std::string(argv[1]) == "bench")
    {
        if (getenv("HONEI_COARSE_CAP")) coarse_cap = strtoul(getenv("HONEI_COARSE_CAP"), 0, 10);
        std::string which(argv[2]), tag(argv[3]);
        unsigned L(atoi(argv[4])), reps(atoi(argv[5])), warmup(argc > 6 ? atoi(argv[6]) : 0);
        if (reps == 0) reps = 1;
        if (tag == "cpu") return bench<tags::CPU>(which, L, reps, warmup, "cpu");
        if (tag == "generic") return bench<tags::CPU::Generic>(which, L, reps, warmup, "generic");
        if (tag == "sse") return bench<tags::CPU::SSE>(which, L, reps, warmup, "sse");
        if (tag == "mc") return bench<tags::CPU::MultiCore::SSE>(which, L, reps, warmup, "mc");
        fprintf(stderr, "unknown tag '%s'\n", tag.c_str());
        return 2;
    }
    fprintf(stderr, "usage: %s golden <outdir> | bench <cg|mg|ir|spmv> <cpu|generic|sse|mc> <level> <reps>\n", argv[0]);
    return 2;
}
