/*
 * The B200 tag inside a HONEI tree: the tree's own, unchanged solver templates
 * instantiated with tags::B200 (honei_b200/binding) and with tags::CPU on the same
 * data, compared.
 *
 *   feast   the flow of the tree's MGSolverTestQuad (math/mg_TEST.cc:398-463): its
 *           FEAST Q1 data (A_1..A_6, prol_2..prol_6, rhs_6, init_6, sol_6 in the
 *           directory argv[1]) read by MGUtil::load_data, W-cycle with
 *           CGSolver<Tag, NONE> on the coarsest level, RISmoother, Restriction /
 *           Prolongation<PROLMAT>, MGSolver<Tag, Norm<vnt_l_two, true, Tag> >
 *   cg      CGSolver<Tag, methods::NONE> on A_6 with rhs_6 from zero, to 1e-8
 *   size    Product<tags::B200> with a wrong-sized result throws
 *           VectorSizeDoesNotMatch before anything runs
 *
 * The B200 runs go once with the reference-order reductions (same bits expected)
 * and once with the library's tree-ordered ones (same counts within one and the
 * test's own tolerance against sol_6 expected).  Prints one RESULT line (JSON).
 */
#include "b200_operations.hh"

#include <honei/la/dense_vector.hh>
#include <honei/la/sparse_matrix_ell.hh>
#include <honei/math/cg.hh>
#include <honei/math/matrix_io.hh>
#include <honei/math/mg.hh>
#include <honei/math/prolongation.hh>
#include <honei/math/restriction.hh>
#include <honei/math/ri.hh>
#include <honei/math/vector_io.hh>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace honei;

namespace
{
    struct Run
    {
        std::vector<double> x;
        unsigned long iters, coarse;
    };

    std::vector<double> host(const DenseVector<double> & v)
    {
        v.lock(lm_read_only);
        std::vector<double> out(v.elements(), v.elements() + v.size());
        v.unlock(lm_read_only);
        return out;
    }

    template <typename Tag_>
    Run feast_mg(const std::string & dir)
    {
        const unsigned long max_level(6), min_level(1);
        typedef MGUtil<Tag_, SparseMatrixELL<double>, DenseVector<double>, SparseMatrixELL<double>, DenseVector<double>,
                MatrixIO<io_formats::ELL>, VectorIO<io_formats::EXP>, double> Util;
        MGData<SparseMatrixELL<double>, DenseVector<double>, SparseMatrixELL<double>, DenseVector<double>, double>
            data(Util::load_data(dir, max_level, double(0.7), "jac"));
        Util::configure(data, 100, 100, 4, 4, min_level, double(1e-8));
        OperatorList ol(MGCycleCreation<Tag_, methods::CYCLE::W::STATIC, CGSolver<Tag_, methods::NONE>, RISmoother<Tag_>,
                Restriction<Tag_, methods::PROLMAT>, Prolongation<Tag_, methods::PROLMAT>, double>::value(data));
        MGSolver<Tag_, Norm<vnt_l_two, true, Tag_> >::value(data, ol);
        Run r;
        r.x = host(data.x.at(MGDataIndex::internal_index_A(max_level)));
        r.iters = data.used_iters;
        r.coarse = data.used_iters_coarse;
        return r;
    }

    template <typename Tag_>
    Run cg(const std::string & dir)
    {
        SparseMatrixELL<double> A(MatrixIO<io_formats::ELL>::read_matrix(dir + "A_6.ell", double(0)));
        DenseVector<double> b(VectorIO<io_formats::EXP>::read_vector(dir + "rhs_6", double(0)));
        DenseVector<double> x(b.size(), double(0)), dummy(1);
        Run r;
        CGSolver<Tag_, methods::NONE>::value(A, dummy, b, x, 2000ul, r.iters, 1e-8);
        r.coarse = 0;
        r.x = host(x);
        return r;
    }

    bool same_bits(const Run & a, const Run & b)
    {
        return a.x.size() == b.x.size() && std::memcmp(&a.x[0], &b.x[0], a.x.size() * sizeof(double)) == 0 &&
            a.iters == b.iters && a.coarse == b.coarse;
    }

    double max_diff(const Run & a, const Run & b)
    {
        double m(0);
        for (unsigned long i(0) ; i < a.x.size() && i < b.x.size() ; ++i)
            m = std::max(m, std::fabs(a.x[i] - b.x[i]));
        return m;
    }

    /* the check of math/mg_TEST.cc:445-461: every entry within its eps of sol_6 */
    bool test_tolerance(const Run & r, const std::string & dir)
    {
        DenseVector<double> ref(VectorIO<io_formats::EXP>::read_vector(dir + "sol_6", double(0)));
        const double base_eps(1 / std::pow(10., 1.)), add_eps(base_eps / std::pow(10., 2.));
        const double m((add_eps - base_eps) / double(4)), b(base_eps - double(4) * m);
        const double eps((m * sizeof(double) + b) * double(8));
        for (unsigned long i(0) ; i < ref.size() ; ++i)
            if (! (std::fabs(r.x[i] - ref[i]) <= eps))
                return false;
        return true;
    }
}

int main(int argc, char ** argv)
{
    if (argc < 2)
    {
        std::fprintf(stderr, "usage: %s <directory with the FEAST Q1 data, ending in />\n", argv[0]);
        return 2;
    }
    const std::string dir(argv[1]);
    try
    {
        const Run cpu(feast_mg<tags::CPU>(dir));
        b200::set_exact_reductions(true);
        const Run b_exact(feast_mg<tags::B200>(dir));
        b200::set_exact_reductions(false);
        const Run b_tree(feast_mg<tags::B200>(dir));

        const Run cg_cpu(cg<tags::CPU>(dir));
        b200::set_exact_reductions(true);
        const Run cg_exact(cg<tags::B200>(dir));
        b200::set_exact_reductions(false);
        const Run cg_tree(cg<tags::B200>(dir));

        bool size_throws(false);
        {
            SparseMatrixELL<double> A(MatrixIO<io_formats::ELL>::read_matrix(dir + "A_2.ell", double(0)));
            DenseVector<double> x(A.columns(), double(1)), y(A.rows() + 1, double(0));
            try
            {
                Product<tags::B200>::value(y, A, x);
            }
            catch (VectorSizeDoesNotMatch &)
            {
                size_throws = true;
            }
        }
        std::printf("RESULT {\"feast_cpu_iters\": %lu, \"feast_cpu_coarse\": %lu, \"feast_exact_iters\": %lu, "
                "\"feast_exact_coarse\": %lu, \"feast_exact_same_bits\": %s, \"feast_tree_iters\": %lu, "
                "\"feast_tree_max_diff\": %.3g, \"feast_cpu_test_ok\": %s, \"feast_tree_test_ok\": %s, "
                "\"cg_cpu_iters\": %lu, \"cg_exact_iters\": %lu, \"cg_exact_same_bits\": %s, \"cg_tree_iters\": %lu, "
                "\"cg_tree_max_diff\": %.3g, \"size_check_throws\": %s}\n",
                cpu.iters, cpu.coarse, b_exact.iters, b_exact.coarse, same_bits(cpu, b_exact) ? "true" : "false",
                b_tree.iters, max_diff(cpu, b_tree), test_tolerance(cpu, dir) ? "true" : "false",
                test_tolerance(b_tree, dir) ? "true" : "false", cg_cpu.iters, cg_exact.iters,
                same_bits(cg_cpu, cg_exact) ? "true" : "false", cg_tree.iters, max_diff(cg_cpu, cg_tree),
                size_throws ? "true" : "false");
    }
    catch (std::exception & e)
    {
        std::fprintf(stderr, "binding_test: %s\n", e.what());
        return 1;
    }
    return 0;
}
