/*
 * Operators of the B200 tag for a HONEI tree: full specialisations of the tree's
 * tag-dispatched templates over the C ABI of libhonei_b200 (include/honei_b200.h).
 * Each one checks sizes like the tree's own backends (throwing
 * VectorSizeDoesNotMatch before anything runs), locks its containers in the B200
 * memory (the MemoryArbiter uploads on first use and keeps the device copy valid,
 * util/memory_arbiter-impl.hh:410-470), makes one library call on the default
 * stream and unlocks.  The solver templates (CGSolver, RISmoother, MGSolver with its
 * OperatorList cycle, the MG utilities) instantiate unchanged over these.
 *
 *   Product<tags::B200>      y = A x (SparseMatrixELL, la/product.hh:148-206),
 *                            r = a (.) b (la/product.hh:1198-1204)
 *   Defect<tags::B200>       r = rhs - A x (math/defect.hh:357-383)
 *   Sum / Difference / Scale / ScaledSum          (la/sum.hh, la/difference.hh,
 *                            la/scale.hh, la/scaled_sum.hh:73-110)
 *   DotProduct / Norm<vnt_l_two, root>            (la/dot_product.hh:72-89,
 *                            la/norm.hh:290-381)
 *   copy<tags::B200>, fill<tags::B200>: through the MemoryArbiter and the B200
 *                            memory backend (b200_backend.cc)
 *
 * A SparseMatrixELL is converted to the device layout once and kept, keyed by its
 * value array: the arbiter drops the device copy (and so the converted matrix)
 * when the host writes the array or the matrix is destroyed.
 *
 * Reductions: by default the library's tree-ordered dot (fast, deterministic);
 * with b200::set_exact_reductions(true) (or HB2_BINDING_EXACT=1 in the
 * environment) the reference's tags::CPU order, one fma chain, so a solver's
 * iterates match tags::CPU bit for bit (products, defects and updates already do
 * in both modes).
 */
#pragma once
#ifndef HONEI_B200_BINDING_OPERATIONS_HH
#define HONEI_B200_BINDING_OPERATIONS_HH 1

#include "b200_tag.hh"
#include "honei_b200.h"

#include <honei/la/dense_vector.hh>
#include <honei/la/difference.hh>
#include <honei/la/dot_product.hh>
#include <honei/la/norm.hh>
#include <honei/la/product.hh>
#include <honei/la/scale.hh>
#include <honei/la/scaled_sum.hh>
#include <honei/la/sparse_matrix_ell.hh>
#include <honei/la/sum.hh>
#include <honei/math/defect.hh>
#include <honei/util/exception.hh>

namespace honei
{
    namespace b200
    {
        /* a library status to the tree's exceptions */
        void check(int status, const char * what);

        /* the device form of A (created on first use, kept while A's values are) */
        hb2_ell ell(const SparseMatrixELL<float> & a);
        hb2_ell ell(const SparseMatrixELL<double> & a);

        bool exact_reductions();
        void set_exact_reductions(bool exact);

        template <typename DT_> struct DType;
        template <> struct DType<float> { static hb2_dtype value() { return HB2_F32; } };
        template <> struct DType<double> { static hb2_dtype value() { return HB2_F64; } };

        /* a container's device address for the duration of one call */
        template <typename DT_>
        class Locked
        {
            private:
                const DenseVectorContinuousBase<DT_> & _v;
                LockMode _mode;
                void * _dev;

            public:
                Locked(const DenseVectorContinuousBase<DT_> & v, LockMode mode) :
                    _v(v), _mode(mode), _dev(v.lock(mode, tags::B200::memory_value))
                {
                }

                ~Locked()
                {
                    _v.unlock(_mode);
                }

                void * operator() () const
                {
                    return _dev;
                }
        };

        template <typename DT_>
        DT_ dot(const DenseVectorContinuousBase<DT_> & x, const DenseVectorContinuousBase<DT_> & y, int root)
        {
            if (x.size() != y.size())
                throw VectorSizeDoesNotMatch(y.size(), x.size());
            double result(0);
            Locked<DT_> xd(x, lm_read_only), yd(y, lm_read_only);
            if (exact_reductions())
                check(hb2_dot_ordered(DType<DT_>::value(), xd(), yd(), x.size(), root, 0, &result, 0), "DotProduct");
            else if (root)
                check(hb2_norm_l2(DType<DT_>::value(), xd(), x.size(), 1, 0, &result, 0), "Norm");
            else
                check(hb2_dot(DType<DT_>::value(), xd(), yd(), x.size(), 0, &result, 0), "DotProduct");
            return DT_(result);
        }
    }

    template <> struct Product<tags::B200>
    {
        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & y, const SparseMatrixELL<DT_> & a, const DenseVector<DT_> & x)
        {
            if (x.size() != a.columns())
                throw VectorSizeDoesNotMatch(x.size(), a.columns());
            if (y.size() != a.rows())
                throw VectorSizeDoesNotMatch(y.size(), a.rows());
            hb2_ell m(b200::ell(a));
            b200::Locked<DT_> xd(x, lm_read_only), yd(y, lm_write_only);
            b200::check(hb2_product_ell(m, xd(), yd(), 0), "Product");
            return y;
        }

        template <typename DT_>
        static DenseVectorContinuousBase<DT_> & value(DenseVectorContinuousBase<DT_> & r,
                const DenseVectorContinuousBase<DT_> & a, const DenseVectorContinuousBase<DT_> & b)
        {
            if (a.size() != b.size())
                throw VectorSizeDoesNotMatch(b.size(), a.size());
            if (r.size() != a.size())
                throw VectorSizeDoesNotMatch(r.size(), a.size());
            b200::Locked<DT_> ad(a, lm_read_only), bd(b, lm_read_only), rd(r, lm_write_only);
            b200::check(hb2_element_product(b200::DType<DT_>::value(), rd(), ad(), bd(), r.size(), 0), "ElementProduct");
            return r;
        }
    };

    template <> struct Defect<tags::B200>
    {
        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & r, const DenseVector<DT_> & rhs, const SparseMatrixELL<DT_> & a,
                const DenseVector<DT_> & x)
        {
            if (x.size() != a.columns())
                throw VectorSizeDoesNotMatch(x.size(), a.columns());
            if (rhs.size() != a.rows())
                throw VectorSizeDoesNotMatch(rhs.size(), a.rows());
            if (r.size() != a.rows())
                throw VectorSizeDoesNotMatch(r.size(), a.rows());
            hb2_ell m(b200::ell(a));
            b200::Locked<DT_> bd(rhs, lm_read_only), xd(x, lm_read_only), rd(r, lm_write_only);
            b200::check(hb2_defect_ell(m, bd(), xd(), rd(), 0, 0), "Defect");
            return r;
        }
    };

    template <> struct Sum<tags::B200>
    {
        template <typename DT_>
        static DenseVectorContinuousBase<DT_> & value(DenseVectorContinuousBase<DT_> & a,
                const DenseVectorContinuousBase<DT_> & b)
        {
            if (a.size() != b.size())
                throw VectorSizeDoesNotMatch(b.size(), a.size());
            b200::Locked<DT_> bd(b, lm_read_only), ad(a, lm_read_and_write);
            b200::check(hb2_sum(b200::DType<DT_>::value(), ad(), bd(), a.size(), 0), "Sum");
            return a;
        }
    };

    template <> struct Difference<tags::B200>
    {
        template <typename DT_>
        static DenseVectorContinuousBase<DT_> & value(DenseVectorContinuousBase<DT_> & a,
                const DenseVectorContinuousBase<DT_> & b)
        {
            if (a.size() != b.size())
                throw VectorSizeDoesNotMatch(b.size(), a.size());
            b200::Locked<DT_> bd(b, lm_read_only), ad(a, lm_read_and_write);
            b200::check(hb2_difference(b200::DType<DT_>::value(), ad(), bd(), a.size(), 0), "Difference");
            return a;
        }
    };

    template <> struct Scale<tags::B200>
    {
        template <typename DT_>
        static DenseVectorContinuousBase<DT_> & value(DenseVectorContinuousBase<DT_> & x, const DT_ a)
        {
            b200::Locked<DT_> xd(x, lm_read_and_write);
            b200::check(hb2_scale(b200::DType<DT_>::value(), xd(), double(a), x.size(), 0), "Scale");
            return x;
        }
    };

    template <> struct ScaledSum<tags::B200>
    {
        /* x += b y */
        template <typename DT_>
        static DenseVectorContinuousBase<DT_> & value(DenseVectorContinuousBase<DT_> & x,
                const DenseVectorContinuousBase<DT_> & y, const DT_ b)
        {
            if (x.size() != y.size())
                throw VectorSizeDoesNotMatch(y.size(), x.size());
            b200::Locked<DT_> yd(y, lm_read_only), xd(x, lm_read_and_write);
            b200::check(hb2_scaled_sum(b200::DType<DT_>::value(), xd(), yd(), double(b), x.size(), 0), "ScaledSum");
            return x;
        }

        /* r = b y + x */
        template <typename DT_>
        static DenseVectorContinuousBase<DT_> & value(DenseVectorContinuousBase<DT_> & r,
                const DenseVectorContinuousBase<DT_> & x, const DenseVectorContinuousBase<DT_> & y, const DT_ b)
        {
            if (x.size() != y.size())
                throw VectorSizeDoesNotMatch(y.size(), x.size());
            if (r.size() != x.size())
                throw VectorSizeDoesNotMatch(r.size(), x.size());
            b200::Locked<DT_> xd(x, lm_read_only), yd(y, lm_read_only), rd(r, lm_write_only);
            b200::check(hb2_scaled_sum3(b200::DType<DT_>::value(), rd(), xd(), yd(), double(b), r.size(), 0), "ScaledSum");
            return r;
        }
    };

    template <> struct DotProduct<tags::B200>
    {
        template <typename DT_>
        static DT_ value(const DenseVectorContinuousBase<DT_> & x, const DenseVectorContinuousBase<DT_> & y)
        {
            return b200::dot(x, y, 0);
        }
    };

    template <> struct Norm<vnt_l_two, false, tags::B200>
    {
        template <typename DT_>
        static DT_ value(const DenseVectorContinuousBase<DT_> & x)
        {
            return b200::dot(x, x, 0);
        }
    };

    template <> struct Norm<vnt_l_two, true, tags::B200>
    {
        template <typename DT_>
        static DT_ value(const DenseVectorContinuousBase<DT_> & x)
        {
            return b200::dot(x, x, 1);
        }
    };
}

#endif
