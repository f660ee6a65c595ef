/* honei_b200.hh -- HONEI's operator and solver templates for the B200 tag, in C++,
 * on top of the C ABI of honei_b200.h.  Header-only (C++17); link libhonei_b200.so
 * and the CUDA runtime, with which the containers allocate device memory.
 *
 * Names, argument order and meaning follow the reference's templates:
 *   Product<Tag>::value(result, A, x)            la/product.hh:148-206 (SparseMatrixELL),
 *                                                371-403 (BandedMatrixQx<Q1Type>)
 *   Defect<Tag>::value(result, rhs, A, x)        math/defect.hh:357-383 (ELL), 194-198 (Q1)
 *   ScaledSum<Tag>::value(x, y, b)               la/scaled_sum.hh:73-88: x += b y
 *   ScaledSum<Tag>::value(r, x, y, b)            la/scaled_sum.hh:91-110: r = b y + x
 *   Sum / Difference / Scale / ElementProduct    la/sum.hh, la/difference.hh, la/scale.hh,
 *                                                la/product.hh:1198-1204
 *   DotProduct<Tag>::value(x, y)                 la/dot_product.hh:72-89
 *   Norm<vnt_l_two, root, Tag>::value(x)         la/norm.hh:290-305 (squared), 363-381 (root)
 *   RISmoother<Tag>::value(A, P, b, x, temps, max_iters)             math/ri.hh:97-133
 *   CGSolver<Tag, methods::NONE>::value(A, P, b, x, max_iters, used_iters, eps)
 *                                                math/cg.hh:64-135
 *   MGSolver<Tag, Norm<...>>::value(data, b, x)  math/mg.hh:1094-1127 (the V-cycle
 *                                                OperatorList lives inside MGData here)
 *   IRSolver<Outer, Inner, Norm>::value(A, b, x, inner, eps, max_iters, used_iters)
 *                                                math/ir.hh:42-80
 *   Prolongation / Restriction<Tag, NONE|PROLMAT>::value(fine|coarse, coarse|fine, mask, matrix)
 *                                                math/prolongation.hh:42-155, math/restriction.hh:41-185
 *   Transposition<Tag>::value(A)                 math/transposition.hh:36-50
 *   MatrixIO<io_formats::ELL>::read_matrix / write_matrix      math/matrix_io.hh:433-560
 *   SparseMatrixCSR Product / Defect             la/product.hh:208-244, math/defect.hh:385-420
 *   CGSolver<Tag, methods::VAR>, BiCGStabSolver<Tag, methods::VAR>, CGSmoother<Tag>
 *                                                math/cg.hh:142-290, math/bicgstab.hh:60-210
 *   Multigrid<Tag, OuterTag, NONE, JAC, CYCLE::V, FIXED|MIXED>::value(system, b, x,
 *                                                max_levels, conv_rad, info)
 *                                                math/multigrid.hh:781-825, 2252-2394
 * Size mismatches throw VectorSizeDoesNotMatch / MatrixRowsDoNotMatch /
 * MatrixColumnsDoNotMatch before anything is launched (la/vector_error.hh:48,
 * la/matrix_error.hh:46-75); a failing library call throws InternalError with the
 * library's message (util/exception.hh:142), NotFinite for a NaN defect norm.
 *
 * Containers live in device memory and keep the reference's shallow-copy semantics
 * (copies share the array, clone() copies it, la/dense_vector.hh); host data moves
 * through the host-array constructors and to_host().  Every call runs on the CUDA
 * default stream and, where it returns a host value, synchronises it. */
#pragma once

#include <cuda_runtime_api.h>

#include "honei_b200.h"

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace honei_b200
{
    namespace tags
    {
        /* the tag of this backend (honei/util/tags.hh defines the reference's tags) */
        struct B200
        {
        };
    }

    namespace methods
    {
        struct NONE
        {
        };
        struct PROLMAT
        {
        };
        struct VAR
        {
        };
        struct JAC
        {
        };
        struct FIXED
        {
        };
        struct MIXED
        {
        };
        namespace CYCLE
        {
            struct V
            {
            };
        }
    }

    namespace io_formats
    {
        struct ELL
        {
        };
    }

    enum VectorNormType
    {
        vnt_l_two = 2
    };

    // ------------------------------------------------------------------ errors
    class Exception : public std::runtime_error
    {
        public:
            explicit Exception(const std::string & message) : std::runtime_error(message) {}
    };

    class InternalError : public Exception
    {
        public:
            explicit InternalError(const std::string & message) : Exception("Internal error: " + message) {}
    };

    class NotFinite : public InternalError
    {
        public:
            explicit NotFinite(const std::string & message) : InternalError(message) {}
    };

    class VectorSizeDoesNotMatch : public Exception
    {
        public:
            VectorSizeDoesNotMatch(uint64_t size, uint64_t expected) :
                Exception("vector size " + std::to_string(size) + " does not match the expected size " +
                          std::to_string(expected))
            {
            }
    };

    class MatrixRowsDoNotMatch : public Exception
    {
        public:
            MatrixRowsDoNotMatch(uint64_t rows, uint64_t expected) :
                Exception("matrix rows " + std::to_string(rows) + " do not match the expected " +
                          std::to_string(expected))
            {
            }
    };

    class MatrixColumnsDoNotMatch : public Exception
    {
        public:
            MatrixColumnsDoNotMatch(uint64_t columns, uint64_t expected) :
                Exception("matrix columns " + std::to_string(columns) + " do not match the expected " +
                          std::to_string(expected))
            {
            }
    };

    namespace detail
    {
        inline void check(int status, const char * what)
        {
            if (status == HB2_OK) return;
            const std::string message = std::string(what) + ": " + hb2_last_error();
            if (status == HB2_ERR_NOT_FINITE) throw NotFinite(message);
            throw InternalError(message);
        }

        inline void check_cuda(cudaError_t e, const char * what)
        {
            if (e != cudaSuccess) throw InternalError(std::string(what) + ": " + cudaGetErrorString(e));
        }

        inline void check_size(uint64_t size, uint64_t expected)
        {
            if (size != expected) throw VectorSizeDoesNotMatch(size, expected);
        }

        template <typename DT_> struct Dtype;
        template <> struct Dtype<double> { static constexpr hb2_dtype value = HB2_F64; };
        template <> struct Dtype<float> { static constexpr hb2_dtype value = HB2_F32; };

        /* one device allocation, freed with its last owner */
        class DeviceArray
        {
            public:
                explicit DeviceArray(size_t bytes) : _p(nullptr)
                {
                    if (bytes) check_cuda(cudaMalloc(&_p, bytes), "cudaMalloc");
                }
                ~DeviceArray() { if (_p) cudaFree(_p); }
                DeviceArray(const DeviceArray &) = delete;
                DeviceArray & operator=(const DeviceArray &) = delete;
                void * get() const { return _p; }

            private:
                void * _p;
        };
    }

    // ------------------------------------------------------------------ containers
    /* DenseVector<DT_> (la/dense_vector.hh) resident on the device */
    template <typename DT_>
    class DenseVector
    {
        public:
            explicit DenseVector(uint64_t size, DT_ value = DT_(0)) :
                _size(size), _a(std::make_shared<detail::DeviceArray>(size * sizeof(DT_)))
            {
                detail::check(hb2_fill(detail::Dtype<DT_>::value, _a->get(), (double)value, size, nullptr), "fill");
            }

            explicit DenseVector(const std::vector<DT_> & host) :
                _size(host.size()), _a(std::make_shared<detail::DeviceArray>(host.size() * sizeof(DT_)))
            {
                if (_size)
                    detail::check_cuda(cudaMemcpy(_a->get(), host.data(), _size * sizeof(DT_), cudaMemcpyHostToDevice),
                                       "DenseVector upload");
            }

            uint64_t size() const { return _size; }
            DT_ * elements() const { return static_cast<DT_ *>(_a->get()); }

            std::vector<DT_> to_host() const
            {
                std::vector<DT_> h(_size);
                if (_size)
                    detail::check_cuda(cudaMemcpy(h.data(), _a->get(), _size * sizeof(DT_), cudaMemcpyDeviceToHost),
                                       "DenseVector download");
                return h;
            }

            /* an independent copy (DenseVector::copy() of the reference) */
            DenseVector clone() const
            {
                DenseVector c(_size);
                detail::check(hb2_copy(detail::Dtype<DT_>::value, c.elements(), elements(), _size, nullptr), "copy");
                return c;
            }

        private:
            uint64_t _size;
            std::shared_ptr<detail::DeviceArray> _a;
    };

    /* SparseMatrixELL<DT_> (la/sparse_matrix_ell.hh) in the device layout the library
     * chooses; the reference arrays go in through the raw-array constructor
     * (la/sparse_matrix_ell-impl.hh:132-184) and come back through export_arrays(). */
    template <typename DT_>
    class SparseMatrixELL
    {
        public:
            SparseMatrixELL(uint64_t rows, uint64_t columns, uint64_t stride, uint64_t num_cols_per_row,
                            const std::vector<uint64_t> & Aj, const std::vector<DT_> & Ax,
                            const std::vector<uint64_t> & Arl, uint64_t threads = 1)
            {
                hb2_ell h = nullptr;
                detail::check(hb2_ell_create(&h, detail::Dtype<DT_>::value, rows, columns, stride, num_cols_per_row,
                                             threads, Aj.data(), Ax.data(), Arl.data(), 1, nullptr),
                              "SparseMatrixELL");
                _h = std::shared_ptr<hb2_ell_s>(h, [](hb2_ell p) { hb2_ell_destroy(p); });
            }

            /* FillMatrix<Tag, POISSON, DIRICHLET_0> (math/fill_matrix.hh:37-79) of level L,
             * converted to ELL (la/sparse_matrix_ell-impl.hh:75-122), assembled on the device */
            static SparseMatrixELL poisson_q1(unsigned level, double aniso = 1.0)
            {
                hb2_ell h = nullptr;
                detail::check(hb2_ell_create_q1(&h, detail::Dtype<DT_>::value, level, aniso, nullptr), "poisson_q1");
                return SparseMatrixELL(h);
            }

            /* takes ownership of a matrix handle made by the C ABI */
            static SparseMatrixELL adopt(hb2_ell h) { return SparseMatrixELL(h); }

            uint64_t rows() const { info(); return _rows; }
            uint64_t columns() const { info(); return _cols; }
            uint64_t stride() const { info(); return _stride; }
            uint64_t num_cols_per_row() const { info(); return _K; }
            uint64_t threads() const { info(); return _T; }
            hb2_ell handle() const { return _h.get(); }

            void export_arrays(std::vector<uint64_t> & Aj, std::vector<DT_> & Ax, std::vector<uint64_t> & Arl) const
            {
                info();
                Aj.assign(_K * _stride, 0);
                Ax.assign(_K * _stride, DT_(0));
                Arl.assign(_rows, 0);
                detail::check(hb2_ell_export(handle(), Aj.data(), Ax.data(), Arl.data()), "export");
            }

        private:
            explicit SparseMatrixELL(hb2_ell h) : _h(h, [](hb2_ell p) { hb2_ell_destroy(p); }) {}

            void info() const
            {
                uint64_t bytes = 0;
                detail::check(hb2_ell_info(handle(), &_rows, &_cols, &_stride, &_K, &_T, &bytes), "info");
            }

            std::shared_ptr<hb2_ell_s> _h;
            mutable uint64_t _rows = 0, _cols = 0, _stride = 0, _K = 0, _T = 0;
    };

    /* BandedMatrixQx<Q1Type, DT_> (la/banded_matrix_qx.hh): nine bands LL..UU of size n */
    template <typename DT_>
    class BandedMatrixQx
    {
        public:
            /* band-major host array (band b, row i at b * n + i) */
            BandedMatrixQx(uint64_t size, const std::vector<DT_> & bands) : _n(size)
            {
                if (bands.size() != 9 * size) throw VectorSizeDoesNotMatch(bands.size(), 9 * size);
                hb2_q1 h = nullptr;
                detail::check(hb2_q1_create(&h, detail::Dtype<DT_>::value, size, bands.data(), 1, nullptr),
                              "BandedMatrixQx");
                _h = std::shared_ptr<hb2_q1_s>(h, [](hb2_q1 p) { hb2_q1_destroy(p); });
            }

            static BandedMatrixQx poisson_q1(unsigned level, double aniso = 1.0)
            {
                hb2_q1 h = nullptr;
                detail::check(hb2_q1_create_poisson(&h, detail::Dtype<DT_>::value, level, aniso, nullptr),
                              "poisson_q1");
                const uint64_t m = (1ull << level) + 1;
                return BandedMatrixQx(h, m * m);
            }

            uint64_t rows() const { return _n; }
            uint64_t columns() const { return _n; }
            hb2_q1 handle() const { return _h.get(); }

        private:
            BandedMatrixQx(hb2_q1 h, uint64_t n) : _n(n), _h(h, [](hb2_q1 p) { hb2_q1_destroy(p); }) {}

            uint64_t _n;
            std::shared_ptr<hb2_q1_s> _h;
    };

    /* SparseMatrixCSR<DT_> (la/sparse_matrix_csr-impl.hh:40-71): Ar (rows + 1 block offsets),
     * Aj (first column of each block), Ax (blocksize values per block) */
    template <typename DT_>
    class SparseMatrixCSR
    {
        public:
            SparseMatrixCSR(uint64_t rows, uint64_t columns, uint64_t blocksize, const std::vector<uint64_t> & Ar,
                            const std::vector<uint64_t> & Aj, const std::vector<DT_> & Ax)
            {
                if (Ar.size() != rows + 1) throw VectorSizeDoesNotMatch(Ar.size(), rows + 1);
                hb2_csr h = nullptr;
                detail::check(hb2_csr_create(&h, detail::Dtype<DT_>::value, rows, columns, blocksize, Ar.data(),
                                             Aj.data(), Ax.data(), 1, nullptr),
                              "SparseMatrixCSR");
                _h = std::shared_ptr<hb2_csr_s>(h, [](hb2_csr p) { hb2_csr_destroy(p); });
            }

            /* SparseMatrixCSR(SparseMatrix(ELL)) with csr::blocksize */
            static SparseMatrixCSR from_ell(const SparseMatrixELL<DT_> & A, uint64_t blocksize = 1)
            {
                hb2_csr h = nullptr;
                detail::check(hb2_csr_from_ell(&h, A.handle(), blocksize, nullptr), "SparseMatrixCSR");
                return SparseMatrixCSR(h);
            }

            uint64_t rows() const { uint64_t r, c, bs, nb, bytes; info(r, c, bs, nb, bytes); return r; }
            uint64_t columns() const { uint64_t r, c, bs, nb, bytes; info(r, c, bs, nb, bytes); return c; }
            uint64_t blocksize() const { uint64_t r, c, bs, nb, bytes; info(r, c, bs, nb, bytes); return bs; }
            hb2_csr handle() const { return _h.get(); }

            void export_arrays(std::vector<uint64_t> & Ar, std::vector<uint64_t> & Aj, std::vector<DT_> & Ax) const
            {
                uint64_t r, c, bs, nb, bytes;
                info(r, c, bs, nb, bytes);
                Ar.assign(r + 1, 0);
                Aj.assign(nb, 0);
                Ax.assign(nb * bs, DT_(0));
                detail::check(hb2_csr_export(handle(), Ar.data(), Aj.data(), Ax.data()), "export");
            }

        private:
            explicit SparseMatrixCSR(hb2_csr h) : _h(h, [](hb2_csr p) { hb2_csr_destroy(p); }) {}

            void info(uint64_t & r, uint64_t & c, uint64_t & bs, uint64_t & nb, uint64_t & bytes) const
            {
                detail::check(hb2_csr_info(handle(), &r, &c, &bs, &nb, &bytes), "info");
            }

            std::shared_ptr<hb2_csr_s> _h;
    };

    /* ProlongationMatrix (level fine_level - 1 -> fine_level, identity index maps,
     * math/prolongation_matrix.hh:44-100) and its Transposition, the restriction */
    template <typename DT_>
    std::pair<SparseMatrixELL<DT_>, SparseMatrixELL<DT_>> q1_transfer(unsigned fine_level);

    // ------------------------------------------------------------------ operators
    template <typename Tag_> struct Product;
    template <typename Tag_> struct Defect;
    template <typename Tag_> struct ScaledSum;
    template <typename Tag_> struct Sum;
    template <typename Tag_> struct Difference;
    template <typename Tag_> struct Scale;
    template <typename Tag_> struct ElementProduct;
    template <typename Tag_> struct DotProduct;
    template <VectorNormType NormType_, bool root_, typename Tag_> struct Norm;

    template <>
    struct Product<tags::B200>
    {
        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & result, const SparseMatrixELL<DT_> & a,
                                        const DenseVector<DT_> & b)
        {
            detail::check_size(b.size(), a.columns());
            detail::check_size(result.size(), a.rows());
            detail::check(hb2_product_ell(a.handle(), b.elements(), result.elements(), nullptr), "Product (ELL)");
            return result;
        }

        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & result, const BandedMatrixQx<DT_> & a,
                                        const DenseVector<DT_> & b)
        {
            detail::check_size(b.size(), a.columns());
            detail::check_size(result.size(), a.rows());
            detail::check(hb2_product_q1(a.handle(), b.elements(), result.elements(), nullptr), "Product (Q1)");
            return result;
        }

        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & result, const SparseMatrixCSR<DT_> & a,
                                        const DenseVector<DT_> & b)
        {
            detail::check_size(b.size(), a.columns());
            detail::check_size(result.size(), a.rows());
            detail::check(hb2_product_csr(a.handle(), b.elements(), result.elements(), nullptr), "Product (CSR)");
            return result;
        }
    };

    template <>
    struct Defect<tags::B200>
    {
        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & result, const DenseVector<DT_> & right_hand_side,
                                        const SparseMatrixELL<DT_> & system, const DenseVector<DT_> & x)
        {
            detail::check_size(x.size(), system.columns());
            if (right_hand_side.size() != system.rows())
                throw MatrixRowsDoNotMatch(system.rows(), right_hand_side.size());
            detail::check_size(result.size(), system.rows());
            detail::check(hb2_defect_ell(system.handle(), right_hand_side.elements(), x.elements(), result.elements(),
                                         nullptr, nullptr),
                          "Defect (ELL)");
            return result;
        }

        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & result, const DenseVector<DT_> & right_hand_side,
                                        const BandedMatrixQx<DT_> & system, const DenseVector<DT_> & x)
        {
            detail::check_size(x.size(), system.columns());
            if (right_hand_side.size() != system.rows())
                throw MatrixRowsDoNotMatch(system.rows(), right_hand_side.size());
            detail::check_size(result.size(), system.rows());
            detail::check(hb2_defect_q1(system.handle(), right_hand_side.elements(), x.elements(), result.elements(),
                                        nullptr),
                          "Defect (Q1)");
            return result;
        }

        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & result, const DenseVector<DT_> & right_hand_side,
                                        const SparseMatrixCSR<DT_> & system, const DenseVector<DT_> & x)
        {
            detail::check_size(x.size(), system.columns());
            if (right_hand_side.size() != system.rows())
                throw MatrixRowsDoNotMatch(system.rows(), right_hand_side.size());
            detail::check_size(result.size(), system.rows());
            detail::check(hb2_defect_csr(system.handle(), right_hand_side.elements(), x.elements(), result.elements(),
                                         nullptr),
                          "Defect (CSR)");
            return result;
        }
    };

    template <>
    struct ScaledSum<tags::B200>
    {
        /* x += b y */
        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & x, const DenseVector<DT_> & y, DT_ b)
        {
            detail::check_size(y.size(), x.size());
            detail::check(hb2_scaled_sum(detail::Dtype<DT_>::value, x.elements(), y.elements(), (double)b, x.size(),
                                         nullptr),
                          "ScaledSum");
            return x;
        }

        /* result = b y + x */
        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & result, const DenseVector<DT_> & x,
                                        const DenseVector<DT_> & y, DT_ b)
        {
            detail::check_size(x.size(), result.size());
            detail::check_size(y.size(), result.size());
            detail::check(hb2_scaled_sum3(detail::Dtype<DT_>::value, result.elements(), x.elements(), y.elements(),
                                          (double)b, result.size(), nullptr),
                          "ScaledSum");
            return result;
        }
    };

    template <>
    struct Sum<tags::B200>
    {
        /* x += y */
        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & x, const DenseVector<DT_> & y)
        {
            detail::check_size(y.size(), x.size());
            detail::check(hb2_sum(detail::Dtype<DT_>::value, x.elements(), y.elements(), x.size(), nullptr), "Sum");
            return x;
        }
    };

    template <>
    struct Difference<tags::B200>
    {
        /* x -= y */
        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & x, const DenseVector<DT_> & y)
        {
            detail::check_size(y.size(), x.size());
            detail::check(hb2_difference(detail::Dtype<DT_>::value, x.elements(), y.elements(), x.size(), nullptr),
                          "Difference");
            return x;
        }
    };

    template <>
    struct Scale<tags::B200>
    {
        /* x *= a */
        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & x, DT_ a)
        {
            detail::check(hb2_scale(detail::Dtype<DT_>::value, x.elements(), (double)a, x.size(), nullptr), "Scale");
            return x;
        }
    };

    template <>
    struct ElementProduct<tags::B200>
    {
        /* result = a (.) b */
        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & result, const DenseVector<DT_> & a,
                                        const DenseVector<DT_> & b)
        {
            detail::check_size(a.size(), result.size());
            detail::check_size(b.size(), result.size());
            detail::check(hb2_element_product(detail::Dtype<DT_>::value, result.elements(), a.elements(),
                                              b.elements(), result.size(), nullptr),
                          "ElementProduct");
            return result;
        }
    };

    template <>
    struct DotProduct<tags::B200>
    {
        template <typename DT_>
        static DT_ value(const DenseVector<DT_> & x, const DenseVector<DT_> & y)
        {
            detail::check_size(y.size(), x.size());
            double r = 0.0;
            detail::check(hb2_dot(detail::Dtype<DT_>::value, x.elements(), y.elements(), x.size(), nullptr, &r,
                                  nullptr),
                          "DotProduct");
            return (DT_)r;
        }
    };

    template <bool root_>
    struct Norm<vnt_l_two, root_, tags::B200>
    {
        template <typename DT_>
        static DT_ value(const DenseVector<DT_> & x)
        {
            double r = 0.0;
            detail::check(hb2_norm_l2(detail::Dtype<DT_>::value, x.elements(), x.size(), root_ ? 1 : 0, nullptr, &r,
                                      nullptr),
                          "Norm");
            return (DT_)r;
        }
    };

    // ------------------------------------------------------------------ solvers
    template <typename Tag_> struct RISmoother;
    template <typename Tag_, typename Method_> struct CGSolver;
    template <typename Tag_, typename NormType_> struct MGSolver;
    template <typename OuterTag_, typename InnerTag_, typename NormType_> struct IRSolver;

    template <>
    struct RISmoother<tags::B200>
    {
        /* PreconFill "jac" (math/mg.hh:266-273): P = omega / diag(A) */
        template <typename DT_>
        static DenseVector<DT_> jacobi_precon(const SparseMatrixELL<DT_> & A, double omega = 0.7)
        {
            DenseVector<DT_> P(A.rows());
            detail::check(hb2_jacobi_precon(A.handle(), omega, P.elements(), nullptr), "PreconFill");
            return P;
        }

        /* max_iters sweeps x += P (.) (b - A x); temp_vecs[0] (if given) is the
         * scratch vector of the sweeps */
        template <typename DT_>
        static void value(const SparseMatrixELL<DT_> & A, const DenseVector<DT_> & P, const DenseVector<DT_> & b,
                          DenseVector<DT_> & x, std::vector<DenseVector<DT_>> & temp_vecs, uint64_t max_iters)
        {
            detail::check_size(x.size(), A.columns());
            detail::check_size(b.size(), A.rows());
            detail::check_size(P.size(), A.rows());
            DenseVector<DT_> tmp = temp_vecs.empty() ? DenseVector<DT_>(x.size()) : temp_vecs[0];
            detail::check_size(tmp.size(), x.size());
            detail::check(hb2_jacobi_ell(A.handle(), P.elements(), b.elements(), x.elements(), tmp.elements(),
                                         max_iters, nullptr),
                          "RISmoother");
        }
    };

    template <>
    struct CGSolver<tags::B200, methods::NONE>
    {
        /* P is unused, as in the reference's methods::NONE solver */
        template <typename DT_, typename PreconContType_>
        static DenseVector<DT_> & value(const SparseMatrixELL<DT_> & A, const PreconContType_ &,
                                        const DenseVector<DT_> & b, DenseVector<DT_> & x, uint64_t max_iters,
                                        uint64_t & used_iters, DT_ eps_relative = DT_(1e-8))
        {
            detail::check_size(b.size(), A.rows());
            detail::check_size(x.size(), A.columns());
            double defect = 0.0;
            detail::check(hb2_cg_solve(A.handle(), b.elements(), x.elements(), max_iters, (double)eps_relative,
                                       &used_iters, &defect, nullptr),
                          "CGSolver");
            return x;
        }
    };

    /* MG parameters of the reference's Poisson solves (V(4,4), omega 0.7, coarse CG in
     * the reference's dot order) */
    inline hb2_mg_params mg_params(double eps = 1e-10, uint64_t max_iters = 100, uint64_t max_iters_coarse = 100)
    {
        hb2_mg_params p;
        p.n_pre_smooth = 4;
        p.n_post_smooth = 4;
        p.max_iters = max_iters;
        p.max_iters_coarse = max_iters_coarse;
        p.eps_relative = eps;
        p.coarse_eps = eps;
        p.omega = 0.7;
        p.coarse_exact = 1;
        p.no_fused_levels = 0;
        p.coarse_fp64 = 0;
        p.cycle = 0;
        return p;
    }

    /* MGData (math/mg.hh:57-240) of a Q1 Poisson hierarchy with its V-cycle, resident
     * on the device; the solver statistics of the last solve are kept here */
    template <typename DT_>
    class MGData
    {
        public:
            static MGData poisson_q1(unsigned min_level, unsigned max_level, const hb2_mg_params & params,
                                     double aniso = 1.0)
            {
                hb2_mg h = nullptr;
                detail::check(hb2_mg_create_q1(&h, detail::Dtype<DT_>::value, min_level, max_level, aniso, &params,
                                               nullptr),
                              "MGData");
                const uint64_t m = (1ull << max_level) + 1;
                return MGData(h, m * m);
            }

            uint64_t size() const { return _n; }
            hb2_mg handle() const { return _h.get(); }

            uint64_t used_iters = 0, used_iters_coarse = 0;
            double rnorm_initial = 0.0, rnorm_current = 0.0;

        private:
            MGData(hb2_mg h, uint64_t n) : _n(n), _h(h, [](hb2_mg p) { hb2_mg_destroy(p); }) {}

            uint64_t _n;
            std::shared_ptr<hb2_mg_s> _h;
    };

    template <bool root_>
    struct MGSolver<tags::B200, Norm<vnt_l_two, root_, tags::B200>>
    {
        template <typename DT_>
        static void value(MGData<DT_> & data, const DenseVector<DT_> & b, DenseVector<DT_> & x)
        {
            detail::check_size(b.size(), data.size());
            detail::check_size(x.size(), data.size());
            double stats[4] = {0, 0, 0, 0};
            const int st = hb2_mg_solve(data.handle(), b.elements(), x.elements(), stats, nullptr);
            // the statistics are filled also when the solve ends on a NaN defect norm
            data.used_iters = (uint64_t)stats[0];
            data.rnorm_initial = stats[1];
            data.rnorm_current = stats[2];
            data.used_iters_coarse = (uint64_t)stats[3];
            detail::check(st, "MGSolver");
        }
    };

    template <bool root_>
    struct IRSolver<tags::B200, tags::B200, Norm<vnt_l_two, root_, tags::B200>>
    {
        /* FP64 outer defect, update and norm around the inner MG solve of `inner`
         * (an FP32 hierarchy for mixed precision) */
        template <typename InnerDT_>
        static void value(const SparseMatrixELL<double> & A, const DenseVector<double> & b, DenseVector<double> & x,
                          MGData<InnerDT_> & inner, double eps, uint64_t max_iters, uint64_t & used_iters)
        {
            detail::check_size(b.size(), A.rows());
            detail::check_size(x.size(), A.columns());
            detail::check_size(inner.size(), A.rows());
            double stats[4] = {0, 0, 0, 0};
            const int st = hb2_ir_solve(A.handle(), inner.handle(), b.elements(), x.elements(), eps, max_iters, 0,
                                        stats, nullptr);
            used_iters = (uint64_t)stats[0];
            detail::check(st, "IRSolver");
        }
    };

    // ------------------------------------------------------------------ grid transfer
    template <typename DT_>
    std::pair<SparseMatrixELL<DT_>, SparseMatrixELL<DT_>> q1_transfer(unsigned fine_level)
    {
        hb2_ell p = nullptr, r = nullptr;
        detail::check(hb2_ell_create_transfer(&p, &r, detail::Dtype<DT_>::value, fine_level, nullptr), "q1_transfer");
        return std::make_pair(SparseMatrixELL<DT_>::adopt(p), SparseMatrixELL<DT_>::adopt(r));
    }

    /* the 8 boundary entries of a macro (edges and corners): 2 = Dirichlet, 1 = Neumann */
    inline std::vector<uint64_t> all_dirichlet() { return std::vector<uint64_t>(8, 2); }

    template <typename Tag_, typename Method_> struct Prolongation;
    template <typename Tag_, typename Method_> struct Restriction;

    template <>
    struct Prolongation<tags::B200, methods::NONE>
    {
        /* matrix-free bilinear prolongation (level sizes (2^l + 1)^2) and the mask's
         * Dirichlet boundaries; the matrix argument is unused as in the reference */
        template <typename DT_, typename MatrixType_>
        static DenseVector<DT_> & value(DenseVector<DT_> & fine, const DenseVector<DT_> & coarse,
                                        const std::vector<uint64_t> & mask, const MatrixType_ &)
        {
            detail::check_size(mask.size(), 8);
            detail::check(hb2_prolongation(detail::Dtype<DT_>::value, fine.elements(), fine.size(), coarse.elements(),
                                           coarse.size(), mask.data(), nullptr),
                          "Prolongation");
            return fine;
        }
    };

    template <>
    struct Prolongation<tags::B200, methods::PROLMAT>
    {
        /* fine = prolmat coarse; the mask is unused as in the reference */
        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & fine, const DenseVector<DT_> & coarse,
                                        const std::vector<uint64_t> &, const SparseMatrixELL<DT_> & prolmat)
        {
            return Product<tags::B200>::value(fine, prolmat, coarse);
        }
    };

    template <>
    struct Restriction<tags::B200, methods::NONE>
    {
        template <typename DT_, typename MatrixType_>
        static DenseVector<DT_> & value(DenseVector<DT_> & coarse, const DenseVector<DT_> & fine,
                                        const std::vector<uint64_t> & mask, const MatrixType_ &)
        {
            detail::check_size(mask.size(), 8);
            detail::check(hb2_restriction(detail::Dtype<DT_>::value, coarse.elements(), coarse.size(), fine.elements(),
                                          fine.size(), mask.data(), nullptr),
                          "Restriction");
            return coarse;
        }
    };

    template <>
    struct Restriction<tags::B200, methods::PROLMAT>
    {
        template <typename DT_>
        static DenseVector<DT_> & value(DenseVector<DT_> & coarse, const DenseVector<DT_> & fine,
                                        const std::vector<uint64_t> &, const SparseMatrixELL<DT_> & resmat)
        {
            return Product<tags::B200>::value(coarse, resmat, fine);
        }
    };

    template <typename Tag_> struct Transposition;

    template <>
    struct Transposition<tags::B200>
    {
        template <typename DT_>
        static SparseMatrixELL<DT_> value(const SparseMatrixELL<DT_> & a)
        {
            hb2_ell h = nullptr;
            detail::check(hb2_ell_transpose(&h, a.handle(), nullptr), "Transposition");
            return SparseMatrixELL<DT_>::adopt(h);
        }
    };

    // ------------------------------------------------------------------ files
    template <typename Format_> struct MatrixIO;

    template <>
    struct MatrixIO<io_formats::ELL>
    {
        /* the reference's binary ELL file, values rounded to DT_ */
        template <typename DT_>
        static SparseMatrixELL<DT_> read_matrix(const std::string & input, DT_)
        {
            hb2_ell h = nullptr;
            detail::check(hb2_ell_read(&h, input.c_str(), detail::Dtype<DT_>::value, nullptr), "MatrixIO::read_matrix");
            return SparseMatrixELL<DT_>::adopt(h);
        }

        static void write_matrix(const std::string & output, const SparseMatrixELL<double> & smatrix)
        {
            detail::check(hb2_ell_write(smatrix.handle(), output.c_str()), "MatrixIO::write_matrix");
        }
    };

    // ------------------------------------------------------------------ Krylov solvers (FP64)
    template <typename Tag_, typename Method_> struct BiCGStabSolver;
    template <typename Tag_> struct CGSmoother;

    namespace detail
    {
        /* one solve of a hb2_krylov handle built for (A, P); P an element-wise vector or an ELL matrix */
        inline void krylov(int method, const SparseMatrixELL<double> & A, hb2_ell Pm, const double * Pd,
                           const DenseVector<double> & b, DenseVector<double> & x, uint64_t max_iters,
                           double eps_relative, uint64_t & used_iters, const char * what)
        {
            check_size(b.size(), A.rows());
            check_size(x.size(), A.columns());
            hb2_krylov K = nullptr;
            check(hb2_krylov_create(&K, method, A.handle(), Pm, Pd, max_iters, eps_relative, nullptr), what);
            std::unique_ptr<hb2_krylov_s, int (*)(hb2_krylov)> keep(K, hb2_krylov_destroy);
            double defect = 0.0;
            check(hb2_krylov_solve(K, b.elements(), x.elements(), &used_iters, &defect, nullptr), what);
        }
    }

    template <>
    struct CGSolver<tags::B200, methods::VAR>
    {
        /* P (.) r as the preconditioner */
        static DenseVector<double> & value(const SparseMatrixELL<double> & A, const DenseVector<double> & P,
                                           const DenseVector<double> & b, DenseVector<double> & x,
                                           uint64_t max_iters, uint64_t & used_iters, double eps_relative = 1e-8)
        {
            detail::check_size(P.size(), A.rows());
            detail::krylov(HB2_CG_VAR, A, nullptr, P.elements(), b, x, max_iters, eps_relative, used_iters,
                           "CGSolver<VAR>");
            return x;
        }

        /* P r (an ELL matrix, e.g. an SPAI) as the preconditioner */
        static DenseVector<double> & value(const SparseMatrixELL<double> & A, const SparseMatrixELL<double> & P,
                                           const DenseVector<double> & b, DenseVector<double> & x,
                                           uint64_t max_iters, uint64_t & used_iters, double eps_relative = 1e-8)
        {
            if (P.rows() != A.rows()) throw MatrixRowsDoNotMatch(P.rows(), A.rows());
            detail::krylov(HB2_CG_VAR, A, P.handle(), nullptr, b, x, max_iters, eps_relative, used_iters,
                           "CGSolver<VAR>");
            return x;
        }
    };

    template <>
    struct BiCGStabSolver<tags::B200, methods::VAR>
    {
        /* used_iters as the reference counts them (iterations + 1) */
        static DenseVector<double> & value(const SparseMatrixELL<double> & A, const DenseVector<double> & P,
                                           const DenseVector<double> & b, DenseVector<double> & x,
                                           uint64_t max_iters, uint64_t & used_iters, double eps_relative = 1e-8)
        {
            detail::check_size(P.size(), A.rows());
            detail::krylov(HB2_BICGSTAB_VAR, A, nullptr, P.elements(), b, x, max_iters, eps_relative, used_iters,
                           "BiCGStabSolver<VAR>");
            return x;
        }
    };

    template <>
    struct CGSmoother<tags::B200>
    {
        /* exactly max_iters preconditioned CG steps from x; temp_vecs are unused (the
         * solver keeps its vectors on the device) */
        static DenseVector<double> & value(const SparseMatrixELL<double> & A, const DenseVector<double> & P,
                                           const DenseVector<double> & b, DenseVector<double> & x,
                                           std::vector<DenseVector<double>> &, uint64_t max_iters)
        {
            detail::check_size(P.size(), A.rows());
            uint64_t used = 0;
            detail::krylov(HB2_CG_SMOOTHER, A, nullptr, P.elements(), b, x, max_iters, 0.0, used, "CGSmoother");
            return x;
        }
    };

    // ------------------------------------------------------------------ legacy banded multigrid
    /* MGInfo's configuration (math/multigrid.hh:65-149), defaults of the reference's
     * banded tests */
    inline hb2_lmg_params mg_info_params(uint64_t n_max_iter = 16, bool initial_zero = true, double tolerance = 1e-8,
                                         uint64_t n_pre_smooth = 2)
    {
        hb2_lmg_params p;
        p.n_max_iter = n_max_iter;
        p.initial_zero = initial_zero ? 1 : 0;
        p.convergence_check = 0;
        p.is_smoother = 0;
        p.tolerance = tolerance;
        p.n_pre_smooth = n_pre_smooth;
        p.adapt_correction_factor = 1.0;
        p.omega = 0.7;
        for (int i = 0; i < 8; ++i) p.macro_border_mask[i] = 2;
        p.adaptive = 0;
        return p;
    }

    /* MGInfo with its levels' banded operators (coarsest first, levels min_level ..),
     * resident on the device with the solver's graph; cycles / defect of the last solve */
    template <typename DT_>
    class MGInfo
    {
        public:
            MGInfo(unsigned min_level, const std::vector<BandedMatrixQx<DT_>> & a,
                   const hb2_lmg_params & params = mg_info_params()) :
                _a(a), _n(a.empty() ? 0 : a.back().rows())
            {
                std::vector<hb2_q1> h;
                for (const auto & m : a) h.push_back(m.handle());
                hb2_lmg g = nullptr;
                detail::check(hb2_lmg_create(&g, min_level, min_level + (unsigned)a.size() - 1, h.data(), &params,
                                             nullptr),
                              "MGInfo");
                _h = std::shared_ptr<hb2_lmg_s>(g, [](hb2_lmg p) { hb2_lmg_destroy(p); });
            }

            uint64_t size() const { return _n; }
            hb2_lmg handle() const { return _h.get(); }

            uint64_t cycles = 0, outer_steps = 0;
            double defect = 0.0;

        private:
            std::vector<BandedMatrixQx<DT_>> _a;
            uint64_t _n;
            std::shared_ptr<hb2_lmg_s> _h;
    };

    template <typename Tag_, typename OuterTag_, typename ProlType_, typename SmootherType_, typename CycleType_,
              typename Mode_>
    struct Multigrid;

    template <>
    struct Multigrid<tags::B200, tags::B200, methods::NONE, methods::JAC, methods::CYCLE::V, methods::FIXED>
    {
        /* x: initial guess in, result out; max_levels and conv_rad are unused as in the
         * reference (the levels are the info's) */
        template <typename DT_>
        static void value(const BandedMatrixQx<DT_> & system, const DenseVector<DT_> & right_hand_side,
                          DenseVector<DT_> & x, unsigned long, DT_, MGInfo<DT_> & info)
        {
            detail::check_size(system.rows(), info.size());
            detail::check_size(right_hand_side.size(), info.size());
            detail::check_size(x.size(), info.size());
            uint64_t cycles = 0;
            double defect = 0.0;
            detail::check(hb2_lmg_solve(info.handle(), right_hand_side.elements(), x.elements(), &cycles, &defect,
                                        nullptr),
                          "Multigrid<FIXED>");
            info.cycles = cycles;
            info.defect = defect;
        }
    };

    template <>
    struct Multigrid<tags::B200, tags::B200, methods::NONE, methods::JAC, methods::CYCLE::V, methods::MIXED>
    {
        /* FP64 defect correction around the FP32 hierarchy of info (the reference has no
         * cap on the outer steps; max_outer bounds them and NotFinite reports reaching it) */
        static void value(const BandedMatrixQx<double> & system, const DenseVector<double> & right_hand_side,
                          DenseVector<double> & x, unsigned long, double, MGInfo<float> & info,
                          uint64_t max_outer = 1000)
        {
            detail::check_size(system.rows(), info.size());
            detail::check_size(right_hand_side.size(), info.size());
            detail::check_size(x.size(), info.size());
            uint64_t outer = 0, inner = 0;
            double defect = 0.0;
            const int st = hb2_lmg_solve_mixed(info.handle(), system.handle(), right_hand_side.elements(),
                                               x.elements(), max_outer, &outer, &inner, &defect, nullptr);
            info.outer_steps = outer;
            info.cycles = inner;
            info.defect = defect;
            detail::check(st, "Multigrid<MIXED>");
        }
    };
}
