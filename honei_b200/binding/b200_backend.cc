/*
 * The B200 memory backend and the glue of the operator shims (b200_operations.hh)
 * for a HONEI tree: device memory for containers locked with
 * tags::B200::memory_value, following the tree's backend interface
 * (util/memory_backend.hh) and its registration (the pattern of
 * backends/cuda/memory_backend.cc:670).  The MemoryArbiter decides when data
 * moves (util/memory_arbiter-impl.hh:410-470); this backend only moves bytes and
 * keeps the device copy of each memory id.
 *
 * A SparseMatrixELL's value array is registered here too, but holds the library's
 * converted matrix (b200::ell) instead of a raw copy: when the arbiter drops the
 * device copy (the host wrote the array, or it was destroyed), the converted matrix
 * goes with it.
 */
#include "b200_operations.hh"

#include <honei/util/instantiation_policy-impl.hh>
#include <honei/util/memory_arbiter.hh>
#include <honei/util/memory_backend.hh>

#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <map>
#include <string>

namespace honei
{
    const std::string tags::B200::name = "b200";

    template <> class MemoryBackend<tags::B200> :
        public MemoryBackendBase,
        public InstantiationPolicy<MemoryBackend<tags::B200>, Singleton>
    {
        private:
            std::map<void *, void *> _dev;        // memory id -> device copy
            std::map<void *, hb2_ell> _matrix;    // value-array memory id -> converted matrix

            static void cuda(cudaError_t e, const char * what)
            {
                if (e != cudaSuccess)
                    throw InternalError(std::string("B200 memory backend: ") + what + ": " + cudaGetErrorString(e));
            }

            void * device(void * memid)
            {
                std::map<void *, void *>::iterator i(_dev.find(memid));
                if (i == _dev.end())
                    throw InternalError("B200 memory backend: no device copy of this memory id");
                return i->second;
            }

        public:
            virtual ~MemoryBackend()
            {
            }

            virtual void * upload(void * memid, void * address, unsigned long bytes)
            {
                if (_matrix.count(memid))
                    return address;          // held as the converted matrix
                std::map<void *, void *>::iterator i(_dev.find(memid));
                if (i != _dev.end())
                    return i->second;        // still valid: the arbiter frees stale copies first
                void * d(alloc(memid, address, bytes));
                cuda(cudaMemcpy(d, address, bytes, cudaMemcpyHostToDevice), "upload");
                return d;
            }

            virtual void download(void * memid, void * address, unsigned long bytes)
            {
                if (_matrix.count(memid))
                    return;                  // the host values were never changed on the device
                cuda(cudaMemcpy(address, device(memid), bytes, cudaMemcpyDeviceToHost), "download");
            }

            virtual void * alloc(void * memid, void * /*address*/, unsigned long bytes)
            {
                std::map<void *, void *>::iterator i(_dev.find(memid));
                if (i != _dev.end())
                    return i->second;
                void * d(0);
                cuda(cudaMalloc(&d, bytes ? bytes : 16), "alloc");
                _dev[memid] = d;
                return d;
            }

            virtual void free(void * memid)
            {
                std::map<void *, hb2_ell>::iterator m(_matrix.find(memid));
                if (m != _matrix.end())
                {
                    hb2_ell_destroy(m->second);
                    _matrix.erase(m);
                }
                std::map<void *, void *>::iterator i(_dev.find(memid));
                if (i != _dev.end())
                {
                    cudaFree(i->second);
                    _dev.erase(i);
                }
            }

            virtual void copy(void * src_id, void * /*src_address*/, void * dest_id, void * /*dest_address*/,
                    unsigned long bytes)
            {
                cuda(cudaMemcpy(device(dest_id), device(src_id), bytes, cudaMemcpyDeviceToDevice), "copy");
            }

            virtual void convert_float_double(void * src_id, void * /*src_address*/, void * dest_id,
                    void * /*dest_address*/, unsigned long bytes)
            {
                b200::check(hb2_convert(HB2_F64, device(dest_id), HB2_F32, device(src_id), bytes / sizeof(float), 0),
                        "convert");
            }

            virtual void convert_double_float(void * src_id, void * /*src_address*/, void * dest_id,
                    void * /*dest_address*/, unsigned long bytes)
            {
                b200::check(hb2_convert(HB2_F32, device(dest_id), HB2_F64, device(src_id), bytes / sizeof(double), 0),
                        "convert");
            }

            virtual void fill(void * memid, void * /*address*/, unsigned long bytes, float proto)
            {
                b200::check(hb2_fill(HB2_F32, device(memid), proto, bytes / sizeof(float), 0), "fill");
            }

            virtual void fill(void * memid, void * /*address*/, unsigned long bytes, double proto)
            {
                b200::check(hb2_fill(HB2_F64, device(memid), proto, bytes / sizeof(double), 0), "fill");
            }

            virtual bool knows(void * memid, void * /*address*/)
            {
                return _dev.count(memid) != 0 || _matrix.count(memid) != 0;
            }

            hb2_ell matrix(void * memid)
            {
                std::map<void *, hb2_ell>::iterator m(_matrix.find(memid));
                return m == _matrix.end() ? 0 : m->second;
            }

            void keep_matrix(void * memid, hb2_ell m)
            {
                _matrix[memid] = m;
            }
    };

    static MemoryBackendRegistrator b200_backend_registrator(tags::B200::memory_value,
            MemoryBackend<tags::B200>::instance());

    namespace b200
    {
        void check(int status, const char * what)
        {
            if (status == HB2_OK)
                return;
            const std::string msg(std::string(what) + ": " + hb2_last_error());
            if (status == HB2_ERR_SIZE)
                throw VectorSizeDoesNotMatch(0, 0);
            throw InternalError(msg);
        }

        namespace
        {
            bool exact_flag()
            {
                const char * v(std::getenv("HB2_BINDING_EXACT"));
                return v && std::strcmp(v, "1") == 0;
            }

            bool g_exact(exact_flag());

            template <typename DT_>
            hb2_ell convert(const SparseMatrixELL<DT_> & a)
            {
                MemoryBackend<tags::B200> * backend(MemoryBackend<tags::B200>::instance());
                void * key(a.Ax().memid());
                hb2_ell m(backend->matrix(key));
                if (m)
                    return m;
                a.Aj().lock(lm_read_only);
                a.Ax().lock(lm_read_only);
                a.Arl().lock(lm_read_only);
                const int st(hb2_ell_create(&m, DType<DT_>::value(), a.rows(), a.columns(), a.stride(),
                            a.num_cols_per_row(), a.threads(), a.Aj().elements(), a.Ax().elements(),
                            a.Arl().elements(), 1, 0));
                a.Arl().unlock(lm_read_only);
                a.Ax().unlock(lm_read_only);
                a.Aj().unlock(lm_read_only);
                check(st, "SparseMatrixELL upload");
                backend->keep_matrix(key, m);
                // the arbiter now counts this backend as a reader of the value array
                // and tells it when the array changes or goes
                a.Ax().lock(lm_read_only, tags::B200::memory_value);
                a.Ax().unlock(lm_read_only);
                return m;
            }
        }

        hb2_ell ell(const SparseMatrixELL<float> & a)
        {
            return convert(a);
        }

        hb2_ell ell(const SparseMatrixELL<double> & a)
        {
            return convert(a);
        }

        bool exact_reductions()
        {
            return g_exact;
        }

        void set_exact_reductions(bool exact)
        {
            g_exact = exact;
        }
    }
}
