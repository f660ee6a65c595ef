// Files and the transposition of SparseMatrixELL.
//
// hb2_ell_read / hb2_ell_write are MatrixIO<io_formats::ELL> (math/matrix_io.hh:433-560):
// a header of five little-endian uint64 (size = num_cols_per_row * stride, rows,
// columns, stride, num_cols_per_row), then `size` uint64 column indices and
// `size` doubles, in the reference's slot layout with one thread per row.  A read
// matrix gets the row lengths the reference's raw-array constructor computes
// (la/sparse_matrix_ell-impl.hh:185-208: the slots up to the first zero value)
// and is converted to the device layout by hb2_ell_create.
//
// hb2_ell_transpose is Transposition<Tag>::value (math/transposition.hh:36-50):
// A^T as the reference builds it -- A's nonzeros visited row by row, each stored
// at (column, row), and the result assembled into ELL with every row's entries
// in ascending column order, stride = rows rounded up to 32, num_cols_per_row =
// the longest row.  Host code: matrices read from files are small set-up data.
#include "hb2_common.cuh"
#include "hb2_internal.hh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

using namespace hb2;

namespace
{
    struct FileCloser
    {
        FILE * f;
        ~FileCloser() { if (f) fclose(f); }
    };

    // row lengths of the reference's raw-array constructor (one thread per row)
    void row_lengths(uint64_t rows, uint64_t stride, uint64_t size, const double * Ax, std::vector<uint64_t> & Arl)
    {
        Arl.assign(rows, 0);
        for (uint64_t r = 0; r < rows; ++r)
        {
            uint64_t count = 0;
            for (uint64_t i = r; i < size; i += stride)
            {
                if (Ax[i] == 0.0) break;
                ++count;
            }
            Arl[r] = count;
        }
    }
}

extern "C" int hb2_ell_read(hb2_ell * out, const char * path, hb2_dtype dtype, cudaStream_t stream)
{
    if (! out || ! path) return fail(HB2_ERR_ARG, "hb2_ell_read: null argument");
    FileCloser fc = {fopen(path, "rb")};
    if (! fc.f) return fail(HB2_ERR_ARG, std::string("hb2_ell_read: file ") + path + " not found");
    uint64_t head[5];
    if (fread(head, sizeof(uint64_t), 5, fc.f) != 5) return fail(HB2_ERR_ARG, "hb2_ell_read: fread error (header)");
    const uint64_t size = head[0], rows = head[1], cols = head[2], stride = head[3], ncpr = head[4];
    if (ncpr == 0 || stride < rows || size != ncpr * stride || cols > 0x7fffffffULL)
        return fail(HB2_ERR_ARG, "hb2_ell_read: inconsistent header");
    std::vector<uint64_t> Aj(size);
    std::vector<double> Ax(size);
    if (fread(Aj.data(), sizeof(uint64_t), size, fc.f) != size) return fail(HB2_ERR_ARG, "hb2_ell_read: fread error (Aj)");
    if (fread(Ax.data(), sizeof(double), size, fc.f) != size) return fail(HB2_ERR_ARG, "hb2_ell_read: fread error (Ax)");
    std::vector<uint64_t> Arl;
    row_lengths(rows, stride, size, Ax.data(), Arl);
    if (dtype == HB2_F64)
        return hb2_ell_create(out, dtype, rows, cols, stride, ncpr, 1, Aj.data(), Ax.data(), Arl.data(), 1, stream);
    // convert<tags::CPU>(axc, ax): values rounded to the element type
    std::vector<float> Af(size);
    for (uint64_t i = 0; i < size; ++i) Af[i] = (float)Ax[i];
    return hb2_ell_create(out, dtype, rows, cols, stride, ncpr, 1, Aj.data(), Af.data(), Arl.data(), 1, stream);
}

extern "C" int hb2_ell_write(hb2_ell A, const char * path)
{
    if (! A || ! path) return fail(HB2_ERR_ARG, "hb2_ell_write: null argument");
    if (A->dtype != HB2_F64) return fail(HB2_ERR_UNSUPPORTED, "hb2_ell_write: only double ELL output is supported");
    if (A->ref_T != 1) return fail(HB2_ERR_UNSUPPORTED, "hb2_ell_write: only the one-thread-per-row layout is supported");
    const uint64_t size = A->ref_K * A->ref_stride;
    std::vector<uint64_t> Aj(size), Arl(std::max<uint64_t>(A->rows, 1));
    std::vector<double> Ax(size);
    int st = hb2_ell_export(A, Aj.data(), Ax.data(), Arl.data());
    if (st) return st;
    FileCloser fc = {fopen(path, "wb")};
    if (! fc.f) return fail(HB2_ERR_ARG, std::string("hb2_ell_write: cannot open ") + path);
    const uint64_t head[5] = {size, A->rows, A->cols, A->ref_stride, A->ref_K};
    if (fwrite(head, sizeof(uint64_t), 5, fc.f) != 5 || fwrite(Aj.data(), sizeof(uint64_t), size, fc.f) != size ||
        fwrite(Ax.data(), sizeof(double), size, fc.f) != size)
        return fail(HB2_ERR_ARG, "hb2_ell_write: fwrite error");
    return HB2_OK;
}

namespace
{
    template <typename T>
    int transpose_typed(hb2_ell * out, hb2_ell A, cudaStream_t stream)
    {
        const uint64_t K = A->ref_K, T_ = A->ref_T, stride = A->ref_stride, size = K * stride;
        std::vector<uint64_t> Aj(size), Arl(std::max<uint64_t>(A->rows, 1));
        std::vector<T> Ax(size);
        int st = hb2_ell_export(A, Aj.data(), Ax.data(), Arl.data());
        if (st) return st;
        // nonzeros of A row by row, in the reference's visiting order, stored at (column, row)
        const uint64_t rows_t = A->cols, cols_t = A->rows;
        std::vector<std::vector<std::pair<uint64_t, T>>> trow(rows_t);
        for (uint64_t r = 0; r < A->rows; ++r)
        {
            // the row's entries sorted by column, as the reference's SparseMatrix holds them
            std::vector<std::pair<uint64_t, T>> row;
            for (uint64_t k = 0; k < Arl[r] * T_; ++k)
            {
                const uint64_t i = (k % T_) + r * T_ + (k / T_) * stride;
                if (Ax[i] != T(0)) row.push_back(std::make_pair(Aj[i], Ax[i]));
            }
            std::stable_sort(row.begin(), row.end(),
                             [](const std::pair<uint64_t, T> & a, const std::pair<uint64_t, T> & b) { return a.first < b.first; });
            for (const auto & e : row) trow[e.first].push_back(std::make_pair(r, e.second));
        }
        uint64_t kt = 1;
        for (const auto & row : trow) kt = std::max<uint64_t>(kt, row.size());
        const uint64_t stride_t = 32 * ((rows_t + 31) / 32);
        std::vector<uint64_t> Ajt(kt * stride_t, 0), Arlt(std::max<uint64_t>(rows_t, 1), 0);
        std::vector<T> Axt(kt * stride_t, T(0));
        for (uint64_t r = 0; r < rows_t; ++r)
        {
            Arlt[r] = trow[r].size();
            for (uint64_t k = 0; k < trow[r].size(); ++k)
            {
                Ajt[k * stride_t + r] = trow[r][k].first;
                Axt[k * stride_t + r] = trow[r][k].second;
            }
        }
        return hb2_ell_create(out, (hb2_dtype)A->dtype, rows_t, cols_t, stride_t, kt, 1, Ajt.data(), Axt.data(),
                              Arlt.data(), 1, stream);
    }
}

extern "C" int hb2_ell_transpose(hb2_ell * out, hb2_ell A, cudaStream_t stream)
{
    if (! out || ! A) return fail(HB2_ERR_ARG, "hb2_ell_transpose: null argument");
    return A->dtype == HB2_F64 ? transpose_typed<double>(out, A, stream) : transpose_typed<float>(out, A, stream);
}
