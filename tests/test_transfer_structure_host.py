"""The row structure the Q1 transfer kernels assume (q1_prolong_row / q1_restrict_row in
honei_b200/csrc/hb2_common.cuh), checked against the oracle's ProlongationMatrix and its
Transposition: every row's columns, in slot order, and its weights.  The kernels sum these
rows like the ELL kernels, so this is what makes them bit-identical to the matrix
products (the GPU side: test_q1_transfer_kernels_match_matrix_products)."""
import numpy as np
import pytest


def structured_prolongation(L):
    """(columns, weights) per fine row, slot order, as the kernel derives them."""
    mf, mc = (1 << L) + 1, (1 << (L - 1)) + 1
    rows = []
    for r in range(mf * mf):
        i, j = divmod(r, mf)
        I, J = i // 2, j // 2
        base = I * mc + J
        if i % 2 == 0 and j % 2 == 0:
            rows.append(([base], [1.0]))
        elif i % 2 == 0:
            rows.append(([base, base + 1], [0.5, 0.5]))
        elif j % 2 == 0:
            rows.append(([base, base + mc], [0.5, 0.5]))
        else:
            rows.append(([base, base + 1, base + mc, base + mc + 1], [0.25] * 4))
    return rows


def structured_restriction(L):
    mf, mc = (1 << L) + 1, (1 << (L - 1)) + 1
    rows = []
    for r in range(mc * mc):
        I, J = divmod(r, mc)
        cols, w = [], []
        for di in (-1, 0, 1):
            i = 2 * I + di
            if not 0 <= i < mf:
                continue
            for dj in (-1, 0, 1):
                j = 2 * J + dj
                if not 0 <= j < mf:
                    continue
                cols.append(i * mf + j)
                w.append((1.0 if di == 0 else 0.5) * (1.0 if dj == 0 else 0.5))
        rows.append((cols, w))
    return rows


def matrix_rows(E):
    out = []
    for r in range(E.rows):
        k = np.arange(int(E.Arl[r]))
        idx = k * E.stride + r
        out.append((E.Aj[idx].astype(np.int64).tolist(), E.Ax[idx].astype(np.float64).tolist()))
    return out


@pytest.mark.parametrize("L", [2, 3, 4, 6])
def test_transfer_rows_match_the_matrices(oracle, L):
    P, R = oracle.transfer_ell(L)
    assert matrix_rows(P) == structured_prolongation(L)
    assert matrix_rows(R) == structured_restriction(L)


def test_structured_rows_give_the_matrix_products(oracle):
    """The rows summed in slot order from zero, products and sums rounded separately,
    give the oracle's ELL products bit for bit."""
    L = 5
    P, R = oracle.transfer_ell(L)
    c, f = oracle.uniform(P.cols, 3), oracle.uniform(P.rows, 4)
    for rows, x, E in ((structured_prolongation(L), c, P), (structured_restriction(L), f, R)):
        y = np.empty(len(rows))
        for r, (cols, w) in enumerate(rows):
            s = 0.0
            for col, wt in zip(cols, w):
                s = s + wt * x[col]     # Python floats: IEEE double, no contraction
            y[r] = s
        assert np.array_equal(y.view(np.uint64), oracle.ell_spmv(E, x).view(np.uint64))
