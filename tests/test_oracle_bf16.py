"""The oracle's restatement of the BF16-stored matrix (hb2_ell_create_bf16; no
counterpart in the reference): its rounding pinned against torch's float32 ->
bfloat16 conversion (round to nearest even), the scale choice, the row sums of the
compensated form and the product's error against the FP64 product."""
import numpy as np
import pytest
import torch

from honei_b200 import inputs


def test_bf16_round_matches_torch_on_float32_values(oracle):
    """Doubles that are float32 values (so torch's float32 -> bfloat16 conversion
    rounds them once): random magnitudes, exact ties, subnormals, the overflow edge"""
    rng = np.random.default_rng(5)
    f = np.concatenate([
        (rng.standard_normal(20000) * np.exp2(rng.integers(-60, 60, 20000))).astype(np.float32),
        # ties: 8 significant bits + one half-ulp bit, either parity
        (np.float32(1.0) + np.float32(2.0 ** -8) * np.arange(1, 200, 2, dtype=np.float32)).astype(np.float32),
        np.array([2.0 ** -130, 2.0 ** -133 * 1.5, 2.0 ** -134, 3.0e38, 3.3895e38, -0.0, 1.0], np.float32),
    ])
    ours = oracle.bf16_round(f.astype(np.float64))
    theirs = torch.from_numpy(f).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(ours, theirs)


def test_bf16_round_of_doubles_rounds_once(oracle):
    """A double just above a tie rounds up, just below rounds down (no double
    rounding through float32)"""
    tie = 1.0 + 2.0 ** -8            # halfway between 1 and 1 + 2^-7
    assert oracle.bf16_round(np.array([tie]))[0] == 1.0
    assert oracle.bf16_round(np.array([tie + 2.0 ** -40]))[0] == 1.0 + 2.0 ** -7
    assert oracle.bf16_round(np.array([tie - 2.0 ** -40]))[0] == 1.0


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_q1_scale_three_is_exact(oracle, dt):
    A = oracle.q1_ell(6, dt)
    for comp in (False, True):
        s, err = oracle.ell_bf16_scale(A, comp)
        # 3 * 8/3 and 3 * -1/3 round to 8 and -1 (exactly from FP64; FP32's 8/3 is
        # off by less than one FP32 unit)
        assert s == 3.0 and err <= (0.0 if dt == np.float64 else 2.0 ** -23)
    x = oracle.uniform(A.rows, 3, np.float32)
    y = oracle.ell_bf16_spmv(A, 3.0, False, x).astype(np.float64)
    A3 = oracle.Ell(A.rows, A.cols, A.stride, A.K, 1, A.Aj, np.round(A.Ax.astype(np.float64) * 3), A.Arl)
    ref = oracle.ell_spmv(A3, x.astype(np.float64)) / 3
    absA3 = oracle.Ell(A.rows, A.cols, A.stride, A.K, 1, A.Aj, np.abs(A3.Ax), A.Arl)
    # exact integer entries (8, -1, 3): only the FP32 sums and the division round
    bound = oracle.ell_spmv(absA3, np.abs(x).astype(np.float64)) / 3 * 11 * np.finfo(np.float32).eps
    assert np.all(np.abs(y - ref) <= bound)


def coef_ell(oracle, L, seed=7, dt=np.float64):
    rows, cols, stride, K, Aj, Ax, Arl = inputs.q1_coefficient_operator(inputs.element_coefficients(L, seed), dt)
    return oracle.Ell(rows, cols, stride, K, 1, Aj, Ax, Arl)


def test_compensated_form_keeps_row_sums(oracle):
    """sum_j q_ij + d_i = s * sum_j a_ij up to d's single FP32 rounding"""
    A = coef_ell(oracle, 6)
    s, err = oracle.ell_bf16_scale(A, True)
    assert err < 2.0 ** -8
    v = oracle.ell_bf16_values(A, s, True).astype(np.float64).reshape(A.K, A.stride) * s
    a = A.Ax.reshape(A.K, A.stride)
    rows_v, rows_a = v.sum(axis=0), a.sum(axis=0) * s
    d = np.abs(v).max(axis=0)
    assert np.all(np.abs(rows_v - rows_a) <= 4 * np.finfo(np.float32).eps * d)
    # the pure form does not keep them
    vp = oracle.ell_bf16_values(A, s, False).astype(np.float64).reshape(A.K, A.stride) * s
    assert np.abs(vp.sum(axis=0) - rows_a).max() > 100 * np.abs(rows_v - rows_a).max()


@pytest.mark.parametrize("comp", [False, True])
def test_bf16_product_error_against_fp64(oracle, comp):
    """|A_bf16 x - A x| <= (2^-8 + n_slots eps32) sum |a_ij x_j| per row"""
    A = coef_ell(oracle, 7)
    s, err = oracle.ell_bf16_scale(A, comp)
    x = oracle.uniform(A.rows, 9, np.float32)
    y = oracle.ell_bf16_spmv(A, s, comp, x).astype(np.float64)
    ref = oracle.ell_spmv(A, x.astype(np.float64))
    absA = oracle.Ell(A.rows, A.cols, A.stride, A.K, 1, A.Aj, np.abs(A.Ax), A.Arl)
    ax = np.abs(x).astype(np.float64)
    # entry errors <= err |a_ij| (the compensated diagonal carries its row's, paid
    # with |x_i|), FP32 sums and the division
    reach = oracle.ell_spmv(absA, ax) + (ax * oracle.ell_spmv(absA, np.ones(A.cols)) if comp else 0.0)
    bound = reach * (err + 12 * np.finfo(np.float32).eps)
    assert np.all(np.abs(y - ref) <= bound + 1e-30)


@pytest.mark.parametrize("level", [1, 2, 4, 6])
def test_feast_matrices_are_exact_in_bf16_at_scale_three(oracle, feast, level):
    """The reference's FEAST Q1 matrices (math/mg_TEST.cc:398-463, its ELL files):
    3 a is within 1e-7 of an integer of magnitude at most 12 for every entry, so the
    FP32 copies stored at s = 3 round no further than FP32 already did (largest
    relative error 2^-25), pure and compensated alike, and the stored values read back
    in FP32 are (float)(k / 3) -- why the BF16 inner hierarchies take the FP32 one's
    steps on the FEAST system (tests/test_gpu_bf16.py)."""
    A = feast.ell(oracle, f"A_{level}")
    k = np.round(3 * A.Ax)
    assert np.abs(3 * A.Ax - k).max() < 1e-7 and np.abs(k).max() <= 12
    A32 = oracle.Ell(A.rows, A.cols, A.stride, A.K, A.T, A.Aj, A.Ax.astype(np.float32), A.Arl)
    for comp in (False, True):
        s, err = oracle.ell_bf16_scale(A32, comp)
        assert s == 3.0 and err <= 2.0 ** -25
    assert np.array_equal(oracle.ell_bf16_values(A32, 3.0, False), (k / 3).astype(np.float32))
