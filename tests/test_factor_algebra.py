"""The algebra of the block factor's in-place Gauss-Jordan inversion, restated
on the CPU (`csrc/vb_thomas.cu`, gj_factor_atmosphere): implicit threshold
partial pivoting (no row exchanges; the pivot row is the lowest row whose
magnitude matches the column maximum in the top 24 bits of its FP64 pattern,
pivot_key32), pivot rows left
unnormalised during the elimination and scaled by 1/pivot at the end, the
result stored permuted (B^{-1}[q(i)][p_m] = T[i][m]), and the two
orientations: elimination on A^T (the Ros2 step and forward solves, which
need the right residual |A X - I| that the reference's lu_solve(LU, I) has)
or on A (the adjoint's transposed solves, which need |X A - I|). The GPU
kernel itself is compared with the oracle in the -m gpu tests."""
import numpy as np
import pytest


def pivot_row(col, cand):
    """The kernel's pivot choice among the candidate rows `cand` of a column:
    key = (top 24 bits of |v|, i.e. the sign-cleared high word >> 7) << 8 |
    (255 - row), NaN as magnitude 0; the row of the largest key."""
    v = np.abs(col[cand]).astype(np.float64)
    hi = (v.view(np.uint64) >> np.uint64(32)) & np.uint64(0x7fffffff)
    mag = np.where(np.isnan(v), np.uint64(0), hi >> np.uint64(7)).astype(np.int64)
    key = (mag << 8) | (255 - cand)
    return int(cand[np.argmax(key)])


def gauss_jordan_inverse(A, transposed):
    """X = A^{-1} by the kernel's sequence of operations."""
    Bm = (A.T if transposed else A).astype(np.float64).copy()
    n = Bm.shape[0]
    used = np.zeros(n, bool)
    q = np.zeros(n, int)       # step whose pivot row is row i
    pivs = np.zeros(n, int)    # pivot row of step k
    rps = np.zeros(n)          # 1 / pivot of row i
    for k in range(n):
        cand = np.flatnonzero(~used)
        p = pivot_row(Bm[:, k], cand)
        rp = 1.0 / Bm[p, k]
        m = np.where(np.arange(n) != p, Bm[:, k] * rp, 0.0)
        Bm -= np.outer(m, Bm[p])                         # pivot row unchanged (m_p = 0)
        Bm[:, k] = -m
        Bm[p, k] = 1.0
        used[p], q[p], pivs[k], rps[p] = True, k, p, rp
    T = Bm * rps[:, None]
    Binv = np.empty_like(T)
    Binv[q[:, None], pivs[None, :]] = T                  # B^{-1}[q(i)][p_m] = T[i][m]
    return Binv.T if transposed else Binv


@pytest.mark.parametrize("n", [1, 2, 5, 32, 69, 89])
@pytest.mark.parametrize("transposed", [True, False])
def test_matches_inverse(n, transposed):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)) + np.diag(rng.uniform(1.0, 2.0, n))
    X = gauss_jordan_inverse(A, transposed)
    R = np.linalg.inv(A)
    assert np.abs(X - R).max() <= 1e-12 * np.abs(R).max()


def test_ties_go_to_the_lowest_row():
    # column 0 has equal magnitudes in rows 1 and 2: row 1 must pivot first
    A = np.array([[0.5, 1.0, 0.0], [-2.0, 0.0, 1.0], [2.0, 3.0, 1.0]])
    X = gauss_jordan_inverse(A, transposed=False)
    assert np.abs(X @ A - np.eye(3)).max() < 1e-15
    # the permutation bookkeeping holds for any tie order; the choice itself is
    # the lowest row, as LAPACK's idamax
    assert pivot_row(A[:, 0], np.array([1, 2])) == 1


def test_threshold_pivot_choice():
    """Magnitudes equal in their top 24 bits count as ties (the lowest row
    wins); a larger exponent or a leading-mantissa difference wins outright;
    pivoted rows and NaN never beat a candidate with a finite magnitude."""
    rows = np.array([3, 5, 7])
    near = 1.0 + 2.0 ** -20                         # same top 24 bits as 1.0
    assert pivot_row(np.array([0, 0, 0, 1.0, 0, -near, 0, 0.5]), rows) == 3
    assert pivot_row(np.array([0, 0, 0, 1.0, 0, -(1.0 + 2.0 ** -12), 0, 0.5]), rows) == 5
    assert pivot_row(np.array([0, 0, 0, 1e-30, 0, 1e-29, 0, np.nan]), rows) == 5
    assert pivot_row(np.array([0, 0, 0, np.nan, 0, 0.0, 0, np.nan]), rows) == 3
    # within the threshold the choice is a pivot at least (1 - 2^-13) of the maximum
    rng = np.random.default_rng(0)
    for _ in range(200):
        col = rng.standard_normal(40) * 10.0 ** rng.integers(-3, 3, 40)
        cand = np.sort(rng.choice(40, 25, replace=False))
        p = pivot_row(col, cand)
        assert abs(col[p]) >= (1 - 2.0 ** -13) * np.abs(col[cand]).max()


def test_orientation_on_the_stiff_config0_chain():
    """The specified config-0 draw (k log-uniform in [1e-40, 1e-8], dt=1e-6):
    the block-Thomas chain over its 120 stage-1 blocks with Gauss-Jordan
    inverses, each inverse feeding the next Schur update, then the solve by
    inverse products. Eliminating on A^T (the kernel's choice for the step)
    keeps the solve's normwise backward error at rounding level; eliminating
    on A itself leaves it about 600 times larger (4e-12 against 7e-15)."""
    from conftest import load_pkg
    from oracle import ros2 as orc
    syn = load_pkg("synthetic")
    case = syn.config0()
    diag, sup_n, sub_n, rhs, _ = orc.lhs_blocks(case.y, case.k, case.dt, case.atm, case.net.tables)
    nz = diag.shape[0]

    def chain_solve(transposed):
        invs, A = [], diag[0]
        for j in range(nz):
            if j > 0:
                A = diag[j] - (sub_n[j - 1][:, None] * sup_n[j - 1][None, :]) * invs[-1]   # solver.py:47
            invs.append(gauss_jordan_inverse(A, transposed))
        rm = [rhs[0]]
        for j in range(1, nz):
            rm.append(rhs[j] - sub_n[j - 1] * (invs[j - 1] @ rm[-1]))
        x = [None] * nz
        x[-1] = invs[-1] @ rm[-1]
        for j in range(nz - 2, -1, -1):
            x[j] = invs[j] @ (rm[j] - sup_n[j] * x[j + 1])
        return np.stack(x)

    def backward_error(x):
        r = np.einsum("zij,zj->zi", diag, x)
        r[:-1] += sup_n * x[1:]
        r[1:] += sub_n * x[:-1]
        r -= rhs
        norm_a = max(np.abs(diag).sum(axis=2).max(), 1.0)
        return np.abs(r).max() / (norm_a * np.abs(x).max() + np.abs(rhs).max())

    with np.errstate(all="ignore"):
        bt = backward_error(chain_solve(True))
        bn = backward_error(chain_solve(False))
    print(f"solve backward error: elimination on A^T {bt:.2e}, on A {bn:.2e}")
    assert bt <= 1e-13
    assert bn >= 100 * bt
