"""The drop-in linear-solver policy (mac_csc_factorize / mac_csc_solve, the
member functions of Policy_Solve_Linear_Umfpack, src/Policy_Solve_Linear_Umfpack.h:28-70)
on matrices other than the reference's pressure matrix.

Umfpack is a general sparse LU: it solves any non-singular matrix the caller
assembles. The device policy solves the reference's symmetric pressure
matrix by CG and every other matrix by BiCGStab on a row-major copy; these
tests check the second path against a direct solve (scipy spsolve, FP64) and
that malformed CSC arrays are refused.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ctx(rtol=1e-12):
    from mac_b200.gpu import Context
    from mac_b200.state import Params
    return Context(Params(h=(0.05, 0.05, 0.05)), max_bricks=64, max_particles=1024, rtol=rtol, max_iters=5000)


def _convection_diffusion(n, peclet, seed):
    """7-point diffusion plus first-order upwind convection on an n^3 grid
    with Dirichlet walls: non-symmetric, diagonally dominant."""
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    N = n ** 3
    idx = np.arange(N).reshape(n, n, n)
    rows, cols, vals = [], [], []
    vel = rng.uniform(-1, 1, 3) * peclet
    for a in range(3):
        for s in (-1, 1):
            src = [slice(None)] * 3
            dst = [slice(None)] * 3
            src[a] = slice(1, None) if s < 0 else slice(None, -1)
            dst[a] = slice(None, -1) if s < 0 else slice(1, None)
            i, j = idx[tuple(src)].ravel(), idx[tuple(dst)].ravel()
            up = max(0.0, -s * vel[a])
            rows.append(i)
            cols.append(j)
            vals.append(np.full(i.size, 1.0 + up))
    diag = np.full(N, -6.0 - np.abs(vel).sum())
    rows.append(np.arange(N))
    cols.append(np.arange(N))
    vals.append(diag)
    A = sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    A.sort_indices()
    return A


def test_nonsymmetric_matrix_is_solved_by_bicgstab():
    import scipy.sparse.linalg as spl
    A = _convection_diffusion(12, 3.0, seed=7)
    assert abs(A - A.T).max() > 0.5
    b = np.random.default_rng(8).uniform(-1, 1, A.shape[0])
    want = spl.spsolve(A, b)
    with _ctx() as ctx:
        got = ctx.csc_solve(A.indptr, A.indices, A.data, b)
        st = ctx.stats()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-9
    assert np.linalg.norm(A @ got - b) / np.linalg.norm(b) <= 1e-11
    assert 0 < st["iterations"] < 5000


def test_positive_diagonal_matrix_goes_to_the_general_path():
    # the negation of a pressure-like matrix: symmetric, positive diagonal
    import scipy.sparse.linalg as spl
    A = -_convection_diffusion(8, 0.0, seed=1)
    b = np.random.default_rng(2).uniform(-1, 1, A.shape[0])
    want = spl.spsolve(A.tocsc(), b)
    A = A.tocsc()
    A.sort_indices()
    with _ctx() as ctx:
        got = ctx.csc_solve(A.indptr, A.indices, A.data, b)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-9


def test_malformed_csc_is_refused():
    from mac_b200.gpu import MacError
    with _ctx() as ctx:
        with pytest.raises(MacError):
            # row index 5 in a 3x3 matrix
            ctx.csc_solve(np.array([0, 1, 2, 3]), np.array([0, 5, 2]), np.array([-1.0, -1.0, -1.0]), np.ones(3))
        with pytest.raises(MacError):
            # decreasing offsets
            ctx.csc_solve(np.array([0, 2, 1, 3]), np.array([0, 1, 2]), np.array([-1.0, -1.0, -1.0]), np.ones(3))
