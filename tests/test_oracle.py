"""Pins for the CPU oracle (no GPU): the reference has no tests or golden
vectors for this path, so the oracle is checked against the reference's own
tables and compiled C++ cores (tests/golden/, made by make_golden.py), a dense
O(V^2) Toeplitz direct sum, algebraic identities and scipy."""
import json
import os

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle import vie as ov

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def parity_G(rng, L, M, N):
    G = rng.standard_normal((L, M, N, 6)) + 1j * rng.standard_normal((L, M, N, 6))
    G[0, :, :, 1] = 0
    G[:, 0, :, 1] = 0
    G[0, :, :, 2] = 0
    G[:, :, 0, 2] = 0
    G[:, 0, :, 4] = 0
    G[:, :, 0, 4] = 0
    return G


def test_gauss_rules_match_reference_tables():
    from oracle.assembly import gauss_1d
    tab = json.load(open(os.path.join(GOLD, "gauss_1d.json")))
    for n, d in tab.items():
        w, x = gauss_1d(int(n))
        assert np.max(np.abs(x - np.array(d["xtab"]))) < 4e-16
        assert np.max(np.abs(w - np.array(d["weight"]))) < 4e-15


@pytest.mark.parametrize("shape", [(4, 3, 3), (5, 4, 2), (3, 3, 5)])
def test_circulant_matvec_equals_dense_toeplitz_sum(shape):
    rng = np.random.default_rng(0)
    L, M, N = shape
    G = rng.standard_normal((L, M, N, 6)) + 1j * rng.standard_normal((L, M, N, 6))
    fN = ov.fN_from_toeplitz(G)
    Mc = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    J = rng.standard_normal((L, M, N, 3)) + 1j * rng.standard_normal((L, M, N, 3))
    idx = np.arange(1, 3 * L * M * N + 1)
    y = ov.mv_AN_const(J.reshape(-1, order="F"), fN, np.ones(shape), Mc, 0.3, "notransp", idx)
    NJ = ov.dense_toeplitz_matvec(G, J)
    ref = (0.3 * J - Mc[..., None] * NJ).reshape(-1, order="F")
    assert rel(y, ref) < 1e-13


def test_golden_tiny_case_reproduced():
    d = np.load(os.path.join(GOLD, "tiny_case.npz"))
    G, J = d["G"], d["J"]
    L, M, N, _ = G.shape
    fN = ov.fN_from_toeplitz(G)
    idx = np.arange(1, 3 * L * M * N + 1)
    y = ov.mv_AN_const(J.reshape(-1, order="F"), fN, np.ones((L, M, N)), d["Mc"], float(d["Gram"]),
                       "notransp", idx)
    assert rel(y, d["y"]) < 1e-13
    ref = (float(d["Gram"]) * J - d["Mc"][..., None] * d["dense_NJ"]).reshape(-1, order="F")
    assert rel(y, ref) < 1e-12


def test_transp_branch_is_the_adjoint():
    rng = np.random.default_rng(1)
    L, M, N = 5, 4, 3
    G = parity_G(rng, L, M, N)
    fN = ov.fN_from_toeplitz(G)
    Mr = rng.standard_normal((L, M, N)) + 2 + 1j * rng.standard_normal((L, M, N))
    Mc = rng.standard_normal((L, M, N)) + 1j * rng.standard_normal((L, M, N))
    idx = np.arange(1, 3 * L * M * N + 1)
    x = rng.standard_normal(idx.size) + 1j * rng.standard_normal(idx.size)
    y = rng.standard_normal(idx.size) + 1j * rng.standard_normal(idx.size)
    Ax = ov.mv_AN_const(x, fN, Mr, Mc, 0.7, "notransp", idx)
    Aty = ov.mv_AN_const(y, fN, Mr, Mc, 0.7, "transp", idx)
    assert abs(np.vdot(y, Ax) - np.vdot(Aty, x)) < 1e-12 * abs(np.vdot(y, Ax))


def test_fN_parity_symmetry():
    """The transformed circulant of a parity-structured tensor satisfies
    fN(-k) = s fN(k) per axis (the octant storage of the device operator)."""
    rng = np.random.default_rng(2)
    G = parity_G(rng, 6, 5, 4)
    fN = ov.fN_from_toeplitz(G)
    sx = ov.GP_COEFF["L"]
    sy = ov.GP_COEFF["M"]
    sz = ov.GP_COEFF["N"]
    m = fN[::-1, ::-1, ::-1, :]
    m = np.roll(m, 1, axis=(0, 1, 2))  # index -k
    s = sx * sy * sz
    assert np.max(np.abs(m * s - fN)) < 1e-12 * np.max(np.abs(fN))


def test_sparse_unsorted_idx_is_scatter_gather():
    rng = np.random.default_rng(3)
    L, M, N = 4, 3, 3
    G = parity_G(rng, L, M, N)
    fN = ov.fN_from_toeplitz(G)
    Mc = rng.standard_normal((L, M, N)) + 0j
    full = np.arange(1, 3 * L * M * N + 1)
    idx = rng.permutation(full)[:40]
    J = rng.standard_normal(40) + 1j * rng.standard_normal(40)
    Jf = np.zeros(full.size, complex)
    Jf[idx - 1] = J
    yf = ov.mv_AN_const(Jf, fN, np.ones((L, M, N)), Mc, 1.0, "notransp", full)
    y = ov.mv_AN_const(J, fN, np.ones((L, M, N)), Mc, 1.0, "notransp", idx)
    assert rel(y, yf[idx - 1]) < 1e-14


def test_pgmres_matches_scipy_on_known_spectrum():
    rng = np.random.default_rng(4)
    n = 120
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    lam = 1 + rng.uniform(0, 4, n) + 0.5j * rng.standard_normal(n)
    A = (Q * lam) @ Q.conj().T
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x, flag, relres, it, resvec = ov.pgmres(lambda v: A @ v, b, 20, 1e-10, 20)
    assert flag == 0 and relres <= 1e-10
    xs, info = spla.gmres(A, b, rtol=1e-12, restart=20, maxiter=100)
    assert rel(x, xs) < 1e-8
    assert rel(x, np.linalg.solve(A, b)) < 1e-8
    assert resvec[0] == 1.0 and np.all(np.diff(resvec[: it[0] + 1]) <= 1e-12)


def test_pgmres_zero_rhs_and_maxit():
    A = np.eye(5) * 2.0
    x, flag, relres, it, resvec = ov.pgmres(lambda v: A @ v, np.ones(5), 3, 1e-30, 1)
    assert it[1] == 1 and flag == 1 or relres < 1e-15


def test_level1_blocks_pairing_identity():
    """B_{L-i} = D B_i D (D = -1 on the x rows) for a tensor whose xy and xz
    components vanish on the x = 0 plane - the identity behind the device
    preconditioner's mode pairing."""
    rng = np.random.default_rng(5)
    L, M, N = 7, 3, 2
    G = parity_G(rng, L, M, N)
    circ, _ = ov.level_1_parallel_func_N(G, L, M, N, 1.0)
    face3 = ov.face_from_Mr(2.0 + rng.uniform(0, 1, (L, M, N)))
    B = ov.level1_blocks(circ, face3, 1.0)
    MN = M * N
    d = np.ones(3 * MN)
    d[:MN] = -1
    for i in range(1, L):
        assert np.max(np.abs(B[L - i] - d[:, None] * B[i] * d[None, :])) < 1e-12 * np.max(
            np.abs(B[i]))


def test_chan_mvp_idx_is_blockwise_solve():
    rng = np.random.default_rng(6)
    L, M, N = 5, 2, 2
    G = parity_G(rng, L, M, N)
    circ, _ = ov.level_1_parallel_func_N(G, L, M, N, 2.0)
    face3 = ov.face_from_Mr(2.0 + rng.uniform(0, 1, (L, M, N)))
    B = ov.level1_blocks(circ, face3, 2.0)
    Binv = ov.level1_inverse_blocks(circ, face3, 2.0)
    idx = np.arange(1, 3 * L * M * N + 1)
    J = rng.standard_normal(idx.size) + 1j * rng.standard_normal(idx.size)
    y = ov.chan_mvp_idx(Binv, J, L, M, N, idx)
    # forward: fft along x, block multiply, ifft must return J
    t = np.fft.fft(y.reshape((L, 3 * M * N), order="F"), axis=0)
    back = np.stack([B[i] @ t[i] for i in range(L)])
    back = np.fft.ifft(back, axis=0).reshape(-1, order="F")
    assert rel(back, J) < 1e-12


def test_jvie2_scaling():
    rng = np.random.default_rng(7)
    e_r = 1 + rng.uniform(0, 4, (3, 3, 2)) - 0.1j * rng.uniform(0, 1, (3, 3, 2))
    e_r[0, 0, 0] = 1.0
    Einc = rng.standard_normal((3, 3, 2, 3)) + 1j * rng.standard_normal((3, 3, 2, 3))
    Mr, Mc, idx, b = ov.jvie2_system(Einc, e_r, 8e-24, 2.8e14)
    assert np.all(Mr == 1)
    assert np.allclose(Mc, (e_r - 1) / e_r)
    assert idx.size == 3 * (e_r.size - 1)
