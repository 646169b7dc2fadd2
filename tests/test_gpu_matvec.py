"""GPU parity of the fused FFT-circulant matvec against the CPU oracle.

Tolerances (relative, 2-norm over the output vector): complex128 1e-12,
complex64 1e-5 -- the matvec bars of the benchmark definition.
"""
import numpy as np
import pytest

from oracle import vie as ov
import voxphoton_b200 as vb
from voxphoton_b200 import geometry as geo

pytestmark = pytest.mark.gpu

TOL128 = 1e-12
TOL64 = 1e-5


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def rand_c(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def rand_toeplitz(rng, L, M, N):
    """A random Toeplitz tensor with the parity structure of a physical G
    (xy vanishes on the x=0 and y=0 planes, xz on x=0 and z=0, yz on y=0 and z=0)."""
    G = rand_c(rng, L, M, N, 6)
    G[0, :, :, 1] = 0
    G[:, 0, :, 1] = 0
    G[0, :, :, 2] = 0
    G[:, :, 0, 2] = 0
    G[:, 0, :, 4] = 0
    G[:, :, 0, 4] = 0
    return G


@pytest.mark.parametrize("shape", [(7, 5, 3), (13, 11, 2), (16, 9, 6), (30, 4, 5)])
def test_matvec_random_full_support(shape):
    rng = np.random.default_rng(0)
    L, M, N = shape
    G = rand_toeplitz(rng, L, M, N)
    fN = ov.fN_from_toeplitz(G)
    Mc = rand_c(rng, L, M, N)
    Gram = 0.37
    idx = np.arange(1, 3 * L * M * N + 1)
    J = rand_c(rng, idx.size)
    ref = ov.mv_AN_const(J, fN, np.ones((L, M, N)), Mc, Gram, "notransp", idx)
    for src in ("G", "fN"):
        kw = {"G": G} if src == "G" else {"fN": fN}
        op = vb.Operator(Mc, Gram, idx, **kw)
        assert rel(op.mv_AN(J), ref) < TOL128
        assert rel(op.mv_AN(J, prec="c64"), ref) < TOL64
        op.close()


def test_matvec_sparse_support_transp_and_Mr():
    rng = np.random.default_rng(1)
    L, M, N = 12, 7, 5
    V = L * M * N
    G = rand_toeplitz(rng, L, M, N)
    fN = ov.fN_from_toeplitz(G)
    Mr = rand_c(rng, L, M, N) + 2.0
    Mc = rand_c(rng, L, M, N)
    Gram = 1.7
    # unsorted, sparse support (the reference accepts any idx order)
    idx = rng.permutation(3 * V)[: (3 * V) // 3] + 1
    J = rand_c(rng, idx.size)
    op = vb.Operator(Mc, Gram, idx, fN=fN, Mr=Mr)
    for flag in ("notransp", "transp"):
        ref = ov.mv_AN_const(J, fN, Mr, Mc, Gram, flag, idx)
        assert rel(op.mv_AN(J, flag), ref) < TOL128
        assert rel(op.mv_AN(J, flag, prec="c64"), ref) < TOL64
    op.close()


def test_mv_L_const():
    rng = np.random.default_rng(2)
    L, M, N = 9, 6, 4
    G = rand_toeplitz(rng, L, M, N)
    fN = ov.fN_from_toeplitz(G)
    idx = np.arange(1, 3 * L * M * N + 1)
    J = rand_c(rng, idx.size)
    ref = ov.mv_L_const(J, fN, (L, M, N), 0.5, idx)
    out = vb.mv_L_const(J, fN, np.zeros((L, M, N, 3)), 0.5, idx)
    assert rel(out, ref) < TOL128


def test_mv_AN_const_oneshot_signature():
    rng = np.random.default_rng(3)
    L, M, N = 6, 5, 4
    G = rand_toeplitz(rng, L, M, N)
    fN = ov.fN_from_toeplitz(G)
    Mc = rand_c(rng, L, M, N)
    idx = np.arange(1, 3 * L * M * N + 1)
    J = rand_c(rng, idx.size)
    ref = ov.mv_AN_const(J, fN, np.ones((L, M, N)), Mc, 2.0, "notransp", idx)
    out = vb.mv_AN_const(J, fN, np.ones((L, M, N)), Mc, 2.0, "notransp", idx, 1)
    assert rel(out, ref) < TOL128


def test_strip_cfg1_ten_seeded_inputs():
    """Straight strip, 100 x 25 x 11 at 20 nm, physical operator, 10 inputs (seed 0)."""
    p = geo.strip()
    G = vb.assemble_toeplitz(p.shape, p.ko, p.res)
    fN = ov.fN_from_toeplitz(G)
    Mop = p.Mop()
    idx = p.idxS3()
    op = vb.Operator(Mop, p.Gram, idx, fN=fN)
    rng = np.random.default_rng(0)
    ones = np.ones(p.shape)
    for _ in range(10):
        J = rng.standard_normal(idx.size) + 1j * rng.standard_normal(idx.size)
        ref = ov.mv_AN_const(J, fN, ones, Mop, p.Gram, "notransp", idx)
        assert rel(op.mv_AN(J), ref) < TOL128
        assert rel(op.mv_AN(J, prec="c64"), ref) < TOL64
    op.close()


def test_single_voxel_support_and_empty_like_input():
    rng = np.random.default_rng(4)
    L, M, N = 5, 4, 3
    G = rand_toeplitz(rng, L, M, N)
    fN = ov.fN_from_toeplitz(G)
    Mc = rand_c(rng, L, M, N)
    idx = np.array([17])
    op = vb.Operator(Mc, 1.0, idx, fN=fN)
    J = np.array([1.0 - 2.0j])
    ref = ov.mv_AN_const(J, fN, np.ones((L, M, N)), Mc, 1.0, "notransp", idx)
    assert rel(op.mv_AN(J), ref) < TOL128
    # zero input gives exactly zero
    assert np.all(op.mv_AN(np.zeros(1)) == 0)
    op.close()


def test_bad_arguments_raise():
    L, M, N = 4, 4, 4
    Mc = np.ones((L, M, N))
    G = np.zeros((L, M, N, 6), dtype=complex)
    with pytest.raises(vb.vie._lib.VoxError):
        vb.Operator(Mc, 1.0, [0], G=G)          # idx is 1-based
    with pytest.raises(vb.vie._lib.VoxError):
        vb.Operator(Mc, 1.0, [1, 1], G=G)       # duplicate position
    with pytest.raises(vb.vie._lib.VoxError):
        vb.Operator(Mc, 1.0, [3 * L * M * N + 1], G=G)


def test_matvec_split_planes_for_tall_grids():
    # 8 x 430 x 11: a padded plane of 3N = 33 rows x Py (864) values exceeds
    # shared memory in both precisions, so kernel 2 runs in its split form
    from voxphoton_b200 import geometry as geo
    rng = np.random.default_rng(11)
    L, M, N = 8, 430, 11
    res = 20e-9
    ko = 2 * np.pi * geo.N_EXT / 1550e-9
    G = vb.assemble_toeplitz((L, M, N), ko, res)
    Mc = 0.3 + 0.1j + 0.05 * rng.standard_normal((L, M, N))
    Mr = 1.0 + 0.1 * rng.standard_normal((L, M, N))
    keep = rng.random(L * M * N) < 0.7
    s = np.flatnonzero(keep) + 1
    V = L * M * N
    idx = np.concatenate([s, V + s, 2 * V + s])
    op = vb.Operator(Mc, res ** 3, idx, G=G, Mr=Mr)
    fN = ov.fN_from_toeplitz(G)
    for t in ("notransp", "transp"):
        x = rng.standard_normal(idx.size) + 1j * rng.standard_normal(idx.size)
        ref = ov.mv_AN_const(x, fN, Mr, Mc, res ** 3, t, idx)
        y = op.mv_AN(x, t, prec="c128")
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-12
        y32 = op.mv_AN(x, t, prec="c64")
        assert np.linalg.norm(y32 - ref) / np.linalg.norm(ref) < 1e-5
    op.close()
