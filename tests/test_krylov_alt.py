"""The reference's other Krylov drivers: GMRES with deflated restarting
(pgmresDR.m) and BiCGStab (JVIE_Solver_const.m:470-504).  The oracle's
restatements are checked on the CPU against a dense solve; the device drivers
against the oracle on the same problems."""
import numpy as np
import pytest

import voxphoton_b200 as vb
from oracle import vie as ov
from voxphoton_b200 import geometry as geo


def small_grating():
    return geo.bragg(periods=4, len_abs=0.4e-6, res=40e-9, height=120e-9)


@pytest.fixture(scope="module")
def system():
    p = small_grating()
    idx = p.idxS3()
    G = vb.assemble_toeplitz(p.shape, p.ko, p.res)
    fN = ov.fN_from_toeplitz(G)
    A = lambda v: ov.mv_AN_const(v, fN, np.ones(p.shape), p.Mop(), p.Gram, "notransp", idx)
    L, M, N = p.shape
    circ, _ = ov.level_1_parallel_func_N(G, L, M, N, p.Gram)
    blocks = ov.level1_inverse_blocks(circ, ov.face_from_Mr(p.e_r), p.Gram)
    prec = lambda v: ov.chan_mvp_idx(blocks, v, L, M, N, idx)
    b = ov.jvie2_system(geo.plane_wave(p), p.e_r, p.Gram, p.freq)[3]
    return p, G, idx, A, prec, b


def _dense(A, n):
    return np.stack([A(e) for e in np.eye(n, dtype=complex)], axis=1)


def test_oracle_pgmresDR_converges_and_deflation_pays(system):
    p, G, idx, A, prec, b = system
    x, flag, relres, it, rv = ov.pgmresDR(A, b, 10, 1e-8, 60, 4)
    assert flag == 0 and relres <= 1e-8
    # the same restart without deflation needs more iterations
    _, f0, _, it0, rv0 = ov.pgmres(A, b, 10, 1e-8, 60)
    assert len(rv) < len(rv0)
    # left preconditioned: the preconditioned residual reaches tol (the true
    # relative residual, which sets flag as in pgmresDR.m, stays close to it)
    # and its history is monotone
    x1, f1, r1, it1, rv1 = ov.pgmresDR(A, b, 10, 1e-8, 60, 4, L1=prec)
    assert rv1[-1] <= 1e-8 and r1 < 1e-7
    assert np.all(np.diff(rv1) <= 1e-12)
    assert np.linalg.norm(x1 - x) / np.linalg.norm(x) < 1e-6


def test_oracle_bicgstab_matches_a_dense_solve():
    rng = np.random.default_rng(0)
    n = 60
    Ad = np.eye(n) * 4 + (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / 3
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    Md = np.diag(np.diag(Ad))
    x, flag, relres, it, rv = ov.bicgstab(lambda v: Ad @ v, b, 1e-12, 200,
                                          M=lambda v: np.linalg.solve(Md, v))
    assert flag == 0 and relres <= 1e-12
    assert np.allclose(x, np.linalg.solve(Ad, b), rtol=1e-10, atol=1e-10)
    assert len(rv) == int(2 * it) + 1


def test_oracle_pgmresDR_first_cycle_is_pgmres(system):
    """One cycle of GMRES-DR is plain GMRES(restart) with one-pass CGS."""
    p, G, idx, A, prec, b = system
    _, _, _, _, rv = ov.pgmresDR(A, b, 15, 1e-30, 0, 4)
    _, _, _, _, rv0 = ov.pgmres(A, b, 15, 1e-30, 1)
    assert np.allclose(rv, rv0, rtol=1e-8, atol=0)


@pytest.mark.gpu
def test_device_pgmresDR_matches_oracle(system):
    p, G, idx, A, prec, b = system
    op = vb.Operator(p.Mop(), p.Gram, idx, G=G)
    pc = vb.Preconditioner.level1(op, G, p.e_r)
    for kw, okw in (({}, {}), ({"L1": pc}, {"L1": prec}), ({"R1": pc}, {"R1": prec})):
        x, flag, relres, it, rv = vb.pgmresDR(op, b, 10, 1e-8, 60, 4, **kw)
        xo, fo, ro, ito, rvo = ov.pgmresDR(A, b, 10, 1e-8, 60, 4, **okw)
        assert flag == fo and list(it) == list(ito) and len(rv) == len(rvo)
        assert np.allclose(rv, rvo, rtol=1e-6, atol=1e-14)
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8
        assert abs(relres - ro) <= 1e-3 * ro
    pc.close()
    op.close()


@pytest.mark.gpu
def test_device_bicgstab_matches_oracle(system):
    p, G, idx, A, prec, b = system
    op = vb.Operator(p.Mop(), p.Gram, idx, G=G)
    pc = vb.Preconditioner.level1(op, G, p.e_r)
    for M, Mo in ((None, None), (pc, prec)):
        x, flag, relres, it, rv = vb.bicgstab(op, b, 1e-8, 300, M=M)
        xo, fo, ro, ito, rvo = ov.bicgstab(A, b, 1e-8, 300, M=Mo)
        # BiCGStab's residual is not monotone: rounding can move the step at
        # which it first crosses tol by a half step or so
        assert flag == fo == 0 and abs(it - ito) <= 1.0
        k = min(len(rv), len(rvo), 20)
        assert np.allclose(rv[:k], rvo[:k], rtol=1e-6, atol=0)
        assert relres <= 1e-8
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-6
    pc.close()
    op.close()
