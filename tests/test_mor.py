"""Reduced-order wavelength sweep (Bragg_MOR_script.m:84-142 and the sweep loop
of example_Bragg_1500nm_to_1600nm.m:85-100): the oracle's restatement pinned
by properties on the CPU, the device block kernels against numpy, and the
device ReducedModel against the oracle on a small grating."""
import numpy as np
import pytest

import voxphoton_b200 as vb
from oracle import mor as om
from oracle import vie as ov
from voxphoton_b200 import geometry as geo
from voxphoton_b200 import mor
from voxphoton_b200._lib import PREC, check, lib
from voxphoton_b200.serving import legendre_nodes

BAND = (1500e-9, 1600e-9)
TOL = 1e-10


def small_grating():
    return geo.bragg(periods=4, len_abs=0.4e-6, res=40e-9, height=120e-9)


def test_lagrange_weights_reproduce_polynomials():
    rng = np.random.default_rng(0)
    s = legendre_nodes(*BAND, 5)
    c = rng.standard_normal(5)
    x0 = 1550e-9
    poly = lambda S: sum(c[k] * ((S - x0) / 50e-9) ** k for k in range(5))
    dpoly = lambda S: sum(k * c[k] * ((S - x0) / 50e-9) ** (k - 1) / 50e-9 for k in range(1, 5))
    vals = [poly(si) for si in s]
    for S in (1500e-9, 1523.4e-9, 1550e-9, s[1], 1600e-9):
        assert np.isclose(om.lagrange_int(vals, S, s), poly(S), rtol=1e-10, atol=1e-12)
        assert np.isclose(om.lagrange_int_deriv(vals, S, s), dpoly(S), rtol=1e-8,
                          atol=1e-6 * np.abs(dpoly(S)).max())
        # the package's weights are the same loops
        assert np.allclose(mor.lagrange_weights(S, s) @ vals, om.lagrange_int(vals, S, s),
                           rtol=1e-14, atol=0)
        assert np.allclose(mor.lagrange_deriv_weights(S, s) @ vals,
                           om.lagrange_int_deriv(vals, S, s), rtol=1e-12, atol=0)
    # weights at a node are the unit vector there
    assert np.array_equal(mor.lagrange_weights(s[2], s), np.eye(5)[2])


class OracleSweep:
    """The oracle's reduced model of the small grating: nG nodes, `order`
    vectors per node, per-node level-1 preconditioners as the script."""

    def __init__(self, nG=3, order=3, tol=TOL):
        p = small_grating()
        self.p = p
        self.s = legendre_nodes(*BAND, nG)
        self.idx = p.idxS3()
        self.Mop = p.Mop()
        ones = np.ones(p.shape)
        self.G = [vb.assemble_toeplitz(p.shape, p.with_wavelength(l).ko, p.res) for l in self.s]
        self.fN = [ov.fN_from_toeplitz(G) for G in self.G]
        Gram = p.Gram
        idx, Mop = self.idx, self.Mop
        L, M, N = p.shape

        def A_of(f):
            return lambda J: ov.mv_AN_const(J, f, ones, Mop, Gram, "notransp", idx)

        face3 = ov.face_from_Mr(p.e_r)
        self.MVP_A = [A_of(f) for f in self.fN]
        fNd = [om.lagrange_int_deriv(self.fN, si, self.s) for si in self.s]
        self.MVP_E = [lambda J, f=f: A_of(f)(J) - Gram * J for f in fNd]
        self.prec = []
        for G in self.G:
            circ, _ = ov.level_1_parallel_func_N(G, L, M, N, Gram)
            blocks = ov.level1_inverse_blocks(circ, face3, Gram)
            self.prec.append(lambda J, b=blocks: ov.chan_mvp_idx(b, J, L, M, N, idx))
        self.VRHS = [self.rhs(l) for l in self.s]
        self.xSol, self.V, self.H, self.its = om.mor_basis(self.MVP_A, self.prec, self.MVP_E,
                                                           self.VRHS, order, tol)
        self.P, self.Q = om.mor_project(self.V, self.MVP_A)

    def rhs(self, lam):
        pl = self.p.with_wavelength(lam)
        return ov.jvie2_system(geo.plane_wave(pl), pl.e_r, pl.Gram, pl.freq)[3]

    def direct(self, lam, tol=1e-12):
        """The full solve with the interpolated operator lagrange_int(fN, S, s)."""
        f = om.lagrange_int(self.fN, lam, self.s)
        A = lambda J: ov.mv_AN_const(J, f, np.ones(self.p.shape), self.Mop, self.p.Gram,
                                     "notransp", self.idx)
        x, flag, *_ = ov.pgmres(A, self.rhs(lam), 400, tol, 1, L1=self.prec[len(self.s) // 2])
        return x


@pytest.fixture(scope="module")
def oracle_sweep():
    return OracleSweep()


def test_oracle_basis_is_orthonormal_and_spans_the_node_solutions(oracle_sweep):
    o = oracle_sweep
    P = o.P
    assert np.allclose(P.conj().T @ P, np.eye(P.shape[1]), atol=1e-12)
    for x in o.xSol:
        assert np.linalg.norm(x - P @ (P.conj().T @ x)) / np.linalg.norm(x) < 1e-12
    for Vt in o.V:
        assert np.allclose(Vt.conj().T @ Vt, np.eye(Vt.shape[1]), atol=1e-12)


def test_oracle_reduced_solution_reproduces_node_solves(oracle_sweep):
    o = oracle_sweep
    for i, S in enumerate(o.s):
        x, _ = om.mor_solve(o.P, o.Q, o.s, S, o.VRHS[i])
        assert np.linalg.norm(x - o.xSol[i]) / np.linalg.norm(o.xSol[i]) < 1e-7


def test_oracle_reduced_solution_between_nodes(oracle_sweep):
    """Between the nodes the reduced model is an approximation: on this
    grating it stays within 1e-3 of the full solve of the interpolated
    operator."""
    o = oracle_sweep
    for S in (1512e-9, 1547e-9, 1589e-9):
        x, _ = om.mor_solve(o.P, o.Q, o.s, S, o.rhs(S))
        xd = o.direct(S)
        assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-3


@pytest.mark.gpu
def test_block_kernels_match_numpy():
    import torch
    rng = np.random.default_rng(3)
    for n, a, b in ((1, 1, 1), (1000, 25, 25), (4097, 32, 7), (70001, 5, 40), (333, 40, 33)):
        Xh = rng.standard_normal((a, n)) + 1j * rng.standard_normal((a, n))
        Yh = rng.standard_normal((b, n)) + 1j * rng.standard_normal((b, n))
        X = torch.from_numpy(Xh).cuda()
        Y = torch.from_numpy(Yh).cuda()
        C = mor.block_dot(X, Y).cpu().numpy()
        ref = Xh.conj() @ Yh.T
        assert np.abs(C - ref).max() <= 1e-12 * np.abs(ref).max()
        assert np.array_equal(C, mor.block_dot(X, Y).cpu().numpy())   # fixed order
        W = rng.standard_normal((a, b)) + 1j * rng.standard_normal((a, b))
        Z = mor.block_update(X, W).cpu().numpy()
        assert np.allclose(Z, (Xh.T @ W).T, rtol=1e-12, atol=1e-12 * np.abs(Z).max())
        Y2 = mor.block_update(X, W, Y.clone(), beta=-0.5).cpu().numpy()
        assert np.allclose(Y2, -0.5 * Yh + (Xh.T @ W).T, rtol=1e-12,
                           atol=1e-12 * np.abs(Y2).max())
    # strided block views (rows of a wider array)
    Xh = rng.standard_normal((6, 3000)) + 1j * rng.standard_normal((6, 3000))
    X = torch.from_numpy(Xh).cuda()
    C = mor.block_dot(X[::2, :2500], X[1::2, :2500]).cpu().numpy()
    assert np.allclose(C, Xh[::2, :2500].conj() @ Xh[1::2, :2500].T, rtol=1e-12, atol=1e-10)


@pytest.mark.gpu
def test_batched_matvec_matches_each_member_alone(oracle_sweep):
    import torch
    o = oracle_sweep
    p = o.p
    nodes = [vb.Operator(o.Mop, p.Gram, o.idx, G=G) for G in o.G]
    opB = vb.Operator(o.Mop, p.Gram, o.idx, G=o.G[0], members=len(nodes))
    for i in range(len(nodes)):
        opB.interp(nodes, np.eye(len(nodes))[i], member=i)
    rng = np.random.default_rng(4)
    n = o.idx.size
    xh = rng.standard_normal((len(nodes), n)) + 1j * rng.standard_normal((len(nodes), n))
    x = torch.from_numpy(xh).cuda()
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    check(lib().vox_mv_AN_batch_device(opB.handle, 0, PREC["c128"], len(nodes),
                                       mor._ptr(x), mor._ptr(y), None))
    torch.cuda.synchronize()
    yb = y.cpu().numpy()
    for i, op in enumerate(nodes):
        solo = op.mv_AN(xh[i])
        assert np.array_equal(yb[i], solo)
        ref = o.MVP_A[i](xh[i])
        assert np.linalg.norm(solo - ref) / np.linalg.norm(ref) < 1e-12
    for op in nodes + [opB]:
        op.close()


@pytest.mark.gpu
def test_reduced_model_matches_oracle(oracle_sweep):
    o = oracle_sweep
    p = o.p
    nodes = [vb.Operator(o.Mop, p.Gram, o.idx, G=G) for G in o.G]
    pc = vb.Preconditioner.level1(nodes[len(nodes) // 2], o.G[len(nodes) // 2], p.e_r)
    rm = mor.ReducedModel(nodes, o.s, o.Mop, p.Gram, o.idx, o.G[0], np.array(o.VRHS), pc=pc,
                          order=3, tol=TOL, inner_tol=1e-3, maxit_inner=40)
    assert all(i.flag == 0 for info in rm.infos for i in info)
    # node solutions within the solve tolerance of the oracle's
    xs = rm.xSol.cpu().numpy()
    for i in range(len(nodes)):
        assert np.linalg.norm(xs[i] - o.xSol[i]) / np.linalg.norm(o.xSol[i]) < 1e-7
    # the same span: the oracle's basis lies in the device's
    P = rm.P.cpu().numpy().T
    assert P.shape == o.P.shape
    assert np.allclose(P.conj().T @ P, np.eye(P.shape[1]), atol=1e-12)
    assert np.linalg.norm(o.P - P @ (P.conj().T @ o.P)) < 1e-6
    # reduced solutions at and between the nodes
    lams = np.array([o.s[0], 1512e-9, 1547e-9, o.s[1], 1589e-9])
    B = np.array([o.rhs(l) for l in lams])
    X, _ = rm.solve(lams, B)
    X = X.cpu().numpy()
    for c, S in enumerate(lams):
        xo, _ = om.mor_solve(o.P, o.Q, o.s, S, B[c])
        assert np.linalg.norm(X[c] - xo) / np.linalg.norm(xo) < 1e-6
    rm.close()
    pc.close()
    for op in nodes:
        op.close()
