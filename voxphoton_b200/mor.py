"""Reduced-order model of a wavelength sweep, built and evaluated on the device
(Bragg_MOR_script.m:1-142, example_Bragg_1500nm_to_1600nm.m:77-114,
lagrange_int.m:1-12, lagrange_int_deriv.m:1-21).

The reference solves the JVIE-II system at nG Legendre wavelengths s_i, grows
at each node an Arnoldi basis of `order` vectors whose new directions are
solves against the wavelength derivative of the operator
(MVP_E{i} = mv_AN(., fN'(s_i)) - Gram, with fN' the derivative of the
Lagrange interpolant of fN), puts the nG * order vectors side by side as P,
orthonormalises P by an economy SVD, projects Q{i} = P' A_i P, and then, for
every wavelength S of the sweep, solves only the small system
lagrange_int(Q, S, s) x = P' Vrhs(S) and lifts x back with P.

Here the nG node systems are the members of batched operators: the first
solves, every derivative product, every Arnoldi solve and every projection
product run for all nodes in one launch (vox_mv_AN_batch_device,
vox_solve_refined_batch_device).  The tall-skinny products P' Y and P X use
vox_block_dot / vox_block_update (FP64 sums in a fixed order); the dense
work of size nG * order (eigen-decomposition, the reduced solves) is FP64
numpy on the host, as small as the reference's.

Basis: the reference's `[U,S,V] = svd(P,0); P = U` keeps every direction.
The reduced solution P (P'AP)^-1 P' b depends only on the span of P, so any
orthonormal basis of that span gives it; this one is P W with W from the
eigen-decomposition of P'P, taken twice (the second pass restores
orthogonality lost to rounding), dropping directions whose singular value is
below `rank_tol` times the largest (numerically absent from the span).
"""

from __future__ import annotations

import contextlib
import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib
from .vie import Operator

__all__ = ["lagrange_weights", "lagrange_deriv_weights", "block_dot", "block_update",
           "ReducedModel"]


def lagrange_weights(S, s):
    """lagrange_int.m:1-12: weights l_i(S) of the Lagrange basis on nodes s."""
    s = np.asarray(s, dtype=float)
    w = np.ones(s.size)
    for i in range(s.size):
        for j in range(s.size):
            if j != i:
                w[i] *= (S - s[j]) / (s[i] - s[j])
    return w


def lagrange_deriv_weights(S, s):
    """lagrange_int_deriv.m:1-21: weights l_i'(S), same loop order."""
    s = np.asarray(s, dtype=float)
    n = s.size
    w = np.zeros(n)
    for i in range(n):
        acc = 0.0
        for j in range(n):
            if j != i:
                ld = 1.0
                for k in range(n):
                    if k != i and k != j:
                        ld *= (S - s[k]) / (s[i] - s[k])
                acc += ld / (s[i] - s[j])
        w[i] = acc
    return w


def _torch():
    import torch
    return torch


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(t):
    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


@contextlib.contextmanager
def device_stream(dev, ops=()):
    """Run the enclosed torch work and libvox calls in order on one CUDA
    stream: torch's current stream when it is a created stream, else a new
    side stream ordered after it (libvox's operators run on non-blocking
    streams, which the legacy default stream does not order against).  The
    operators in `ops` are pointed at that stream for the duration."""
    torch = _torch()
    cur = torch.cuda.current_stream(dev)
    s = cur if cur.cuda_stream != 0 else torch.cuda.Stream(device=dev)
    if s is not cur:
        s.wait_stream(cur)
    prev = [getattr(op, "stream_ptr", 0) for op in ops]
    try:
        with torch.cuda.stream(s):
            for op in ops:
                op.set_stream(s.cuda_stream)
            yield s
    finally:
        for op, p in zip(ops, prev):
            op.set_stream(p)
        if s is not cur:
            cur.wait_stream(s)


def _block(t):
    """A (cols, n) complex128 CUDA tensor whose rows are the block's columns."""
    torch = _torch()
    if t.dtype != torch.complex128 or not t.is_cuda or t.dim() != 2 or t.stride(1) != 1:
        raise ValueError("blocks are (columns, n) complex128 CUDA tensors, rows contiguous")
    return t


def block_dot(X, Y):
    """X^H Y for blocks X (a, n) and Y (b, n): an (a, b) complex128 CUDA tensor
    (vox_block_dot; more than 32 columns are done 32 at a time)."""
    torch = _torch()
    X, Y = _block(X), _block(Y)
    a, n = X.shape
    b = Y.shape[0]
    if Y.shape[1] != n:
        raise ValueError("blocks differ in length")
    C = torch.empty((a, b), dtype=torch.complex128, device=X.device)
    for i0 in range(0, a, 32):
        i1 = min(a, i0 + 32)
        for j0 in range(0, b, 32):
            j1 = min(b, j0 + 32)
            Ct = torch.empty((j1 - j0, i1 - i0), dtype=torch.complex128, device=X.device)
            check(lib().vox_block_dot(n, i1 - i0, j1 - j0, _ptr(X[i0:i1]), X.stride(0),
                                      _ptr(Y[j0:j1]), Y.stride(0), _ptr(Ct), _stream(X)))
            C[i0:i1, j0:j1] = Ct.T
    return C


def block_update(X, W, Y=None, beta=0.0):
    """Y <- beta Y + X W for X (a, n) and W (a, b): returns Y (b, n)
    (vox_block_update; W is moved to the device; more than 32 columns of W
    are done 32 at a time)."""
    torch = _torch()
    X = _block(X)
    a, n = X.shape
    W = torch.as_tensor(np.asarray(W, dtype=np.complex128) if not torch.is_tensor(W) else W,
                        dtype=torch.complex128, device=X.device)
    if W.shape[0] != a:
        raise ValueError("W must have as many rows as X has columns")
    b = W.shape[1]
    if Y is None:
        Y = torch.empty((b, n), dtype=torch.complex128, device=X.device)
        beta = 0.0
    Y = _block(Y)
    for j0 in range(0, b, 32):
        j1 = min(b, j0 + 32)
        for i0 in range(0, a, 32):
            i1 = min(a, i0 + 32)
            # device layout W[i + a j]: the transposed (b, a) tensor, row-major
            Wt = W[i0:i1, j0:j1].T.contiguous()
            bt = beta if i0 == 0 else 1.0
            check(lib().vox_block_update(n, i1 - i0, j1 - j0, _ptr(X[i0:i1]), X.stride(0),
                                         _ptr(Wt), float(bt), _ptr(Y[j0:j1]), Y.stride(0),
                                         _stream(X)))
    return Y


class ReducedModel:
    """Bragg_MOR_script.m:84-142 on batched device operators.

    node_ops: the nG Operators at the node wavelengths ``nodes`` (their member
    0 holds fN(s_i)); Mc, Gram, idx, G: the arguments they were made from (G
    only shapes the batched operators, whose fN are then interpolated from
    node_ops); VRHS: (nG, n) right-hand sides at the nodes; pc: a
    preconditioner of one node operator, shared by every node (the reference
    builds one per node; either only changes iteration counts).

    After construction: ``P`` (r, n) is the orthonormal basis on the device,
    ``Q`` the nG projected operators (r x r, FP64 host), ``xSol`` (nG, n) the
    node solutions, ``infos`` the solves' vox_gmres_info records.
    """

    def __init__(self, node_ops, nodes, Mc, Gram, idx, G, VRHS, pc=None, order=5, tol=1e-4,
                 restart=50, maxit_inner=40, inner_tol=1e-3, side="left", rank_tol=1e-13,
                 device=0):
        torch = _torch()
        nG = len(node_ops)
        if nG < 1 or nG > 8:
            raise ValueError("1..8 node operators")
        self.nodes = np.asarray(nodes, dtype=float)
        self.order = int(order)
        self.Gram = float(Gram)
        self.nG = nG
        dev = torch.device("cuda", device)
        self.opA = Operator(Mc, Gram, idx, G=G, members=nG, device=device)
        self.opE = Operator(Mc, Gram, idx, G=G, members=nG, device=device)
        for i in range(nG):
            e = np.zeros(nG)
            e[i] = 1.0
            self.opA.interp(node_ops, e, member=i)                        # fN{i}
            self.opE.interp(node_ops, lagrange_deriv_weights(self.nodes[i], self.nodes),
                            member=i)                                     # fN_deriv{i}
        self.pc = pc.share(self.opA) if pc is not None else None
        with device_stream(dev, (self.opA, self.opE)):
            self._build(VRHS, dev, side, tol, restart, maxit_inner, inner_tol, rank_tol)

    def _build(self, VRHS, dev, side, tol, restart, maxit_inner, inner_tol, rank_tol):
        torch = _torch()
        nG = self.nG
        pc = self.pc
        n = self.opA.n
        self.n = n
        kw = dict(pc=self.pc, side=side if pc is not None else None, tol=tol, restart=restart,
                  maxit_inner=maxit_inner, inner_tol=inner_tol)
        torch.cuda.synchronize(dev)
        B = torch.as_tensor(VRHS, dtype=torch.complex128).to(dev).contiguous()
        if B.shape != (nG, n):
            raise ValueError(f"VRHS must be ({nG}, {n})")
        self.infos = []
        # xSol{iG} (Bragg_MOR_script.m:86-95)
        X = torch.empty_like(B)
        self.infos.append(self._solve(B, X, kw))
        self.xSol = X
        # Arnoldi at each node (:97-125): V[i, k] is Vtemp(:, k+1) of node i
        V = torch.empty((nG, self.order, n), dtype=torch.complex128, device=dev)
        nrm = torch.linalg.vector_norm(X, dim=1)
        V[:, 0] = X / nrm[:, None]
        T = torch.empty_like(B)
        Y = torch.empty_like(B)
        self.H = np.zeros((nG, self.order, self.order - 1 if self.order > 1 else 1), complex)
        for k in range(1, self.order):
            # v_temp = -/+ MVP_E{i}(Vtemp(:, n)), n = k (1-based): '-' for odd n
            src = V[:, k - 1].contiguous()
            check(lib().vox_mv_AN_batch_device(self.opA_E, 0, _lib.PREC["c128"], nG,
                                               _ptr(src), _ptr(T), _stream(T)))
            T -= self.Gram * src
            if k % 2 == 1:
                T.neg_()
            self.infos.append(self._solve(T, Y, kw))
            for i in range(nG):
                v = Y[i:i + 1]
                for j in range(k):                          # modified Gram-Schmidt
                    h = block_dot(V[i, j:j + 1], v)
                    self.H[i, j, k - 1] = h.item()
                    block_update(V[i, j:j + 1], -h, v, beta=1.0)
                hn = torch.linalg.vector_norm(v).item()
                self.H[i, k, k - 1] = hn
                V[i, k] = v[0] / hn
        self.V = V
        # P = [V{1} ... V{nG}], orthonormalised (:127-132)
        P = V.reshape(nG * self.order, n)
        for _ in range(2):
            P = self._orthonormalise(P, rank_tol)
        self.P = P
        del V, T, Y
        self.V = None
        # Q{iG} = P' A_iG P (:134-142): one batched product per column of P
        r = P.shape[0]
        AP = torch.empty((r, nG, n), dtype=torch.complex128, device=dev)
        rep = torch.empty((nG, n), dtype=torch.complex128, device=dev)
        for c in range(r):
            rep.copy_(P[c].expand(nG, n))
            out = AP[c]
            check(lib().vox_mv_AN_batch_device(self.opA.handle, 0, _lib.PREC["c128"], nG,
                                               _ptr(rep), _ptr(out), _stream(rep)))
        self.Q = []
        for i in range(nG):
            self.Q.append(block_dot(P, AP[:, i]).cpu().numpy())
        del AP, rep
        torch.cuda.synchronize(dev)

    @property
    def opA_E(self):
        return self.opE.handle

    def _solve(self, B, X, kw):
        """The batched refined solve (on the operators' stream, the build's)."""
        return self.opA.solve_refined_batch_device(B.data_ptr(), X.data_ptr(), self.nG, **kw)

    @staticmethod
    def _orthonormalise(P, rank_tol):
        G = block_dot(P, P).cpu().numpy()
        G = 0.5 * (G + G.conj().T)
        lam, U = np.linalg.eigh(G)
        keep = lam > (rank_tol ** 2) * lam.max()
        W = U[:, keep] / np.sqrt(lam[keep])
        W = W[:, ::-1].copy()                     # largest singular value first
        return block_update(P, W)

    @property
    def rank(self):
        return self.P.shape[0]

    def reduced_matrix(self, S):
        """lagrange_int(Q, S, s)."""
        w = lagrange_weights(S, self.nodes)
        return sum(wi * Qi for wi, Qi in zip(w, self.Q))

    def solve(self, lams, Vrhs):
        """example_Bragg_1500nm_to_1600nm.m:97-100 for every wavelength in
        lams: Vrhs is (count, n) on the device (or host); returns the lifted
        solutions P x (count, n) on the device and the reduced coefficients."""
        torch = _torch()
        with device_stream(self.P.device):
            Vrhs = torch.as_tensor(Vrhs, dtype=torch.complex128).to(self.P.device).contiguous()
            R = block_dot(self.P, Vrhs).cpu().numpy()          # RHS = P' Vrhs, (r, count)
            Xt = np.empty_like(R)
            for c, S in enumerate(np.asarray(lams, dtype=float)):
                Xt[:, c] = np.linalg.solve(self.reduced_matrix(S), R[:, c])
            return block_update(self.P, Xt), Xt

    def close(self):
        if self.pc is not None:
            self.pc.close()
            self.pc = None
        for op in (self.opA, self.opE):
            op.close()
        self.P = None
