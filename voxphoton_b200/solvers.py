"""The reference's other Krylov drivers on device vectors: GMRES with deflated
restarting (pgmresDR.m:73-282, pgmresDR_iter.m:22-142, getHarmVecs1.m,
getHarmVecs2.m) and BiCGStab (the built-in bicgstab that
JVIE_Solver_const.m:470-504 calls).

Both keep every n-vector in device memory in complex128, as the reference
solves in double precision: products with A and the preconditioner are
libvox's device matvec (vox_mv_AN_device) and preconditioner
(vox_precond_apply_device); inner products and block updates are
vox_block_dot / vox_block_update (FP64 sums in a fixed order).  The small
dense algebra of each cycle (least squares, harmonic Ritz eigenproblems, QR)
is FP64 numpy/scipy on the host, of the size the reference hands to MATLAB.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import check, lib
from .mor import _ptr, _stream, block_dot, block_update, device_stream


def _torch():
    import torch
    return torch


class _DeviceOps:
    """y = L1 A R1 x on (1, n) complex128 CUDA rows."""

    def __init__(self, A, L1=None, R1=None, L2=None, R2=None):
        if L2 is not None or R2 is not None:
            raise NotImplementedError("second preconditioners (L2, R2) are not supported")
        for pc in (L1, R1):
            if pc is not None and getattr(pc, "handle", None) is None:
                raise TypeError("preconditioners are Preconditioner handles")
        self.A, self.L1, self.R1 = A, L1, R1
        torch = _torch()
        self.dev = torch.device("cuda", A.device)
        self.n = A.n
        self._tmp = torch.empty((1, self.n), dtype=torch.complex128, device=self.dev)

    def pc(self, pc, x, out):
        check(lib().vox_precond_apply_device(pc.handle, _ptr(x), _ptr(out), _stream(x)))
        return out

    def mv(self, x, out):
        check(lib().vox_mv_AN_device(self.A.handle, 0, _lib.VOX_C128, _ptr(x), _ptr(out),
                                     _stream(x)))
        return out

    def step(self, x, out):
        """out = L1 A R1 x (pgmresDR_iter.m:60-96 without L2/R2)."""
        src = x
        if self.R1 is not None:
            src = self.pc(self.R1, x, self._tmp)
        if self.L1 is not None:
            mid = _torch().empty_like(out)
            self.mv(src, mid)
            return self.pc(self.L1, mid, out)
        return self.mv(src, out)

    def right(self, x):
        if self.R1 is None:
            return x
        out = _torch().empty_like(x)
        return self.pc(self.R1, x, out)

    def left(self, x):
        if self.L1 is None:
            return x
        out = _torch().empty_like(x)
        return self.pc(self.L1, x, out)


def _norm(v):
    return float(np.sqrt(block_dot(v, v).real.item()))


def _scaled(v, s, out):
    """out = s v for (1, n) rows."""
    return block_update(v, np.array([[s]], dtype=np.complex128), out)


def _cat_dot(blocks, v):
    """[B1; B2; ...]^H v for row blocks (the reference's [C V]' * r)."""
    return np.concatenate([block_dot(b, v).cpu().numpy() for b in blocks if b.shape[0] > 0])


def _cat_update(blocks, W, Y, beta):
    """Y = beta Y + [B1 B2 ...] W (W split by the blocks' row counts)."""
    i = 0
    for b in blocks:
        k = b.shape[0]
        if k == 0:
            continue
        block_update(b, W[i:i + k], Y, beta=beta)
        beta = 1.0
        i += k
    return Y


def pgmresDR_iter(ops, r, m, C, tol):
    """pgmresDR_iter.m:22-142 on device rows: Arnoldi on (I - C C') L A R from
    r with one-pass classical Gram-Schmidt.  Returns (V, H, B, k, resvec), V
    a (k+1, n) device block, H / B host arrays."""
    torch = _torch()
    n = ops.n
    V = torch.empty((m + 1, n), dtype=torch.complex128, device=r.device)
    rn = _norm(r)
    _scaled(r, 1.0 / rn, V[0:1])
    kc = 0 if C is None else C.shape[0]
    B = np.zeros((kc, m), dtype=complex)
    H = np.zeros((m + 1, m), dtype=complex)
    resvec = np.zeros(m)
    w = torch.empty((1, n), dtype=torch.complex128, device=r.device)
    for k in range(1, m + 1):
        ops.step(V[k - 1:k], w)
        if kc:
            bk = block_dot(C, w)
            block_update(C, -bk, w, beta=1.0)
            B[:, k - 1] = bk.cpu().numpy()[:, 0]
        h = block_dot(V[:k], w)
        block_update(V[:k], -h, w, beta=1.0)
        H[:k, k - 1] = h.cpu().numpy()[:, 0]
        H[k, k - 1] = _norm(w)
        _scaled(w, 1.0 / H[k, k - 1].real, V[k:k + 1])
        rhs = np.zeros(k + 1, dtype=complex)
        rhs[0] = rn
        y = np.linalg.lstsq(H[:k + 1, :k], rhs, rcond=None)[0]
        resvec[k - 1] = np.linalg.norm(rhs - H[:k + 1, :k] @ y)
        if resvec[k - 1] < tol:
            return V[:k + 1], H[:k + 1, :k], B[:, :k], k, resvec[:k]
    return V, H, B, m, resvec


def _harm_vecs1(m, k, H):
    """getHarmVecs1.m: the k harmonic Ritz vectors of smallest magnitude."""
    Hm = H[:m, :]
    T = np.linalg.solve(Hm.conj().T, np.eye(m))
    T[:m, :m - 1] = 0
    T = Hm + H[m, m - 1] ** 2 * T
    vals, vecs = np.linalg.eig(T)
    return vecs[:, np.argsort(np.abs(vals), kind="stable")][:, :k]


def _harm_vecs2(m, k, H2, CU, VU):
    """getHarmVecs2.m with C'U and V'U computed on the device."""
    import scipy.linalg
    Bm = H2.conj().T @ H2
    W = np.zeros((m + 1, m), dtype=complex)
    W[:k, :k] = CU
    W[k:m + 1, :k] = VU
    W[k:m, k:m] = np.eye(m - k)
    vals, vecs = scipy.linalg.eig(H2.conj().T @ W, Bm)
    return vecs[:, np.argsort(np.abs(vals), kind="stable")][:, m - k:m]


def pgmresDR(A, b, restart=None, tol=None, maxit=None, ritz=None, L1=None, L2=None, R1=None,
             R2=None, x0=None):
    """[x, flag, relres, iter, resvec] = pgmresDR(A, b, restart, tol, maxit,
    ritz, L1, L2, R1, R2, x0) (pgmresDR.m:73-282) with A an Operator and
    L1 / R1 Preconditioner handles, all vectors on the device in complex128.
    b and x0 may be host arrays or (n,) complex128 CUDA tensors; x is
    returned as a host array."""
    torch = _torch()
    with device_stream(torch.device("cuda", A.device), (A,)):
        return _pgmresDR(A, b, restart, tol, maxit, ritz, L1, L2, R1, R2, x0)


def _pgmresDR(A, b, restart, tol, maxit, ritz, L1, L2, R1, R2, x0):
    torch = _torch()
    restart = 50 if restart is None else int(restart)
    tol = 1e-3 if tol is None else float(tol)
    maxit = 10 if maxit is None else int(maxit)
    ritz = min(10, round(restart / 2)) if ritz is None else min(int(ritz), restart - 1)
    ops = _DeviceOps(A, L1, R1, L2, R2)
    n = ops.n
    dev = ops.dev
    bd = torch.as_tensor(np.asarray(b) if not torch.is_tensor(b) else b,
                         dtype=torch.complex128).to(dev).reshape(1, n)
    x0d = None if x0 is None else torch.as_tensor(
        np.asarray(x0) if not torch.is_tensor(x0) else x0,
        dtype=torch.complex128).to(dev).reshape(1, n)
    r = bd.clone()
    if x0d is not None:
        ax = ops.mv(x0d, torch.empty_like(bd))
        r -= ax
    bp = bd
    if L1 is not None:
        r = ops.left(r)
        bp = ops.left(bd)
    bnorm = _norm(bp)
    resvec = np.zeros(restart * (maxit + 1) + 1)
    it = 0
    outit = 0
    resvec[it] = _norm(r) / bnorm
    V, H, _, p, rv = pgmresDR_iter(ops, r, restart, None, tol * bnorm)
    resvec[it + 1:it + 1 + p] = rv / bnorm
    it += p
    y = np.linalg.lstsq(H, block_dot(V, r).cpu().numpy()[:, 0], rcond=None)[0]
    x = block_update(V[:p], y[:, None])
    block_update(V, -(H @ y)[:, None], r, beta=1.0)
    U = C = None
    if resvec[it] > tol:
        P = _harm_vecs1(p, p - 1 if ritz > p - 1 else ritz, H)
        U = block_update(V[:p], P)
        Cq, R = np.linalg.qr(H @ P)
        C = block_update(V, Cq)
        U = block_update(U, np.linalg.inv(R))                  # U / R
    while resvec[it] > tol and outit < maxit:
        outit += 1
        V, H, B, p, rv = pgmresDR_iter(ops, r, restart, C, tol * bnorm)
        resvec[it + 1:it + 1 + p] = rv / bnorm
        it += p
        k = U.shape[0]
        d = np.sqrt(np.real(np.diag(block_dot(U, U).cpu().numpy())))
        D = np.diag(1.0 / d)
        U = block_update(U, D.astype(complex))
        H2 = np.zeros((k + H.shape[0], k + H.shape[1]), dtype=complex)
        H2[:k, :k] = D
        H2[:k, k:] = B
        H2[k:, k:] = H
        y = np.linalg.lstsq(H2, _cat_dot([C, V], r)[:, 0], rcond=None)[0]
        _cat_update([U, V[:p]], y[:, None], x, beta=1.0)
        _cat_update([C, V], -(H2 @ y)[:, None], r, beta=1.0)
        if resvec[it] > tol:
            CU = block_dot(C, U).cpu().numpy()
            VU = block_dot(V, U).cpu().numpy()
            P = _harm_vecs2(p + k, k, H2, CU, VU)
            Unew = torch.empty((k, n), dtype=torch.complex128, device=dev)
            _cat_update([U, V[:p]], P, Unew, beta=0.0)
            Q, R = np.linalg.qr(H2 @ P)
            Cnew = torch.empty((k, n), dtype=torch.complex128, device=dev)
            _cat_update([C, V], Q, Cnew, beta=0.0)
            C = Cnew
            U = block_update(Unew, np.linalg.inv(R))
    x = ops.right(x)
    if x0d is not None:
        x = x + x0d
    resvec = resvec[:it + 1]
    ax = ops.mv(x, torch.empty_like(x))
    relres = _norm(bd - ax) / _norm(bd)
    flag = 0 if relres <= tol else 1
    return x.reshape(-1).cpu().numpy(), flag, relres, [p, outit], resvec


def bicgstab(A, b, tol=1e-6, maxit=20, M=None, x0=None):
    """[x, flag, relres, iter, resvec] = bicgstab(A, b, tol, maxit, M) on the
    device in complex128: the published preconditioned BiCGStab (van der
    Vorst 1992) that MATLAB's built-in implements, M applied as M \\ v (a
    Preconditioner handle).  The residual is tested after each half step;
    resvec holds ||r|| per half step; flag 0 converged, 1 maxit reached,
    4 breakdown."""
    torch = _torch()
    with device_stream(torch.device("cuda", A.device), (A,)):
        return _bicgstab(A, b, tol, maxit, M, x0)


def _bicgstab(A, b, tol, maxit, M, x0):
    torch = _torch()
    ops = _DeviceOps(A)
    n = ops.n
    dev = ops.dev
    row = lambda: torch.empty((1, n), dtype=torch.complex128, device=dev)
    bd = torch.as_tensor(np.asarray(b) if not torch.is_tensor(b) else b,
                         dtype=torch.complex128).to(dev).reshape(1, n)
    nb = _norm(bd)
    x = torch.zeros_like(bd)
    r = bd.clone()
    if x0 is not None:
        x = torch.as_tensor(np.asarray(x0) if not torch.is_tensor(x0) else x0,
                            dtype=torch.complex128).to(dev).reshape(1, n).clone()
        r -= ops.mv(x, row())
    rt = r.clone()
    resvec = [_norm(r)]

    def relres_of(x):
        return _norm(bd - ops.mv(x, row())) / nb

    def out(flag, it):
        return x.reshape(-1).cpu().numpy(), flag, relres_of(x), it, np.array(resvec)

    if resvec[0] <= tol * nb:
        return out(0, 0.0)
    precond = (lambda v: ops.pc(M, v, row())) if M is not None else (lambda v: v)
    dot = lambda a, c: complex(block_dot(a, c).item())
    rho_prev = alpha = omega = 1.0
    p = torch.zeros_like(bd)
    v = torch.zeros_like(bd)
    for i in range(1, maxit + 1):
        rho = dot(rt, r)
        if rho == 0:
            return out(4, i - 1.0)
        if i == 1:
            p = r.clone()
        else:
            beta = (rho / rho_prev) * (alpha / omega)
            p = r + beta * (p - omega * v)
        ph = precond(p)
        v = ops.mv(ph, row())
        alpha = rho / dot(rt, v)
        s = r - alpha * v
        x = x + alpha * ph
        resvec.append(_norm(s))
        if resvec[-1] <= tol * nb:
            return out(0, i - 0.5)
        sh = precond(s)
        t = ops.mv(sh, row())
        tt = dot(t, t)
        if tt == 0:
            return out(4, i - 0.5)
        omega = dot(t, s) / tt
        x = x + omega * sh
        r = s - omega * t
        resvec.append(_norm(r))
        if resvec[-1] <= tol * nb:
            return out(0, float(i))
        if omega == 0:
            return out(4, float(i))
        rho_prev = rho
    rr = relres_of(x)
    return x.reshape(-1).cpu().numpy(), 0 if rr <= tol else 1, rr, float(maxit), np.array(resvec)
