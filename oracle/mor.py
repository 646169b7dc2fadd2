"""CPU restatement of the reference's reduced-order wavelength sweep (TEST
INFRASTRUCTURE ONLY: the checker for voxphoton_b200.mor; only ``tests/`` may
import it).

Follows Bragg_MOR_script.m:84-142 (node solves, per-node Arnoldi on the
derivative operator, economy SVD of the stacked bases, projected operators)
and example_Bragg_1500nm_to_1600nm.m:85-100 (reduced solve per wavelength),
with lagrange_int.m:1-12 and lagrange_int_deriv.m:1-21 for the wavelength
interpolation of fN.  MATLAB's built-in unrestarted ``gmres(A, b, [], tol,
1000, M)`` is the oracle's pgmres with a restart long enough not to restart
on the small test problems and the same left preconditioner handle.

Parity status: the reference ships no reduced-model outputs, so this module
is pinned through its parts (the oracle matvec, preconditioner and pgmres,
each checked elsewhere) and by properties: Lagrange weights reproduce
polynomials of degree < nG and their derivatives, and the reduced solution at
a node wavelength reproduces that node's solve (Galerkin projection onto a
space that contains it).
"""
from __future__ import annotations

import numpy as np

from . import vie as ov


def lagrange_int(fN, S, s):
    """lagrange_int.m:1-12: sum_i l_i(S) fN{i}."""
    n = len(s)
    P = 0
    for i in range(n):
        L = 1.0
        for j in range(n):
            if j != i:
                L = L * (S - s[j]) / (s[i] - s[j])
        P = P + L * fN[i]
    return P


def lagrange_int_deriv(fN, S, s):
    """lagrange_int_deriv.m:1-21: sum_i l_i'(S) fN{i}."""
    n = len(s)
    P = 0
    for i in range(n):
        L = 0.0
        for j in range(n):
            if j != i:
                Ld = 1.0
                for k in range(n):
                    if k != i and k != j:
                        Ld = Ld * (S - s[k]) / (s[i] - s[k])
                L = L + 1.0 / (s[i] - s[j]) * Ld
        P = P + L * fN[i]
    return P


def _gmres(A, b, tol, M, restart):
    """gmres(A, b, [], tol, 1000, M): left-preconditioned, not restarted."""
    x, flag, relres, it, rv = ov.pgmres(A, b, restart, tol, 1, L1=M)
    return x, flag, len(rv)


def mor_basis(MVP_A, prec_A, MVP_E, VRHS, order, tol, restart=400):
    """Bragg_MOR_script.m:84-125: xSol{iG} and the Arnoldi bases V{iG}.
    MVP_A, prec_A, MVP_E: per-node callables; VRHS: per-node right-hand sides.
    Returns (xSol, V, H, iterations)."""
    nG = len(MVP_A)
    xSol, V, H, its = [], [], [], []
    for iG in range(nG):
        x, _, k = _gmres(MVP_A[iG], VRHS[iG], tol, prec_A[iG], restart)
        xSol.append(x)
        its.append(k)
    numIt = order - 1
    for iG in range(nG):
        b = xSol[iG]
        Vt = np.zeros((b.size, numIt + 1), dtype=complex)
        h = np.zeros((numIt + 1, max(numIt, 1)), dtype=complex)
        Vt[:, 0] = b / np.linalg.norm(b)
        for n in range(1, numIt + 1):
            if n % 2 == 1:
                v_temp = -MVP_E[iG](Vt[:, n - 1])
            else:
                v_temp = MVP_E[iG](Vt[:, n - 1])
            v, _, k = _gmres(MVP_A[iG], v_temp, tol, prec_A[iG], restart)
            its.append(k)
            for j in range(n):
                h[j, n - 1] = np.vdot(Vt[:, j], v)
                v = v - h[j, n - 1] * Vt[:, j]
            h[n, n - 1] = np.linalg.norm(v)
            Vt[:, n] = v / h[n, n - 1]
        V.append(Vt)
        H.append(h)
    return xSol, V, H, its


def mor_project(V, MVP_A):
    """Bragg_MOR_script.m:127-142: P = U of svd([V{1} ... V{nG}], 0) and
    Q{iG} = P' * MVP_A{iG}(P)."""
    P = np.concatenate(V, axis=1)
    U, _, _ = np.linalg.svd(P, full_matrices=False)
    P = U
    Q = []
    for A in MVP_A:
        AP = np.stack([A(P[:, i]) for i in range(P.shape[1])], axis=1)
        Q.append(P.conj().T @ AP)
    return P, Q


def mor_solve(P, Q, s, S, Vrhs):
    """example_Bragg_1500nm_to_1600nm.m:97-100: x = P * (lagrange_int(Q,S,s) \\ (P' Vrhs))."""
    RHS = P.conj().T @ Vrhs
    x_temp = np.linalg.solve(lagrange_int(Q, S, s), RHS)
    return P @ x_temp, x_temp
