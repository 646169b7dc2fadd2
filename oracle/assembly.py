"""Oracle for the operator setup: Toeplitz Green-tensor assembly (TEST INFRASTRUCTURE ONLY).

Restates assembly_nop_const.m:1-174 (far / medium / near cubature, DEMCEM
singular corrections, 6x6 face projection) in numpy.  The per-cell face-pair
cubature and the DEMCEM singular integrals are the reference's own C++ cores
(mexcubatures/cubature_nop_const.cpp, direct_ws_{st,ea,va}_const.cpp), compiled
by oracle/Makefile into oracle/_ref/libvoxref.so.  Only tests and the CPU
baseline use this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def ref_lib():
    """Load oracle/_ref/libvoxref.so (built by `make -C oracle`)."""
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_ref", "libvoxref.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/_ref/libvoxref.so missing: run `make -C oracle`")
        lib = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.voxref_cubature_nop.argtypes = [ctypes.c_int, dp, dp, dp, dp, dp, dp,
                                            ctypes.c_double, ctypes.c_double, dp, dp]
        lib.voxref_direct_ws_st.argtypes = [dp, dp, dp, ctypes.c_double, ctypes.c_int, dp, dp, dp]
        lib.voxref_direct_ws_ea.argtypes = [dp, dp, dp, dp, ctypes.c_double, ctypes.c_int, dp, dp, dp]
        lib.voxref_direct_ws_va.argtypes = [dp, dp, dp, dp, dp, ctypes.c_double, ctypes.c_int,
                                            dp, dp, dp]
        lib.voxref_cell_loop.argtypes = [ctypes.c_int] * 7 + [dp, dp, dp, dp, ctypes.c_double,
                                                               ctypes.c_double, dp, dp]
        _LIB = lib
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def gauss_1d(n):
    """gauss_1d.m: Gauss-Legendre on [-1,1]; returns (weight, xtab) like MATLAB."""
    x, w = np.polynomial.legendre.leggauss(n)
    return w, x


def gauss_2d(Np):
    """gauss_2d.m:1-19: tensor rule on [0,1]^2, I outer / J inner, weights / 4."""
    w1, x1 = gauss_1d(Np)
    W = np.outer(w1, w1).reshape(-1) / 4.0
    U = np.repeat((x1 + 1) / 2, Np)
    V = np.tile((x1 + 1) / 2, Np)
    return Np * Np, W, U, V


def cube_faces(dx, dy, dz):
    """cube_faces.m:1-39: R_faces(3,4,6), faces -x,+x,-y,+y,-z,+z."""
    R = np.zeros((3, 4, 6))
    R[:, :, 0] = np.array([[0, 0, 0], [0, dy, 0], [0, dy, dz], [0, 0, dz]]).T
    R[:, :, 1] = np.array([[dx, 0, 0], [dx, dy, 0], [dx, dy, dz], [dx, 0, dz]]).T
    R[:, :, 2] = np.array([[0, 0, 0], [dx, 0, 0], [dx, 0, dz], [0, 0, dz]]).T
    R[:, :, 3] = np.array([[0, dy, 0], [dx, dy, 0], [dx, dy, dz], [0, dy, dz]]).T
    R[:, :, 4] = np.array([[0, 0, 0], [dx, 0, 0], [dx, dy, 0], [0, dy, 0]]).T
    R[:, :, 5] = np.array([[0, 0, dz], [dx, 0, dz], [dx, dy, dz], [0, dy, dz]]).T
    return R


def vector_projection():
    """vector_projection.m:1-25: P(k,l,comp) = (n_k x e_a).(n_l x e_b)."""
    ex, ey, ez = np.eye(3)
    KL = np.array([-ex, ex, -ey, ey, -ez, ez])
    pairs = [(ex, ex), (ex, ey), (ex, ez), (ey, ey), (ey, ez), (ez, ez)]
    P = np.zeros((6, 6, 6))
    for kk in range(6):
        for ll in range(6):
            for c, (a, b) in enumerate(pairs):
                P[kk, ll, c] = np.dot(np.cross(KL[kk], a), np.cross(KL[ll], b))
    return P


_IDX_OBS = np.array([1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 5, 5, 6]) - 1
_IDX_SRC = np.array([1, 2, 3, 4, 5, 6, 1, 3, 4, 5, 6, 3, 4, 5, 6, 3, 5, 6, 5, 6, 5]) - 1
# (dst, src) pairs of the symmetric fill (cubature_nop_sym_near.m:66-84)
_SYM_FILL = [((1, 1), (0, 0)), ((2, 0), (1, 3)), ((2, 1), (0, 3)), ((3, 0), (1, 2)),
             ((3, 1), (0, 2)), ((3, 3), (2, 2)), ((4, 0), (1, 5)), ((4, 1), (0, 5)),
             ((4, 2), (3, 5)), ((4, 3), (2, 5)), ((5, 0), (1, 4)), ((5, 1), (0, 4)),
             ((5, 2), (3, 4)), ((5, 3), (2, 4)), ((5, 5), (4, 4))]


def cubature_nop_sym_near(Np, wp, up, vp, r_m, r_n, R_faces, ko, dx):
    """cubature_nop_sym_near.m:1-88 (numpy; same maths as the C++ far cubature)."""
    I = np.zeros((6, 6), dtype=complex)
    W = np.outer(wp, wp)
    for io, js in zip(_IDX_OBS, _IDX_SRC):
        rp1, rp2, rp4 = R_faces[:, 0, io], R_faces[:, 1, io], R_faces[:, 3, io]
        rq1, rq2, rq4 = R_faces[:, 0, js], R_faces[:, 1, js], R_faces[:, 3, js]
        a_p, b_p = rp2 - rp1, rp4 - rp1
        a_q, b_q = rq2 - rq1, rq4 - rq1
        rrp = rp1[:, None] + np.outer(a_p, up) + np.outer(b_p, vp) + np.asarray(r_m)[:, None]
        rrq = rq1[:, None] + np.outer(a_q, up) + np.outer(b_q, vp) + np.asarray(r_n)[:, None]
        R = np.sqrt(((rrp[:, :, None] - rrq[:, None, :]) ** 2).sum(axis=0))
        # touching panels give R = 0 (Inf/NaN), exactly as in MATLAB; those
        # entries are replaced by the singular values in nearby_correct
        with np.errstate(divide="ignore", invalid="ignore"):
            G = np.exp(-1j * ko * R) / R
            I[io, js] = np.sum(W * G)
    for (d0, d1), (s0, s1) in _SYM_FILL:
        I[d0, d1] = I[s0, s1]
    return dx ** 4 * I


def cubature_nop_ref(Np, wp, up, vp, r_m, r_n, R_faces, ko, dx):
    """The reference C++ core cubature_nop_const.cpp:8-125 (via libvoxref)."""
    lib = ref_lib()
    re = np.zeros(36)
    im = np.zeros(36)
    Rf = _f64(R_faces.reshape(-1, order="F"))
    lib.voxref_cubature_nop(int(Np), _p(_f64(wp)), _p(_f64(up)), _p(_f64(vp)), _p(_f64(r_m)),
                            _p(_f64(r_n)), _p(Rf), float(ko), float(dx), _p(re), _p(im))
    return (re + 1j * im).reshape((6, 6), order="F")


def _st(r1, r2, r3, ko, Np, z, w):
    out = np.zeros(2)
    ref_lib().voxref_direct_ws_st(_p(_f64(r1)), _p(_f64(r2)), _p(_f64(r3)), float(ko), int(Np),
                                  _p(_f64(z)), _p(_f64(w)), _p(out))
    return out[0] + 1j * out[1]


def _ea(r1, r2, r3, r4, ko, Np, z, w):
    out = np.zeros(2)
    ref_lib().voxref_direct_ws_ea(_p(_f64(r1)), _p(_f64(r2)), _p(_f64(r3)), _p(_f64(r4)),
                                  float(ko), int(Np), _p(_f64(z)), _p(_f64(w)), _p(out))
    return out[0] + 1j * out[1]


def _va(r1, r2, r3, r4, r5, ko, Np, z, w):
    out = np.zeros(2)
    ref_lib().voxref_direct_ws_va(_p(_f64(r1)), _p(_f64(r2)), _p(_f64(r3)), _p(_f64(r4)),
                                  _p(_f64(r5)), float(ko), int(Np), _p(_f64(z)), _p(_f64(w)),
                                  _p(out))
    return out[0] + 1j * out[1]


def singular_st_const(Np, ko, dx, dy):
    """singular_st_const.m:22-39 (DEMCEM branch): square = 2 triangles."""
    w, z = gauss_1d(Np)
    r1, r2, r3, r4 = [0, 0, 0], [dx, 0, 0], [dx, dy, 0], [0, dy, 0]
    return (_st(r1, r2, r3, ko, Np, z, w) + _ea(r1, r3, r2, r4, ko, Np, z, w)
            + _ea(r1, r3, r4, r2, ko, Np, z, w) + _st(r1, r3, r4, ko, Np, z, w))


def singular_ea_const(Np, ko, dx, dy, dz):
    """singular_ea_const.m:78-108 (DEMCEM): coplanar (c) and orthogonal (o) edge-adjacent."""
    w, z = gauss_1d(Np)
    r1, r2, r3, r4 = [0, 0, 0], [dx, 0, 0], [dx, dy, 0], [0, dy, 0]
    r5, r6 = [2 * dx, 0, 0], [2 * dx, dy, 0]
    r5o, r6o = [dx, 0, dz], [dx, dy, dz]
    EAc = (_ea(r2, r3, r1, r5, ko, Np, z, w) + _va(r3, r1, r2, r5, r6, ko, Np, z, w)
           + _va(r3, r4, r1, r2, r5, ko, Np, z, w) + _va(r3, r4, r1, r5, r6, ko, Np, z, w))
    EAo = (_ea(r2, r3, r1, r5o, ko, Np, z, w) + _va(r3, r1, r2, r5o, r6o, ko, Np, z, w)
           + _va(r3, r4, r1, r2, r5o, ko, Np, z, w) + _va(r3, r4, r1, r5o, r6o, ko, Np, z, w))
    return EAc, EAo


def singular_va_const(Np, ko, dx, dy, dz):
    """singular_va_const.m:149-173 (DEMCEM): coplanar and orthogonal vertex-adjacent."""
    w, z = gauss_1d(Np)
    r1, r2, r3, r4 = [0, 0, 0], [dx, 0, 0], [dx, dy, 0], [0, dy, 0]
    r5, r6, r7 = [2 * dx, dy, 0], [2 * dx, 2 * dy, 0], [dx, 2 * dy, 0]
    r5o, r6o, r7o = [dx, dy, dz], [dx, 2 * dy, dz], [dx, 2 * dy, 0]
    VAc = (_va(r3, r1, r2, r5, r6, ko, Np, z, w) + _va(r3, r1, r2, r6, r7, ko, Np, z, w)
           + _va(r3, r4, r1, r5, r6, ko, Np, z, w) + _va(r3, r4, r1, r6, r7, ko, Np, z, w))
    VAo = (_va(r3, r1, r2, r5o, r6o, ko, Np, z, w) + _va(r3, r1, r2, r6o, r7o, ko, Np, z, w)
           + _va(r3, r4, r1, r5o, r6o, ko, Np, z, w) + _va(r3, r4, r1, r6o, r7o, ko, Np, z, w))
    return VAc, VAo


def _near_tables(ST, EAc, EAo, VAc, VAo):
    """nearby_correct.m:73-199: (C, P) per near cell; P==1 keeps the cubature."""
    Z = 0.0
    t = {}
    t[(1, 1, 1)] = (
        [[ST, Z, EAo, EAo, EAo, EAo], [Z, ST, EAo, EAo, EAo, EAo], [EAo, EAo, ST, Z, EAo, EAo],
         [EAo, EAo, Z, ST, EAo, EAo], [EAo, EAo, EAo, EAo, ST, Z], [EAo, EAo, EAo, EAo, Z, ST]],
        [[0, 1, 0, 0, 0, 0], [1, 0, 0, 0, 0, 0], [0, 0, 0, 1, 0, 0], [0, 0, 1, 0, 0, 0],
         [0, 0, 0, 0, 0, 1], [0, 0, 0, 0, 1, 0]])
    t[(2, 1, 1)] = (
        [[Z, ST, EAo, EAo, EAo, EAo], [Z] * 6, [Z, EAo, EAc, Z, VAo, VAo],
         [Z, EAo, Z, EAc, VAo, VAo], [Z, EAo, VAo, VAo, EAc, Z], [Z, EAo, VAo, VAo, Z, EAc]],
        [[1, 0, 0, 0, 0, 0], [1] * 6, [1, 0, 0, 1, 0, 0], [1, 0, 1, 0, 0, 0],
         [1, 0, 0, 0, 0, 1], [1, 0, 0, 0, 1, 0]])
    t[(2, 1, 2)] = (
        [[Z, EAc, VAo, VAo, Z, EAo], [Z] * 6, [Z, VAo, VAc, Z, Z, VAo], [Z, VAo, Z, VAc, Z, VAo],
         [Z, EAo, VAo, VAo, Z, EAc], [Z] * 6],
        [[1, 0, 0, 0, 1, 0], [1] * 6, [1, 0, 0, 1, 1, 0], [1, 0, 1, 0, 1, 0],
         [1, 0, 0, 0, 1, 0], [1] * 6])
    t[(1, 1, 2)] = (
        [[EAc, Z, VAo, VAo, Z, EAo], [Z, EAc, VAo, VAo, Z, EAo], [VAo, VAo, EAc, Z, Z, EAo],
         [VAo, VAo, Z, EAc, Z, EAo], [EAo, EAo, EAo, EAo, Z, ST], [Z] * 6],
        [[0, 1, 0, 0, 1, 0], [1, 0, 0, 0, 1, 0], [0, 0, 0, 1, 1, 0], [0, 0, 1, 0, 1, 0],
         [0, 0, 0, 0, 1, 0], [1] * 6])
    t[(1, 2, 1)] = (
        [[EAc, Z, Z, EAo, VAo, VAo], [Z, EAc, Z, EAo, VAo, VAo], [EAo, EAo, Z, ST, EAo, EAo],
         [Z] * 6, [VAo, VAo, Z, EAo, EAc, Z], [VAo, VAo, Z, EAo, Z, EAc]],
        [[0, 1, 1, 0, 0, 0], [1, 0, 1, 0, 0, 0], [0, 0, 1, 0, 0, 0], [1] * 6,
         [0, 0, 1, 0, 0, 1], [0, 0, 1, 0, 1, 0]])
    t[(2, 2, 1)] = (
        [[Z, EAc, Z, EAo, VAo, VAo], [Z] * 6, [Z, EAo, Z, EAc, VAo, VAo], [Z] * 6,
         [Z, VAo, Z, VAo, VAc, Z], [Z, VAo, Z, VAo, Z, VAc]],
        [[1, 0, 1, 0, 0, 0], [1] * 6, [1, 0, 1, 0, 0, 0], [1] * 6, [1, 0, 1, 0, 0, 1],
         [1, 0, 1, 0, 1, 0]])
    t[(1, 2, 2)] = (
        [[VAc, Z, Z, VAo, Z, VAo], [Z, VAc, Z, VAo, Z, VAo], [VAo, VAo, Z, EAc, Z, EAo], [Z] * 6,
         [VAo, VAo, Z, EAo, Z, EAc], [Z] * 6],
        [[0, 1, 1, 0, 1, 0], [1, 0, 1, 0, 1, 0], [0, 0, 1, 0, 1, 0], [1] * 6, [0, 0, 1, 0, 1, 0],
         [1] * 6])
    t[(2, 2, 2)] = (
        [[Z, VAc, Z, VAo, Z, VAo], [Z] * 6, [Z, VAo, Z, VAc, Z, VAo], [Z] * 6,
         [Z, VAo, Z, VAo, Z, VAc], [Z] * 6],
        [[1, 0, 1, 0, 1, 0], [1] * 6, [1, 0, 1, 0, 1, 0], [1] * 6, [1, 0, 1, 0, 1, 0], [1] * 6])
    return {k: (np.array(c, dtype=complex), np.array(p, dtype=float)) for k, (c, p) in t.items()}


def nearby_correct(m, I_non_correct, ST, EAc, EAo, VAc, VAo):
    """nearby_correct.m:1-211: entries with P == 0 take the singular values."""
    C, P = _near_tables(ST, EAc, EAo, VAc, VAo)[tuple(m)]
    return np.where(P == 0.0, C, I_non_correct)


def assembly_nop_const(shape3, ko, dx, singular="DEMCEM"):
    """assembly_nop_const.m:1-174 -> G_mn(L,M,N,6) complex128."""
    if singular != "DEMCEM":
        raise ValueError("only the DEMCEM branch is restated")
    L, M, N = shape3
    dy = dz = dx
    R_faces = cube_faces(dx, dy, dz)
    Np_DEMCEM, Np_near, Np_medium, Np_far = 20, 20, 10, 4
    nL, nM, nN = min(5, L), min(5, M), min(5, N)
    lib = ref_lib()
    V = L * M * N
    J_re = np.zeros(V * 36)
    J_im = np.zeros(V * 36)
    Rf = _f64(R_faces.reshape(-1, order="F"))
    for Npt, (aL, aM, aN) in ((Np_far, (L, M, N)), (Np_medium, (nL, nM, nN))):
        _, wp, up, vp = gauss_2d(Npt)
        lib.voxref_cell_loop(L, M, N, aL, aM, aN, Npt * Npt, _p(_f64(wp)), _p(_f64(up)),
                             _p(_f64(vp)), _p(Rf), float(ko), float(dx), _p(J_re), _p(J_im))
    J = (J_re + 1j * J_im).reshape((L, M, N, 6, 6), order="F")
    _, wp, up, vp = gauss_2d(Np_near)
    ST = singular_st_const(Np_DEMCEM, ko, dx, dy)
    EAc, EAo = singular_ea_const(Np_DEMCEM, ko, dx, dy, dz)
    VAc, VAo = singular_va_const(Np_DEMCEM, ko, dx, dy, dz)
    near = [(1, 1, 1), (1, 1, 2)] if L == 1 else [
        (mx, my, mz) for mz in (1, 2) for my in (1, 2) for mx in (1, 2)]
    for m in near:
        r_m = (np.array(m) - 1) * np.array([dx, dy, dz])
        I_nc = cubature_nop_sym_near(Np_near, wp, up, vp, r_m, np.zeros(3), R_faces, ko, dx)
        J[m[0] - 1, m[1] - 1, m[2] - 1] = nearby_correct(m, I_nc, ST, EAc, EAo, VAc, VAo)
    P = vector_projection()
    G = np.einsum("xyzij,ijk->xyzk", J, P)
    return G / (4 * np.pi)
