"""MATLAB-facing mirror of VoxPhoton's VIE hot path over libvox.

Names, argument meaning and return values follow the reference functions:

* ``Operator(...)``           -- the device-resident operator behind the
  ``mv_AN_const(JIn0, fN, Mr, Mc, Gram, transp_flag, idx, GPU_flag)`` handle
  (piecewise_constant/src_vie/src_mvp/mv_AN_const.m:1); the one-time upload of
  JVIE_Solver_const.m:277-284.
* ``mv_AN_const(...)``        -- one-shot call with the reference signature.
* ``mv_L_const(...)``         -- mv_L_const.m:1.
* ``Preconditioner.level1``   -- level_1_parallel_func_N.m:1 + Bragg_MOR_script.m:61-72.
* ``chan_mvp_idx(...)``       -- chan_mvp_idx.m:2.
* ``pgmres(...)``             -- pgmres.m:70, returning (x, flag, relres, iter, resvec).

All compute runs in libvox (hand-written sm_100a CUDA); this module only
marshals MATLAB-layout arrays.
"""
from __future__ import annotations

import ctypes
import weakref

import numpy as np

from . import _lib
from ._lib import check, dptr, fortran_flat, lib, split


def _idx_array(idx):
    a = np.ascontiguousarray(np.asarray(idx, dtype=np.float64).reshape(-1))
    return a


class Operator:
    """Device-resident JVIE-II operator A = Gram*Mr - Mc*N (one per wavelength).

    Give either ``fN`` (2L x 2M x 2N x 6, the circulant FFT from
    getOPERATORS_SAM) or ``G`` (L x M x N x 6 Toeplitz, opToeplitz).
    ``Mr=None`` means Mr == 1 (the JVIE-II form).  ``members=K`` makes a
    batched operator: K independent copies of fN and of the solve state on one
    grid and support (vox_op_create_batch), solved together by
    ``solve_refined_batch``.
    """

    def __init__(self, Mc, Gram, idx, fN=None, G=None, Mr=None, precisions=("c128", "c64"),
                 device=0, members=1):
        Mc = np.asarray(Mc)
        if Mc.ndim != 3:
            raise ValueError("Mc must be L x M x N")
        L, M, N = Mc.shape
        self.shape = (L, M, N)
        self.Gram = float(Gram)
        self._keep = []
        d = _lib.OpDesc()
        d.L, d.M, d.N = L, M, N
        if (fN is None) == (G is None):
            raise ValueError("give exactly one of fN or G")
        if fN is not None:
            fN = np.asarray(fN)
            d.LfN, d.MfN, d.NfN = fN.shape[:3]
            re, im = split(fortran_flat(fN))
            d.fN_re, d.fN_im = dptr(re), dptr(im)
            self._keep += [re, im]
        else:
            G = np.asarray(G)
            if G.shape != (L, M, N, 6):
                raise ValueError("G must be L x M x N x 6")
            re, im = split(fortran_flat(G))
            d.G_re, d.G_im = dptr(re), dptr(im)
            self._keep += [re, im]
        if Mr is not None:
            re, im = split(fortran_flat(Mr))
            d.Mr_re, d.Mr_im = dptr(re), dptr(im)
            self._keep += [re, im]
        re, im = split(fortran_flat(Mc))
        d.Mc_re, d.Mc_im = dptr(re), dptr(im)
        self._keep += [re, im]
        d.gram = self.Gram
        ia = _idx_array(idx)
        d.idx, d.n_idx = dptr(ia), ia.size
        self._keep.append(ia)
        d.precisions = (1 if "c128" in precisions else 0) | (2 if "c64" in precisions else 0)
        d.device = device
        self.device = int(device)
        h = ctypes.c_void_p()
        if members == 1:
            check(lib().vox_op_create(ctypes.byref(d), ctypes.byref(h)))
        else:
            check(lib().vox_op_create_batch(ctypes.byref(d), int(members), ctypes.byref(h)))
        self._h = h
        self.members = int(members)
        self._keep = []
        self._pcs = weakref.WeakSet()
        self.n = ia.size
        self.idx = ia

    @property
    def handle(self):
        return self._h

    def info(self):
        px, py, pz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        n = ctypes.c_longlong()
        check(lib().vox_op_info(self._h, ctypes.byref(px), ctypes.byref(py), ctypes.byref(pz),
                                ctypes.byref(n)))
        fl = ctypes.c_int()
        check(lib().vox_op_flags(self._h, ctypes.byref(fl)))
        return {"Px": px.value, "Py": py.value, "Pz": pz.value, "n": n.value,
                "octant_fN": bool(fl.value & 1)}

    def close(self):
        """Free the device operator (and the preconditioners built on it)."""
        if getattr(self, "_h", None):
            for pc in list(getattr(self, "_pcs", ())):
                pc.close()
            lib().vox_op_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _mv(self, fn, x, *pre):
        re, im = split(x, self.n)
        ore = np.empty(self.n)
        oim = np.empty(self.n)
        check(fn(self._h, *pre, dptr(re), dptr(im), dptr(ore), dptr(oim)))
        return ore + 1j * oim

    def mv_AN(self, JIn0, transp_flag="notransp", prec="c128"):
        t = {"notransp": 0, "transp": 1}[transp_flag]
        return self._mv(lib().vox_mv_AN, JIn0, t, _lib.PREC[prec])

    def mv_L(self, JIn0, prec="c128"):
        return self._mv(lib().vox_mv_L, JIn0, _lib.PREC[prec])

    def __call__(self, JIn0):
        return self.mv_AN(JIn0)

    # ----------------------------------------------- device-resident calls
    def interp(self, srcs, weights, member=0):
        """fN <- sum_i weights[i] * srcs[i].fN on the device (lagrange_int.m),
        for one member of a batched operator."""
        arr = (ctypes.c_void_p * len(srcs))(*[s.handle for s in srcs])
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
        check(lib().vox_op_interp_member(self._h, int(member), arr, dptr(w), len(srcs)))

    def set_stream(self, stream_ptr):
        """Run on the caller's cudaStream_t (an int handle; 0 restores the op's)."""
        check(lib().vox_op_set_stream(self._h, ctypes.c_void_p(stream_ptr or None)))
        self.stream_ptr = stream_ptr or 0

    def launches(self):
        v = ctypes.c_longlong()
        check(lib().vox_op_stats(self._h, ctypes.byref(v)))
        return v.value

    def profile_stages(self, pc=None, prec="c64", restart=50, kgs=25, reps=20):
        """Per-kernel device ms of one GMRES iteration (see vox_profile_stages)."""
        out = np.zeros(10)
        check(lib().vox_profile_stages(self._h, pc.handle if pc else None, _lib.PREC[prec],
                                       restart, kgs, reps, dptr(out)))
        names = ["mv_xfwd", "mv_plane", "mv_xinv", "pc_xfwd", "pc_solve", "pc_xinv",
                 "gs_dots", "gs_update_dots", "gs_update_norm", "gs_scale"]
        return dict(zip(names, out.tolist()))

    def solve_refined_device(self, b_ptr, x_ptr, pc=None, side=None, tol=1e-5, restart=50,
                             maxit_inner=20, inner_tol=1e-3, max_refine=10):
        """vox_solve_refined_device on device pointers (interleaved complex128)."""
        info = _lib.GmresInfo()
        check(lib().vox_solve_refined_device(
            self._h, pc.handle if pc else None, _lib.SIDE[side] if pc else 0,
            ctypes.c_void_p(b_ptr), tol, restart, maxit_inner, inner_tol, max_refine,
            ctypes.c_void_p(x_ptr), ctypes.byref(info)))
        return info

    def solve_refined_batch_device(self, b_ptr, x_ptr, count, pc=None, side=None, tol=1e-5,
                                   restart=50, maxit_inner=20, inner_tol=1e-3, max_refine=10):
        """vox_solve_refined_batch_device: `count` right-hand sides (member-major
        interleaved complex128 device vectors) on members 0..count-1."""
        infos = (_lib.GmresInfo * count)()
        check(lib().vox_solve_refined_batch_device(
            self._h, pc.handle if pc else None, _lib.SIDE[side] if pc else 0, int(count),
            ctypes.c_void_p(b_ptr), tol, restart, maxit_inner, inner_tol, max_refine,
            ctypes.c_void_p(x_ptr), infos))
        return list(infos)

    def pgmres_device(self, b_ptr, x_ptr, pc=None, side=None, prec="c128", restart=50,
                      tol=1e-5, maxit=20):
        """vox_pgmres_device on device pointers (interleaved complex128 in/out)."""
        info = _lib.GmresInfo()
        check(lib().vox_pgmres_device(
            self._h, pc.handle if pc else None, _lib.SIDE[side] if pc else 0, _lib.PREC[prec],
            ctypes.c_void_p(b_ptr), restart, tol, maxit, ctypes.c_void_p(x_ptr),
            ctypes.byref(info)))
        return info


def mv_AN_const(JIn0, fN, Mr, Mc, Gram, transp_flag, idx, GPU_flag=1, prec="c128"):
    """mv_AN_const.m:1 with the reference's arguments (uploads fN each call;
    keep an ``Operator`` for repeated products)."""
    Mr_arg = None if np.all(np.asarray(Mr) == 1) else Mr
    op = Operator(Mc, Gram, idx, fN=fN, Mr=Mr_arg, precisions=(prec,))
    try:
        return op.mv_AN(JIn0, transp_flag, prec)
    finally:
        op.close()


def mv_L_const(JIn0, fN, r, Gram, idx, GPU_flag=1, prec="c128"):
    """mv_L_const.m:1: (N - Gram) J at the positions idx."""
    L, M, N = np.asarray(r).shape[:3]
    op = Operator(np.ones((L, M, N)), Gram, idx, fN=fN, precisions=(prec,))
    try:
        return op.mv_L(JIn0, prec)
    finally:
        op.close()


def face3_from_Mr(Mr):
    """Bragg_MOR_script.m:64-66: face = (m-1)/m, m = real(mean over x of Mr)."""
    Mr = np.asarray(Mr)
    hey = np.real(Mr.sum(axis=0) / Mr.shape[0])
    f = ((hey - 1) / hey).reshape(-1, order="F")
    return np.ascontiguousarray(np.concatenate([f, f, f]), dtype=np.float64)


class Preconditioner:
    """Level-1 circulant preconditioner on the device (chan_mvp_idx)."""

    def __init__(self, op: Operator, handle):
        self.op = op
        self._h = handle
        op._pcs.add(self)

    @classmethod
    def level1(cls, op: Operator, G, Mr_mean_source):
        """Build from the Toeplitz tensor G (L x M x N x 6) and the permittivity
        Mr used for the x-averaged face factor (Bragg_MOR_script.m:61-72)."""
        re, im = split(fortran_flat(G))
        f3 = face3_from_Mr(Mr_mean_source)
        h = ctypes.c_void_p()
        check(lib().vox_precond_create_level1(op.handle, dptr(re), dptr(im), dptr(f3),
                                              ctypes.byref(h)))
        return cls(op, h)

    @classmethod
    def from_blocks(cls, op: Operator, inv_blocks):
        """chan_mvp_idx with caller-supplied inverse blocks (list of L matrices)."""
        B = np.stack([np.asarray(b) for b in inv_blocks])  # L x n3 x n3
        flat = np.concatenate([fortran_flat(b) for b in B])
        re, im = split(flat)
        h = ctypes.c_void_p()
        check(lib().vox_precond_create_blocks(op.handle, dptr(re), dptr(im), ctypes.byref(h)))
        return cls(op, h)

    @classmethod
    def box(cls, op: Operator, level, x0, y0, Ls, Ms, G_box, Mc_box, Mr1=1.0, mask=None,
            scale=-1.0):
        """Level-1 (level_1_parallel_func) or level-2 (level_2_parallel_func)
        circulant preconditioner on the box x0:x0+Ls, y0:y0+Ms (all z) of op's
        grid: G_box its Toeplitz tensor, Mc_box its contrast, mask the box
        voxels it acts on (default: all of op's unknowns in the box); scale -1
        is the resonator script's negation."""
        re, im = split(fortran_flat(np.asarray(G_box)))
        mre, mim = split(fortran_flat(np.asarray(Mc_box)))
        mk = None
        if mask is not None:
            mk = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8).reshape(-1, order="F"))
        h = ctypes.c_void_p()
        check(lib().vox_precond_create_box(
            op.handle, int(level), int(x0), int(y0), int(Ls), int(Ms),
            mk.ctypes.data_as(ctypes.c_void_p) if mk is not None else None,
            dptr(re), dptr(im), dptr(mre), dptr(mim), float(Mr1), float(scale), ctypes.byref(h)))
        return cls(op, h)

    @classmethod
    def sum(cls, op: Operator, parts):
        """prec_fun_disk_idx: each part on its unknowns, identity elsewhere (the
        parts are owned by the sum from now on)."""
        arr = (ctypes.c_void_p * len(parts))(*[q.handle for q in parts])
        h = ctypes.c_void_p()
        check(lib().vox_precond_create_sum(op.handle, arr, len(parts), ctypes.byref(h)))
        for q in parts:
            op._pcs.discard(q)
            q._h = None
        return cls(op, h)

    @classmethod
    def disk(cls, op: Operator, G, p, regions=None):
        """resonator_MOR_scripts.m:94-198: level 1 on the bus box with the
        contrast at its centre (Mc_WG(round(L_WG/2),1,1)), level 2 on the disk
        square with the disk material's contrast ((e_r-1)/e_r, e_r the scalar
        Si permittivity of the script) acting on the disk's voxels, both
        inverses negated, identity elsewhere (prec_fun_disk_idx)."""
        from . import geometry as geo
        r = regions or geo.microdisk_regions(p)
        G = np.asarray(G)
        Mc = p.Mop()
        L, M, N = p.shape
        yb0, Mw = r["bus"]
        Mc_c = Mc[int(np.floor(L / 2 + 0.5)) - 1, yb0, 0]
        bus = cls.box(op, 1, 0, yb0, L, Mw, G[:L, :Mw, :N, :], np.full((L, Mw, N), Mc_c),
                      1.0, None, -1.0)
        x0, Ls, y0, Ms = r["square"]
        sq = np.zeros(Ls * Ms * N, dtype=bool)
        sq[r["idx_disk_in_sq"] - 1] = True
        mask = sq.reshape((Ls, Ms, N), order="F")
        e_si = geo.EPS_SI / geo.EPS_SIO2
        disk = cls.box(op, 2, x0, y0, Ls, Ms, G[:Ls, :Ms, :N, :],
                       np.full((Ls, Ms, N), (e_si - 1) / e_si), 1.0, mask, -1.0)
        return cls.sum(op, [bus, disk])

    @property
    def handle(self):
        return self._h

    def share(self, op: Operator):
        """A handle on the same factors bound to `op` (same grid and idx), with its
        own work buffers, for concurrent solves on another operator/stream."""
        h = ctypes.c_void_p()
        check(lib().vox_precond_share(self._h, op.handle, ctypes.byref(h)))
        return Preconditioner(op, h)

    def info(self):
        nf, ld, pr = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().vox_precond_info(self._h, ctypes.byref(nf), ctypes.byref(ld),
                                     ctypes.byref(pr)))
        return {"n_blocks": nf.value, "ld": ld.value, "paired": bool(pr.value)}

    def apply(self, JIn, prec="c128"):
        re, im = split(JIn, self.op.n)
        ore = np.empty(self.op.n)
        oim = np.empty(self.op.n)
        check(lib().vox_precond_apply(self._h, _lib.PREC[prec], dptr(re), dptr(im), dptr(ore),
                                      dptr(oim)))
        return ore + 1j * oim

    __call__ = apply

    def close(self):
        if getattr(self, "_h", None):
            if getattr(self.op, "_h", None):
                lib().vox_precond_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def chan_mvp_idx(inv_blocks, JIn, L, M, N, idx, op=None):
    """chan_mvp_idx.m:2 (builds a temporary preconditioner from inv_blocks)."""
    if op is None:
        raise ValueError("an Operator on the same grid/idx is required for the index map")
    pc = Preconditioner.from_blocks(op, inv_blocks)
    try:
        return pc.apply(JIn)
    finally:
        pc.close()


def _info(resvec_cap):
    info = _lib.GmresInfo()
    buf = np.zeros(max(1, resvec_cap))
    info.resvec = dptr(buf)
    info.resvec_cap = buf.size
    return info, buf


def pgmres(A: Operator, b, restart=None, tol=None, maxit=None, L1=None, R1=None, prec="c128"):
    """pgmres.m:70 on the device: returns (x, flag, relres, iter, resvec).

    ``L1`` / ``R1`` are left / right preconditioners (``Preconditioner``)."""
    restart = 50 if restart is None else int(restart)
    tol = 1e-3 if tol is None else float(tol)
    maxit = 10 if maxit is None else int(maxit)
    if L1 is not None and R1 is not None:
        raise ValueError("give at most one of L1 or R1")
    pc = L1 if L1 is not None else R1
    side = 1 if L1 is not None else (2 if R1 is not None else 0)
    re, im = split(b, A.n)
    xre = np.empty(A.n)
    xim = np.empty(A.n)
    info, buf = _info(restart * maxit + 1)
    check(lib().vox_pgmres(A.handle, pc.handle if pc else None, side, _lib.PREC[prec], dptr(re),
                           dptr(im), restart, tol, maxit, dptr(xre), dptr(xim),
                           ctypes.byref(info)))
    resvec = buf[:min(info.n_resvec, buf.size)].copy()
    return (xre + 1j * xim, info.flag, info.relres, [info.iter_inner, info.iter_outer], resvec)


def solve_refined(A: Operator, b, tol=1e-5, restart=50, maxit_inner=20, inner_tol=1e-3,
                  max_refine=10, L1=None, R1=None):
    """complex64 GMRES inside FP64 iterative refinement; returns (x, info dict)."""
    pc = L1 if L1 is not None else R1
    side = 1 if L1 is not None else (2 if R1 is not None else 0)
    re, im = split(b, A.n)
    xre = np.empty(A.n)
    xim = np.empty(A.n)
    info, buf = _info(restart * maxit_inner * max_refine + max_refine + 1)
    check(lib().vox_solve_refined(A.handle, pc.handle if pc else None, side, dptr(re), dptr(im),
                                  tol, restart, maxit_inner, inner_tol, max_refine, dptr(xre),
                                  dptr(xim), ctypes.byref(info)))
    return xre + 1j * xim, {
        "flag": info.flag, "relres": info.relres, "iters": info.total_iters,
        "refinements": info.refinements, "seconds": info.seconds,
        "resvec": buf[:min(info.n_resvec, buf.size)].copy()}


class Lane:
    """Continuous batching on a batched operator (vox_lane_*): every member
    runs its own complex64 + FP64-refinement solve, all members' Arnoldi steps
    share one launch per kernel (each member at its own point of its own
    cycle), and a member takes a new right-hand side as soon as its previous
    solve is collected.  Each result equals solve_refined on that member
    alone."""

    def __init__(self, op: Operator, pc=None, side="left", tol=1e-5, restart=50, maxit_inner=40,
                 inner_tol=0.0, max_refine=10):
        h = ctypes.c_void_p()
        check(lib().vox_lane_create(op.handle, pc.handle if pc else None,
                                    _lib.SIDE[side] if pc else 0, tol, restart, maxit_inner,
                                    inner_tol, max_refine, ctypes.byref(h)))
        self._h = h
        self.op = op
        self.members = op.members
        self._cap = restart * maxit_inner * max_refine + max_refine + 1
        self._done = (ctypes.c_int * op.members)()
        op._lanes = getattr(op, "_lanes", []) + [self]

    def submit(self, member, b):
        """Start a solve of b (host vector) on a free member."""
        re, im = split(b, self.op.n)
        check(lib().vox_lane_submit(self._h, int(member), dptr(re), dptr(im)))

    def submit_device(self, member, b_ptr, x_ptr):
        """Start a solve with device vectors (interleaved complex128)."""
        check(lib().vox_lane_submit_device(self._h, int(member), ctypes.c_void_p(b_ptr),
                                           ctypes.c_void_p(x_ptr)))

    def step(self):
        """Advance every solving member (VOX_LANE_STEPS Arnoldi steps with the
        members' cycles out of phase, default 2; whole restart cycles for
        restart > 50 or VOX_LANE_STEPS=0), refine the members whose inner solve
        ended; returns the members that finished."""
        nd = ctypes.c_int()
        check(lib().vox_lane_step(self._h, self._done, ctypes.byref(nd)))
        return [self._done[i] for i in range(nd.value)]

    def collect(self, member, host=True):
        """(x or None, info dict) of a finished member, which becomes free."""
        info, buf = _info(self._cap)
        n = self.op.n
        xre = np.empty(n) if host else None
        xim = np.empty(n) if host else None
        check(lib().vox_lane_collect(self._h, int(member), dptr(xre) if host else None,
                                     dptr(xim) if host else None, ctypes.byref(info)))
        x = xre + 1j * xim if host else None
        return x, {"flag": info.flag, "relres": info.relres, "iters": info.total_iters,
                   "refinements": info.refinements,
                   "resvec": buf[:min(info.n_resvec, buf.size)].copy()}

    def state(self):
        st = (ctypes.c_int * self.members)()
        check(lib().vox_lane_state(self._h, st))
        return list(st)

    def close(self):
        if getattr(self, "_h", None) and getattr(self.op, "_h", None):
            lib().vox_lane_destroy(self._h)
        self._h = None


def solve_refined_batch(A: Operator, bs, tol=1e-5, restart=50, maxit_inner=20, inner_tol=1e-3,
                        max_refine=10, L1=None, R1=None):
    """solve_refined for several right-hand sides at once on the members of a
    batched operator (member i solves bs[i]); returns [(x, info dict)]."""
    pc = L1 if L1 is not None else R1
    side = 1 if L1 is not None else (2 if R1 is not None else 0)
    count = len(bs)
    B = np.stack([np.asarray(b, dtype=np.complex128).reshape(-1) for b in bs])
    if B.shape[1] != A.n:
        raise ValueError("right-hand sides must have length n")
    re = np.ascontiguousarray(B.real)
    im = np.ascontiguousarray(B.imag)
    xre = np.empty((count, A.n))
    xim = np.empty((count, A.n))
    cap = restart * maxit_inner * max_refine + max_refine + 1
    infos = (_lib.GmresInfo * count)()
    bufs = [np.zeros(cap) for _ in range(count)]
    for i in range(count):
        infos[i].resvec = dptr(bufs[i])
        infos[i].resvec_cap = cap
    check(lib().vox_solve_refined_batch(A.handle, pc.handle if pc else None, side, count,
                                        dptr(re), dptr(im), tol, restart, maxit_inner, inner_tol,
                                        max_refine, dptr(xre), dptr(xim), infos))
    out = []
    for i in range(count):
        inf = infos[i]
        out.append((xre[i] + 1j * xim[i], {
            "flag": inf.flag, "relres": inf.relres, "iters": inf.total_iters,
            "refinements": inf.refinements, "seconds": inf.seconds,
            "resvec": bufs[i][:min(inf.n_resvec, cap)].copy()}))
    return out


def E_field_Nop_const(J, op_full: Operator, Gram, freq, Einc=None, prec="c128"):
    """E_field_Nop_const.m:59-84: the total field on the whole grid,
    Etot = Einc + (N J - Gram J) / (Gram j omega eo).

    J: L x M x N x 3 polarisation currents (zero outside the scatterer).
    op_full: an Operator whose support is the whole grid (idx = 1..3LMN, as the
    reference passes to mv_L_const) holding this wavelength's fN."""
    J = np.asarray(J)
    L, M, N, _ = J.shape
    if op_full.n != 3 * L * M * N:
        raise ValueError("op_full must be built on the whole grid (idx = 1..3*L*M*N)")
    mu = 4 * np.pi * 1e-7
    co = 299792458.0
    eo = 1.0 / co ** 2 / mu
    omega = 2 * np.pi * freq
    E = op_full.mv_L(J.reshape(-1, order="F"), prec=prec).reshape((L, M, N, 3), order="F")
    E = E / (Gram * 1j * omega * eo)
    return E if Einc is None else Einc + E


def transmitted_power(E, res, len_abs, delW):
    """example_Bragg_1500nm_to_1600nm.m:107-113: sum of |E|^2 over the voxel
    slice x = L - round((len_abs + 450 nm) / res) (1-based), trimmed by
    round(delW / 2) / res voxels at each y edge.  The rounding is of a length
    in metres, as in the reference, so for nanometre corrugations nothing is
    trimmed."""
    E = np.asarray(E)
    L, M = E.shape[:2]
    x_thru = L - int(np.round((len_abs + 450e-9) / res))
    vox = int(np.round(np.round(delW / 2) / res))
    e = E[x_thru - 1, vox:M - vox, :, :]
    return float(np.sum((e * np.conj(e)).real))


def jvie_rhs(e_r, Einc, Gram, freq, idx):
    """JVIE_Solver_const.m:151-157 + :243-251: Vrhs at the positions idx."""
    e_r = np.asarray(e_r)
    L, M, N = e_r.shape
    er_re, er_im = split(fortran_flat(e_r))
    e_re, e_im = split(fortran_flat(Einc))
    ia = _idx_array(idx)
    ore = np.empty(ia.size)
    oim = np.empty(ia.size)
    check(lib().vox_jvie_rhs(L, M, N, dptr(er_re), dptr(er_im), dptr(e_re), dptr(e_im),
                             float(Gram), float(freq), dptr(ia), ia.size, dptr(ore), dptr(oim)))
    return ore + 1j * oim


def assemble_toeplitz(shape3, ko, dx, nthreads=0, device=None):
    """assembly_nop_const(r, ko, dx, 'DEMCEM'): G (L x M x N x 6).  On the host
    (C++, nthreads) by default; with device=<ordinal> the regular face-pair
    cubature runs on that GPU (vox_assemble_toeplitz_device)."""
    L, M, N = shape3
    V = L * M * N
    re = np.empty(6 * V)
    im = np.empty(6 * V)
    if device is None:
        check(lib().vox_assemble_toeplitz(L, M, N, float(ko), float(dx), int(nthreads),
                                          dptr(re), dptr(im)))
    else:
        check(lib().vox_assemble_toeplitz_device(L, M, N, float(ko), float(dx), int(device),
                                                 dptr(re), dptr(im)))
    return (re + 1j * im).reshape((L, M, N, 6), order="F")


def singular_integrals(ko, dx, order=32):
    """(ST, EAc, EAo, VAc, VAo) face-pair integrals of exp(-j ko R)/R."""
    out = np.empty(10)
    check(lib().vox_singular_integrals(float(ko), float(dx), int(order), dptr(out)))
    return tuple(out[0::2] + 1j * out[1::2])


def JVIE_Solver_const(Einc, e_r, r, freq, fN=None, tol=None, form=None, solver=None,
                      precond=None, max_it=None, inner_it=None, outer_it=None, ritz=None,
                      gpu_flag=None, logfile=None, G=None, prec="c128"):
    """[Je, flag, relres, iter, resvec, solvert, vsol] = JVIE_Solver_const(Einc, e_r, r,
    freq, fN, tol, form, solver, precond, max_it, inner_it, outer_it, ritz, gpu_flag,
    logfile) (JVIE_Solver_const.m:1-535) on the device.

    Einc: L x M x N x 3, e_r: L x M x N, r: the voxel centres (L x M x N x 3; the
    voxel edge is r(1,1,2,3) - r(1,1,1,3), as :140), fN the N operator (or
    ``G=`` its Toeplitz tensor).  Defaults and clamps as the reference: tol 1e-3,
    form 2, solver 'B' (BiCGStab), max_it 1000, inner_it 50, outer_it 200, ritz 5.
    solver 'G' runs vox_jvie_solve (restarted GMRES; ``prec="c64"`` gives the
    complex64 + FP64-refinement solve); 'D' runs pgmresDR and 'B' bicgstab
    (voxphoton_b200.solvers) on an operator built the same way.  Only form 2
    (JVIE-II) is implemented; its preconditioner fP = Gram * I leaves GMRES's
    iterates unchanged, so 'L' / 'R' solve unpreconditioned.  gpu_flag selects
    the device (ordinal gpu_flag - 1; 0 is refused: there is no CPU path);
    logfile is accepted and ignored."""
    import time as _time
    Einc = np.asarray(Einc)
    e_r = np.asarray(e_r)
    L, M, N = e_r.shape
    tol = 1e-3 if (tol is None or tol < 1e-15 or tol >= 1) else float(tol)
    form = 2 if form is None else int(form)
    solver = "B" if solver is None else solver
    if solver not in ("G", "D"):
        solver = "B"
    if precond not in ("L", "R"):
        precond = None
    max_it = 1000 if max_it is None else int(max_it)
    inner_it = 50 if (inner_it is None or inner_it < 1) else int(inner_it)
    outer_it = 200 if (outer_it is None or outer_it < 1) else int(outer_it)
    ritz = 5 if (ritz is None or ritz < 1) else int(ritz)
    gpu_flag = 1 if gpu_flag is None else int(gpu_flag)
    if gpu_flag < 1:
        raise ValueError("gpu_flag 0 asks for the CPU path, which this library does not have")
    device = gpu_flag - 1
    if form != 2:
        raise NotImplementedError("only the JVIE-II formulation (form 2) is implemented")
    if (fN is None) == (G is None):
        raise ValueError("give exactly one of fN or G")
    r = np.asarray(r)
    dx = float(r[0, 0, 1, 2] - r[0, 0, 0, 2])
    Gram = dx ** 3
    t0 = _time.perf_counter()
    V = L * M * N
    idx = np.flatnonzero(np.abs(fortran_flat(e_r) - 1.0) > 1e-12) + 1
    idx3 = np.concatenate([idx, V + idx, 2 * V + idx])
    if solver == "G":
        d = _lib.JvieDesc()
        d.L, d.M, d.N = L, M, N
        e_re, e_im = split(fortran_flat(Einc))
        r_re, r_im = split(fortran_flat(e_r))
        d.Einc_re, d.Einc_im, d.er_re, d.er_im = dptr(e_re), dptr(e_im), dptr(r_re), dptr(r_im)
        d.dx, d.freq = dx, float(freq)
        if fN is not None:
            fN = np.asarray(fN)
            d.LfN, d.MfN, d.NfN = fN.shape[:3]
            f_re, f_im = split(fortran_flat(fN))
            d.fN_re, d.fN_im = dptr(f_re), dptr(f_im)
        else:
            f_re, f_im = split(fortran_flat(np.asarray(G)))
            d.G_re, d.G_im = dptr(f_re), dptr(f_im)
        d.tol = tol
        d.form = 2
        d.solver = b"G"
        d.precond = precond.encode() if precond else b"\0"
        d.inner_it, d.outer_it = inner_it, outer_it
        d.prec = _lib.PREC[prec]
        d.device = device
        info, buf = _info(inner_it * outer_it * 10 + 11)
        Je_re = np.empty(3 * V)
        Je_im = np.empty(3 * V)
        check(lib().vox_jvie_solve(ctypes.byref(d), dptr(Je_re), dptr(Je_im), ctypes.byref(info)))
        del e_re, e_im, r_re, r_im, f_re, f_im
        Je = (Je_re + 1j * Je_im).reshape((L, M, N, 3), order="F")
        resvec = buf[:min(info.n_resvec, buf.size)].copy()
        vsol = Je.reshape(-1, order="F")[idx3 - 1]
        return (Je, info.flag, info.relres, [info.iter_inner, info.iter_outer], resvec,
                _time.perf_counter() - t0, vsol)
    # GMRES-DR / BiCGStab on an operator built as :133-157, 243-251
    from .solvers import bicgstab, pgmresDR
    b = jvie_rhs(e_r, Einc, Gram, freq, idx3)
    op = Operator((e_r - 1.0) / e_r, Gram, idx3, fN=fN, G=G, precisions=("c128",),
                  device=device)
    try:
        if solver == "D":
            x, flag, relres, it, resvec = pgmresDR(op, b, inner_it, tol, outer_it, ritz)
        else:
            x, flag, relres, it, resvec = bicgstab(op, b, tol, max_it)
    finally:
        op.close()
    Je = np.zeros(3 * V, dtype=complex)
    Je[idx3 - 1] = x
    return (Je.reshape((L, M, N, 3), order="F"), flag, relres, it, resvec,
            _time.perf_counter() - t0, x)
