"""Request loop for broadband sweeps: frequency solves of several device
lengths arriving as a stream, served concurrently on one GPU.

Per device length (a "family") the loop keeps resident on the device:

* the operator at nG Legendre wavelengths over the sweep band - the reference's
  own sweep mechanism (Si_in_SiO2_parameters.m:11-14 nodes, lagrange_int.m:1-12
  interpolation of fN in wavelength, example_Bragg_1500nm_to_1600nm.m:104);
* one level-1 circulant preconditioner built at the band centre and shared by
  every wavelength of that length (vox_precond_share: one factor copy, per-slot
  work buffers);
* a number of solve slots, each an operator + GMRES state + its own CUDA
  stream.  The number of slots is set by the HBM footprint of one slot
  against a memory budget ("admission by footprint").

A request (length, wavelength) waits until it has arrived and a slot of its
length is free; the slot then interpolates fN to the request's wavelength on
the device (vox_op_interp), forms the right-hand side for the plane wave at
that wavelength and runs the complex64 + FP64-refinement solve (or the plain
complex128 GMRES for the baseline) through the C-ABI with host buffers.  Slots
run in host threads (the C calls release the GIL), so solves of different
lengths and wavelengths overlap on the GPU.  Latency = completion - arrival.
"""
from __future__ import annotations

import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import geometry as geo
from .vie import Operator, Preconditioner, assemble_toeplitz


def legendre_nodes(lam_lo, lam_hi, nG):
    """Si_in_SiO2_parameters.m:11-14: s = s_mid + (s_plus - s_minus)/2 * xG."""
    x, _ = np.polynomial.legendre.leggauss(nG)
    mid = 0.5 * (lam_lo + lam_hi)
    return mid + 0.5 * (lam_hi - lam_lo) * x


def lagrange_weights(S, s):
    """lagrange_int.m:1-12: weights L_i(S) of the Lagrange basis on nodes s."""
    s = np.asarray(s, dtype=float)
    w = np.ones(s.size)
    for i in range(s.size):
        for j in range(s.size):
            if j != i:
                w[i] *= (S - s[j]) / (s[i] - s[j])
    return w


@dataclass
class Request:
    rid: int
    key: object
    lam: float
    arrival: float  # seconds after the stream starts


@dataclass
class Result:
    rid: int
    key: object
    lam: float
    arrival: float
    start: float
    done: float
    iters: int
    relres: float
    flag: int
    x: object = None  # the solution, when ServeConfig.keep_x

    @property
    def latency(self):
        return self.done - self.arrival


def shard_requests(items, world, rank):
    """Replica sharding across GPUs: rank r serves items r, r+world, ... (the
    solves are independent; no collective is involved)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return list(items[rank::world])


def poisson_stream(keys_lams, rate, seed=0):
    """Requests in a seeded random order with exponential inter-arrival times."""
    rng = np.random.default_rng(seed)
    order = rng.permutation(len(keys_lams))
    t = np.cumsum(rng.exponential(1.0 / rate, size=len(keys_lams)))
    return [Request(int(i), keys_lams[k][0], keys_lams[k][1], float(t[i]))
            for i, k in enumerate(order)]


class _RhsBuilder:
    """Plane-wave right-hand side of the JVIE-II system at any wavelength.

    For k along x the voxel-averaged plane wave (PlaneWave_Excitation.m:67-98)
    factors as Eo_c * fx(x; k) * dy * dz / dx^3, so
    Vrhs_i = j w eo Gram (Mc/Mr)_i Eo_c fx(x_i; k) dy dz / dx^3
    (JVIE_Solver_const.m:151-157, 243-251) is a per-x factor times a fixed
    per-unknown coefficient."""

    def __init__(self, p: geo.Problem, idx, Eo=(0.0, 1.0, 0.0)):
        L, M, N = p.shape
        V = L * M * N
        i0 = np.asarray(idx, dtype=np.int64) - 1
        comp = i0 // V
        cell = i0 % V
        self.xi = cell % L
        mop = p.Mop().reshape(-1, order="F")[cell]
        dx = p.res
        self.coef = p.Gram * mop * np.asarray(Eo)[comp] * dx * dx / dx ** 3
        self.x = p.centres[0]
        self.dx = dx

    def __call__(self, freq):
        ko = 2 * np.pi * freq / geo.C0
        k = ko
        fx = np.exp(-1j * k * self.x) * (np.exp(-1j * k * self.dx / 2)
                                         - np.exp(1j * k * self.dx / 2)) / (-1j * k)
        omega = 2 * np.pi * freq
        return 1j * omega * geo.EPS0 * self.coef * fx[self.xi]


class Family:
    """Resident state of one device length."""

    def __init__(self, key, problem: geo.Problem, band, nG=5, precond=True, device=0):
        self.key = key
        self.p = problem
        self.nodes = legendre_nodes(band[0], band[1], nG)
        self.idx = problem.idxS3()
        self.mop = problem.Mop()
        t0 = time.time()
        self.node_ops = []
        Gc = None
        for j, lam in enumerate(self.nodes):
            pj = problem.with_wavelength(lam)
            G = assemble_toeplitz(pj.shape, pj.ko, pj.res)
            self.node_ops.append(Operator(self.mop, pj.Gram, self.idx, G=G, device=device))
            if j == nG // 2:
                Gc = G
        self.assembly_s = time.time() - t0
        t0 = time.time()
        self.pc = None
        if precond:
            self.pc = Preconditioner.level1(self.node_ops[nG // 2], Gc, problem.e_r)
        self.precond_s = time.time() - t0
        self.rhs = _RhsBuilder(problem, self.idx)
        self._Gc = Gc
        self.device = device
        self.slots = []

    def add_slot(self):
        op = Operator(self.mop, self.p.Gram, self.idx, G=self._Gc, device=self.device)
        pc = self.pc.share(op) if self.pc is not None else None
        self.slots.append((op, pc))
        return self.slots[-1]

    def close(self):
        for op, pc in self.slots:
            if pc is not None:
                pc.close()
            op.close()
        if self.pc is not None:
            self.pc.close()
        for op in self.node_ops:
            op.close()


@dataclass
class ServeConfig:
    tol: float = 1e-5
    restart: int = 50
    maxit_inner: int = 40
    mode: str = "mixed"          # "mixed" (c64 + FP64 refinement) or "fp64" (plain c128 GMRES)
    maxit_fp64: int = 40
    keep_x: bool = False         # return each solution with its result


class SweepServer:
    """Serves a request stream over several families with per-family slots."""

    def __init__(self, families, cfg: ServeConfig = None):
        self.families = {f.key: f for f in families}
        self.cfg = cfg or ServeConfig()

    def _solve(self, fam: Family, op, pc, req: Request):
        import ctypes
        from . import _lib
        lib = _lib.lib()
        w = lagrange_weights(req.lam, fam.nodes)
        op.interp(fam.node_ops, w)
        freq = geo.C0 / req.lam * geo.N_EXT
        b = fam.rhs(freq)
        bre = np.ascontiguousarray(b.real)
        bim = np.ascontiguousarray(b.imag)
        xre = np.empty(op.n)
        xim = np.empty(op.n)
        info = _lib.GmresInfo()
        side = 1 if pc is not None else 0
        pch = pc.handle if pc is not None else None
        c = self.cfg
        if c.mode == "mixed":
            _lib.check(lib.vox_solve_refined(op.handle, pch, side, _lib.dptr(bre), _lib.dptr(bim),
                                             c.tol, c.restart, c.maxit_inner, 0.0, 10,
                                             _lib.dptr(xre), _lib.dptr(xim), ctypes.byref(info)))
        else:
            _lib.check(lib.vox_pgmres(op.handle, pch, side, _lib.VOX_C128, _lib.dptr(bre),
                                      _lib.dptr(bim), c.restart, c.tol, c.maxit_fp64,
                                      _lib.dptr(xre), _lib.dptr(xim), ctypes.byref(info)))
        return info, (xre + 1j * xim if c.keep_x else None)

    def solve_one(self, fam: Family, req: Request, slot=0):
        """One request on one slot of its family, on the calling thread."""
        op, pc = fam.slots[slot]
        t0 = time.perf_counter()
        info, x = self._solve(fam, op, pc, req)
        t1 = time.perf_counter()
        return Result(req.rid, req.key, req.lam, 0.0, 0.0, t1 - t0, info.total_iters,
                      info.relres, info.flag, x)

    def serve(self, requests, realtime=True):
        """Run the stream; returns (results, wall seconds)."""
        queues = {k: deque() for k in self.families}
        for r in sorted(requests, key=lambda r: r.arrival):
            queues[r.key].append(r)
        locks = {k: threading.Lock() for k in self.families}
        results = []
        res_lock = threading.Lock()
        t0 = time.perf_counter()
        errors = []

        def worker(fam, op, pc):
            q = queues[fam.key]
            while True:
                with locks[fam.key]:
                    if not q:
                        return
                    req = q.popleft()
                now = time.perf_counter() - t0
                if realtime and req.arrival > now:
                    time.sleep(req.arrival - now)
                start = time.perf_counter() - t0
                try:
                    info, x = self._solve(fam, op, pc, req)
                except Exception as e:  # surfaced after the threads join
                    errors.append(e)
                    return
                done = time.perf_counter() - t0
                with res_lock:
                    results.append(Result(req.rid, req.key, req.lam, req.arrival if realtime
                                          else 0.0, start, done, info.total_iters, info.relres,
                                          info.flag, x))

        threads = [threading.Thread(target=worker, args=(fam, op, pc), daemon=True)
                   for fam in self.families.values() for (op, pc) in fam.slots]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        wall = time.perf_counter() - t0
        if errors:
            raise errors[0]
        return sorted(results, key=lambda r: r.rid), wall


def summarize(results, wall):
    lat = np.array([r.latency for r in results])
    return {"solves": len(results), "wall_s": wall, "solves_per_s": len(results) / wall,
            "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_iters": float(np.mean([r.iters for r in results])),
            "max_relres": float(np.max([r.relres for r in results])),
            "flags": int(np.sum([r.flag for r in results]))}
