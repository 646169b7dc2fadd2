"""Request loop for broadband sweeps: frequency solves of several device
lengths arriving as a stream, served concurrently on one GPU.

Per device length (a "family") the loop keeps resident on the device:

* the operator at nG Legendre wavelengths over the sweep band - the reference's
  own sweep mechanism (Si_in_SiO2_parameters.m:11-14 nodes, lagrange_int.m:1-12
  interpolation of fN in wavelength, example_Bragg_1500nm_to_1600nm.m:104);
* one level-1 circulant preconditioner built at the band centre and shared by
  every wavelength of that length (vox_precond_share: one factor copy, per-slot
  work buffers);
* solve slots ("lanes"), each a batched operator of K members
  (vox_op_create_batch: K copies of fN and of the GMRES state) + its own CUDA
  stream.  With a pool budget (SweepServer pool_bytes) lanes are admitted by
  their measured HBM footprint as the queues of the lengths fill, and idle
  lanes of lengths with nothing waiting are retired to make room.

A request (length, wavelength) waits until it has arrived and a lane of its
length is free.  The lane then takes every request of its length that has
arrived by then, up to K (continuous batching: requests that arrive while the
lanes are busy join the next batch), interpolates each member's fN to its
request's wavelength on the device (vox_op_interp_member), forms the
right-hand sides for the plane wave at those wavelengths and runs the
complex64 + FP64-refinement solve of the whole batch in lockstep
(vox_solve_refined_batch: one launch per kernel for all members, the
preconditioner's factors streamed once for all of them) through the C-ABI
with host buffers.  Each result is identical to solving that request alone.
Lanes run in host threads (the C calls release the GIL), so batches of
different lengths overlap on the GPU.  Latency = completion - arrival.  The
plain complex128 GMRES baseline solves one request at a time.
"""
from __future__ import annotations

import threading
import time
from collections import deque
from dataclasses import dataclass

import numpy as np

from . import _lib
from . import geometry as geo
from .vie import Lane, Operator, Preconditioner, assemble_toeplitz


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
    refinements: int = 0  # FP64 refinement steps (mixed-precision solves)

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

    def fill_device(self, freqs, out):
        """The right-hand sides at every frequency of freqs into the rows of
        out, a (len(freqs), n) complex128 CUDA tensor (synthetic input built
        in place, without host copies of n-vectors)."""
        import torch
        dev = out.device
        if getattr(self, "_dev", None) is None or self._dev[0] != dev:
            self._dev = (dev, torch.from_numpy(self.xi).to(dev),
                         torch.from_numpy(self.coef.astype(np.complex128)).to(dev))
        _, xi, coef = self._dev
        for r, freq in enumerate(freqs):
            k = 2 * np.pi * freq / geo.C0
            fx = np.exp(-1j * k * self.x) * (np.exp(-1j * k * self.dx / 2)
                                             - np.exp(1j * k * self.dx / 2)) / (-1j * k)
            fx = fx * (1j * 2 * np.pi * freq * geo.EPS0)
            out[r].copy_(coef * torch.from_numpy(fx).to(dev)[xi])
        return out


class Family:
    """Resident state of one device length."""

    def __init__(self, key, problem: geo.Problem, band, nG=5, precond=True, device=0, members=1,
                 G_nodes=None):
        """G_nodes: the Toeplitz tensors at the nG nodes, if already assembled;
        precond: "level1" (or True) for the level-1 circulant preconditioner,
        "disk" for the resonator's bus + disk composite, None for none."""
        self.key = key
        self.members = int(members)
        self.p = problem
        self.nodes = legendre_nodes(band[0], band[1], nG)
        self.idx = problem.idxS3()
        self.mop = problem.Mop()
        t0 = time.time()
        self.node_ops = []
        Gc = None
        for j, lam in enumerate(self.nodes):
            pj = problem.with_wavelength(lam)
            G = G_nodes[j] if G_nodes is not None else assemble_toeplitz(pj.shape, pj.ko, pj.res,
                                                                         device=device)
            self.node_ops.append(Operator(self.mop, pj.Gram, self.idx, G=G, device=device))
            if j == nG // 2:
                Gc = G
        self.assembly_s = time.time() - t0
        t0 = time.time()
        self.pc = None
        if precond == "disk":
            self.pc = Preconditioner.disk(self.node_ops[nG // 2], Gc, problem)
        elif precond:
            self.pc = Preconditioner.level1(self.node_ops[nG // 2], Gc, problem.e_r)
        self.precond_s = time.time() - t0
        self.rhs = _RhsBuilder(problem, self.idx)
        self._Gc = Gc
        self.device = device
        self.slots = []

    def add_slot(self, stream=None):
        """One more lane: a batched operator of `members` members, on its own
        CUDA stream (a torch.cuda.Stream when given, needed for device-resident
        right-hand sides)."""
        op = Operator(self.mop, self.p.Gram, self.idx, G=self._Gc, device=self.device,
                      members=self.members)
        op.torch_stream = stream
        if stream is not None:
            op.set_stream(stream.cuda_stream)
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
    side: str = "left"           # preconditioning of the mixed-precision inner solves
                                 # ("left" as the reference's L1, or "right")
    batching: str = "continuous"  # "continuous" (a member slot is refilled as soon as
                                  # its solve ends) or "lockstep" (a lane's batch
                                  # starts and ends together)
    inner_tol: float = 0.0       # relative target of each complex64 inner solve; 0 aims
                                 # each one at the remaining FP64 target directly


class _LaneCtx:
    """One continuously batched lane of a family inside the HBM pool."""

    def __init__(self, fam, op, pc, lane, nbytes):
        self.fam = fam
        self.op = op
        self.pc = pc
        self.lane = lane
        self.nbytes = nbytes
        self.inflight = {}      # member -> (request, start time)
        self.retire = False     # asked to leave the pool once idle
        self.stop = False       # the stream is over
        self.thread = None


class SweepServer:
    """Serves a request stream over several families with per-family slots.

    pool_bytes (continuous batching only): admission by HBM footprint.  The
    lanes of every family share one device-memory budget; a family whose
    arrived requests outnumber its free member slots gets a new lane when the
    lane's measured footprint fits in what is left (and max_lanes allows),
    and otherwise an idle lane of a family with nothing waiting is retired to
    make room (every family keeps one), so lanes move between device lengths
    as the mix of the stream changes.  JVIE_Solver_const.m:200-201 admits a
    solve to the GPU when its estimated memory fits the device; here every
    lane is admitted the same way."""

    def __init__(self, families, cfg: ServeConfig = None, pool_bytes=None, max_lanes=None):
        self.families = {f.key: f for f in families}
        self.cfg = cfg or ServeConfig()
        self._bufs = {}
        self._lanes = {}
        self.pool_bytes = pool_bytes
        self.max_lanes = max_lanes  # per family, on top of the byte budget (None: no cap)
        self.lane_bytes = {}     # family key -> measured bytes of one lane
        self._pool = []          # _LaneCtx of every lane in the pool
        self.pool_events = []    # ("add" | "retire", family key, bytes, time)

    def _solve_batch(self, fam: Family, op, pc, reqs):
        """Mixed-precision solves of reqs (len <= members) in lockstep on one
        lane; returns [(info, x)]."""
        import ctypes
        from . import _lib
        if self.cfg.mode != "mixed":
            return [self._solve(fam, op, pc, r) for r in reqs]
        lib = _lib.lib()
        n = op.n
        count = len(reqs)
        bre = np.empty((count, n))
        bim = np.empty((count, n))
        for i, req in enumerate(reqs):
            op.interp(fam.node_ops, lagrange_weights(req.lam, fam.nodes), member=i)
            b = fam.rhs(geo.C0 / req.lam * geo.N_EXT)
            bre[i] = b.real
            bim[i] = b.imag
        xre = np.empty((count, n))
        xim = np.empty((count, n))
        infos = (_lib.GmresInfo * count)()
        c = self.cfg
        side = (1 if c.side == "left" else 2) if pc is not None else 0
        _lib.check(lib.vox_solve_refined_batch(op.handle, pc.handle if pc is not None else None,
                                               side, count, _lib.dptr(bre), _lib.dptr(bim),
                                               c.tol, c.restart, c.maxit_inner, c.inner_tol, 10,
                                               _lib.dptr(xre), _lib.dptr(xim), infos))
        return [(infos[i], (xre[i] + 1j * xim[i]) if c.keep_x else None) for i in range(count)]

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
        c = self.cfg
        side = (1 if c.side == "left" else 2) if pc is not None else 0
        pch = pc.handle if pc is not None else None
        if c.mode == "mixed":
            _lib.check(lib.vox_solve_refined(op.handle, pch, side, _lib.dptr(bre), _lib.dptr(bim),
                                             c.tol, c.restart, c.maxit_inner, c.inner_tol, 10,
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

    def _solve_batch_device(self, fam: Family, op, pc, reqs, dev_b, dev_x):
        """As _solve_batch with right-hand sides and solutions in device memory
        (dev_b / dev_x: request id -> complex128 torch tensor), staged through the
        lane's buffers on the lane's stream."""
        import torch
        c = self.cfg
        n = op.n
        s = op.torch_stream
        key = id(op)
        with torch.cuda.stream(s):
            if key not in self._bufs:
                self._bufs[key] = (torch.empty(op.members * n, dtype=torch.complex128,
                                               device="cuda"),
                                   torch.empty(op.members * n, dtype=torch.complex128,
                                               device="cuda"))
            bbuf, xbuf = self._bufs[key]
            for i, req in enumerate(reqs):
                op.interp(fam.node_ops, lagrange_weights(req.lam, fam.nodes), member=i)
                bbuf[i * n:(i + 1) * n].copy_(dev_b[req.rid])
            infos = op.solve_refined_batch_device(
                bbuf.data_ptr(), xbuf.data_ptr(), len(reqs), pc=pc, side=c.side,
                tol=c.tol, restart=c.restart, maxit_inner=c.maxit_inner, inner_tol=c.inner_tol,
                max_refine=10)
            for i, req in enumerate(reqs):
                dev_x[req.rid].copy_(xbuf[i * n:(i + 1) * n])
        return [(inf, None) for inf in infos]

    def prepare_device(self):
        """Allocate every lane's staging buffers for device-resident serving."""
        import torch
        for fam in self.families.values():
            for op, pc in fam.slots:
                with torch.cuda.stream(op.torch_stream):
                    self._bufs[id(op)] = (
                        torch.empty(op.members * op.n, dtype=torch.complex128, device="cuda"),
                        torch.empty(op.members * op.n, dtype=torch.complex128, device="cuda"))

    def warm(self):
        """One full batch on every lane of every family (captures each lane's
        restart-cycle graph before any timed work)."""
        for fam in self.families.values():
            lam = float(np.mean(fam.nodes))
            reqs = [Request(-1, fam.key, lam, 0.0)] * fam.members
            for op, pc in fam.slots:
                self._solve_batch(fam, op, pc, reqs)

    def _lane(self, fam: Family, op, pc):
        key = id(op)
        if key not in self._lanes:
            c = self.cfg
            self._lanes[key] = Lane(op, pc, side=c.side, tol=c.tol, restart=c.restart,
                                    maxit_inner=c.maxit_inner, inner_tol=c.inner_tol,
                                    max_refine=10)
        return self._lanes[key]

    def close(self):
        for ln in self._lanes.values():
            ln.close()
        self._lanes = {}

    # ------------------------------------------------------- HBM pool
    def pool_used(self):
        return sum(c.nbytes for c in self._pool)

    def pool_summary(self):
        """Lanes per family now, bytes admitted per lane, lanes added and retired."""
        out = {}
        for fam in self.families.values():
            k = fam.key
            out[str(k)] = {"lanes": sum(1 for c in self._pool if c.fam is fam),
                           "lane_bytes": self.lane_bytes.get(k),
                           "added": sum(1 for e in self.pool_events if e[0] == "add" and e[1] == k),
                           "retired": sum(1 for e in self.pool_events
                                          if e[0] == "retire" and e[1] == k)}
        return {"budget_bytes": self.pool_bytes, "used_bytes": self.pool_used(),
                "families": out}

    def pool_peak(self):
        """Largest sum of admitted lane bytes over the pool's history."""
        used = peak = 0
        for ev, _, nb, _ in self.pool_events:
            used += nb if ev == "add" else -nb
            peak = max(peak, used)
        return peak

    def _new_lane(self, fam):
        """A lane for fam inside the pool: batched operator, shared
        preconditioner handle, lane state and its own stream; its bytes are
        measured once per family (operator, work, Krylov arenas)."""
        import torch
        torch.cuda.synchronize()
        held0 = _lib.mem_in_use(fam.device)
        op, pc = fam.add_slot(torch.cuda.Stream())
        lane = self._lane(fam, op, pc)
        if fam.key not in self.lane_bytes:
            # one warm solve allocates the lane's arenas and captures its graph;
            # the library's own count of device bytes, so the CUDA context,
            # modules loaded on first use and torch's pool do not enter it
            lam = float(np.mean(fam.nodes))
            op.interp(fam.node_ops, lagrange_weights(lam, fam.nodes), member=0)
            lane.submit(0, fam.rhs(geo.C0 / lam * geo.N_EXT))
            while not lane.step():
                pass
            lane.collect(0, host=False)
            torch.cuda.synchronize()
            self.lane_bytes[fam.key] = max(_lib.mem_in_use(fam.device) - held0, 1)
        ctx = _LaneCtx(fam, op, pc, lane, self.lane_bytes[fam.key])
        self._pool.append(ctx)
        self.pool_events.append(("add", fam.key, ctx.nbytes, time.perf_counter()))
        return ctx

    def _drop_lane(self, ctx):
        """Free a lane that has left the pool (its worker has stopped)."""
        self._lanes.pop(id(ctx.op), None)
        ctx.lane.close()
        if ctx.pc is not None:
            ctx.pc.close()
        ctx.op.close()
        ctx.fam.slots = [sl for sl in ctx.fam.slots if sl[0] is not ctx.op]
        self._pool.remove(ctx)
        self.pool_events.append(("retire", ctx.fam.key, ctx.nbytes, time.perf_counter()))

    def prepare_pool(self, lanes_per_family=1):
        """At least lanes_per_family lanes per family in the pool (each lane
        measured and warm), within the budget."""
        for fam in self.families.values():
            while sum(1 for c in self._pool if c.fam is fam) < lanes_per_family:
                if self._pool and self.pool_used() + self.lane_bytes.get(fam.key, 0) > \
                        self.pool_bytes:
                    break
                self._new_lane(fam)

    def close_pool(self):
        for ctx in list(self._pool):
            self._drop_lane(ctx)

    def _serve_pool(self, requests, realtime, device_io):
        """Continuous batching with lanes admitted and retired by footprint."""
        queues = {k: deque() for k in self.families}
        for r in sorted(requests, key=lambda r: r.arrival):
            queues[r.key].append(r)
        qlock = threading.Lock()
        results = []
        res_lock = threading.Lock()
        errors = []
        t0 = time.perf_counter()
        pending = [len(requests)]

        def arrived(key, now):
            return sum(1 for r in queues[key] if not realtime or r.arrival <= now)

        def worker(ctx):
            fam, op, lane = ctx.fam, ctx.op, ctx.lane
            q = queues[fam.key]
            try:
                while True:
                    free = [m for m in range(lane.members) if m not in ctx.inflight]
                    admit = []
                    with qlock:
                        if not ctx.retire:
                            now = time.perf_counter() - t0
                            while free and q and (not realtime or q[0].arrival <= now):
                                admit.append((free.pop(0), q.popleft()))
                    for m, req in admit:
                        op.interp(fam.node_ops, lagrange_weights(req.lam, fam.nodes), member=m)
                        if device_io is not None:
                            dev_b, dev_x = device_io
                            lane.submit_device(m, dev_b[req.rid].data_ptr(),
                                               dev_x[req.rid].data_ptr())
                        else:
                            lane.submit(m, fam.rhs(geo.C0 / req.lam * geo.N_EXT))
                        ctx.inflight[m] = (req, time.perf_counter() - t0)
                    if not ctx.inflight:
                        if ctx.retire or ctx.stop:
                            return
                        time.sleep(2e-4)
                        continue
                    for m in lane.step():
                        req, start = ctx.inflight.pop(m)
                        x, info = lane.collect(m, host=device_io is None)
                        done = time.perf_counter() - t0
                        with res_lock:
                            results.append(Result(req.rid, req.key, req.lam,
                                                  req.arrival if realtime else 0.0, start, done,
                                                  info["iters"], info["relres"], info["flag"],
                                                  x if self.cfg.keep_x else None,
                                                  info.get("refinements", 0)))
                            pending[0] -= 1
            except Exception as e:  # surfaced after the threads join
                errors.append(e)

        def start(ctx):
            ctx.stop = ctx.retire = False
            ctx.thread = threading.Thread(target=worker, args=(ctx,), daemon=True)
            ctx.thread.start()

        for ctx in self._pool:
            start(ctx)
        try:
            while pending[0] > 0 and not errors:
                now = time.perf_counter() - t0
                for fam in self.families.values():
                    mine = [c for c in self._pool if c.fam is fam and not c.retire]
                    with qlock:
                        want = arrived(fam.key, now)
                    free_slots = sum(c.lane.members - len(c.inflight) for c in mine)
                    if want <= free_slots or want == 0:
                        continue
                    if self.max_lanes is not None and len(mine) >= self.max_lanes:
                        continue
                    need = self.lane_bytes.get(fam.key)
                    if need is None or self.pool_used() + need > self.pool_bytes:
                        # retire an idle lane of a family with nothing waiting
                        # (every family keeps one lane, warm for its next request)
                        for c in self._pool:
                            if c.fam is fam or c.retire or c.inflight:
                                continue
                            if sum(1 for o in self._pool if o.fam is c.fam) <= 1:
                                continue
                            with qlock:
                                waiting = arrived(c.fam.key, now)
                            if waiting == 0:
                                c.retire = True
                                c.thread.join()
                                self._drop_lane(c)
                                break
                    if need is None or self.pool_used() + need <= self.pool_bytes:
                        start(self._new_lane(fam))
                time.sleep(1e-3)
        finally:
            for ctx in self._pool:
                ctx.stop = True
            for ctx in self._pool:
                if ctx.thread is not None:
                    ctx.thread.join()
        wall = time.perf_counter() - t0
        if errors:
            raise errors[0]
        return sorted(results, key=lambda r: r.rid), wall

    def serve(self, requests, realtime=True, device_io=None):
        """Run the stream; returns (results, wall seconds).  device_io =
        (dev_b, dev_x) serves right-hand sides already in device memory and
        leaves the solutions there."""
        if self.pool_bytes is not None and self.cfg.batching == "continuous" and \
                self.cfg.mode == "mixed":
            return self._serve_pool(requests, realtime, device_io)
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
            K = getattr(op, "members", 1)
            while True:
                with locks[fam.key]:
                    if not q:
                        return
                    first = q.popleft()
                now = time.perf_counter() - t0
                if realtime and first.arrival > now:
                    time.sleep(first.arrival - now)
                # every request of this length that has arrived by now, up to K
                batch = [first]
                with locks[fam.key]:
                    now = time.perf_counter() - t0
                    while q and len(batch) < K and (not realtime or q[0].arrival <= now):
                        batch.append(q.popleft())
                start = time.perf_counter() - t0
                try:
                    if device_io is not None:
                        out = self._solve_batch_device(fam, op, pc, batch, *device_io)
                    else:
                        out = self._solve_batch(fam, op, pc, batch)
                except Exception as e:  # surfaced after the threads join
                    errors.append(e)
                    return
                done = time.perf_counter() - t0
                with res_lock:
                    for req, (info, x) in zip(batch, out):
                        results.append(Result(req.rid, req.key, req.lam,
                                              req.arrival if realtime else 0.0, start, done,
                                              info.total_iters, info.relres, info.flag, x))

        def lane_worker(fam, op, pc):
            # continuous batching: admit arrived requests into free members,
            # run one restart cycle of every solving member, collect the
            # finished ones, repeat
            q = queues[fam.key]
            lane = self._lane(fam, op, pc)
            inflight = {}  # member -> (request, start time)
            try:
                while True:
                    free = [m for m in range(lane.members) if m not in inflight]
                    admit = []
                    with locks[fam.key]:
                        now = time.perf_counter() - t0
                        while free and q and (not realtime or q[0].arrival <= now):
                            admit.append((free.pop(0), q.popleft()))
                        nxt = q[0].arrival if q else None
                    for m, req in admit:
                        op.interp(fam.node_ops, lagrange_weights(req.lam, fam.nodes), member=m)
                        if device_io is not None:
                            dev_b, dev_x = device_io
                            lane.submit_device(m, dev_b[req.rid].data_ptr(),
                                               dev_x[req.rid].data_ptr())
                        else:
                            lane.submit(m, fam.rhs(geo.C0 / req.lam * geo.N_EXT))
                        inflight[m] = (req, time.perf_counter() - t0)
                    if not inflight:
                        if nxt is None:
                            return
                        time.sleep(max(0.0, nxt - (time.perf_counter() - t0)))
                        continue
                    for m in lane.step():
                        req, start = inflight.pop(m)
                        x, info = lane.collect(m, host=device_io is None)
                        done = time.perf_counter() - t0
                        with res_lock:
                            results.append(Result(req.rid, req.key, req.lam,
                                                  req.arrival if realtime else 0.0, start, done,
                                                  info["iters"], info["relres"], info["flag"],
                                                  x if self.cfg.keep_x else None,
                                                  info.get("refinements", 0)))
            except Exception as e:  # surfaced after the threads join
                errors.append(e)

        target = lane_worker if (self.cfg.batching == "continuous" and self.cfg.mode == "mixed") \
            else worker
        threads = [threading.Thread(target=target, args=(fam, op, pc), daemon=True)
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
            "mean_refinements": float(np.mean([r.refinements for r in results])),
            "flags": int(np.sum([r.flag for r in results]))}
