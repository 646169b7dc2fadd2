"""Benchmark: GMRES solves/s of the JVIE-II frequency solve on B200.

Workload (default, `--workload sweep`): the mixed-length Bragg sweep - gratings
of 20, 40, 60, 80 and 100 periods (520-1800 x 30 x 11 at 20 nm), 201
wavelengths over 1500-1600 nm each = 1005 solves arriving as a seeded Poisson
stream, complex64 GMRES(50) + FP64 refinement to 1e-5 relative residual
||b - A x|| / ||b|| on continuously batched lanes, against the plain complex128
drop-in solved one request at a time.  Synthetic, seeded geometry; operators
assembled by libvox; everything in the timed region runs in libvox's sm_100a
kernels.  Other workloads: microdisk, mor, bragg20, bragg20-p<N>, strip,
bragg10 (single solves).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vox|reference]
                    [--workload sweep|microdisk|mor|bragg20|strip|bragg10]

--impl reference: the reference's CPU path (the numpy oracle; MATLAB is
absent) on the host cores, whole solves.  N > 1 (torchrun): independent
replicas, one per GPU (the solve does not shard); value = total solves /
max-over-ranks device time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GMRES solves/s + p50/p99 latency: FP32+refine vs FP64 on B200 at 1e-5 residual"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (sweep: the whole 1005-solve stream divided into K "
                         "steps, default 20; other workloads: K solves, default 10)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vox", choices=["vox", "reference"])
    ap.add_argument("--workload", default="sweep",
                    help="sweep (default) | microdisk | mor | stages | bragg20 | bragg20-p<N> | "
                         "strip | bragg10")
    ap.add_argument("--precond", default="level1", choices=["none", "level1"])
    ap.add_argument("--tol", type=float, default=1e-5)
    ap.add_argument("--restart", type=int, default=50)
    ap.add_argument("--inner-tol", type=float, default=0.0,
                    help="complex64 inner GMRES tolerance (0: aim at the target directly, "
                         "f * tol * ||b|| / ||r|| with the library's f; negative: f = -value)")
    ap.add_argument("--fp64-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg")
    ap.add_argument("--no-stages", action="store_true", help="skip per-kernel timing")
    ap.add_argument("--sweep-periods", default="20,40,60,80,100")
    ap.add_argument("--sweep-lambdas", type=int, default=201)
    ap.add_argument("--sweep-rate", type=float, default=200.0,
                    help="Poisson arrival rate (requests/s) of the sweep stream")
    ap.add_argument("--sweep-slots", type=int, default=1,
                    help="most lanes per device length in the HBM pool (more lanes share "
                         "the GPU's L2 and measured slower on the sweep)")
    ap.add_argument("--sweep-members", type=int, default=4,
                    help="solves per lane advanced in lockstep (batched operator members)")
    ap.add_argument("--sweep-side", default="right", choices=["left", "right"],
                    help="preconditioning side of the mixed-precision inner solves")
    ap.add_argument("--sweep-batching", default="continuous", choices=["continuous", "lockstep"],
                    help="member slots refilled as solves finish, or whole batches")
    ap.add_argument("--sweep-fp64", type=int, default=50,
                    help="requests solved one at a time in plain complex128 for the baseline")
    ap.add_argument("--disk-restart", type=int, default=128,
                    help="GMRES restart length of the microdisk workload (the resonator "
                         "stagnates under GMRES(50))")
    ap.add_argument("--disk-fp64", type=int, default=3,
                    help="microdisk wavelengths solved by the plain FP64 drop-in")
    ap.add_argument("--mor-config", default="bragg20",
                    help="grating of the reduced-order sweep (bragg20 = 1160 x 30 x 11)")
    ap.add_argument("--mor-order", type=int, default=5)
    ap.add_argument("--mor-tol", type=float, default=1e-4,
                    help="tolerance of the model's solves (the script's 1e-4)")
    ap.add_argument("--mor-check", type=int, default=5,
                    help="wavelengths compared against full solves")
    ap.add_argument("--stage-periods", type=int, default=60,
                    help="stages workload: grating periods (60 = 1160 x 30 x 11)")
    ap.add_argument("--stage-prec", default="c64", choices=["c64", "c128"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-clocks", action="store_true",
                    help="do not spawn the nvidia-smi clock sampler (profiler runs)")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [s.strip() for s in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": ["no samples"]}
        # median over samples under load (clock above idle floor)
        load = [s for s in sm if s > 0.5 * (smax or max(sm))] or sm
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_traffic(kernel, alg_bytes):
    """DRAM bytes per launch of stage `kernel` from the committed ncu summaries
    (a line 'traffic_ratio <stage> <r>' in profiles/*.md: measured dram bytes /
    algorithmic bytes on the captured case), scaled to this launch's algorithmic
    bytes (traffic grows with the tiles streamed); None when no capture covers
    the stage."""
    import glob
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            for line in f:
                parts = line.strip().strip("`").split()
                if len(parts) == 3 and parts[0] == "traffic_ratio" and parts[1] == kernel:
                    return float(parts[2]) * alg_bytes
    return None


def build_problem(name):
    from voxphoton_b200 import geometry as geo
    import voxphoton_b200 as vb
    p = geo.bragg_config(name)
    t = time.time()
    G = vb.assemble_toeplitz(p.shape, p.ko, p.res)
    t_asm = time.time() - t
    Einc = geo.plane_wave(p)
    idx = p.idxS3()
    b = vb.jvie_rhs(p.e_r, Einc, p.Gram, p.freq, idx)
    return p, G, idx, b, t_asm


def kernel_bytes(op_info, shape, n, pc_info, k, c=8):
    """Algorithmic bytes per launch of each stage for one member, c bytes per
    complex value (8: complex64, 16: complex128); int32 index maps."""
    L, M, N = shape
    V = L * M * N
    Px, Py, Pz = op_info["Px"], op_info["Py"], op_info["Pz"]
    T = Px * 3 * N * M * c
    n3 = 3 * M * N
    if op_info.get("octant_fN"):
        fN_bytes = 6 * (Px // 2 + 1) * (Py // 2 + 1) * (Pz // 2 + 1) * c
    else:
        fN_bytes = 6 * Px * Py * Pz * c
    b = {
        "mv_xfwd": n * c + 3 * V * 4 + T,
        "mv_plane": 2 * T + fN_bytes,
        "mv_xinv": T + 2 * n * c + 3 * V * 4 + V * c,
        "gs_dots": (k + 1) * n * c + n * c,
        "gs_update_dots": (k + 1) * n * c + 2 * n * c,
        "gs_update_norm": (k + 1) * n * c + 2 * n * c,
        "gs_scale": 2 * n * c,
    }
    if pc_info:
        # the stored inverse blocks (n3 x n3 each, read once for both paired
        # modes and every member), the transformed vectors in and out
        nf = pc_info["n_blocks"]
        b["pc_xfwd"] = n * c + 3 * V * 4 + L * n3 * c
        b["pc_solve"] = nf * n3 * n3 * c + 2 * L * n3 * c
        b["pc_xinv"] = L * n3 * c + 3 * V * 4 + n * c
    return b


def matvec_roofline(op_info, shape, n, pc_info, members, ms, hbm, c=8):
    """The matvec chain's bytes, achieved GB/s and fraction of the HBM peak for
    one launch of `members` members taking `ms` milliseconds, on two byte
    counts: the kernels' own (kernel_bytes: vector, index map, the x-frequency
    planes once each way, the stored fN octant) and the compulsory figure of
    the full padded product, c * (7V + 6P) per member (J in, Mc, out and the
    six fN components over the P = Px Py Pz padded cells)."""
    L, M, N = shape
    V = L * M * N
    P = op_info["Px"] * op_info["Py"] * op_info["Pz"]
    kb = kernel_bytes(op_info, shape, n, pc_info, 20, c)
    own = members * (kb["mv_xfwd"] + kb["mv_plane"] + kb["mv_xinv"])
    full = members * c * (7 * V + 6 * P)
    s = ms * 1e-3
    return {"bytes_per_launch": own, "ms": ms, "achieved": own / s / 1e9,
            "frac": own / s / 1e9 / hbm,
            "compulsory_full_fN": {"bytes_per_launch": full, "achieved": full / s / 1e9,
                                   "frac": full / s / 1e9 / hbm}}


def _cpu_geometry():
    """voxphoton_b200/geometry.py (numpy only) loaded from its file: importing
    the package would load libvox, which the CPU reference path never touches."""
    import importlib.util
    name = "_vox_geometry_cpu"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(
            name, os.path.join(ROOT, "voxphoton_b200", "geometry.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


class OracleGrating:
    """The reference CPU path for one Bragg grating of the sweep, on the oracle
    (numpy complex128 restatement of the reference; libvox is never loaded):

    * Toeplitz tensors at the nG Legendre wavelengths of the band
      (assembly_nop_const.m with the reference's own compiled cubature cores,
      oracle/_ref) and their circulants fN (circulant_nop_const.m,
      fft_operator.m);
    * the level-1 preconditioner at the band centre (level_1_parallel_func_N.m
      + Bragg_MOR_script.m:61-72: one dense inverse per x-mode, all L of them);
    * per request: fN interpolated to its wavelength (lagrange_int.m), the
      plane-wave JVIE-II right-hand side, then
      pgmres(A, b, restart, tol, maxit, L1 = chan_mvp_idx) (pgmres.m:70-181).

    FFTs run on `threads` scipy.fft workers, the dense products on numpy's
    BLAS threads.  Only the pgmres call is timed."""

    def __init__(self, periods, band, threads, nG=5):
        from oracle import assembly as oa
        from oracle import vie as ov
        self.ov = ov
        self.geo = _cpu_geometry()
        ov.set_fft_workers(threads)
        self.threads = threads
        self.p = self.geo.bragg(periods=periods, M=30)
        self.nodes = ov.legendre_wavelengths(band[0], band[1], nG)
        t = time.perf_counter()
        Gc = None
        self.fN = []
        for j, lam in enumerate(self.nodes):
            q = self.p.with_wavelength(lam)
            G = oa.assembly_nop_const(q.shape, q.ko, q.res)
            self.fN.append(ov.fN_from_toeplitz(G))
            if j == nG // 2:
                Gc = G
        L, M, N = self.p.shape
        circ, _ = ov.level_1_parallel_func_N(Gc, L, M, N, self.p.Gram)
        self.inv = ov.level1_inverse_blocks(circ, ov.face_from_Mr(self.p.e_r.astype(complex)),
                                            self.p.Gram)
        self.setup_s = time.perf_counter() - t

    def solve(self, lam, tol, restart, maxit):
        """One request; returns (seconds in pgmres, iterations, relres, flag)."""
        ov = self.ov
        q = self.p.with_wavelength(lam)
        _, Mc, idx, b = ov.jvie2_system(self.geo.plane_wave(q), q.e_r, q.Gram, q.freq)
        fN = ov.lagrange_int(self.fN, lam, self.nodes)
        L, M, N = q.shape
        ones = np.ones(q.shape)

        def A(v):
            return ov.mv_AN_const(v, fN, ones, Mc, q.Gram, "notransp", idx)

        def P(v):
            return ov.chan_mvp_idx(self.inv, v, L, M, N, idx)

        t = time.perf_counter()
        _, flag, relres, _, rv = ov.pgmres(A, b, restart, tol, maxit, L1=P)
        return time.perf_counter() - t, len(rv) - 1, float(relres), int(flag)


def _sweep_items(periods, lams):
    return [(pr, lam) for lam in lams for pr in periods]


def _cpu_sample(reqs, key, count):
    """The first `count` requests of length `key` in arrival order (cycled)."""
    own = [r for r in sorted(reqs, key=lambda r: r.arrival) if r.key == key]
    return [own[i % len(own)] for i in range(count)]


def cpu_baseline_sweep(args, reqs, band, solves=2):
    """The oracle on the host cores: `solves` whole requests of the sweep's
    shortest grating (all threads), as solves/s."""
    from voxphoton_b200 import serving as sv  # noqa: F401  (request type only)
    periods = [int(x) for x in args.sweep_periods.split(",")]
    key = min(periods)
    threads = os.cpu_count() or 1
    og = OracleGrating(key, band, threads)
    ts, its, rr, fl = [], [], [], []
    for r in _cpu_sample(reqs, key, solves):
        dt, k, rel, flag = og.solve(r.lam, args.tol, args.restart, 10)
        ts.append(dt)
        its.append(k)
        rr.append(rel)
        fl.append(flag)
    L, M, N = og.p.shape
    return {"value": len(ts) / sum(ts), "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"{len(ts)} whole requests of the {key}-period grating ({L}x{M}x{N}, the "
                      f"sweep's shortest, so an upper bound on the CPU rate over the sweep): "
                      f"numpy complex128 oracle pgmres(A, b, {args.restart}, {args.tol}, 10, "
                      f"L1 = chan_mvp_idx), operator by lagrange_int over 5 Legendre nodes, "
                      f"level-1 inverse blocks at the band centre; {sum(ts):.1f} s in pgmres, "
                      f"{np.mean(its):.1f} iterations, max relres {max(rr):.2e}, flags "
                      f"{sum(fl)}; setup (assembly with the reference's cubature cores, "
                      f"{L} dense inverses) {og.setup_s:.1f} s, untimed"}


def run_reference(args, world, rank):
    """--impl reference: the reference's CPU path (its oracle restatement:
    MATLAB/Octave are absent) on the host cores, whole solves only.

    Sweep: each step is one whole request of the seeded stream on the
    sweep's shortest grating (20 periods, 520 x 30 x 11), solved as the
    reference does - operator interpolated over 5 Legendre nodes, level-1
    preconditioner (all L dense inverse blocks) at the band centre,
    left-preconditioned pgmres(50) to the tolerance.  The shortest grating
    is the cheapest solve of the sweep, so this rate is an upper bound on the
    CPU path's solves/s over the mixed stream."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    steps = args.steps or 20
    if args.workload != "sweep":
        print(json.dumps({"impl": "reference", "unavailable":
                          f"the CPU reference arm covers the sweep workload only "
                          f"(asked: {args.workload})"}), flush=True)
        return
    band = (1500e-9, 1600e-9)
    periods = [int(x) for x in args.sweep_periods.split(",")]
    key = min(periods)
    lams = np.linspace(band[0], band[1], args.sweep_lambdas)
    reqs = _poisson(_sweep_items(periods, lams), args.sweep_rate, args.seed)
    og = OracleGrating(key, band, threads)
    sample = _cpu_sample(reqs, key, args.warmup + steps)
    for r in sample[:args.warmup]:
        og.solve(r.lam, args.tol, args.restart, 10)
    ts, its, rr, fl = [], [], [], []
    for r in sample[args.warmup:]:
        dt, k, rel, flag = og.solve(r.lam, args.tol, args.restart, 10)
        ts.append(dt)
        its.append(k)
        rr.append(rel)
        fl.append(flag)
    tot = sum(ts)
    val = steps / tot
    L, M, N = og.p.shape
    sample_txt = (f"{steps} whole requests of the {key}-period grating ({L}x{M}x{N}), "
                  f"numpy complex128 oracle, pgmres(A, b, {args.restart}, {args.tol}, 10, "
                  f"L1 = chan_mvp_idx), {threads} threads; {np.mean(its):.1f} iterations per "
                  f"solve, max relres {max(rr):.2e}, flags {sum(fl)}")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "solves/s",
            "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * tot / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": f"sweep: mixed-length Bragg gratings of {periods} periods, "
                                   f"{len(lams)} wavelengths over 1500-1600 nm each = "
                                   f"{len(reqs)} solves; the CPU reference solves whole "
                                   f"requests of its shortest grating ({L}x{M}x{N})",
                       "tol": args.tol, "restart": args.restart,
                       "precond": "level1 at band centre, left (pgmres L1)",
                       "setup_s": round(og.setup_s, 1)},
            "cpu_baseline": {"value": val, "unit": "solves/s", "cores": threads, "kind": "port",
                             "sample": sample_txt},
            "e2e": {"value": val, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _poisson(items, rate, seed):
    """serving.poisson_stream without importing the package (same draws)."""
    from types import SimpleNamespace
    rng = np.random.default_rng(seed)
    order = rng.permutation(len(items))
    t = np.cumsum(rng.exponential(1.0 / rate, size=len(items)))
    return [SimpleNamespace(rid=int(i), key=items[k][0], lam=items[k][1], arrival=float(t[i]))
            for i, k in enumerate(order)]


def _progress(msg, _t0=[time.time()]):
    print(f"[bench {time.time() - _t0[0]:7.1f} s] {msg}", file=sys.stderr, flush=True)


def _assemble_family_nodes(periods, band, device):
    """Toeplitz tensors of every (device length, Legendre node) pair, the
    regular cubature on this rank's GPU (vox_assemble_toeplitz_device)."""
    import voxphoton_b200 as vb
    from voxphoton_b200 import geometry as geo
    from voxphoton_b200 import serving as sv
    nodes = sv.legendre_nodes(band[0], band[1], 5)
    out = {}
    for pr in periods:
        for j in range(len(nodes)):
            q = geo.bragg(periods=pr, M=30).with_wavelength(nodes[j])
            out[(pr, j)] = vb.assemble_toeplitz(q.shape, q.ko, q.res, device=device)
    return out


def run_sweep(args, world, rank, local):
    """Mixed-length Bragg sweep served as a Poisson request stream.

    The stream is always the whole sweep: 5 gratings x 201 wavelengths over
    1500-1600 nm = 1005 solves per GPU (each rank serves its own copy:
    replicas, weak scaling); --steps K only divides it (one step = 1005/K
    solves, ms_per_step = stream time / K) and --warmup W serves W steps' worth
    of extra requests before timing.  After a common warm-up, two legs are
    timed back to back on the same warm lanes:

    * e2e (first): the stream through the host-buffer C-ABI (vox_lane_submit /
      vox_lane_collect), right-hand sides formed on the host and copied in,
      solutions copied out, inside the timed region;
    * value (second): the same stream with every right-hand side already in
      HBM (vox_lane_submit_device), solutions left there."""
    import torch
    import voxphoton_b200 as vb
    from voxphoton_b200 import geometry as geo
    from voxphoton_b200 import serving as sv
    torch.cuda.set_device(local)
    periods = [int(x) for x in args.sweep_periods.split(",")]
    band = (1500e-9, 1600e-9)
    lams = np.linspace(band[0], band[1], args.sweep_lambdas)
    items = _sweep_items(periods, lams)
    total = len(items)
    steps = args.steps if args.steps else 20
    per_step = total / steps
    t = time.time()
    Gs = _assemble_family_nodes(periods, band, local)
    fams = [sv.Family(pr, geo.bragg(periods=pr, M=30), band, nG=5, device=local,
                      members=args.sweep_members, G_nodes=[Gs[(pr, j)] for j in range(5)])
            for pr in periods]
    setup_s = time.time() - t
    _progress("setup")
    # admission by HBM footprint: one device-memory pool for the lanes of
    # every length (80 % of what is free after setup, less room for the
    # device-resident right-hand sides and solutions); lanes are admitted (and retired) by their measured bytes as
    # the queues of the lengths fill, up to --sweep-slots lanes per length
    torch.cuda.synchronize()
    free0, total_mem = torch.cuda.mem_get_info()
    io_bytes = 2 * 16 * len(lams) * sum(f.idx.size for f in fams)
    budget = int(0.8 * (free0 - io_bytes))
    reqs = sv.poisson_stream(items, rate=args.sweep_rate, seed=args.seed + rank)
    cfg = sv.ServeConfig(tol=args.tol, side=args.sweep_side, batching=args.sweep_batching,
                         inner_tol=args.inner_tol)
    srv = sv.SweepServer(fams, cfg, pool_bytes=budget, max_lanes=args.sweep_slots)
    srv.prepare_pool(1)
    # common warm-up: W steps' worth of requests at wavelengths between the
    # sweep's (admits the lanes the queues ask for and captures their graphs)
    n_warm = max(len(periods), int(round(args.warmup * per_step)))
    wl = np.linspace(band[0], band[1], n_warm // len(periods) + 2)[1:-1]
    srv.serve([sv.Request(-1 - i, pr, lam, 0.0)
               for i, (pr, lam) in enumerate(_sweep_items(periods, wl))], realtime=False)
    torch.cuda.synchronize()
    _progress(f"warm ({n_warm} requests)")
    fam_of = {f.key: f for f in fams}
    clocks = None if args.no_clocks else Clocks(local)
    if clocks:
        clocks.start()
    # leg 1: e2e through the host-buffer C-ABI
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e2.record()
    res_h, wall_h = srv.serve(reqs, realtime=True)
    torch.cuda.synchronize()
    e3.record()
    torch.cuda.synchronize()
    e2e_s = e2.elapsed_time(e3) / 1e3
    summ_h = sv.summarize(res_h, wall_h)
    _progress(f"host-buffer stream: {len(reqs)} solves in {e2e_s:.2f} s")
    # every request's right-hand side resident in HBM before the second leg
    dev_b = {}
    for r in reqs:
        b = fam_of[r.key].rhs(geo.C0 / r.lam * geo.N_EXT)
        dev_b[r.rid] = torch.from_numpy(b).to("cuda")
    dev_x = {r.rid: torch.empty_like(dev_b[r.rid]) for r in reqs}
    torch.cuda.synchronize()
    # leg 2: device-resident
    lane_ops = [op for f in fams for op, _ in f.slots]
    l0 = sum(op.launches() for op in lane_ops)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    res_dev, wall_dev = srv.serve(reqs, realtime=True, device_io=(dev_b, dev_x))
    torch.cuda.synchronize()
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else {"sm_mhz": None, "sm_max_mhz": None,
                                        "reasons": ["not sampled (--no-clocks)"]}
    dev_s = e0.elapsed_time(e1) / 1e3
    lane_ops_end = [op for f in fams for op, _ in f.slots]
    launches = (sum(op.launches() for op in lane_ops_end if op in lane_ops) - l0 +
                sum(op.launches() for op in lane_ops_end if op not in lane_ops) +
                10 * len(reqs))
    pool = srv.pool_summary()
    pool["peak_bytes"] = srv.pool_peak()
    summ_dev = sv.summarize(res_dev, wall_dev)
    _progress(f"device-resident stream: {len(reqs)} solves in {dev_s:.2f} s")
    # roofline of the dominant kernel: the inverse-block apply of one lane of
    # the 1160 x 30 x 11 grating at the lane's width (stage timing by CUDA
    # events on the lane's stream)
    fmid = fam_of[periods[len(periods) // 2]]
    op_m, pc_m = fmid.slots[0]
    stage = op_m.profile_stages(pc_m, prec="c64", restart=args.restart, kgs=20, reps=10)
    info_m = pc_m.info()
    L, M, N = fmid.p.shape
    n3 = 3 * M * N
    K = args.sweep_members
    alg = info_m["n_blocks"] * n3 * n3 * 8 + 2 * K * L * n3 * 8
    hbm, src = peaks()
    ach = alg / (stage["pc_solve"] * 1e-3) / 1e9
    mv_ms = stage["mv_xfwd"] + stage["mv_plane"] + stage["mv_xinv"]
    mv_roof = matvec_roofline(op_m.info(), fmid.p.shape, fmid.idx.size, info_m, K, mv_ms, hbm)
    roof = {"bound": "hbm", "kernel": f"pc_solve (k_pc_inv_stream, {K} members, "
                                      f"{L}x{M}x{N})",
            "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
            "traffic": measured_traffic("pc_solve", alg), "peak_source": src,
            "bytes_per_launch": alg, "ms_per_launch": stage["pc_solve"],
            "stage_ms": stage,
            "matvec": {"kernels": "k_xfwd + k_plane64 + k_xinv", "members": K, **mv_roof}}
    # the lanes are done: free them and the staged vectors before the baseline
    del dev_b, dev_x
    srv.close_pool()
    srv.close()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    _progress("lanes released")
    # plain complex128 GMRES (left-preconditioned pgmres, the drop-in), strictly
    # one solve at a time on one thread, on one single-member operator per
    # length, on a seeded subset of the stream; each length's complex128 cycle
    # graph is captured by an untimed first solve
    for f in fams:
        op1 = vb.Operator(f.mop, f.p.Gram, f.idx, G=f._Gc, device=local)
        f.slots = [(op1, f.pc.share(op1))]
    rng = np.random.default_rng(args.seed)
    sub = [reqs[i] for i in rng.choice(len(reqs), size=min(len(reqs), args.sweep_fp64),
                                       replace=False)]

    def fp64_serial_run(side):
        srv64 = sv.SweepServer(fams, sv.ServeConfig(tol=args.tol, mode="fp64", side=side))
        for f in fams:
            srv64.solve_one(f, sv.Request(-1, f.key, lams[len(lams) // 2], 0.0))
        torch.cuda.synchronize()
        out = []
        t64 = time.perf_counter()
        for r in sub:
            out.append(srv64.solve_one(fam_of[r.key], r))
        wall = time.perf_counter() - t64
        return sv.summarize(out, wall), len(out) / wall
    # the drop-in: left-preconditioned, stops on the preconditioned residual
    fp64, fp64_serial = fp64_serial_run("left")
    # right-preconditioned: stops on the true residual, so it meets 1e-5 as
    # the mixed-precision solves do
    fp64r, fp64r_serial = fp64_serial_run("right")
    _progress("fp64 baselines")
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([dev_s, e2e_s], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dev_s, e2e_s = (float(v) for v in tt.tolist())
    value = len(reqs) * world / dev_s
    e2e_val = len(reqs) * world / e2e_s
    for f in fams:
        f.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sweep(args, reqs, band)
        _progress("cpu baseline")
    if rank == 0:
        nbar = int(np.mean([fam_of[r.key].idx.size for r in reqs]))
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
                "steps": steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * dev_s / steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "c64", "data": "synthetic",
                "config": {"workload": f"sweep: mixed-length Bragg gratings of {periods} periods "
                                       f"(grids {[list(f.p.shape) for f in fams]}, 20 nm voxels), "
                                       f"{len(lams)} wavelengths over 1500-1600 nm each = "
                                       f"{len(reqs)} solves per GPU, seeded Poisson arrivals at "
                                       f"{args.sweep_rate}/s (seed {args.seed + rank}), sizes "
                                       f"interleaved; one step = {per_step:.2f} solves of the "
                                       f"stream",
                           "tol": args.tol, "restart": args.restart,
                           "solver": f"complex64 GMRES + FP64 refinement, {args.sweep_batching} "
                                     f"batching",
                           "admission": "HBM pool", "members_per_lane": K,
                           "max_lanes_per_length": args.sweep_slots,
                           "pool": pool, "setup_s": round(setup_s, 1),
                           "warmup_requests": n_warm,
                           "legs": "common warm-up, then e2e (host buffers) first and the "
                                   "device-resident stream second, on the same lanes",
                           "operator": "Lagrange interpolation of fN over 5 Legendre wavelengths",
                           "precond": f"level1 at band centre, shared per length, "
                                      f"{args.sweep_side} (inner solves)",
                           "l2": "inputs larger than L2 (inverse blocks 1.7-7 GB per length, "
                                 "Krylov arenas 0.4-3 GB per lane)",
                           "parallelism": f"replicas x{world}"},
                "latency_ms": {"p50": summ_dev["p50_ms"], "p99": summ_dev["p99_ms"]},
                "serving": summ_dev,
                "fp64_plain_serial": {"solves_per_s": fp64_serial, "sampled": len(sub),
                                      "preconditioning": "left (pgmres L1, the drop-in)",
                                      "mean_iters": fp64["mean_iters"],
                                      "max_relres": fp64["max_relres"],
                                      "flags": fp64["flags"]},
                "fp64_true_residual_serial": {"solves_per_s": fp64r_serial, "sampled": len(sub),
                                              "preconditioning": "right (pgmres R1)",
                                              "mean_iters": fp64r["mean_iters"],
                                              "max_relres": fp64r["max_relres"],
                                              "flags": fp64r["flags"]},
                "speedup_vs_fp64_serial": value / world / fp64_serial,
                "speedup_vs_fp64_true_residual_serial": value / world / fp64r_serial,
                "e2e": {"value": e2e_val, "unit": "solves/s",
                        "h2d_bytes_per_step": int(nbar * 16 * per_step),
                        "d2h_bytes_per_step": int(nbar * 16 * per_step),
                        "latency_ms": {"p50": summ_h["p50_ms"], "p99": summ_h["p99_ms"]},
                        "max_relres": summ_h["max_relres"], "flags": summ_h["flags"],
                        "mean_iters": summ_h["mean_iters"]},
                "gpu_launches": int(launches),
                "roofline": roof,
                "cpu_baseline": cpu,
                "clocks": clk}
        print(json.dumps(line), flush=True)


def run_stages(args, world, rank, local):
    """Per-kernel device time of one GMRES iteration (vox_profile_stages) on a
    batched operator of one grating of the sweep: --stage-periods periods,
    --sweep-members members, --stage-prec precision, level-1 preconditioner,
    restart 50, Gram-Schmidt at a basis of 21 vectors.  The small, repeatable
    case the ncu captures in profiles/ are taken on."""
    import torch
    import voxphoton_b200 as vb
    from voxphoton_b200 import geometry as geo
    torch.cuda.set_device(local)
    p = geo.bragg(periods=args.stage_periods, M=30)
    G = vb.assemble_toeplitz(p.shape, p.ko, p.res, device=local)
    idx = p.idxS3()
    op1 = vb.Operator(p.Mop(), p.Gram, idx, G=G, device=local)
    pc1 = vb.Preconditioner.level1(op1, G, p.e_r)
    K = args.sweep_members
    op = vb.Operator(p.Mop(), p.Gram, idx, G=G, device=local, members=K)
    pc = pc1.share(op)
    stage = op.profile_stages(pc, prec=args.stage_prec, restart=args.restart, kgs=20,
                              reps=max(1, args.steps or 10))
    info, pinfo = op.info(), pc.info()
    L, M, N = p.shape
    n3 = 3 * M * N
    c = 8 if args.stage_prec == "c64" else 16
    nbytes = {k: v * K for k, v in kernel_bytes(info, p.shape, idx.size, pinfo, 20, c).items()}
    # the blocks are streamed once for every member of the launch
    nbytes["pc_solve"] = pinfo["n_blocks"] * n3 * n3 * c + 2 * K * L * n3 * c
    hbm, src = peaks()
    if rank == 0:
        print(json.dumps({"workload": f"stages: grating of {args.stage_periods} periods "
                                      f"({L}x{M}x{N}), {K} members, {args.stage_prec}",
                          "stage_ms": stage,
                          "bytes": nbytes,
                          "frac_of_hbm": {k: (nbytes[k] / (stage[k] * 1e-3) / 1e9 / hbm)
                                          for k in nbytes if stage.get(k, 0) > 0},
                          "peak_gbs": hbm, "peak_source": src, "op": info, "pc": pinfo}),
              flush=True)
    pc.close()
    op.close()
    pc1.close()
    op1.close()


def run_microdisk(args, world, rank, local):
    """Large resonator served broadband: Si microdisk (radius 5 um) side-coupled
    to a bus waveguide, 560 x 540 x 11 at 20 nm, 41 wavelengths over
    1540-1560 nm submitted together, the resonator's composite preconditioner
    (level 1 on the bus, level 2 on the disk: prec_fun_disk_idx), complex64 +
    FP64 refinement on lanes of batched operators vs the plain complex128
    drop-in.  One step = one solve.  The excitation is a y-polarised plane wave
    along the bus (the reference's script uses a dipole source)."""
    import torch
    import voxphoton_b200 as vb
    from voxphoton_b200 import geometry as geo
    from voxphoton_b200 import serving as sv
    torch.cuda.set_device(local)
    band = (1540e-9, 1560e-9)
    steps = args.steps if args.steps else 41
    lams = np.linspace(band[0], band[1], steps)
    p = geo.microdisk()
    t = time.time()
    fam = sv.Family("disk", p, band, nG=5, precond="disk", device=local,
                    members=args.sweep_members)
    setup_s = time.time() - t
    _progress(f"setup {setup_s:.1f} s")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    fam.add_slot(torch.cuda.Stream())
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    # the lane's Krylov arenas are allocated at its first solve: count them here
    # (complex64 basis of restart + 6 columns, complex128 refinement vectors)
    arena = args.sweep_members * fam.idx.size * ((args.disk_restart + 6) * 8 + 8 * 16)
    lane_bytes = max(free0 - free1, 1) + arena
    io_bytes = 2 * 16 * steps * fam.idx.size
    nslots = int(max(1, min(args.sweep_slots, 0.6 * (free1 - io_bytes) // lane_bytes)))
    while len(fam.slots) < nslots:
        fam.add_slot(torch.cuda.Stream())
    reqs = [sv.Request(i, "disk", float(l), 0.0) for i, l in enumerate(lams)]
    R = args.disk_restart
    maxit = max(2, 1600 // R)
    srv = sv.SweepServer([fam], sv.ServeConfig(tol=args.tol, side=args.sweep_side, restart=R,
                                               maxit_inner=maxit, inner_tol=args.inner_tol))
    srv.prepare_device()
    srv.warm()
    _progress("warm")
    dev_b = {r.rid: torch.from_numpy(fam.rhs(geo.C0 / r.lam * geo.N_EXT)).to("cuda")
             for r in reqs}
    dev_x = {r.rid: torch.empty_like(dev_b[r.rid]) for r in reqs}
    lane_ops = [op for op, _ in fam.slots]
    l0 = sum(op.launches() for op in lane_ops)
    clocks = None if args.no_clocks else Clocks(local)
    if clocks:
        clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    res, wall = srv.serve(reqs, realtime=False, device_io=(dev_b, dev_x))
    torch.cuda.synchronize()
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else {"sm_mhz": None, "sm_max_mhz": None,
                                        "reasons": ["not sampled (--no-clocks)"]}
    dev_s = e0.elapsed_time(e1) / 1e3
    lane_ops_end = [op for op, _ in fam.slots]
    launches = (sum(op.launches() for op in lane_ops_end if op in lane_ops) - l0 +
                sum(op.launches() for op in lane_ops_end if op not in lane_ops) +
                10 * len(reqs))
    summ = sv.summarize(res, wall)
    _progress(f"device-resident: {len(reqs)} solves in {dev_s:.2f} s")
    res_h, wall_h = srv.serve(reqs, realtime=False)
    torch.cuda.synchronize()
    summ_h = sv.summarize(res_h, wall_h)
    _progress(f"host-buffer: {wall_h:.2f} s")
    # matvec stages of one lane (all members) against their bytes
    op_m, pc_m = fam.slots[0]
    stage = op_m.profile_stages(pc_m, prec="c64", restart=R, kgs=R // 2, reps=3)
    info = op_m.info()
    L, M, N = p.shape
    K = args.sweep_members
    c = 8
    T = info["Px"] * 3 * N * M * c
    fN_b = 6 * (info["Px"] // 2 + 1) * (info["Py"] // 2 + 1) * (info["Pz"] // 2 + 1) * c
    n = fam.idx.size
    V = L * M * N
    mv_bytes = K * ((n * c + 12 * V + T) + (2 * T + fN_b) + (T + 2 * n * c + 12 * V + V * c))
    mv_ms = stage["mv_xfwd"] + stage["mv_plane"] + stage["mv_xinv"]
    hbm, src = peaks()
    ach = mv_bytes / (mv_ms * 1e-3) / 1e9
    srv.close()
    del dev_b, dev_x
    srv._bufs.clear()
    for op, pc in fam.slots:
        pc.close()
        op.close()
    fam.slots = []
    torch.cuda.empty_cache()
    op1 = vb.Operator(fam.mop, p.Gram, fam.idx, G=fam._Gc, device=local)
    fam.slots = [(op1, fam.pc.share(op1))]
    srv64 = sv.SweepServer([fam], sv.ServeConfig(tol=args.tol, mode="fp64", restart=R,
                                                 maxit_fp64=maxit))
    sub = reqs[::max(1, len(reqs) // max(1, args.disk_fp64))][:max(1, args.disk_fp64)]
    t64 = time.perf_counter()
    res64 = [srv64.solve_one(fam, r) for r in sub]
    wall64 = time.perf_counter() - t64
    fp64 = sv.summarize(res64, wall64)
    _progress("fp64 baseline")
    value = len(reqs) / dev_s
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
                "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * dev_s / steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "c64", "data": "synthetic",
                "config": {"workload": f"microdisk: Si disk r = 5 um + bus waveguide, "
                                       f"{L}x{M}x{N} at 20 nm, {steps} wavelengths over "
                                       f"1540-1560 nm submitted together",
                           "n_unknowns": int(n), "tol": args.tol, "restart": R,
                           "precond": "bus level 1 + disk level 2 (prec_fun_disk_idx), "
                                      "at band centre",
                           "lanes": nslots, "members_per_lane": K,
                           "lane_bytes": int(lane_bytes), "setup_s": round(setup_s, 1),
                           "parallelism": f"replicas x{world}"},
                "latency_ms": {"p50": summ["p50_ms"], "p99": summ["p99_ms"]},
                "serving": summ,
                "fp64_plain_serial": {"solves_per_s": len(res64) / wall64, "sampled": len(sub),
                                      "mean_iters": fp64["mean_iters"],
                                      "max_relres": fp64["max_relres"], "flags": fp64["flags"]},
                "speedup_vs_fp64_serial": value / (len(res64) / wall64),
                "e2e": {"value": len(reqs) / wall_h, "unit": "solves/s",
                        "h2d_bytes_per_step": int(n * 16), "d2h_bytes_per_step": int(n * 16)},
                "gpu_launches": int(launches),
                "roofline": {"bound": "hbm", "kernel": f"matvec (k_xfwd + kernel 2 + k_xinv), "
                                                       f"{K} members",
                             "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                             "traffic": None, "peak_source": src,
                             "bytes_per_launch": mv_bytes, "ms_per_launch": mv_ms,
                             "stage_ms": stage},
                "cpu_baseline": None,
                "clocks": clk}
        print(json.dumps(line), flush=True)
    fam.close()


def run_mor(args, world, rank, local):
    """Reduced-order wavelength sweep of one Bragg grating (Bragg_MOR_script.m:
    84-142 and example_Bragg_1500nm_to_1600nm.m:85-100): 5 Legendre nodes x
    order 5 solves at the script's 1e-4, then the reduced solve at every
    wavelength of the sweep (0.1 nm steps over 1500-1600 nm, as the script's
    free_wavelength).  One step = one wavelength.  Timed: the whole model
    build (solves, Arnoldi, basis, projections) plus the projection of every
    right-hand side, the reduced solves and the lift of every solution, with
    the right-hand sides resident in HBM."""
    import torch
    import voxphoton_b200 as vb
    from voxphoton_b200 import geometry as geo
    from voxphoton_b200 import mor
    from voxphoton_b200 import serving as sv
    torch.cuda.set_device(local)
    band = (1500e-9, 1600e-9)
    steps = args.steps if args.steps else 1001
    lams = np.linspace(band[0], band[1], steps)
    p = geo.bragg_config(args.mor_config)
    t = time.time()
    fam = sv.Family("mor", p, band, nG=5, precond="level1", device=local)
    setup_s = time.time() - t
    _progress(f"setup {setup_s:.1f} s")
    n = fam.idx.size
    dev = torch.device("cuda", local)
    VRHS = torch.empty((5, n), dtype=torch.complex128, device=dev)
    fam.rhs.fill_device([geo.C0 / l * geo.N_EXT for l in fam.nodes], VRHS)
    B = torch.empty((steps, n), dtype=torch.complex128, device=dev)
    fam.rhs.fill_device([geo.C0 / l * geo.N_EXT for l in lams], B)
    kw = dict(order=args.mor_order, tol=args.mor_tol, restart=args.restart, maxit_inner=40)

    def build():
        return mor.ReducedModel(fam.node_ops, fam.nodes, fam.mop, p.Gram, fam.idx, fam._Gc,
                                VRHS, pc=fam.pc, **kw)

    def online(rm):
        X = torch.empty_like(B)
        for c0 in range(0, steps, 128):
            c1 = min(steps, c0 + 128)
            Xc, _ = rm.solve(lams[c0:c1], B[c0:c1])
            X[c0:c1].copy_(Xc)
        return X

    rm = build()                                  # warm-up: graphs, arenas, allocator
    online(rm)
    rm.close()
    torch.cuda.synchronize()
    clocks = None if args.no_clocks else Clocks(local)
    if clocks:
        clocks.start()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    e0.record()
    rm = build()
    e1.record()
    X = online(rm)
    e2.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    clk = clocks.stop() if clocks else {"sm_mhz": None, "sm_max_mhz": None,
                                        "reasons": ["not sampled (--no-clocks)"]}
    build_s = e0.elapsed_time(e1) / 1e3
    online_s = e1.elapsed_time(e2) / 1e3
    _progress(f"model of rank {rm.rank} in {build_s:.2f} s, {steps} wavelengths in "
              f"{online_s * 1e3:.1f} ms")
    # accuracy: the reduced solutions against full solves at sampled wavelengths
    op1 = vb.Operator(fam.mop, p.Gram, fam.idx, G=fam._Gc, device=local)
    pc1 = fam.pc.share(op1)
    errs, rres = [], []
    for c in np.linspace(0, steps - 1, args.mor_check).astype(int):
        op1.interp(fam.node_ops, sv.lagrange_weights(lams[c], fam.nodes))
        b = B[c].cpu().numpy()
        xd, info = vb.solve_refined(op1, b, tol=1e-9, L1=pc1, maxit_inner=40)
        xm = X[c].cpu().numpy()
        errs.append(float(np.linalg.norm(xm - xd) / np.linalg.norm(xd)))
        rres.append(float(np.linalg.norm(op1.mv_AN(xm) - b) / np.linalg.norm(b)))
    pc1.close()
    op1.close()
    iters = [i.total_iters for info in rm.infos for i in info]
    # online HBM bytes: P read twice per 128-wavelength chunk, B read, X written
    r = rm.rank
    chunks = (steps + 127) // 128
    online_bytes = 2 * chunks * r * n * 16 + 2 * steps * n * 16
    hbm, src = peaks()
    ach = online_bytes / online_s / 1e9
    if rank == 0:
        line = {"metric": "reduced-order sweep: wavelengths/s including the model build",
                "value": steps / (build_s + online_s), "unit": "wavelengths/s",
                "n_gpus": world, "steps": steps, "warmup": 1,
                "ms_per_step": 1e3 * (build_s + online_s) / steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c64+c128",
                "data": "synthetic",
                "config": {"workload": f"MOR sweep of {p.name} {p.shape[0]}x{p.shape[1]}x"
                                       f"{p.shape[2]} ({args.mor_config}), {steps} wavelengths "
                                       f"over 1500-1600 nm",
                           "nG": 5, "order": args.mor_order, "rank": r, "tol": args.mor_tol,
                           "n_unknowns": int(n), "setup_s": round(setup_s, 1),
                           "precond": "level1 at band centre, shared by the nodes",
                           "l2": "inputs larger than L2 (right-hand sides "
                                 f"{steps * n * 16 / 1e9:.1f} GB)"},
                "build_s": build_s, "online_ms": online_s * 1e3,
                "node_solves": len(iters), "mean_iters": float(np.mean(iters)),
                "accuracy": {"sampled": len(errs), "max_rel_err_vs_full_solve": max(errs),
                             "max_true_relres": max(rres)},
                "e2e": {"value": steps / wall, "unit": "wavelengths/s",
                        "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                        "note": "host wall clock of the same timed region"},
                "roofline": {"bound": "hbm", "kernel": "online phase (k_block_dot_partial + "
                                                       "k_block_update)",
                             "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                             "traffic": None, "peak_source": src,
                             "bytes": online_bytes},
                "cpu_baseline": None, "clocks": clk}
        print(json.dumps(line), flush=True)
    rm.close()
    fam.close()


def main():
    args = parse()
    if args.steps is None and args.workload not in ("sweep", "microdisk", "mor", "stages"):
        args.steps = 10
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.workload == "microdisk":
        run_microdisk(args, world, rank, local)
        return
    if args.workload == "mor":
        run_mor(args, world, rank, local)
        return
    if args.workload == "stages":
        run_stages(args, world, rank, local)
        return
    if args.workload == "sweep":
        if world > 1:
            import torch
            import torch.distributed as dist
            from datetime import timedelta
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        run_sweep(args, world, rank, local)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    import torch
    import torch.distributed as dist
    import voxphoton_b200 as vb

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    p, G, idx, b, t_asm = build_problem(args.workload)
    n = idx.size
    op = vb.Operator(p.Mop(), p.Gram, idx, G=G, device=local)
    pc = vb.Preconditioner.level1(op, G, p.e_r) if args.precond == "level1" else None
    side = "left" if pc else None
    stream = torch.cuda.Stream()
    op.set_stream(stream.cuda_stream)
    dev = torch.device("cuda", local)
    b_dev = torch.from_numpy(b.astype(np.complex128)).to(dev)
    x_dev = torch.empty_like(b_dev)
    maxit_inner = 40

    def solve_mixed():
        return op.solve_refined_device(b_dev.data_ptr(), x_dev.data_ptr(), pc=pc, side=side,
                                       tol=args.tol, restart=args.restart,
                                       maxit_inner=maxit_inner, inner_tol=args.inner_tol,
                                       max_refine=10)

    torch.cuda.synchronize()
    for _ in range(args.warmup):
        info = solve_mixed()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = None if args.no_clocks else Clocks(local)
    if clocks:
        clocks.start()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    launches0 = op.launches()
    torch.cuda.synchronize()
    ev[0].record(stream)
    iters, relres = [], []
    for s in range(args.steps):
        info = solve_mixed()
        ev[s + 1].record(stream)
        iters.append(info.total_iters)
        relres.append(info.relres)
    torch.cuda.synchronize()
    launches = op.launches() - launches0
    ck = clocks.stop() if clocks else {"sm_mhz": None, "sm_max_mhz": None,
                                       "reasons": ["not sampled (--no-clocks)"]}
    lat = np.array([ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)])
    total_ms = float(ev[0].elapsed_time(ev[-1]))
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps / (total_ms / 1e3)

    # plain complex128 GMRES(50) solve, one at a time (the drop-in form)
    fp64 = None
    if args.fp64_steps > 0:
        x64 = torch.empty_like(b_dev)
        op.pgmres_device(b_dev.data_ptr(), x64.data_ptr(), pc=pc, side=side, prec="c128",
                         restart=args.restart, tol=args.tol, maxit=400)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.fp64_steps):
            inf64 = op.pgmres_device(b_dev.data_ptr(), x64.data_ptr(), pc=pc, side=side,
                                     prec="c128", restart=args.restart, tol=args.tol, maxit=400)
        e1.record(stream)
        torch.cuda.synchronize()
        ms64 = e0.elapsed_time(e1) / args.fp64_steps
        fp64 = {"solves_per_s": 1e3 / ms64, "ms_per_solve": ms64, "iters": inf64.total_iters,
                "relres": inf64.relres, "flag": inf64.flag}

    # end to end through the C-ABI with host buffers (H2D of b, D2H of x per step)
    e2e = None
    if args.steps > 0 and not args.no_e2e:
        import ctypes
        from voxphoton_b200 import _lib
        bre = np.ascontiguousarray(b.real)
        bim = np.ascontiguousarray(b.imag)
        xre = np.empty(n)
        xim = np.empty(n)
        inf = _lib.GmresInfo()
        lib = _lib.lib()

        def host_solve():
            _lib.check(lib.vox_solve_refined(
                op.handle, pc.handle if pc else None, 1 if pc else 0, _lib.dptr(bre),
                _lib.dptr(bim), args.tol, args.restart, maxit_inner, args.inner_tol, 10,
                _lib.dptr(xre),
                _lib.dptr(xim), ctypes.byref(inf)))
        host_solve()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            host_solve()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        e2e = {"value": world * args.steps / (ms / 1e3), "unit": "solves/s",
               "h2d_bytes_per_step": int(2 * n * 8), "d2h_bytes_per_step": int(2 * n * 8)}

    # roofline of the dominant kernel, from live CUDA-event timing of each stage
    roof = None
    if not args.no_stages:
        k_avg = max(1, min(args.restart - 1, int(np.mean(iters) // 2) if iters else 25))
        stages = op.profile_stages(pc, "c64", restart=args.restart, kgs=min(k_avg, 25), reps=20)
        nbytes = kernel_bytes(op.info(), p.shape, n, pc.info() if pc else None, min(k_avg, 25))
        dom = max((k for k in nbytes if stages.get(k, 0) > 0), key=lambda k: stages[k])
        peak, peak_kind = peaks()
        achieved = nbytes[dom] / (stages[dom] * 1e-3) / 1e9
        traffic = measured_traffic(dom, nbytes[dom])
        roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "peak_source": peak_kind, "bytes_per_launch": nbytes[dom],
                "ms_per_launch": stages[dom], "stage_ms": stages}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.precond == "none":
        # one whole unpreconditioned oracle solve on all host threads
        from oracle import vie as ov
        threads = os.cpu_count() or 1
        ov.set_fft_workers(threads)
        fN = ov.fN_from_toeplitz(G)
        ones = np.ones(p.shape)
        Mc = p.Mop()
        t = time.perf_counter()
        _, flag, rel, _, rv = ov.pgmres(
            lambda v: ov.mv_AN_const(v, fN, ones, Mc, p.Gram, "notransp", idx), b,
            args.restart, args.tol, 20)
        dt = time.perf_counter() - t
        cpu = {"value": 1.0 / dt, "unit": "solves/s", "cores": threads, "kind": "port",
               "sample": f"one whole solve of the numpy complex128 oracle pgmres(A, b, "
                         f"{args.restart}, {args.tol}, 20): {len(rv) - 1} iterations, relres "
                         f"{rel:.2e}, {dt:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
            "data": "synthetic",
            "config": {"workload": f"{args.workload} Bragg grating 1160x30x11 (20 nm voxels), "
                                   f"lambda 1550 nm, plane-wave RHS" if args.workload == "bragg20"
                       else args.workload,
                       "grid": list(p.shape), "n_unknowns": int(n), "tol": args.tol,
                       "restart": args.restart, "precond": args.precond,
                       "solver": "complex64 GMRES + FP64 refinement",
                       "l2": "working set (fN + Krylov basis) larger than L2",
                       "parallelism": f"replicas x{world}", "assembly_s": round(t_asm, 2)},
            "latency_ms": {"p50": float(np.percentile(lat, 50)),
                           "p99": float(np.percentile(lat, 99)), "mean": float(lat.mean())},
            "iters_per_solve": float(np.mean(iters)), "relres_max": float(np.max(relres)),
            "fp64_plain": fp64,
            "speedup_vs_fp64": (value / world / fp64["solves_per_s"]) if fp64 else None,
            "e2e": e2e, "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu,
            "clocks": ck,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
