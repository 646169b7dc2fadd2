"""Benchmark: GMRES solves/s of the JVIE-II frequency solve on B200.

Workload (default): Bragg grating, 60 periods + 2 um quadratic absorbers,
20 nm voxels -> 1160 x 30 x 11 grid, lambda = 1550 nm, y-polarised plane wave
along the grating.  One step = one complete solve to 1e-5 relative residual
||b - A x|| / ||b|| (FP64), by complex64 GMRES(50) inside FP64 iterative
refinement.  Synthetic, seeded geometry; operator assembled on the host by
libvox; everything in the timed region runs in libvox's sm_100a kernels.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vox|reference]
                    [--precond none|level1] [--workload bragg20|strip|bragg10]

N > 1 (torchrun): independent replicas, one per GPU (the solve does not
shard); value = total solves / max-over-ranks device time.
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
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vox", choices=["vox", "reference"])
    ap.add_argument("--workload", default="bragg20")
    ap.add_argument("--precond", default="level1", choices=["none", "level1"])
    ap.add_argument("--tol", type=float, default=1e-5)
    ap.add_argument("--restart", type=int, default=50)
    ap.add_argument("--inner-tol", type=float, default=0.0,
                    help="complex64 inner GMRES tolerance (0: aim at the target directly)")
    ap.add_argument("--fp64-steps", type=int, default=3)
    ap.add_argument("--cpu-sample-iters", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg")
    ap.add_argument("--no-stages", action="store_true", help="skip per-kernel timing")
    ap.add_argument("--sweep-periods", default="20,40,60,80,100")
    ap.add_argument("--sweep-lambdas", type=int, default=201)
    ap.add_argument("--sweep-rate", type=float, default=200.0,
                    help="Poisson arrival rate (requests/s) of the sweep stream")
    ap.add_argument("--sweep-slots", type=int, default=4)
    ap.add_argument("--sweep-fp64", type=int, default=10,
                    help="requests solved one at a time in plain complex128 for the baseline")
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


def kernel_bytes(op_info, shape, n, pc_info, k):
    """Algorithmic bytes per launch of each stage, complex64 (8 B per value)."""
    L, M, N = shape
    V = L * M * N
    Px, Py, Pz = op_info["Px"], op_info["Py"], op_info["Pz"]
    c = 8
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
        # factors of the factored modes (each read once for both paired modes),
        # the inverted 32x32 diagonal blocks, the transformed vectors in and out
        nf, ld = pc_info["n_factored"], pc_info["ld"]
        nblk = ld // 32
        b["pc_xfwd"] = n * c + 3 * V * 4 + L * n3 * c
        # the tile stream: nb*(nb+1) 32x32 tiles per factored mode (L and U
        # off-diagonal tiles plus the two inverted diagonal blocks per block row)
        b["pc_solve"] = nf * nblk * (nblk + 1) * 32 * 32 * c + 2 * L * n3 * c + nf * n3 * 4
        b["pc_xinv"] = L * n3 * c + 3 * V * 4 + n * c
    return b


def cpu_baseline(p, G, idx, b, iters_per_solve, sample_iters, restart):
    """The oracle (numpy complex128 restatement of mv_AN_const + pgmres_iter)
    timed on a bounded sample: `sample_iters` Arnoldi steps, scaled to one
    solve of `iters_per_solve` steps."""
    from oracle import vie as ov
    try:
        from threadpoolctl import threadpool_limits
        ctx = threadpool_limits(limits=1)
    except Exception:
        ctx = None
    fN = ov.fN_from_toeplitz(G)
    ones = np.ones(p.shape)
    Mc = p.Mop()
    A = lambda v: ov.mv_AN_const(v, fN, ones, Mc, p.Gram, "notransp", idx)
    t = time.perf_counter()
    ov.pgmres_iter(A, np.zeros_like(b), b, sample_iters, None, None, None, None, 0.0)
    dt = time.perf_counter() - t
    if ctx is not None:
        ctx.unregister() if hasattr(ctx, "unregister") else None
    per_iter = dt / sample_iters
    solve_s = per_iter * max(1, iters_per_solve)
    return {"value": 1.0 / solve_s, "unit": "solves/s", "cores": 1, "kind": "port",
            "sample": f"{sample_iters} Arnoldi steps of the numpy complex128 oracle "
                      f"(mv_AN_const + classical Gram-Schmidt, 1 thread) = {dt:.2f} s, "
                      f"scaled to {iters_per_solve} steps per solve"}


def run_reference(args, world, rank):
    """--impl reference: the oracle port of the reference CPU path, all host threads."""
    if rank != 0:
        return
    p, G, idx, b, _ = build_problem(args.workload)
    from oracle import vie as ov
    fN = ov.fN_from_toeplitz(G)
    ones = np.ones(p.shape)
    Mc = p.Mop()
    ncores = os.cpu_count() or 1
    try:
        import scipy.fft as sfft

        def A(v):
            return ov.mv_AN_const(v, fN, ones, Mc, p.Gram, "notransp", idx)
        ov.set_fft_workers(ncores)
    except Exception:
        A = lambda v: ov.mv_AN_const(v, fN, ones, Mc, p.Gram, "notransp", idx)
    sample = max(1, args.cpu_sample_iters)
    iters = int(os.environ.get("VOX_REF_ITERS_PER_SOLVE", "0")) or None
    times = []
    for s in range(args.warmup + args.steps):
        t = time.perf_counter()
        ov.pgmres_iter(A, np.zeros_like(b), b, sample, None, None, None, None, 0.0)
        dt = time.perf_counter() - t
        if s >= args.warmup:
            times.append(dt)
    per_iter = float(np.mean(times)) / sample
    # iterations per solve: a plain complex128 GMRES(50) solve at tol needs this
    # many Arnoldi steps on this workload (measured by the GPU arm; default
    # from the same oracle on a single restart cycle if not given)
    ips = iters or 300
    val = 1.0 / (per_iter * ips)
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "solves/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * per_iter * ips, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": args.workload, "grid": list(p.shape), "n": int(idx.size),
                       "tol": args.tol, "restart": args.restart, "precond": args.precond},
            "cpu_baseline": {"value": val, "unit": "solves/s", "cores": ncores, "kind": "port",
                             "sample": f"{sample} Arnoldi steps per step of the numpy "
                                       f"complex128 oracle (scipy.fft workers={ncores}), "
                                       f"scaled to {ips} steps per solve"},
            "e2e": {"value": val, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_sweep(args, world, rank, local):
    """Mixed-length Bragg sweep served as a Poisson request stream (one GPU per
    rank; ranks take disjoint shares of the stream)."""
    import torch
    from voxphoton_b200 import geometry as geo
    from voxphoton_b200 import serving as sv
    torch.cuda.set_device(local)
    periods = [int(x) for x in args.sweep_periods.split(",")]
    band = (1500e-9, 1600e-9)
    lams = np.linspace(band[0], band[1], args.sweep_lambdas)
    t = time.time()
    fams = [sv.Family(pr, geo.bragg(periods=pr, M=30), band, nG=5, device=local)
            for pr in periods]
    setup_s = time.time() - t
    # admission by HBM footprint: slots per family from one slot's bytes
    free0, total = torch.cuda.mem_get_info()
    fams[-1].add_slot()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    slot_bytes = max(free0 - free1, 1)
    budget = 0.6 * free1
    nslots = int(max(1, min(args.sweep_slots, budget // (slot_bytes * len(fams)))))
    for f in fams:
        while len(f.slots) < nslots:
            f.add_slot()
    mine = sv.shard_requests([(pr, lam) for pr in periods for lam in lams], world, rank)
    reqs = sv.poisson_stream(mine, rate=args.sweep_rate, seed=args.seed + rank)
    # warm-up: one solve on every slot (cycle-graph capture, caches)
    warm = [sv.Request(-1 - i, f.key, lams[len(lams) // 2], 0.0) for i, f in enumerate(fams)]
    srv_w = sv.SweepServer(fams, sv.ServeConfig(tol=args.tol))
    for f, r in zip(fams, warm):
        for s in range(len(f.slots)):
            srv_w.solve_one(f, r, slot=s)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    res, wall = sv.SweepServer(fams, sv.ServeConfig(tol=args.tol)).serve(reqs, realtime=True)
    torch.cuda.synchronize()
    e1.record()
    torch.cuda.synchronize()
    dev_s = e0.elapsed_time(e1) / 1e3
    summ = sv.summarize(res, wall)
    # plain complex128 GMRES, one solve at a time, on a seeded subset
    rng = np.random.default_rng(args.seed)
    sub = [reqs[i] for i in rng.choice(len(reqs), size=min(len(reqs), args.sweep_fp64), replace=False)]
    for f in fams:
        for op, pc in f.slots[1:]:
            pc.close()
            op.close()
        del f.slots[1:]
    # strictly one solve at a time on this thread (the drop-in form); each
    # family's complex128 cycle graph is captured by an untimed first solve
    srv64 = sv.SweepServer(fams, sv.ServeConfig(tol=args.tol, mode="fp64"))
    fam_of = {f.key: f for f in fams}
    for f in fams:
        srv64.solve_one(f, sv.Request(-1, f.key, lams[len(lams) // 2], 0.0))
    torch.cuda.synchronize()
    res64 = []
    t64 = time.perf_counter()
    for r in sub:
        res64.append(srv64.solve_one(fam_of[r.key], r))
    wall64 = time.perf_counter() - t64
    fp64 = sv.summarize(res64, wall64)
    fp64_serial = len(res64) / wall64
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([dev_s], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dev_s = float(tt.item())
    value = len(res) * world / dev_s
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
                "steps": len(res), "warmup": len(warm), "ms_per_step": 1e3 * dev_s / len(res),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "c64", "data": "synthetic",
                "config": {"workload": f"mixed-length Bragg sweep: periods {periods} (grids "
                                       f"{[f.p.shape for f in fams]}), {len(lams)} wavelengths "
                                       f"in 1500-1600 nm each, Poisson arrivals "
                                       f"{args.sweep_rate}/s (seed {args.seed})",
                           "tol": args.tol, "slots_per_length": nslots,
                           "slot_bytes": int(slot_bytes), "setup_s": round(setup_s, 1),
                           "operator": "Lagrange interpolation over 5 Legendre wavelengths",
                           "precond": "level1 at band centre, shared per length"},
                "latency_ms": {"p50": summ["p50_ms"], "p99": summ["p99_ms"]},
                "serving": summ,
                "fp64_plain_serial": {"solves_per_s": fp64_serial, "sampled": len(res64),
                                      "mean_iters": fp64["mean_iters"],
                                      "max_relres": fp64["max_relres"]},
                "speedup_vs_fp64_serial": value / world / fp64_serial,
                "e2e": {"value": value, "unit": "solves/s",
                        "h2d_bytes_per_step": int(np.mean([f.idx.size for f in fams]) * 16),
                        "d2h_bytes_per_step": int(np.mean([f.idx.size for f in fams]) * 16)}}
        print(json.dumps(line), flush=True)
    for f in fams:
        f.close()


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, world, rank)
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
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        iters_solve = fp64["iters"] if fp64 else int(np.mean(iters))
        cpu = cpu_baseline(p, G, idx, b, iters_solve, args.cpu_sample_iters, args.restart)

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
