"""Host-side logic of the sweep serving loop (no GPU): Legendre nodes and
Lagrange weights (the reference's lagrange_int.m), the per-wavelength
right-hand side, request streams and replica sharding across ranks
(world_size 2 with the gloo backend)."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import voxphoton_b200 as vb
from voxphoton_b200 import geometry as geo
from voxphoton_b200 import serving as sv


def test_legendre_nodes_and_lagrange_weights():
    s = sv.legendre_nodes(1500e-9, 1600e-9, 5)
    assert np.all(np.diff(s) > 0) and 1500e-9 < s[0] and s[-1] < 1600e-9
    for S in (1500e-9, 1537e-9, 1600e-9):
        w = sv.lagrange_weights(S, s)
        assert abs(w.sum() - 1) < 1e-12
        # exact for polynomials of degree < 5 in the wavelength
        f = lambda lam: 3 + 2e6 * lam - 1e12 * lam ** 2 + 5e17 * lam ** 4
        assert abs(w @ f(s) - f(S)) < 1e-9 * abs(f(S))
    assert np.allclose(sv.lagrange_weights(s[2], s), np.eye(5)[2])


def test_rhs_builder_matches_plane_wave_and_jvie_rhs():
    p = geo.bragg(periods=2, period=320e-9, len_abs=0.32e-6, res=40e-9, M=16)
    idx = p.idxS3()
    rb = sv._RhsBuilder(p, idx)
    for lam in (1500e-9, 1550e-9, 1600e-9):
        q = p.with_wavelength(lam)
        ref = vb.jvie_rhs(q.e_r, geo.plane_wave(q), q.Gram, q.freq, idx)
        out = rb(q.freq)
        assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 1e-13


def test_poisson_stream_is_seeded_and_complete():
    items = [(k, lam) for k in (1, 2) for lam in (1.0, 2.0, 3.0)]
    a = sv.poisson_stream(items, rate=10.0, seed=3)
    b = sv.poisson_stream(items, rate=10.0, seed=3)
    assert [(r.key, r.lam, r.arrival) for r in a] == [(r.key, r.lam, r.arrival) for r in b]
    assert sorted((r.key, r.lam) for r in a) == sorted(items)
    assert all(np.diff([r.arrival for r in a]) > 0)


def _rank_main(rank, world, port, items, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    mine = sv.shard_requests(items, world, rank)
    # each rank "serves" its share and reports a time; the job time is the max
    t = torch.tensor([float(len(mine))])
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        out.put((float(t.item()), gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_sharding_two_ranks_gloo():
    items = [(k, lam) for k in (20, 40, 60) for lam in range(7)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, items, q)) for r in range(2)]
    for p in procs:
        p.start()
    tmax, shares = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    flat = [x for s in shares for x in s]
    assert sorted(flat) == sorted(items) and len(flat) == len(set(flat))
    assert tmax == max(len(s) for s in shares)
    with pytest.raises(ValueError):
        sv.shard_requests(items, 2, 2)
