"""The resonator's composite preconditioner (prec_fun_disk_idx.m: level 1 on
the bus, level 2 on the disk, identity elsewhere): the oracle's restatement on
a small microdisk, and the device implementation against it."""
import numpy as np
import pytest

import voxphoton_b200 as vb
from oracle import vie as ov
from voxphoton_b200 import geometry as geo


def small_disk():
    return geo.microdisk(radius=0.6e-6, gap=80e-9, bus_width=160e-9, height=80e-9,
                         len_abs=0.32e-6, res=40e-9, L=36, M=24)


def oracle_disk_prec(p, G):
    """resonator_MOR_scripts.m:94-198 with the oracle's restatements."""
    r = geo.microdisk_regions(p)
    L, M, N = p.shape
    V = L * M * N
    Mop = p.Mop()
    yb0, Mw = r["bus"]
    Mc_c = Mop[int(np.floor(L / 2 + 0.5)) - 1, yb0, 0]
    circ_WG = ov.level_1_parallel_func(G[:L, :Mw, :N], np.full((L, Mw, N), Mc_c),
                                       np.ones((L, Mw, N)), L, Mw, N, p.Gram)
    circ_WG = [-c for c in circ_WG]
    x0, Ls, y0, Ms = r["square"]
    e_si = geo.EPS_SI / geo.EPS_SIO2
    circ_D = ov.level_2_parallel_func(G[:Ls, :Ms, :N], np.full((Ls, Ms, N), (e_si - 1) / e_si),
                                      np.ones((Ls, Ms, N)), Ls, Ms, N, p.Gram)
    circ_D = [[-b for b in row] for row in circ_D]
    idxS3 = p.idxS3()
    idx_T = geo.ext3(r["idx_bus"], V)
    idx_R = geo.ext3(r["idx_disk"], V)
    idx_Sq = geo.ext3(r["idx_disk_in_sq"], Ls * Ms * N)
    return lambda J: ov.prec_fun_disk_idx(J, circ_WG, idx_T, idx_R, L, Mw, N, circ_D, Ls, Ms, N,
                                          L, M, N, idxS3, idx_Sq)


@pytest.fixture(scope="module")
def disk_case():
    p = small_disk()
    G = vb.assemble_toeplitz(p.shape, p.ko, p.res)
    return p, G


def test_regions_partition_the_support(disk_case):
    p, G = disk_case
    r = geo.microdisk_regions(p)
    s = set(p.idxS().tolist())
    bus, disk = set(r["idx_bus"].tolist()), set(r["idx_disk"].tolist())
    assert not (bus & disk)
    assert s == (bus | disk)
    x0, Ls, y0, Ms = r["square"]
    assert r["idx_disk_in_sq"].size == len(disk)


def test_oracle_composite_preconditioner_cuts_iterations(disk_case):
    p, G = disk_case
    idx = p.idxS3()
    fN = ov.fN_from_toeplitz(G)
    A = lambda v: ov.mv_AN_const(v, fN, np.ones(p.shape), p.Mop(), p.Gram, "notransp", idx)
    rng = np.random.default_rng(0)
    b = rng.standard_normal(idx.size) + 1j * rng.standard_normal(idx.size)
    prec = oracle_disk_prec(p, G)
    _, f0, r0, it0, _ = ov.pgmres(A, b, 30, 1e-6, 20)
    _, f1, r1, it1, _ = ov.pgmres(A, b, 30, 1e-6, 20, L1=prec)
    n0 = (it0[1] - 1) * 30 + it0[0]
    n1 = (it1[1] - 1) * 30 + it1[0]
    assert f1 == 0 and n1 < n0


@pytest.mark.gpu
def test_disk_preconditioner_apply_matches_oracle(disk_case):
    p, G = disk_case
    idx = p.idxS3()
    op = vb.Operator(p.Mop(), p.Gram, idx, G=G)
    pc = vb.Preconditioner.disk(op, G, p)
    prec = oracle_disk_prec(p, G)
    rng = np.random.default_rng(1)
    for _ in range(2):
        x = rng.standard_normal(idx.size) + 1j * rng.standard_normal(idx.size)
        ref = prec(x)
        y = pc.apply(x, prec="c128")
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-10
        y32 = pc.apply(x, prec="c64")
        assert np.linalg.norm(y32 - ref) / np.linalg.norm(ref) < 1e-4
    pc.close()
    op.close()


@pytest.mark.gpu
def test_disk_preconditioned_pgmres_matches_oracle(disk_case):
    p, G = disk_case
    idx = p.idxS3()
    op = vb.Operator(p.Mop(), p.Gram, idx, G=G)
    pc = vb.Preconditioner.disk(op, G, p)
    b = vb.jvie_rhs(p.e_r, geo.plane_wave(p), p.Gram, p.freq, idx)
    x, flag, relres, it, rv = vb.pgmres(op, b, restart=30, tol=1e-6, maxit=20, L1=pc)
    fN = ov.fN_from_toeplitz(G)
    A = lambda v: ov.mv_AN_const(v, fN, np.ones(p.shape), p.Mop(), p.Gram, "notransp", idx)
    xo, fo, ro, ito, rvo = ov.pgmres(A, b, 30, 1e-6, 20, L1=oracle_disk_prec(p, G))
    assert flag == fo and list(it) == list(ito)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8
    assert np.allclose(rv, rvo, rtol=1e-6, atol=1e-12)
    # the complex64 + FP64-refinement solve with it reaches the tolerance
    xr, info = vb.solve_refined(op, b, tol=1e-6, restart=30, maxit_inner=20, inner_tol=0.0,
                                L1=pc)
    assert info["flag"] == 0 and info["relres"] <= 1e-6
    pc.close()
    op.close()
