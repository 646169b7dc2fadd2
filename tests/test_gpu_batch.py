"""GPU tests of batched operators: K same-shape solves (one device at K
wavelengths) advanced in lockstep by vox_solve_refined_batch, with one launch
per kernel for all members and the preconditioner's factors streamed once for
all of them.  Each member's result must be identical, bit for bit, to the
single-right-hand-side solve of the same system, and meet the tolerance."""
import numpy as np
import pytest

import voxphoton_b200 as vb
from oracle import vie as ov
from voxphoton_b200 import geometry as geo
from voxphoton_b200 import serving as sv

pytestmark = pytest.mark.gpu

NODES = np.array([1500e-9, 1550e-9, 1600e-9])


@pytest.fixture(scope="module")
def family():
    p = geo.bragg(periods=2, period=320e-9, len_abs=0.32e-6, res=40e-9, M=16)
    idx = p.idxS3()
    Gs = [vb.assemble_toeplitz(p.shape, p.with_wavelength(l).ko, p.res) for l in NODES]
    nodes = [vb.Operator(p.Mop(), p.Gram, idx, G=G) for G in Gs]
    pc = vb.Preconditioner.level1(nodes[1], Gs[1], p.e_r)
    rhs = sv._RhsBuilder(p, idx)
    yield p, idx, Gs, nodes, pc, rhs
    pc.close()
    for op in nodes:
        op.close()


def _solo(p, idx, Gs, nodes, pc, lam, b, side="left"):
    op = vb.Operator(p.Mop(), p.Gram, idx, G=Gs[1])
    pcs = pc.share(op)
    op.interp(nodes, sv.lagrange_weights(lam, NODES))
    kw = {"L1": pcs} if side == "left" else {"R1": pcs}
    x, info = vb.solve_refined(op, b, tol=1e-5, restart=50, maxit_inner=40, inner_tol=0.0, **kw)
    pcs.close()
    op.close()
    return x, info


@pytest.mark.parametrize("members,count", [(3, 3), (4, 2), (5, 5)])
def test_batch_members_equal_solo_solves(family, members, count):
    p, idx, Gs, nodes, pc, rhs = family
    lams = np.linspace(1505e-9, 1595e-9, count)
    bs = [rhs(geo.C0 / l * geo.N_EXT) for l in lams]
    op = vb.Operator(p.Mop(), p.Gram, idx, G=Gs[1], members=members)
    pcb = pc.share(op)
    for m, l in enumerate(lams):
        op.interp(nodes, sv.lagrange_weights(l, NODES), member=m)
    out = vb.solve_refined_batch(op, bs, tol=1e-5, restart=50, maxit_inner=40, inner_tol=0.0,
                                 L1=pcb)
    assert len(out) == count
    for (x, info), l, b in zip(out, lams, bs):
        xs, is_ = _solo(p, idx, Gs, nodes, pc, l, b)
        assert info["flag"] == 0 and info["relres"] <= 1e-5
        assert info["iters"] == is_["iters"] and info["refinements"] == is_["refinements"]
        assert np.array_equal(x, xs)
        assert np.array_equal(info["resvec"], is_["resvec"])
    pcb.close()
    op.close()


def test_batch_solution_meets_tolerance_against_the_oracle(family):
    p, idx, Gs, nodes, pc, rhs = family
    lams = [1512e-9, 1583e-9]
    op = vb.Operator(p.Mop(), p.Gram, idx, G=Gs[1], members=2)
    pcb = pc.share(op)
    for m, l in enumerate(lams):
        op.interp(nodes, sv.lagrange_weights(l, NODES), member=m)
    bs = [rhs(geo.C0 / l * geo.N_EXT) for l in lams]
    out = vb.solve_refined_batch(op, bs, tol=1e-5, restart=50, maxit_inner=40, inner_tol=0.0,
                                 L1=pcb)
    for (x, info), l, b in zip(out, lams, bs):
        fN = sum(w * ov.fN_from_toeplitz(G) for w, G in zip(sv.lagrange_weights(l, NODES), Gs))
        Ax = ov.mv_AN_const(x, fN, np.ones(p.shape), p.Mop(), p.Gram, "notransp", idx)
        assert np.linalg.norm(b - Ax) / np.linalg.norm(b) <= 1e-5
    pcb.close()
    op.close()


def test_zero_right_hand_side_in_a_batch(family):
    p, idx, Gs, nodes, pc, rhs = family
    op = vb.Operator(p.Mop(), p.Gram, idx, G=Gs[1], members=2)
    pcb = pc.share(op)
    b = rhs(geo.C0 / 1550e-9 * geo.N_EXT)
    out = vb.solve_refined_batch(op, [np.zeros_like(b), b], tol=1e-5, restart=50,
                                 maxit_inner=40, inner_tol=0.0, L1=pcb)
    (x0, i0), (x1, i1) = out
    assert i0["flag"] == 0 and i0["relres"] == 0.0 and not np.any(x0)
    assert i1["flag"] == 0 and i1["relres"] <= 1e-5
    pcb.close()
    op.close()


def test_batch_count_is_checked(family):
    p, idx, Gs, nodes, pc, rhs = family
    op = vb.Operator(p.Mop(), p.Gram, idx, G=Gs[1], members=2)
    b = rhs(geo.C0 / 1550e-9 * geo.N_EXT)
    with pytest.raises(vb._lib.VoxError):
        vb.solve_refined_batch(op, [b, b, b])
    op.close()
    with pytest.raises(vb._lib.VoxError):
        vb.Operator(p.Mop(), p.Gram, idx, G=Gs[1], members=9)


def test_stage_profile_of_a_batch(family):
    p, idx, Gs, nodes, pc, rhs = family
    op = vb.Operator(p.Mop(), p.Gram, idx, G=Gs[1], members=4)
    pcb = pc.share(op)
    st = op.profile_stages(pcb, prec="c64", restart=20, kgs=5, reps=3)
    # on the two-read Gram-Schmidt path (restart <= 50) the column finish
    # includes the scaling, so gs_scale is not a separate launch
    assert all(v > 0 for k, v in st.items() if k != "gs_scale")
    pcb.close()
    op.close()


@pytest.mark.parametrize("side,steps", [("left", "4"), ("right", "4"), ("right", "1"),
                                        ("right", "7"), ("left", "0"), ("right", "0")])
def test_lane_refills_members_and_matches_solo_solves(family, monkeypatch, side, steps):
    # 5 requests on 3 members: slots are refilled while other members are
    # mid-solve; every result must equal the single-right-hand-side solve.
    # VOX_LANE_STEPS: out-of-phase steps per lane step (0: in-phase cycles)
    monkeypatch.setenv("VOX_LANE_STEPS", steps)
    p, idx, Gs, nodes, pc, rhs = family
    lams = np.linspace(1502e-9, 1598e-9, 5)
    op = vb.Operator(p.Mop(), p.Gram, idx, G=Gs[1], members=3)
    pcb = pc.share(op)
    lane = vb.Lane(op, pcb, side=side, tol=1e-5, restart=50, maxit_inner=40)
    queue = list(range(len(lams)))
    inflight, out = {}, {}
    while queue or inflight:
        for m in range(3):
            if m not in inflight and queue:
                i = queue.pop(0)
                op.interp(nodes, sv.lagrange_weights(lams[i], NODES), member=m)
                lane.submit(m, rhs(geo.C0 / lams[i] * geo.N_EXT))
                inflight[m] = i
        for m in lane.step():
            out[inflight.pop(m)] = lane.collect(m)
    assert sorted(out) == list(range(len(lams)))
    for i, l in enumerate(lams):
        x, info = out[i]
        xs, is_ = _solo(p, idx, Gs, nodes, pc, l, rhs(geo.C0 / l * geo.N_EXT), side=side)
        assert info["flag"] == 0 and info["relres"] <= 1e-5
        assert info["iters"] == is_["iters"] and info["refinements"] == is_["refinements"]
        assert np.array_equal(x, xs)
        assert np.array_equal(info["resvec"], is_["resvec"])
    lane.close()
    pcb.close()
    op.close()


@pytest.fixture(scope="module")
def wide():
    # the sweep's cross-section (30 x 11 cells at 20 nm): level-1 blocks of 990
    # rows (leading dimension 992), where the streamed apply's right-hand sides
    # and ring fill the shared-memory budget at every member count
    p = geo.bragg(periods=2, M=30)
    assert 3 * p.shape[1] * p.shape[2] == 990
    idx = p.idxS3()
    Gs = [vb.assemble_toeplitz(p.shape, p.with_wavelength(l).ko, p.res) for l in NODES]
    nodes = [vb.Operator(p.Mop(), p.Gram, idx, G=G) for G in Gs]
    pc = vb.Preconditioner.level1(nodes[1], Gs[1], p.e_r)
    assert pc.info()["ld"] == 992
    rhs = sv._RhsBuilder(p, idx)
    yield p, idx, Gs, nodes, pc, rhs
    pc.close()
    for op in nodes:
        op.close()


@pytest.mark.parametrize("members", [2, 4, 5])
def test_batch_equals_solo_at_the_sweep_cross_section(wide, members):
    # 2 and 4 members: one apply launch of 4 and 8 columns; 5: a group of 4
    # and a group of 1
    p, idx, Gs, nodes, pc, rhs = wide
    lams = np.linspace(1510e-9, 1590e-9, members)
    bs = [rhs(geo.C0 / l * geo.N_EXT) for l in lams]
    op = vb.Operator(p.Mop(), p.Gram, idx, G=Gs[1], members=members)
    pcb = pc.share(op)
    for m, l in enumerate(lams):
        op.interp(nodes, sv.lagrange_weights(l, NODES), member=m)
    out = vb.solve_refined_batch(op, bs, tol=1e-5, restart=50, maxit_inner=40, inner_tol=0.0,
                                 R1=pcb)
    for (x, info), l, b in zip(out, lams, bs):
        so = vb.Operator(p.Mop(), p.Gram, idx, G=Gs[1])
        pcs = pc.share(so)
        so.interp(nodes, sv.lagrange_weights(l, NODES))
        xs, is_ = vb.solve_refined(so, b, tol=1e-5, restart=50, maxit_inner=40, inner_tol=0.0,
                                   R1=pcs)
        pcs.close()
        so.close()
        assert info["flag"] == 0 and info["relres"] <= 1e-5
        assert info["iters"] == is_["iters"]
        assert np.array_equal(x, xs)
    pcb.close()
    op.close()
