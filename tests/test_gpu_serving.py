"""GPU tests of the sweep serving pieces: operator interpolation in wavelength
(vox_op_interp), shared preconditioner handles (vox_precond_share), and that
every request's result is the same alone and in the concurrent mix (lanes of
two-member batches, so requests are solved together in lockstep)."""
import numpy as np
import pytest

import voxphoton_b200 as vb
from oracle import vie as ov
from voxphoton_b200 import geometry as geo
from voxphoton_b200 import serving as sv

pytestmark = pytest.mark.gpu


def small(periods):
    return geo.bragg(periods=periods, period=320e-9, len_abs=0.32e-6, res=40e-9, M=16)


def test_interp_is_the_lagrange_combination_of_the_nodes():
    p = small(2)
    idx = p.idxS3()
    lams = [1500e-9, 1550e-9, 1600e-9]
    Gs = [vb.assemble_toeplitz(p.shape, p.with_wavelength(l).ko, p.res) for l in lams]
    ops = [vb.Operator(p.Mop(), p.Gram, idx, G=G) for G in Gs]
    dst = vb.Operator(p.Mop(), p.Gram, idx, G=Gs[0])
    rng = np.random.default_rng(0)
    x = rng.standard_normal(idx.size) + 1j * rng.standard_normal(idx.size)
    w = sv.lagrange_weights(1537e-9, lams)
    dst.interp(ops, w)
    y = dst.mv_AN(x)
    ref = sum(wi * op.mv_AN(x) for wi, op in zip(w, ops))  # affine in fN, sum(w) = 1
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-12
    # the interpolated operator equals the oracle with interpolated fN
    fN = sum(wi * ov.fN_from_toeplitz(G) for wi, G in zip(w, Gs))
    yo = ov.mv_AN_const(x, fN, np.ones(p.shape), p.Mop(), p.Gram, "notransp", idx)
    assert np.linalg.norm(y - yo) / np.linalg.norm(yo) < 1e-12
    for op in ops + [dst]:
        op.close()


def test_shared_preconditioner_matches_its_source():
    p = small(2)
    idx = p.idxS3()
    G = vb.assemble_toeplitz(p.shape, p.ko, p.res)
    op1 = vb.Operator(p.Mop(), p.Gram, idx, G=G)
    op2 = vb.Operator(p.Mop(), p.Gram, idx, G=G)
    pc1 = vb.Preconditioner.level1(op1, G, p.e_r)
    pc2 = pc1.share(op2)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(idx.size) + 1j * rng.standard_normal(idx.size)
    a = pc1.apply(x)
    pc1.close()  # the shared factors stay alive with pc2
    b = pc2.apply(x)
    assert np.array_equal(a, b)
    pc2.close()
    op1.close()
    op2.close()


def test_results_are_the_same_alone_and_in_the_mix():
    band = (1500e-9, 1600e-9)
    fams = [sv.Family(k, small(k), band, nG=3, members=2) for k in (2, 4)]
    for f in fams:
        f.add_slot()
        f.add_slot()
    lams = np.linspace(band[0], band[1], 4)
    reqs = sv.poisson_stream([(k, l) for k in (2, 4) for l in lams], rate=1000.0, seed=0)
    cfg = sv.ServeConfig(tol=1e-5, keep_x=True)
    mix, _ = sv.SweepServer(fams, cfg).serve(reqs, realtime=True)
    for f in fams:
        for op, pc in f.slots[1:]:
            pc.close()
            op.close()
        del f.slots[1:]
    alone = {}
    for r in reqs:
        res, _ = sv.SweepServer(fams, cfg).serve([r], realtime=False)
        alone[r.rid] = res[0]
    assert len(mix) == len(reqs)
    for m in mix:
        a = alone[m.rid]
        assert m.flag == 0 and a.flag == 0 and m.relres <= 1e-5
        assert m.iters == a.iters
        assert np.array_equal(m.x, a.x)
    for f in fams:
        f.close()
