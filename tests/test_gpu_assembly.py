"""Green-tensor assembly with the regular face-pair cubature on the GPU
(vox_assemble_toeplitz_device) against the host assembly and the golden case
assembled by the reference's compiled cubature cores."""
import os
import time

import numpy as np
import pytest

import voxphoton_b200 as vb

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.gpu
def test_device_assembly_matches_golden_reference_cores():
    d = np.load(os.path.join(GOLD, "tiny_case.npz"))
    G = vb.assemble_toeplitz(d["G"].shape[:3], float(d["ko"]), float(d["dx"]), device=0)
    assert np.max(np.abs(G - d["G"])) < 1e-12 * np.max(np.abs(d["G"]))


@pytest.mark.gpu
@pytest.mark.parametrize("shape,dx", [((2, 2, 2), 20e-9), ((9, 7, 6), 20e-9),
                                      ((61, 23, 11), 20e-9), ((40, 30, 12), 10e-9)])
def test_device_assembly_matches_host(shape, dx):
    ko = 2 * np.pi / 1550e-9 * 1.444
    t0 = time.perf_counter()
    Gh = vb.assemble_toeplitz(shape, ko, dx)
    t1 = time.perf_counter()
    Gd = vb.assemble_toeplitz(shape, ko, dx, device=0)
    t2 = time.perf_counter()
    scale = np.max(np.abs(Gh), axis=(0, 1, 2))
    err = np.max(np.abs(Gd - Gh), axis=(0, 1, 2)) / scale
    print(f"{shape}: host {t1 - t0:.3f} s, device {t2 - t1:.3f} s, max rel err {err.max():.2e}")
    assert err.max() < 1e-13


@pytest.mark.gpu
def test_device_assembly_of_the_grating_feeds_the_same_operator():
    """The 1160 x 30 x 11 grating: the device-assembled tensor gives the
    host-assembled operator's products to rounding."""
    from voxphoton_b200 import geometry as geo
    p = geo.bragg_config("bragg20")
    Gd = vb.assemble_toeplitz(p.shape, p.ko, p.res, device=0)
    Gh = vb.assemble_toeplitz(p.shape, p.ko, p.res)
    assert np.max(np.abs(Gd - Gh)) < 1e-13 * np.max(np.abs(Gh))
    idx = p.idxS3()
    op_h = vb.Operator(p.Mop(), p.Gram, idx, G=Gh, precisions=("c128",))
    op_d = vb.Operator(p.Mop(), p.Gram, idx, G=Gd, precisions=("c128",))
    rng = np.random.default_rng(0)
    x = rng.standard_normal(idx.size) + 1j * rng.standard_normal(idx.size)
    yh, yd = op_h.mv_AN(x), op_d.mv_AN(x)
    assert np.linalg.norm(yd - yh) / np.linalg.norm(yh) < 1e-13
    op_h.close()
    op_d.close()
