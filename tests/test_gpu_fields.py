"""GPU test of the total-field evaluation E_field_Nop_const (the N operator on
the whole grid through vox_mv_L) and the transmitted power of the reference's
Bragg example, against the oracle."""
import numpy as np
import pytest

import voxphoton_b200 as vb
from oracle import vie as ov
from voxphoton_b200 import geometry as geo

pytestmark = pytest.mark.gpu


def test_total_field_and_transmitted_power_match_oracle():
    p = geo.bragg(periods=2, period=320e-9, len_abs=0.32e-6, res=40e-9, M=16)
    L, M, N = p.shape
    V = L * M * N
    G = vb.assemble_toeplitz(p.shape, p.ko, p.res)
    op_full = vb.Operator(p.Mop(), p.Gram, np.arange(1, 3 * V + 1), G=G)
    rng = np.random.default_rng(3)
    J = np.zeros((L, M, N, 3), dtype=complex)
    mask = np.abs(p.Mop()) > 0
    for c in range(3):
        J[..., c][mask] = rng.standard_normal(mask.sum()) + 1j * rng.standard_normal(mask.sum())
    Einc = geo.plane_wave(p)
    E = vb.E_field_Nop_const(J, op_full, p.Gram, p.freq, Einc)
    Eo = ov.E_field_Nop_const(J, ov.fN_from_toeplitz(G), p.Gram, p.freq, Einc)
    assert np.linalg.norm(E - Eo) / np.linalg.norm(Eo) < 1e-12
    P = vb.transmitted_power(E, p.res, p.meta["len_abs"], 2 * p.meta["corrugation"])
    Po = vb.transmitted_power(Eo, p.res, p.meta["len_abs"], 2 * p.meta["corrugation"])
    assert abs(P - Po) <= 1e-12 * abs(Po)
    # c64 copy of the operator: within the complex64 tolerance
    E32 = vb.E_field_Nop_const(J, op_full, p.Gram, p.freq, Einc, prec="c64")
    assert np.linalg.norm(E32 - Eo) / np.linalg.norm(Eo) < 1e-5
    op_full.close()
