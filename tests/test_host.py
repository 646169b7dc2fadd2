"""Host-side checks of libvox (no GPU): the C-ABI library loads and exports
every entry point declared in include/vox.h; the host operator setup
(Toeplitz assembly with its own singular-integral scheme) matches the
reference's compiled DEMCEM/cubature cores; the RHS and geometry helpers."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

import voxphoton_b200 as vb
from voxphoton_b200 import _lib, geometry as geo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "vox.h")).read()
    declared = set(re.findall(r"\b(vox_[a-z0-9_]+)\s*\(", hdr))
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert declared <= bound, declared - bound
    assert _lib.lib().vox_abi_version() == 1


def test_singular_integrals_match_reference_demcem():
    g = json.load(open(os.path.join(GOLD, "singular.json")))
    for case in g["cases"]:
        mine = vb.singular_integrals(case["ko"], case["dx"], 32)
        ref = np.array(case["re"]) + 1j * np.array(case["im"])
        assert np.max(np.abs(np.array(mine) - ref) / np.abs(ref)) < 1e-12


def test_assembly_matches_golden_reference_cores():
    d = np.load(os.path.join(GOLD, "tiny_case.npz"))
    G = vb.assemble_toeplitz(d["G"].shape[:3], float(d["ko"]), float(d["dx"]))
    assert np.max(np.abs(G - d["G"])) < 1e-12 * np.max(np.abs(d["G"]))


def test_assembly_matches_oracle_with_reference_cores():
    pytest.importorskip("oracle.assembly")
    from oracle import assembly as A
    try:
        A.ref_lib()
    except RuntimeError:
        pytest.skip("oracle/_ref not built")
    dx, ko = 20e-9, 2 * np.pi / 1550e-9 * 1.444
    shape = (9, 7, 6)
    G1 = vb.assemble_toeplitz(shape, ko, dx)
    G2 = A.assembly_nop_const(shape, ko, dx)
    assert np.max(np.abs(G1 - G2)) < 1e-12 * np.max(np.abs(G2))
    # the xy / xz components vanish on x = 0 (device preconditioner pairing)
    assert np.max(np.abs(G1[0, :, :, 1:3])) < 1e-13 * np.max(np.abs(G1))


def test_jvie_rhs_matches_oracle():
    from oracle import vie as ov
    p = geo.bragg(periods=2, period=320e-9, len_abs=0.32e-6, res=40e-9, M=16)
    Einc = geo.plane_wave(p)
    _, _, idx, b = ov.jvie2_system(Einc, p.e_r, p.Gram, p.freq)
    out = vb.jvie_rhs(p.e_r, Einc, p.Gram, p.freq, idx)
    assert np.linalg.norm(out - b) / np.linalg.norm(b) < 1e-14


def test_benchmark_grids():
    assert geo.bragg_config("strip").shape == (100, 25, 11)
    assert geo.bragg_config("bragg20").shape == (1160, 30, 11)
    assert geo.bragg_config("bragg10").shape == (2320, 60, 22)
    assert [geo.bragg(periods=p, M=30).shape[0] for p in (20, 40, 60, 80, 100)] == [
        520, 840, 1160, 1480, 1800]
    assert geo.microdisk().shape == (560, 540, 11)


def test_assembly_rejects_bad_sizes():
    with pytest.raises(_lib.VoxError):
        vb.assemble_toeplitz((1, 4, 4), 1.0, 1e-8)


def test_operator_fails_loudly_without_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(_lib.VoxError):
        vb.Operator(np.ones((4, 4, 4)), 1.0, [1, 2, 3], G=np.zeros((4, 4, 4, 6)))


def test_transmitted_power_slice_follows_the_reference_example():
    # example_Bragg_1500nm_to_1600nm.m:107-113: x = L - round((len_abs+450nm)/res),
    # all of y (round(delW/2) of a length in metres is 0), all z, all components
    import voxphoton_b200 as vb
    rng = np.random.default_rng(0)
    E = rng.standard_normal((40, 6, 3, 3)) + 1j * rng.standard_normal((40, 6, 3, 3))
    P = vb.transmitted_power(E, 20e-9, 0.3e-6, 50e-9)
    x = 40 - int(round((0.3e-6 + 450e-9) / 20e-9))
    assert x == 2
    assert np.isclose(P, np.sum(np.abs(E[x - 1]) ** 2), rtol=1e-14)


def test_wait_limit_setter_validates_and_defaults():
    """The bounded-wait limit (no device work): bad values are refused, 0
    restores the default."""
    lib = _lib.lib()
    assert lib.vox_set_wait_timeout(-1.0) == _lib.VOX_ERR_BAD_ARG
    assert lib.vox_set_wait_timeout(float("nan")) == _lib.VOX_ERR_BAD_ARG
    assert lib.vox_set_wait_timeout(12.5) == _lib.VOX_OK
    assert lib.vox_get_wait_timeout() == 12.5
    assert lib.vox_set_wait_timeout(0.0) == _lib.VOX_OK
    assert lib.vox_get_wait_timeout() > 0


def test_memory_count_checks_its_arguments():
    """vox_mem_in_use (no device work): NULL and out-of-range devices are
    refused; with nothing created the library holds no device bytes."""
    import ctypes
    lib = _lib.lib()
    b = ctypes.c_longlong(-1)
    assert lib.vox_mem_in_use(-1, ctypes.byref(b)) == _lib.VOX_ERR_BAD_ARG
    assert lib.vox_mem_in_use(64, ctypes.byref(b)) == _lib.VOX_ERR_BAD_ARG
    assert lib.vox_mem_in_use(0, None) == _lib.VOX_ERR_BAD_ARG
    assert lib.vox_mem_in_use(0, ctypes.byref(b)) == _lib.VOX_OK and b.value >= 0


def test_jvie_solve_argument_checks_need_no_device():
    """vox_jvie_solve refuses what it does not implement (form 1, solvers other
    than GMRES) and malformed descriptors before any device call."""
    lib = _lib.lib()
    L, M, N = 4, 3, 2
    V = L * M * N
    er = np.full(V, 2.0)
    Einc = np.ones(3 * V)
    G = np.zeros(6 * V)
    out_re, out_im = np.empty(3 * V), np.empty(3 * V)
    d = _lib.JvieDesc()
    d.L, d.M, d.N = L, M, N
    d.Einc_re, d.er_re, d.G_re = _lib.dptr(Einc), _lib.dptr(er), _lib.dptr(G)
    d.dx, d.freq = 20e-9, 2.8e14
    d.form = 1
    st = lib.vox_jvie_solve(ctypes.byref(d), _lib.dptr(out_re), _lib.dptr(out_im), None)
    assert st == _lib.VOX_ERR_UNSUPPORTED
    d.form = 2
    d.solver = b"B"
    st = lib.vox_jvie_solve(ctypes.byref(d), _lib.dptr(out_re), _lib.dptr(out_im), None)
    assert st == _lib.VOX_ERR_UNSUPPORTED
    d.solver = b"G"
    d.fN_re = _lib.dptr(G)  # both fN and G
    st = lib.vox_jvie_solve(ctypes.byref(d), _lib.dptr(out_re), _lib.dptr(out_im), None)
    assert st == _lib.VOX_ERR_BAD_ARG
    d.fN_re = None
    d.dx = 0.0
    st = lib.vox_jvie_solve(ctypes.byref(d), _lib.dptr(out_re), _lib.dptr(out_im), None)
    assert st == _lib.VOX_ERR_BAD_ARG


def test_bench_matvec_roofline_byte_counts():
    # the bench's matvec line on the 1160 x 30 x 11 grating at 4 members: its
    # own bytes and the compulsory full-fN figure c (7V + 6P) per member
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    info = {"Px": 2560, "Py": 64, "Pz": 24, "n": 963600, "octant_fN": True}
    pcinfo = {"n_blocks": 581, "ld": 992, "paired": True}
    r = bench.matvec_roofline(info, (1160, 30, 11), 963600, pcinfo, 4, 0.6, 6536.7)
    V, P = 1160 * 30 * 11, 2560 * 64 * 24
    assert r["compulsory_full_fN"]["bytes_per_launch"] == 4 * 8 * (7 * V + 6 * P)
    assert abs(r["bytes_per_launch"] - 571420608) < 1
    assert abs(r["frac"] - r["bytes_per_launch"] / 0.6e-3 / 1e9 / 6536.7) < 1e-12
