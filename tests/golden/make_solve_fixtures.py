"""Generate tests/golden/bragg_p20_solves.npz: whole GMRES solves of the
20-period Bragg grating of the sweep (520 x 30 x 11 at 20 nm, 1550 nm, the
benchmark's plane-wave excitation) computed by the oracle alone - the numpy
complex128 restatement of pgmres.m, mv_AN_const.m and chan_mvp_idx.m, with the
Green tensor assembled by the reference's own compiled cubature cores
(oracle/_ref, built by `make -C oracle`).  libvox is never loaded here.

Three solves, as the reference runs them (Bragg_MOR_script.m:61-80,
JVIE_Solver_const.m:276-343), all GMRES(50) to 1e-5:
  * left preconditioned by the level-1 circulant (pgmres(...,L1), the drop-in),
  * right preconditioned (pgmres(...,[],[],R1)),
  * unpreconditioned (944 iterations; about 7 minutes of oracle time, which is
    why it is a fixture and not computed inside the GPU test).
For each: the iteration record, the residual history, the final true relres,
the flag, the solution norm and a fixed subsample of the solution, and the
transmitted power of example_Bragg_1500nm_to_1600nm.m:107-113 from the total
field.  The level-1 solves use the full 520 x 30 x 11 grating because the
60-period grating's complex128 inverse blocks (1160 x 990^2, 18 GB, plus the
same again while they are built) are too heavy for a test host.

    make -C oracle && python tests/golden/make_solve_fixtures.py
"""
import importlib.util
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import assembly as oa  # noqa: E402
from oracle import vie as ov  # noqa: E402

OUT = os.path.join(HERE, "bragg_p20_solves.npz")
SUB = 185  # solution subsample stride


def geometry():
    """voxphoton_b200/geometry.py loaded from its file (numpy only), without
    the package (whose import loads libvox)."""
    name = "_vox_geometry_fixture"
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(ROOT, "voxphoton_b200", "geometry.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    geo = geometry()
    ov.set_fft_workers(os.cpu_count() or 1)
    p = geo.bragg(periods=20, M=30)
    L, M, N = p.shape
    V = L * M * N
    t = time.time()
    G = oa.assembly_nop_const(p.shape, p.ko, p.res)
    fN = ov.fN_from_toeplitz(G)
    Einc = geo.plane_wave(p)
    _, Mc, idx, b = ov.jvie2_system(Einc, p.e_r, p.Gram, p.freq)
    circ, _ = ov.level_1_parallel_func_N(G, L, M, N, p.Gram)
    inv = ov.level1_inverse_blocks(circ, ov.face_from_Mr(p.e_r.astype(complex)), p.Gram)
    del circ
    print(f"setup {time.time() - t:.1f} s", flush=True)
    ones = np.ones(p.shape)

    def A(v):
        return ov.mv_AN_const(v, fN, ones, Mc, p.Gram, "notransp", idx)

    def P(v):
        return ov.chan_mvp_idx(inv, v, L, M, N, idx)

    sub = np.arange(0, idx.size, SUB)
    out = {"shape": np.array(p.shape), "lam0": p.lam0, "tol": 1e-5, "restart": 50,
           "sub": sub, "n": idx.size}
    for name, kw, maxit in (("left", {"L1": P}, 10), ("right", {"R1": P}, 10),
                            ("none", {}, 40)):
        t = time.time()
        x, flag, relres, it, resvec = ov.pgmres(A, b, 50, 1e-5, maxit, **kw)
        J = np.zeros(3 * V, dtype=complex)
        J[idx - 1] = x
        E = ov.E_field_Nop_const(J.reshape((L, M, N, 3), order="F"), fN, p.Gram, p.freq, Einc)
        Pt = ov.transmitted_power(E, p.res, p.meta["len_abs"], 2 * p.meta["corrugation"])
        out[f"{name}_iter"] = np.array(it)
        out[f"{name}_resvec"] = resvec
        out[f"{name}_relres"] = relres
        out[f"{name}_flag"] = flag
        out[f"{name}_xnorm"] = np.linalg.norm(x)
        out[f"{name}_xsub"] = x[sub]
        out[f"{name}_power"] = Pt
        print(f"{name}: iter {it}, {len(resvec) - 1} steps, relres {relres:.3e}, flag {flag}, "
              f"P {Pt:.6e}, {time.time() - t:.1f} s", flush=True)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
