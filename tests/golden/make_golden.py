"""Generate the golden fixtures in tests/golden/ (run in a checkout that has
the reference sources and the compiled oracle/_ref library):

    make -C oracle && python tests/golden/make_golden.py

* gauss_1d.json  - the Gauss-Legendre tables of the reference's own
  piecewise_constant/src_vie/src_operators/cubatures/gauss_1d.m for the orders
  the assembly uses (4, 10, 20), parsed from the .m text.
* singular.json  - the five singular face-pair integrals (ST, EAc, EAo, VAc,
  VAo) from the reference's DEMCEM C++ cores (oracle/_ref), for two voxel
  sizes / wavelengths.
* tiny_case.npz  - a 6 x 5 x 4 grid: G_mn assembled with the reference cores
  (oracle.assembly), its circulant FFT fN, a seeded input J, the oracle's
  mv_AN_const output, and the dense O(V^2) Toeplitz direct sum of the same.
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# REFERENCE: the reference project root (the variable oracle/Makefile reads)
REF_GAUSS = os.path.join(os.environ.get("REFERENCE", "/root/reference"),
                         "piecewise_constant/src_vie/src_operators/cubatures/gauss_1d.m")


def parse_gauss(path, orders):
    text = open(path).read()
    out = {}
    for n in orders:
        m = re.search(r"order == %d \)(.*?)(elseif|else\s|end)" % n, text, re.S)
        body = m.group(1)
        x = [float(v.replace(" ", "")) for v in
             re.findall(r"xtab\(\s*\d+\s*\)\s*=\s*([-+ 0-9.eE]+);", body)]
        w = [float(v.replace(" ", "")) for v in
             re.findall(r"weight\(\s*\d+\s*\)\s*=\s*([-+ 0-9.eE]+);", body)]
        assert len(x) == n and len(w) == n, (n, len(x), len(w))
        out[str(n)] = {"xtab": x, "weight": w}
    return out


def main():
    from oracle import assembly as A
    from oracle import vie as ov

    with open(os.path.join(HERE, "gauss_1d.json"), "w") as f:
        json.dump(parse_gauss(REF_GAUSS, (4, 10, 20)), f, indent=1)

    cases = []
    for dx, lam in ((20e-9, 1550e-9), (10e-9, 1500e-9)):
        ko = 2 * np.pi / lam * 1.444
        st = A.singular_st_const(20, ko, dx, dx)
        eac, eao = A.singular_ea_const(20, ko, dx, dx, dx)
        vac, vao = A.singular_va_const(20, ko, dx, dx, dx)
        vals = [st, eac, eao, vac, vao]
        cases.append({"dx": dx, "ko": ko, "re": [v.real for v in vals],
                      "im": [v.imag for v in vals]})
    with open(os.path.join(HERE, "singular.json"), "w") as f:
        json.dump({"order": ["ST", "EAc", "EAo", "VAc", "VAo"], "cases": cases}, f, indent=1)

    shape = (6, 5, 4)
    dx, ko = 20e-9, 2 * np.pi / 1550e-9 * 1.444
    G = A.assembly_nop_const(shape, ko, dx)
    fN = ov.fN_from_toeplitz(G)
    rng = np.random.default_rng(0)
    L, M, N = shape
    J = rng.standard_normal((L, M, N, 3)) + 1j * rng.standard_normal((L, M, N, 3))
    Mc = 0.5 + 0.1j + 0 * J[..., 0]
    Gram = dx ** 3
    idx = np.arange(1, 3 * L * M * N + 1)
    y = ov.mv_AN_const(J.reshape(-1, order="F"), fN, np.ones(shape), Mc, Gram, "notransp", idx)
    nj = ov.dense_toeplitz_matvec(G, J)
    np.savez_compressed(os.path.join(HERE, "tiny_case.npz"), G=G, J=J, Mc=Mc, Gram=Gram,
                        ko=ko, dx=dx, y=y, dense_NJ=nj)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
