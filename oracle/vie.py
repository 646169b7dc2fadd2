"""CPU oracle for the VIE frequency-solve hot path (TEST INFRASTRUCTURE ONLY).

This module is a plain numpy/complex128 restatement of the reference MATLAB
code of VoxPhoton's piecewise-constant JVIE-II solve.  It exists only to check
the CUDA product path: only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it,
and there only as the checker or as the timed CPU baseline.  Nothing in the
``voxphoton_b200`` package imports it.

MATLAB conventions are kept exactly: arrays are column-major (``order='F'``),
index vectors are 1-based, ``fftn(X, siz)`` zero-pads at the end and
``ifftn`` scales by 1/P.  numpy's ``fft.fftn(x, s=...)`` has the same
conventions.

Parity status: the MATLAB built-ins (fftn, inv, mldivide, gmres) are closed
MathWorks code that cannot run here, so at that boundary parity is pinned by
restatement, by a dense O(V^2) Toeplitz direct sum on tiny grids and by
scipy cross-checks (tests/test_oracle.py).
"""
from __future__ import annotations

import numpy as np
from scipy.linalg import toeplitz

# Optional multi-threaded FFT for the timed CPU reference arm (scipy.fft with
# `workers`); the default numpy FFT is single-threaded pocketfft.
_FFT_WORKERS = None


def set_fft_workers(n):
    global _FFT_WORKERS
    _FFT_WORKERS = n


def _fftn(x, s=None):
    if _FFT_WORKERS:
        import scipy.fft as sf
        return sf.fftn(x, s=s, axes=tuple(range(len(s))) if s is not None else None,
                       workers=_FFT_WORKERS)
    return np.fft.fftn(x, s=s, axes=tuple(range(len(s))) if s is not None else None)


def _ifftn(x):
    if _FFT_WORKERS:
        import scipy.fft as sf
        return sf.ifftn(x, workers=_FFT_WORKERS)
    return np.fft.ifftn(x)

# --------------------------------------------------------------------------
# Operator: circulant embedding of the Toeplitz Green tensor
# --------------------------------------------------------------------------

# gperiodic_coeff_nop.m:4-31 -- sign of each of the 6 tensor components
# (xx, xy, xz, yy, yz, zz) when the Toeplitz block is mirrored into an octant.
GP_COEFF = {
    "L": np.array([+1, -1, -1, +1, +1, +1], dtype=float),
    "M": np.array([+1, -1, +1, +1, -1, +1], dtype=float),
    "N": np.array([+1, +1, -1, +1, -1, +1], dtype=float),
    "LM": np.array([+1, +1, -1, +1, -1, +1], dtype=float),
    "LN": np.array([+1, -1, +1, +1, -1, +1], dtype=float),
    "MN": np.array([+1, -1, -1, +1, +1, +1], dtype=float),
    "LMN": np.array([+1, +1, +1, +1, +1, +1], dtype=float),
}


def circulant_nop_const(G_mn: np.ndarray) -> np.ndarray:
    """circulant_nop_const.m:1-42: mirror G_mn(L,M,N,6) into Gp(2L,2M,2N,6).

    Plane L+1 (1-based) of each axis stays zero; octants L+2:2L take the
    reversed Toeplitz entries L:-1:2 times the per-component sign.
    """
    L, M, N, _ = G_mn.shape
    Gp = np.zeros((2 * L, 2 * M, 2 * N, 6), dtype=complex)
    Gp[:L, :M, :N, :] = G_mn
    rL = slice(L - 1, 0, -1)  # MATLAB L:-1:2 (1-based) -> 0-based L-1..1
    rM = slice(M - 1, 0, -1)
    rN = slice(N - 1, 0, -1)
    for ii in range(6):
        Gp[L + 1:, :M, :N, ii] = G_mn[rL, :M, :N, ii] * GP_COEFF["L"][ii]
        Gp[:L, M + 1:, :N, ii] = G_mn[:L, rM, :N, ii] * GP_COEFF["M"][ii]
        Gp[:L, :M, N + 1:, ii] = G_mn[:L, :M, rN, ii] * GP_COEFF["N"][ii]
        Gp[L + 1:, M + 1:, :N, ii] = G_mn[rL, rM, :N, ii] * GP_COEFF["LM"][ii]
        Gp[L + 1:, :M, N + 1:, ii] = G_mn[rL, :M, rN, ii] * GP_COEFF["LN"][ii]
        Gp[:L, M + 1:, N + 1:, ii] = G_mn[:L, rM, rN, ii] * GP_COEFF["MN"][ii]
    Gp[L + 1:, M + 1:, N + 1:, :] = G_mn[rL, rM, rN, :]
    return Gp


def fft_operator(A: np.ndarray) -> np.ndarray:
    """fft_operator.m:1-8: fftn of each of the d components."""
    out = np.empty(A.shape, dtype=complex)
    for p in range(A.shape[3]):
        out[..., p] = np.fft.fftn(A[..., p])
    return out


def fN_from_toeplitz(G_mn: np.ndarray) -> np.ndarray:
    """getOPERATORS_SAM.m:89-91 ('FFTofC'): fN = fft_operator(circulant(G))."""
    return fft_operator(circulant_nop_const(G_mn))


# --------------------------------------------------------------------------
# Matvecs
# --------------------------------------------------------------------------

def _scatter(JIn0, shape3, idx):
    L, M, N = shape3
    full = np.zeros(3 * L * M * N, dtype=complex)
    full[np.asarray(idx, dtype=np.int64) - 1] = JIn0
    return full.reshape((L, M, N, 3), order="F")


def _gather(JOut, idx):
    return JOut.reshape(-1, order="F")[np.asarray(idx, dtype=np.int64) - 1]


def mv_AN_const(JIn0, fN, Mr, Mc, Gram, transp_flag, idx):
    """mv_AN_const.m:1-147 (CPU branch, GPU_flag = 0).

    notransp (:102-134): JOut_c = Gram*Mr*J_c - Mc * ifftn(sum_k fN_ck fftn(J_k))[crop]
    transp   (:66-99):   the adjoint, with conj(Mc) folded into the input.
    """
    LfN, MfN, NfN, _ = fN.shape
    L, M, N = Mr.shape
    JIn = _scatter(JIn0, (L, M, N), idx)
    JOut = np.zeros((L, M, N, 3), dtype=complex)
    s = (LfN, MfN, NfN)
    if transp_flag == "transp":
        Mcc = np.conj(Mc)
        fJ = _fftn(np.conj(Mcc * JIn[..., 0]), s=s)
        J1 = fN[..., 0] * fJ
        J2 = fN[..., 1] * fJ
        J3 = fN[..., 2] * fJ
        fJ = _fftn(np.conj(Mcc * JIn[..., 1]), s=s)
        J1 = J1 + fN[..., 1] * fJ
        J2 = J2 + fN[..., 3] * fJ
        J3 = J3 + fN[..., 4] * fJ
        fJ = _fftn(np.conj(Mcc * JIn[..., 2]), s=s)
        J1 = J1 + fN[..., 2] * fJ
        J2 = J2 + fN[..., 4] * fJ
        J3 = J3 + fN[..., 5] * fJ
        for c, Jc in enumerate((J1, J2, J3)):
            Jc = _ifftn(Jc)
            JOut[..., c] = Gram * np.conj(Mr) * JIn[..., c] - np.conj(Jc[:L, :M, :N])
    elif transp_flag == "notransp":
        fJ = _fftn(JIn[...,0], s=s)
        J1 = fN[..., 0] * fJ
        J2 = fN[..., 1] * fJ
        J3 = fN[..., 2] * fJ
        fJ = _fftn(JIn[...,1], s=s)
        J1 = J1 + fN[..., 1] * fJ
        J2 = J2 + fN[..., 3] * fJ
        J3 = J3 + fN[..., 4] * fJ
        fJ = _fftn(JIn[...,2], s=s)
        J1 = J1 + fN[..., 2] * fJ
        J2 = J2 + fN[..., 4] * fJ
        J3 = J3 + fN[..., 5] * fJ
        for c, Jc in enumerate((J1, J2, J3)):
            Jc = _ifftn(Jc)
            JOut[..., c] = Gram * Mr * JIn[..., c] - Mc * Jc[:L, :M, :N]
    else:
        raise ValueError("transp_flag must be 'transp' or 'notransp'")
    return _gather(JOut, idx)


def mv_L_const(JIn0, fN, shape3, Gram, idx):
    """mv_L_const.m:1-98: JOut_c = ifftn(sum_k fN_ck fftn(J_k))[crop] - Gram*J_c."""
    LfN, MfN, NfN, _ = fN.shape
    L, M, N = shape3
    JIn = _scatter(JIn0, (L, M, N), idx)
    s = (LfN, MfN, NfN)
    fJ = _fftn(JIn[...,0], s=s)
    J1 = fN[..., 0] * fJ
    J2 = fN[..., 1] * fJ
    J3 = fN[..., 2] * fJ
    fJ = _fftn(JIn[...,1], s=s)
    J1 = J1 + fN[..., 1] * fJ
    J2 = J2 + fN[..., 3] * fJ
    J3 = J3 + fN[..., 4] * fJ
    fJ = _fftn(JIn[...,2], s=s)
    J1 = J1 + fN[..., 2] * fJ
    J2 = J2 + fN[..., 4] * fJ
    J3 = J3 + fN[..., 5] * fJ
    JOut = np.zeros((L, M, N, 3), dtype=complex)
    for c, Jc in enumerate((J1, J2, J3)):
        Jc = np.fft.ifftn(Jc)
        JOut[..., c] = Jc[:L, :M, :N] - Gram * JIn[..., c]
    return _gather(JOut, idx)


def E_field_Nop_const(J, fN, Gram, freq, Einc=None):
    """E_field_Nop_const.m:59-84: Etot = Einc + (N J - Gram J)/(Gram j w eo)."""
    mu = 4 * np.pi * 1e-7
    co = 299792458.0
    eo = 1.0 / co ** 2 / mu
    omega = 2 * np.pi * freq
    L, M, N, _ = J.shape
    if Einc is None:
        Einc = np.zeros_like(J)
    if np.count_nonzero(J) == 0:
        return Einc
    idx = np.arange(1, 3 * L * M * N + 1)
    E = mv_L_const(J.reshape(-1, order="F"), fN, (L, M, N), Gram, idx)
    E = E.reshape((L, M, N, 3), order="F")
    return Einc + E / (Gram * 1j * omega * eo)


def dense_toeplitz_matvec(G_mn, J):
    """O(V^2) direct sum of the block-Toeplitz operator (tiny grids only).

    (N J)_c(m) = sum_{m'} sum_k G_{ck}(m - m') J_k(m'), with G(-d) taken from
    the mirrored sign tables of gperiodic_coeff_nop.m.  Used to pin the
    circulant embedding + FFT convolution independently of any FFT.
    """
    L, M, N, _ = G_mn.shape
    comp = np.array([[0, 1, 2], [1, 3, 4], [2, 4, 5]])
    sL, sM, sN = GP_COEFF["L"], GP_COEFF["M"], GP_COEFF["N"]
    out = np.zeros((L, M, N, 3), dtype=complex)
    for x in range(L):
        for y in range(M):
            for z in range(N):
                dx = x - np.arange(L)[:, None, None]
                dy = y - np.arange(M)[None, :, None]
                dz = z - np.arange(N)[None, None, :]
                ax, ay, az = np.abs(dx), np.abs(dy), np.abs(dz)
                for c in range(3):
                    acc = 0.0
                    for k in range(3):
                        p = comp[c, k]
                        sign = (np.where(dx < 0, sL[p], 1.0) * np.where(dy < 0, sM[p], 1.0)
                                * np.where(dz < 0, sN[p], 1.0))
                        acc = acc + np.sum(sign * G_mn[ax, ay, az, p] * J[..., k])
                    out[x, y, z, c] = acc
    return out


# --------------------------------------------------------------------------
# Level-1 circulant preconditioner
# --------------------------------------------------------------------------

def _chan_axis0(A, sign):
    """level_1_parallel_func_N.m:12-19: T. Chan optimal circulant along x.

    c(i) = (L+1-i)/L * A(i) + sign*(i-1)/L * A(L-i+2)  for i = 2..L (1-based),
    c(1) = A(1).
    """
    L = A.shape[0]
    c = np.zeros_like(A)
    c[0] = A[0]
    for i in range(2, L + 1):
        c[i - 1] = (L + 1 - i) / L * A[i - 1] + sign * (i - 1) / L * A[L - i + 1]
    return c


def level_1_parallel_func_N(opToeplitz, L, M, N, Gram):
    """level_1_parallel_func_N.m:1-281 (on_off = 'on').

    Returns (circ, circ_L_opToep): circ is a list of L dense 3MN x 3MN blocks
    (one per x-Fourier mode), circ_L_opToep the x-FFT of the Chan circulants.
    """
    cc = np.fft.fft(_chan_axis0(opToeplitz[..., 0], +1), axis=0)
    CC = np.fft.fft(_chan_axis0(opToeplitz[..., 1], -1), axis=0)
    C3 = np.fft.fft(_chan_axis0(opToeplitz[..., 2], -1), axis=0)
    C4 = np.fft.fft(_chan_axis0(opToeplitz[..., 3], +1), axis=0)
    C5 = np.fft.fft(_chan_axis0(opToeplitz[..., 4], +1), axis=0)
    C6 = np.fft.fft(_chan_axis0(opToeplitz[..., 5], +1), axis=0)
    circ_L = np.stack([cc, -CC, -C3, C4, C5, C6], axis=3)

    MN = M * N
    zblk = toeplitz(np.arange(N))  # cell2mat(chan(toeplitz(1:N))) block index

    def block_toeplitz(chan):
        res = np.zeros((MN, MN), dtype=complex)
        for p in range(N):
            for q in range(N):
                res[p * M:(p + 1) * M, q * M:(q + 1) * M] = chan[zblk[p, q]]
        return res

    circ = []
    for il in range(L):
        temp = np.zeros((3 * MN, 3 * MN), dtype=complex)
        # First block (:119-126)
        chan = [toeplitz(cc[il, :, i], cc[il, :, i]) for i in range(N)]
        temp[:MN, :MN] = block_toeplitz(chan)
        # Second block (:129-137)
        chan = [toeplitz(np.concatenate(([-CC[il, 0, i]], CC[il, 1:, i])), -CC[il, :, i])
                for i in range(N)]
        res = block_toeplitz(chan)
        temp[:MN, MN:2 * MN] = res
        temp[MN:2 * MN, :MN] = res
        # Third block (:140-151): antisymmetrised from the upper triangle
        chan = [toeplitz(-C3[il, :, i], -C3[il, :, i]) for i in range(N)]
        res = block_toeplitz(chan)
        U = np.triu(res)
        res = U - U.T + np.diag(np.diag(U))
        temp[:MN, 2 * MN:] = res
        temp[2 * MN:, :MN] = res
        # Fourth block (:154-161)
        chan = [toeplitz(C4[il, :, i], C4[il, :, i]) for i in range(N)]
        temp[MN:2 * MN, MN:2 * MN] = block_toeplitz(chan)
        # Fifth block (:164-177): symmetrised from the upper triangle
        chan = [toeplitz(np.concatenate(([C5[il, 0, i]], -C5[il, 1:, i])), C5[il, :, i])
                for i in range(N)]
        res = block_toeplitz(chan)
        U = np.triu(res)
        res = U + U.T - np.diag(np.diag(U))
        temp[MN:2 * MN, 2 * MN:] = res
        temp[2 * MN:, MN:2 * MN] = res
        # Sixth block (:180-188)
        chan = [toeplitz(C6[il, :, i], C6[il, :, i]) for i in range(N)]
        temp[2 * MN:, 2 * MN:] = block_toeplitz(chan)
        circ.append(temp)
    return circ, circ_L


def _level1_temp(cc, CC, C3, C4, C5, C6, il, M, N):
    """The 3MN x 3MN block of x-mode il assembled from the x-FFT'd Chan
    circulants (level_1_parallel_func_N.m:113-190, level_1_parallel_func.m:90-165,
    level_2_parallel_func.m:96-166: the same toeplitz / cell2mat / triu steps)."""
    MN = M * N
    zblk = toeplitz(np.arange(N))

    def block_toeplitz(chan):
        res = np.zeros((MN, MN), dtype=complex)
        for p in range(N):
            for q in range(N):
                res[p * M:(p + 1) * M, q * M:(q + 1) * M] = chan[zblk[p, q]]
        return res

    temp = np.zeros((3 * MN, 3 * MN), dtype=complex)
    chan = [toeplitz(cc[il, :, i], cc[il, :, i]) for i in range(N)]
    temp[:MN, :MN] = block_toeplitz(chan)
    chan = [toeplitz(np.concatenate(([-CC[il, 0, i]], CC[il, 1:, i])), -CC[il, :, i])
            for i in range(N)]
    res = block_toeplitz(chan)
    temp[:MN, MN:2 * MN] = res
    temp[MN:2 * MN, :MN] = res
    chan = [toeplitz(-C3[il, :, i], -C3[il, :, i]) for i in range(N)]
    res = block_toeplitz(chan)
    U = np.triu(res)
    res = U - U.T + np.diag(np.diag(U))
    temp[:MN, 2 * MN:] = res
    temp[2 * MN:, :MN] = res
    chan = [toeplitz(C4[il, :, i], C4[il, :, i]) for i in range(N)]
    temp[MN:2 * MN, MN:2 * MN] = block_toeplitz(chan)
    chan = [toeplitz(np.concatenate(([C5[il, 0, i]], -C5[il, 1:, i])), C5[il, :, i])
            for i in range(N)]
    res = block_toeplitz(chan)
    U = np.triu(res)
    res = U + U.T - np.diag(np.diag(U))
    temp[MN:2 * MN, 2 * MN:] = res
    temp[2 * MN:, MN:2 * MN] = res
    chan = [toeplitz(C6[il, :, i], C6[il, :, i]) for i in range(N)]
    temp[2 * MN:, 2 * MN:] = block_toeplitz(chan)
    return temp


def _contrast_spectra(opToeplitz, Mc, Mr, Gram):
    """level_1_parallel_func.m:5-84 / level_2_parallel_func.m:5-84: the six
    components of -Mc .* opToeplitz (elementwise on the grid), Gram*Mr(1) added
    at the origin of the diagonal components, Chan circulant along x and FFT."""
    Mc = np.asarray(Mc)
    A = -Mc[..., None] * opToeplitz
    mr1 = np.asarray(Mr).reshape(-1, order="F")[0]
    for c in (0, 3, 5):
        A[0, 0, 0, c] = Gram * mr1 + A[0, 0, 0, c]
    signs = (+1, -1, -1, +1, +1, +1)
    return [np.fft.fft(_chan_axis0(A[..., c], signs[c]), axis=0) for c in range(6)]


def level_1_parallel_func(opToeplitz, Mc, Mr, L, M, N, Gram):
    """level_1_parallel_func.m:1-255: circ_inv{i} = inv(temp_i), temp_i the
    3MN x 3MN block of x-mode i of -Mc.*G (+ Gram*Mr(1) at the origin)."""
    sp = _contrast_spectra(opToeplitz, Mc, Mr, Gram)
    return [np.linalg.inv(_level1_temp(*sp, il, M, N)) for il in range(L)]


def level_2_parallel_func(opToeplitz, Mc, Mr, L, M, N, Gram):
    """level_2_parallel_func.m:1-193: per x-mode i, the T. Chan circulant along y
    of every M x M sub-block of temp_i, diagonalised by FFT, collapsed to M blocks
    of 3N x 3N (one per y-mode) and inverted: circ_2_inv[i][m]."""
    sp = _contrast_spectra(opToeplitz, Mc, Mr, Gram)
    out = []
    for il in range(L):
        temp = _level1_temp(*sp, il, M, N)
        diag_t = np.zeros((3 * M * N, 3 * M * N), dtype=complex)
        c = np.zeros(M, dtype=complex)
        for k in range(3 * N):          # :170-186, 1-based j, k in the reference
            for j in range(3 * N):
                row_vec = temp[j * M, k * M:(k + 1) * M]
                col_vec = temp[j * M:(j + 1) * M, k * M]
                c[0] = col_vec[0]
                for i in range(2, M + 1):
                    c[i - 1] = (M + 1 - i) / M * col_vec[i - 1] + (i - 1) / M * row_vec[M - i + 1]
                diag_t[j * M:(j + 1) * M, k * M:(k + 1) * M] = np.diag(np.fft.fft(c))
        # :190 diag_block_collapse_temp = reshape(reshape(X.',3*M*M*N,3*N).',3*M*N,3*M*N)
        X = diag_t.T.reshape((3 * M * M * N, 3 * N), order="F").T
        col = X.reshape((3 * M * N, 3 * M * N), order="F")
        out.append([np.linalg.inv(col[m * 3 * N:(m + 1) * 3 * N, m * 3 * N:(m + 1) * 3 * N])
                    for m in range(M)])
    return out


def chan_2_mvp_for_parallel_idx(inv_blocks, JIn, L, M, N, idx):
    """chan_2_mvp_for_parallel_idx.m:2-22: scatter, FFT along x, per x-mode FFT
    along y, per (x, y) mode a 3N x 3N product, inverse FFTs, gather."""
    Vrhs = np.zeros(3 * L * M * N, dtype=complex)
    ii = np.asarray(idx, dtype=np.int64) - 1
    Vrhs[ii] = JIn
    temp = Vrhs.reshape((L, 3 * M * N), order="F")
    temp = np.fft.fft(temp, axis=0).T
    for i in range(L):
        T = temp[:, i].reshape((M, 3 * N), order="F")
        T = np.fft.fft(T, axis=0).T
        for j in range(M):
            T[:, j] = inv_blocks[i][j] @ T[:, j]
        T = np.fft.ifft(T.T, axis=0)
        temp[:, i] = T.reshape(-1, order="F")
    temp = np.fft.ifft(temp.T, axis=0)
    return temp.reshape(-1, order="F")[ii]


def prec_fun_disk_idx(J, circ_WG_inv, idx_T, idx_R, L_WG, M_WG, N_WG, circ_disk_inv, L_D,
                      M_D, N_D, L, M, N, idxS3, idx_Sq):
    """prec_fun_disk_idx.m:1-23: the bus box by the level-1 circulant
    (chan_mvp), the disk by the level-2 circulant on its square, identity
    elsewhere."""
    Jt = np.zeros(3 * L * M * N, dtype=complex)
    s3 = np.asarray(idxS3, dtype=np.int64) - 1
    Jt[s3] = J
    iT = np.asarray(idx_T, dtype=np.int64) - 1
    iR = np.asarray(idx_R, dtype=np.int64) - 1
    JT = chan_mvp(circ_WG_inv, Jt[iT], L_WG, M_WG, N_WG)
    JR = chan_2_mvp_for_parallel_idx(circ_disk_inv, Jt[iR], L_D, M_D, N_D, idx_Sq)
    Jt[iT] = JT
    Jt[iR] = JR
    return Jt[s3]


def face_from_Mr(Mr):
    """Bragg_MOR_script.m:64-66: face = (m-1)/m with m = real(mean_x(Mr))."""
    L = Mr.shape[0]
    hey = np.real(np.sum(Mr, axis=0) / L)
    face = (hey - 1) / hey
    f = face.reshape(-1, order="F")
    return np.concatenate([f, f, f])


def level1_blocks(circ, face3, Gram):
    """Bragg_MOR_script.m:69-72: block_i = Gram*I - diag(face3)*circ_i (not inverted)."""
    n = circ[0].shape[0]
    return [Gram * np.eye(n) - face3[:, None] * c for c in circ]


def level1_inverse_blocks(circ, face3, Gram):
    """Bragg_MOR_script.m:69-72: circ_inv_i = inv(Gram*I - diag(face3)*circ_i)."""
    return [np.linalg.inv(b) for b in level1_blocks(circ, face3, Gram)]


def _fft1(x, axis, inverse=False):
    if _FFT_WORKERS:
        import scipy.fft as sf
        return (sf.ifft if inverse else sf.fft)(x, axis=axis, workers=_FFT_WORKERS)
    return (np.fft.ifft if inverse else np.fft.fft)(x, axis=axis)


def chan_mvp_idx(inv_blocks, JIn, L, M, N, idx):
    """chan_mvp_idx.m:2-17: scatter, fft along x, per-mode dense matvec, ifft, gather."""
    V = np.zeros(3 * L * M * N, dtype=complex)
    V[np.asarray(idx, dtype=np.int64) - 1] = JIn
    temp = V.reshape((L, 3 * M * N), order="F")
    temp = _fft1(temp, 0).T
    for i in range(L):
        temp[:, i] = inv_blocks[i] @ temp[:, i]
    temp = _fft1(temp.T, 0, inverse=True)
    return temp.reshape(-1, order="F")[np.asarray(idx, dtype=np.int64) - 1]


def chan_mvp(inv_blocks, Vrhs, L, M, N):
    """chan_mvp.m:2-12 (no index map)."""
    idx = np.arange(1, 3 * L * M * N + 1)
    return chan_mvp_idx(inv_blocks, Vrhs, L, M, N, idx)


def lagrange_int(fN, S, s):
    """lagrange_int.m:1-12: P = sum_i L_i(S) fN{i}, the Lagrange interpolant of
    the node operators fN{i} (nodes s) at wavelength S."""
    n = len(s)
    P = 0
    for i in range(n):
        Li = 1.0
        for j in range(n):
            if j != i:
                Li = Li * (S - s[j]) / (s[i] - s[j])
        P = P + Li * fN[i]
    return P


def legendre_wavelengths(s_minus, s_plus, nG):
    """Si_in_SiO2_parameters.m:7-14: s = s_mid + (s_plus - s_minus)/2 * xG with
    xG the nG Gauss-Legendre points (gauss_1d.m)."""
    xG, _ = np.polynomial.legendre.leggauss(nG)
    return 0.5 * (s_plus + s_minus) + 0.5 * (s_plus - s_minus) * xG


# --------------------------------------------------------------------------
# GMRES (pgmres.m / pgmres_iter.m)
# --------------------------------------------------------------------------

def _apply(op, x):
    if op is None:
        return x
    if callable(op):
        y = op(x)
    else:
        y = np.linalg.solve(op, x)
    y = np.asarray(y)
    if y.ndim != 1:
        raise ValueError("user supplied function must return a column vector")
    return y


def pgmres_iter(A, x, r, m, L1, L2, R1, R2, tol):
    """pgmres_iter.m:22-150: one restart cycle of (flexible L/R) GMRES.

    Arnoldi with one-pass classical Gram-Schmidt (:106-110); the least-squares
    problem is re-solved with Hc\\rhs each step (:116-120).
    """
    n = r.shape[0]
    V = np.zeros((n, m + 1), dtype=complex)
    V[:, 0] = r / np.linalg.norm(r)
    H = np.zeros((m + 1, m), dtype=complex)
    resvec = np.zeros(m)
    y = None
    res = None
    k = 0
    for k in range(1, m + 1):
        w = V[:, k - 1]
        w = _apply(R1, w)
        w = _apply(R2, w)
        w = _apply(A, w)
        w = _apply(L1, w)
        w = _apply(L2, w)
        H[:k, k - 1] = V[:, :k].conj().T @ w
        w = w - V[:, :k] @ H[:k, k - 1]
        H[k, k - 1] = np.linalg.norm(w)
        V[:, k] = w / H[k, k - 1]
        rhs = np.zeros(k + 1, dtype=complex)
        rhs[0] = np.linalg.norm(r)
        Hc = H[:k + 1, :k]
        y = np.linalg.lstsq(Hc, rhs, rcond=None)[0]
        res = rhs - Hc @ y
        resvec[k - 1] = np.linalg.norm(res)
        if resvec[k - 1] < tol:
            break
    resvec = resvec[:k]
    xupd = V[:, :k] @ y
    xupd = _apply(R1, xupd)
    xupd = _apply(R2, xupd)
    x = x + xupd
    r = V[:, :k + 1] @ res
    return x, r, k, resvec


def pgmres(A, b, restart=None, tol=None, maxit=None, L1=None, L2=None, R1=None, R2=None, x0=None):
    """pgmres.m:70-181. Returns (x, flag, relres, iter=[p, outit], resvec)."""
    restart = 50 if restart is None else restart
    tol = 1e-3 if tol is None else tol
    maxit = 10 if maxit is None else maxit
    b = np.asarray(b, dtype=complex)
    x0 = np.zeros_like(b) if x0 is None else np.asarray(x0, dtype=complex)
    if np.count_nonzero(x0):
        r = b - _apply(A, x0)
    else:
        r = b.copy()
    bp = b
    if L1 is not None:
        r = _apply(L1, r)
        bp = _apply(L1, bp)
    if L2 is not None:
        r = _apply(L2, r)
        bp = _apply(L2, bp)
    bnorm = np.linalg.norm(bp)
    resvec = np.zeros(restart * maxit + 1)
    it = 0
    outit = 0
    resvec[it] = np.linalg.norm(r) / bnorm
    x = x0
    p = 0
    while resvec[it] > tol and outit < maxit:
        outit += 1
        x, r, p, rv = pgmres_iter(A, x, r, restart, L1, L2, R1, R2, tol * bnorm)
        resvec[it + 1:it + 1 + p] = rv / bnorm
        it += p
    resvec = resvec[:it + 1]
    relres = np.linalg.norm(b - _apply(A, x)) / np.linalg.norm(b)
    flag = 0 if relres <= tol else 1
    return x, flag, relres, [p, outit], resvec


# --------------------------------------------------------------------------
# GMRES with deflated restarting (recycled harmonic Ritz subspace)
# --------------------------------------------------------------------------

def _precond_chain(A, L1, L2, R1, R2):
    """The operator of one Arnoldi step: L2 L1 A R1 R2 (pgmresDR_iter.m:60-96)."""
    def op(v):
        w = _apply(R2, v)
        w = _apply(R1, w)
        w = _apply(A, w)
        w = _apply(L1, w)
        return _apply(L2, w)
    return op


def pgmresDR_iter(A, r, m, L1, L2, R1, R2, C, tol):
    """pgmresDR_iter.m:22-142: one cycle of Arnoldi on (I - C C') L A R with
    one-pass classical Gram-Schmidt (:101-106).  Returns (V, H, B, k, resvec)."""
    op = _precond_chain(A, L1, L2, R1, R2)
    n = r.shape[0]
    V = np.zeros((n, m + 1), dtype=complex)
    V[:, 0] = r / np.linalg.norm(r)
    kc = 0 if C is None else C.shape[1]
    B = np.zeros((kc, m), dtype=complex)
    H = np.zeros((m + 1, m), dtype=complex)
    resvec = np.zeros(m)
    for k in range(1, m + 1):
        w = op(V[:, k - 1])
        if kc:
            B[:, k - 1] = C.conj().T @ w
            w = w - C @ B[:, k - 1]
        H[:k, k - 1] = V[:, :k].conj().T @ w
        w = w - V[:, :k] @ H[:k, k - 1]
        H[k, k - 1] = np.linalg.norm(w)
        V[:, k] = w / H[k, k - 1]
        rhs = np.zeros(k + 1, dtype=complex)
        rhs[0] = np.linalg.norm(r)
        y = np.linalg.lstsq(H[:k + 1, :k], rhs, rcond=None)[0]
        res = rhs - H[:k + 1, :k] @ y
        resvec[k - 1] = np.linalg.norm(res)
        if resvec[k - 1] < tol:
            return V[:, :k + 1], H[:k + 1, :k], B[:, :k], k, resvec[:k]
    return V, H, B, m, resvec


def _sort_eig(vals, vecs):
    """sortrows([abs(vals) vecs']): ascending magnitude (stable for ties)."""
    order = np.argsort(np.abs(vals), kind="stable")
    return vecs[:, order]


def getHarmVecs1(m, k, H):
    """getHarmVecs1.m: the k harmonic Ritz vectors of smallest harmonic Ritz
    value of the (m+1) x m Hessenberg H."""
    Hm = H[:m, :]
    T = np.linalg.solve(Hm.conj().T, np.eye(m))
    T[:m, :m - 1] = 0
    T = Hm + H[m, m - 1] ** 2 * T
    vals, vecs = np.linalg.eig(T)
    return _sort_eig(vals, vecs)[:, :k]


def getHarmVecs2(m, k, H2, V, U, C):
    """getHarmVecs2.m: harmonic Ritz vectors of the augmented cycle from the
    generalized problem (H2' W) z = theta (H2' H2) z; the k of largest
    |theta| (the script's last k after an ascending sort)."""
    import scipy.linalg
    Bm = H2.conj().T @ H2
    W = np.zeros((m + 1, m), dtype=complex)
    W[:k, :k] = C.conj().T @ U
    W[k:m + 1, :k] = V.conj().T @ U
    W[k:m, k:m] = np.eye(m - k)
    Am = H2.conj().T @ W
    vals, vecs = scipy.linalg.eig(Am, Bm)
    return _sort_eig(vals, vecs)[:, m - k:m]


def pgmresDR(A, b, restart=None, tol=None, maxit=None, ritz=None, L1=None, L2=None, R1=None,
             R2=None, x0=None):
    """pgmresDR.m:73-282.  Returns (x, flag, relres, iter=[p, outit], resvec)."""
    restart = 50 if restart is None else restart
    tol = 1e-3 if tol is None else tol
    maxit = 10 if maxit is None else maxit
    ritz = min(10, round(restart / 2)) if ritz is None else min(ritz, restart - 1)
    b = np.asarray(b, dtype=complex)
    x0 = np.zeros_like(b) if x0 is None else np.asarray(x0, dtype=complex)
    r = b - _apply(A, x0)
    bp = b
    if L1 is not None:
        r = _apply(L1, r)
        bp = _apply(L1, bp)
    if L2 is not None:
        r = _apply(L2, r)
        bp = _apply(L2, bp)
    bnorm = np.linalg.norm(bp)
    resvec = np.zeros(restart * (maxit + 1) + 1)
    it = 0
    outit = 0
    resvec[it] = np.linalg.norm(r) / bnorm
    V, H, _, p, rv = pgmresDR_iter(A, r, restart, L1, L2, R1, R2, None, tol * bnorm)
    resvec[it + 1:it + 1 + p] = rv / bnorm
    it += p
    y = np.linalg.lstsq(H, V.conj().T @ r, rcond=None)[0]
    x = V[:, :p] @ y
    r = r - V @ (H @ y)
    U = C = None
    if resvec[it] > tol:
        P = getHarmVecs1(p, p - 1 if ritz > p - 1 else ritz, H)
        U = V[:, :p] @ P
        Cq, R = np.linalg.qr(H @ P)
        C = V @ Cq
        U = np.linalg.solve(R.T, U.T).T                         # U / R
    while resvec[it] > tol and outit < maxit:
        outit += 1
        V, H, B, p, rv = pgmresDR_iter(A, r, restart, L1, L2, R1, R2, C, tol * bnorm)
        resvec[it + 1:it + 1 + p] = rv / bnorm
        it += p
        k = U.shape[1]
        d = np.linalg.norm(U, axis=0)
        D = np.diag(1.0 / d)
        U = U @ D
        H2 = np.zeros((k + H.shape[0], k + H.shape[1]), dtype=complex)
        H2[:k, :k] = D
        H2[:k, k:] = B
        H2[k:, k:] = H
        CV = np.concatenate([C, V], axis=1)
        y = np.linalg.lstsq(H2, CV.conj().T @ r, rcond=None)[0]
        x = x + np.concatenate([U, V[:, :p]], axis=1) @ y
        r = r - CV @ (H2 @ y)
        if resvec[it] > tol:
            P = getHarmVecs2(p + k, k, H2, V, U, C)
            U = np.concatenate([U, V[:, :p]], axis=1) @ P
            Q, R = np.linalg.qr(H2 @ P)
            C = CV @ Q
            U = np.linalg.solve(R.T, U.T).T
    x = _apply(R2, x)
    x = _apply(R1, x)
    x = x0 + x
    resvec = resvec[:it + 1]
    relres = np.linalg.norm(b - _apply(A, x)) / np.linalg.norm(b)
    flag = 0 if relres <= tol else 1
    return x, flag, relres, [p, outit], resvec


# --------------------------------------------------------------------------
# BiCGStab (JVIE_Solver_const.m:470-504 calls MATLAB's built-in bicgstab)
# --------------------------------------------------------------------------

def bicgstab(A, b, tol=1e-6, maxit=20, M=None, x0=None):
    """Preconditioned BiCGStab (van der Vorst 1992; the right-preconditioned
    form of Barrett et al., Templates, 1994, with M applied as M \\ v),
    the published algorithm behind MATLAB's bicgstab(A, b, tol, maxit, M):
    the residual is tested after each half step, so iter may end in .5.
    Returns (x, flag, relres, iter, resvec) with resvec the ||r|| history
    (one entry per half step).  flag 0 converged, 1 maxit reached, 4 a scalar
    of the recurrence vanished (breakdown)."""
    b = np.asarray(b, dtype=complex)
    x = np.zeros_like(b) if x0 is None else np.asarray(x0, dtype=complex).copy()
    nb = np.linalg.norm(b)
    r = b - _apply(A, x) if x0 is not None else b.copy()
    rt = r.copy()
    resvec = [np.linalg.norm(r)]
    if resvec[0] <= tol * nb:
        return x, 0, resvec[0] / nb, 0.0, np.array(resvec)
    rho_prev = alpha = omega = 1.0
    p = v = np.zeros_like(b)
    for i in range(1, maxit + 1):
        rho = np.vdot(rt, r)
        if rho == 0:
            return x, 4, np.linalg.norm(b - _apply(A, x)) / nb, i - 1.0, np.array(resvec)
        if i == 1:
            p = r.copy()
        else:
            beta = (rho / rho_prev) * (alpha / omega)
            p = r + beta * (p - omega * v)
        ph = _apply(M, p)
        v = _apply(A, ph)
        alpha = rho / np.vdot(rt, v)
        s = r - alpha * v
        x = x + alpha * ph
        resvec.append(np.linalg.norm(s))
        if resvec[-1] <= tol * nb:
            return x, 0, np.linalg.norm(b - _apply(A, x)) / nb, i - 0.5, np.array(resvec)
        sh = _apply(M, s)
        t = _apply(A, sh)
        tt = np.vdot(t, t)
        if tt == 0:
            return x, 4, np.linalg.norm(b - _apply(A, x)) / nb, i - 0.5, np.array(resvec)
        omega = np.vdot(t, s) / tt
        x = x + omega * sh
        r = s - omega * t
        resvec.append(np.linalg.norm(r))
        if resvec[-1] <= tol * nb:
            return x, 0, np.linalg.norm(b - _apply(A, x)) / nb, float(i), np.array(resvec)
        if omega == 0:
            return x, 4, np.linalg.norm(b - _apply(A, x)) / nb, float(i), np.array(resvec)
        rho_prev = rho
    relres = np.linalg.norm(b - _apply(A, x)) / nb
    return x, 0 if relres <= tol else 1, relres, float(maxit), np.array(resvec)


# --------------------------------------------------------------------------
# JVIE-II right-hand side (JVIE_Solver_const.m:133-157, 243-251)
# --------------------------------------------------------------------------

MU0 = 4 * np.pi * 1e-7
C0 = 299792458.0
EPS0 = 1.0 / C0 ** 2 / MU0


def jvie2_system(Einc, e_r, Gram, freq, idxS=None):
    """Returns (Mr, Mc, idxS3 (1-based), Vrhs) after the JVIE-II scaling.

    JVIE_Solver_const.m:136-157 builds Vrhs = Gram * (j w eo Mc) * Einc at the
    non-air positions; :243-251 divides Mc and Vrhs by Mr and sets Mr = 1.
    """
    L, M, N = e_r.shape
    omega = 2 * np.pi * freq
    Mr = e_r.astype(complex)
    Mc = e_r - 1.0
    nD = L * M * N
    if idxS is None:
        idxS = np.flatnonzero(np.abs(Mc.reshape(-1, order="F")) > 1e-12) + 1
    idxS3 = np.concatenate([idxS, nD + idxS, 2 * nD + idxS])
    tau = 1j * omega * EPS0 * Mc
    tau3 = np.concatenate([tau.reshape(-1, order="F")] * 3)
    Vrhs = Gram * tau3[idxS3 - 1] * Einc.reshape(-1, order="F")[idxS3 - 1]
    MrS = Mr.reshape(-1, order="F")[idxS - 1]
    Vrhs = Vrhs / np.concatenate([MrS, MrS, MrS])
    Mc = Mc / Mr
    Mr = np.ones_like(Mr)
    return Mr, Mc, idxS3, Vrhs


def transmitted_power(E, res, len_abs, delW):
    """example_Bragg_1500nm_to_1600nm.m:107-113: sum of |E|^2 over the x-slice
    xThru = L - round((len_abs + 450e-9)/res) (1-based), trimmed by
    voxFromEdge = round(delW/2)/res voxels at each y edge (the reference
    rounds a length in metres, so nanometre corrugations trim nothing)."""
    L, M = E.shape[:2]
    xThru = L - int(round((len_abs + 450e-9) / res))
    voxFromEdge = int(round(round(delW / 2) / res))
    eThru = E[xThru - 1, voxFromEdge:M - voxFromEdge, :, :]
    return float(np.sum(np.real(eThru * np.conj(eThru))))
