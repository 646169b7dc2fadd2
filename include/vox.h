/*
 * libvox: B200-native piecewise-constant JVIE-II frequency solve.
 *
 * C-ABI boundary for VoxPhoton's hot path.  Each entry point replaces one
 * MATLAB call of the reference (paths relative to the reference project):
 *
 *   vox_op_create        the device upload done once per operator in
 *                        piecewise_constant/src_vie/src_solver/JVIE_Solver_const.m:277-284
 *                        (fN, Mr, Mc sent to the GPU), with the operator itself
 *                        from getOPERATORS_SAM.m:83-91 (fN) or its Toeplitz form
 *   vox_mv_AN            mv_AN_const(JIn0,fN,Mr,Mc,Gram,transp_flag,idx,GPU_flag)
 *                        piecewise_constant/src_vie/src_mvp/mv_AN_const.m:1
 *   vox_mv_L             mv_L_const(JIn0,fN,r,Gram,idx,GPU_flag)
 *                        piecewise_constant/src_vie/src_mvp/mv_L_const.m:1
 *   vox_precond_create_level1 + vox_precond_apply
 *                        level_1_parallel_func_N.m:1 + Bragg_MOR_script.m:61-72 (build)
 *                        and chan_mvp_idx(inv_blocks,JIn,L,M,N,idx)
 *                        piecewise_constant/src_preconditioning/chan_mvp_idx.m:2 (apply)
 *   vox_precond_create_blocks
 *                        chan_mvp_idx with caller-supplied inverse blocks
 *   vox_pgmres           [x,flag,relres,iter,resvec] = pgmres(A,b,restart,tol,maxit,L1,[],R1)
 *                        piecewise_constant/src_numeric/src_iterative/pgmres.m:70
 *   vox_solve_refined    complex64 GMRES inside an FP64 iterative-refinement loop
 *                        (no reference counterpart; meets pgmres.m:175's relres test)
 *   vox_jvie_rhs         Vrhs of JVIE_Solver_const.m:151-157 with the JVIE-II scaling :243-251
 *   vox_assemble_toeplitz  assembly_nop_const.m:1-174 (far/medium/near cubature,
 *                        singular self/edge/vertex terms, face projection) on the host
 *
 * Conventions: complex arrays are split real/imaginary double arrays as in
 * MATLAB's classic mxArray (mxGetPr/mxGetPi); grids are column-major (x
 * fastest); index vectors are 1-based doubles as MATLAB passes them.  The
 * caller owns all host buffers; the library owns device state behind opaque
 * handles.  A handle is used by one host thread at a time.  Every call returns
 * a vox_status; vox_last_error() gives the text of the last failure on the
 * calling thread.
 */
#ifndef VOX_H_
#define VOX_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VOX_ABI_VERSION 1

typedef enum {
  VOX_OK = 0,
  VOX_ERR_BAD_ARG = 1,
  VOX_ERR_OOM = 2,
  VOX_ERR_NOT_CONVERGED = 3,
  VOX_ERR_TIMEOUT = 4,
  VOX_ERR_CUDA = 5,
  VOX_ERR_UNSUPPORTED = 6
} vox_status;
#define VOX_CUDA_ERROR VOX_ERR_CUDA

typedef enum { VOX_C128 = 0, VOX_C64 = 1 } vox_prec;
typedef enum { VOX_NOTRANSP = 0, VOX_TRANSP = 1 } vox_transp;
typedef enum { VOX_PREC_NONE = 0, VOX_PREC_LEFT = 1, VOX_PREC_RIGHT = 2 } vox_side;

typedef struct vox_op_s* vox_op_t;
typedef struct vox_precond_s* vox_precond_t;

typedef struct {
  int L, M, N;               /* domain grid */
  /* Either the FFT-circulant fN (LfN x MfN x NfN x 6, column-major, the
   * array mv_AN_const receives) ... */
  int LfN, MfN, NfN;
  const double* fN_re;
  const double* fN_im;
  /* ... or the Toeplitz tensor G_mn (L x M x N x 6, assembly_nop_const's
   * output).  Exactly one of fN_re / G_re must be non-NULL. */
  const double* G_re;
  const double* G_im;
  const double* Mr_re;       /* L x M x N; NULL => Mr == 1 (JVIE-II) */
  const double* Mr_im;       /* may be NULL (real Mr) */
  const double* Mc_re;       /* L x M x N */
  const double* Mc_im;       /* may be NULL (real Mc) */
  double gram;               /* voxel volume dx^3 */
  const double* idx;         /* n_idx 1-based positions in the 3*L*M*N grid */
  long long n_idx;
  int precisions;            /* bit 0: complex128, bit 1: complex64 (0 => both) */
  int device;                /* CUDA device ordinal */
} vox_op_desc;

/* Non-convergence (pgmres.m:176-180) is info.flag = 1 with VOX_OK; a solver
 * entry point called with info == NULL returns VOX_ERR_NOT_CONVERGED instead,
 * as the caller could not see the flag. */
typedef struct {
  int flag;                  /* 0 converged (relres <= tol), 1 not converged */
  double relres;             /* ||b - A x|| / ||b|| in FP64 (pgmres.m:175) */
  int iter_inner;            /* iterations of the last restart cycle (iter(1)) */
  int iter_outer;            /* restart cycles (iter(2)) */
  int total_iters;           /* Arnoldi steps over all cycles (and refinements) */
  int refinements;           /* FP64 refinement steps (vox_solve_refined) */
  double* resvec;            /* optional caller buffer for the preconditioned */
  long long resvec_cap;      /*   relative residual history (pgmres's resvec) */
  long long n_resvec;        /* entries written */
  double seconds;            /* wall time of the call */
} vox_gmres_info;

const char* vox_last_error(void);
int vox_abi_version(void);
/* Every wait of the library on the device is bounded: it polls against this
 * limit and returns VOX_ERR_TIMEOUT when the work has not finished (the work
 * stays queued; the handles stay usable once it drains).  Process-wide; the
 * default is VOX_WAIT_TIMEOUT_S from the environment, else 600 s; 0 restores
 * the default.  Teardown (the destroy calls) waits without a limit.  The
 * reference has no counterpart (MATLAB blocks on gpuArray results). */
vox_status vox_set_wait_timeout(double seconds);
double vox_get_wait_timeout(void);
/* Device bytes the library holds on `device` (operators, preconditioners,
 * lanes and their arenas), excluding the CUDA context, loaded modules and other
 * libraries' pools: the difference across creating a handle is what that
 * handle holds.  A serving loop admits lanes against an HBM budget with it.
 * The reference has no counterpart (MATLAB's gpuArray memory is implicit). */
vox_status vox_mem_in_use(int device, long long* bytes);

vox_status vox_op_create(const vox_op_desc* desc, vox_op_t* out);
/* An operator with `members` (1..8) independent copies of fN and of all solve
 * state, sharing grid, support idx, Mr, Mc and Gram: the co-resident
 * same-shape solves of a serving loop (e.g. one device at several
 * wavelengths), which vox_solve_refined_batch advances in lockstep with one
 * launch per kernel for all of them.  Every member starts with desc's fN; set
 * a member's operator with vox_op_interp_member.  The single-right-hand-side
 * entry points act on member 0.  No reference counterpart (MATLAB solves one
 * system per call). */
vox_status vox_op_create_batch(const vox_op_desc* desc, int members, vox_op_t* out);
/* Number of members (1 for vox_op_create). */
vox_status vox_op_members(vox_op_t op, int* members);
void vox_op_destroy(vox_op_t op);
/* Sizes chosen for the device matvec: padded grid and vector length. */
vox_status vox_op_info(vox_op_t op, int* Px, int* Py, int* Pz, long long* n);
/* Run this operator's work on the caller's cudaStream_t (NULL restores the
 * operator's own stream).  No reference counterpart (MATLAB has no streams). */
vox_status vox_op_set_stream(vox_op_t op, void* stream);
/* Kernels launched so far by the solver entry points on this operator. */
vox_status vox_op_stats(vox_op_t op, long long* launches);
/* dst.fN = sum_i w[i] * srcs[i].fN on the device (all operators on one grid,
 * padding, storage and precisions): lagrange_int(fN, S, s) of
 * piecewise_constant/src_photonics/lagrange_int.m:1-12, the reference's
 * wavelength interpolation of the operator between Legendre nodes.  Enqueued
 * on dst's stream; Mr, Mc, Gram and idx of dst are unchanged. */
vox_status vox_op_interp(vox_op_t dst, const vox_op_t* srcs, const double* w, int n);
/* The same for one member of a batched dst (the sources' member 0). */
vox_status vox_op_interp_member(vox_op_t dst, int member, const vox_op_t* srcs, const double* w,
                                int n);
/* Storage flags: bit 0 set when fN is kept as one octant (the transformed
 * circulant has the per-axis parity of the Green tensor). */
vox_status vox_op_flags(vox_op_t op, int* flags);
/* Device time (ms, CUDA events on the operator's stream, mean of reps) of each
 * kernel of one GMRES iteration, launched for all members of the operator:
 * [0..2] matvec x-forward / plane / x-inverse,
 * [3..5] preconditioner x-forward / per-mode solve / x-inverse (0 if pc is
 * NULL), [6..9] Gram-Schmidt dots / update+dots / update+norm / scale at a
 * basis of kgs+1 vectors.  ms_out holds 10 doubles. */
vox_status vox_profile_stages(vox_op_t op, vox_precond_t pc, vox_prec prec, int restart, int kgs,
                              int reps, double* ms_out);

/* JOut = A JIn (transp == VOX_NOTRANSP) or A' JIn, on the support idx.
 * Host buffers of length n_idx (split complex). */
vox_status vox_mv_AN(vox_op_t op, int transp, vox_prec prec, const double* in_re,
                     const double* in_im, double* out_re, double* out_im);
/* JOut = (N - Gram) JIn on the support (mv_L_const). */
vox_status vox_mv_L(vox_op_t op, vox_prec prec, const double* in_re, const double* in_im,
                    double* out_re, double* out_im);
/* Device variant: interleaved complex (double2 for C128, float2 for C64)
 * device pointers of length n; stream is a cudaStream_t (NULL = the op's). */
vox_status vox_mv_AN_device(vox_op_t op, int transp, vox_prec prec, const void* in, void* out,
                            void* stream);
/* Same product as vox_mv_AN_device, but allocating nothing: for callers that
 * cannot call cudaMalloc where they need the product (an external memory
 * manager owns all device memory, or allocation is forbidden in that region).
 * No counterpart in the reference.  The two plane intermediates live in a
 * fixed 64 MiB device array inside libvox (held by every GPU that loads the
 * library until exit), so operators needing more than 64 MiB of intermediates
 * (2 * Px * 3MN complex values) are rejected with VOX_ERR_BAD_ARG, and so are
 * operators whose planes are too tall for shared memory (split plane kernels,
 * which need a third intermediate).  The first call on a device looks up the
 * array's device address and keeps it for the life of that device's primary
 * context (do not call it again after cudaDeviceReset in the same process);
 * make that first call before any stream capture.  Every call shares the
 * array: calls that overlap on the GPU (different streams or threads) race.
 * Each call overwrites what it reads, so nothing carries over from the
 * previous call. */
vox_status vox_mv_AN_noalloc(vox_op_t op, int transp, vox_prec prec, const void* in, void* out,
                             void* stream);
/* count products of a batched operator in one launch: member m multiplies
 * in + m*n_idx into out + m*n_idx with its own fN (the reduced-order model's
 * MVP_A{iG} / MVP_E{iG} at all nodes at once, Bragg_MOR_script.m:39-41,
 * 78-80, 137-140).  1 <= count <= members. */
vox_status vox_mv_AN_batch_device(vox_op_t op, int transp, vox_prec prec, int count,
                                  const void* in, void* out, void* stream);

/* Tall-skinny products of the reduced-order model on interleaved complex128
 * device blocks, column-major: X is n x a (column stride ldx), Y n x b (ldy),
 * 1 <= a, b <= 32.
 *   vox_block_dot:    C = X^H Y (a x b device array, leading dimension a);
 *                     Vtemp(:,j)'*v, P'*Qtemp{iG}, P'*Vrhs (Bragg_MOR_script.m:
 *                     114-116, 137-142; example_Bragg_1500nm_to_1600nm.m:97).
 *                     FP64 sums in a fixed order: repeated calls agree bitwise.
 *   vox_block_update: Y = beta*Y + X*W, W a x b (device, leading dimension a);
 *                     v - h*Vtemp(:,j), P*x_temp (example_…:100). Y must not
 *                     overlap X; beta == 0 does not read Y.
 * stream is a cudaStream_t (NULL = the default stream). */
vox_status vox_block_dot(long long n, int a, int b, const void* X, long long ldx, const void* Y,
                         long long ldy, void* C, void* stream);
vox_status vox_block_update(long long n, int a, int b, const void* X, long long ldx,
                            const void* W, double beta, void* Y, long long ldy, void* stream);

/* Level-1 circulant preconditioner (T. Chan circulant along x, per-mode dense
 * blocks inv(Gram*I - diag(face3)*circ_i)); face3 = (m-1)/m with m the x-mean of
 * Mr (length 3*M*N, real).  G_re/G_im: the L x M x N x 6 Toeplitz tensor. */
vox_status vox_precond_create_level1(vox_op_t op, const double* G_re, const double* G_im,
                                     const double* face3, vox_precond_t* out);
/* Preconditioner from caller-supplied inverse blocks: L blocks of (3MN)^2,
 * each column-major, concatenated (chan_mvp_idx's inv_blocks). */
vox_status vox_precond_create_blocks(vox_op_t op, const double* blk_re, const double* blk_im,
                                     vox_precond_t* out);
/* Circulant preconditioner on a box of the grid (x0 <= x < x0+Ls,
 * y0 <= y < y0+Ms, every z): level 1 is level_1_parallel_func
 * (piecewise_constant/src_preconditioning/level_1_parallel_func.m:1-255: per
 * x-mode the inverse of the 3MN block of A = -Mc.*G + Gram*Mr1 at the origin),
 * level 2 is level_2_parallel_func (level_2_parallel_func.m:1-193: a second T.
 * Chan circulant along y, per (x, y)-mode inverse 3N x 3N blocks) applied as
 * chan_2_mvp_for_parallel_idx.m:2-22.  G: the box's Toeplitz tensor
 * (Ls x Ms x N x 6, column-major), Mc: the box's contrast (Ls x Ms x N), mask:
 * which box voxels it acts on (Ls*Ms*N bytes, NULL = all of the operator's
 * unknowns in the box), scale multiplies the inverse (the resonator script
 * negates it: -1).  Level 2 needs 3N <= 64 and M with prime factors <= 64.
 * On its own it acts on the box's unknowns only; combine with
 * vox_precond_create_sum. */
vox_status vox_precond_create_box(vox_op_t op, int level, int x0, int y0, int Ls, int Ms,
                                  const unsigned char* mask, const double* G_re,
                                  const double* G_im, const double* Mc_re, const double* Mc_im,
                                  double Mr1, double scale, vox_precond_t* out);
/* prec_fun_disk_idx (prec_fun_disk_idx.m:1-23): each part applied on its own
 * unknowns, the identity on the unknowns of no part.  The parts (handles made
 * on op) become owned by the sum: destroy only the sum. */
vox_status vox_precond_create_sum(vox_op_t op, const vox_precond_t* parts, int n,
                                  vox_precond_t* out);
void vox_precond_destroy(vox_precond_t p);
/* A second handle on the same factors, bound to `op` (same grid and support
 * idx as the source's operator), with its own work buffers: lets solves on
 * different operators/streams (e.g. the wavelengths of a sweep of one device)
 * apply one preconditioner concurrently.  The factors live until the last
 * handle sharing them is destroyed.  No reference counterpart. */
vox_status vox_precond_share(vox_precond_t src, vox_op_t op, vox_precond_t* out);
/* Stored inverse blocks (L, or L/2+1 when mode L-i is applied with the block
 * of mode i), their leading dimension (3MN rounded up to 32), and whether
 * modes are paired that way (1) or every mode has its own block (0). */
vox_status vox_precond_info(vox_precond_t p, int* n_blocks, int* ld, int* paired);
/* mvp = chan_mvp_idx(inv_blocks, JIn, L, M, N, idx), host buffers of length n_idx. */
vox_status vox_precond_apply(vox_precond_t p, vox_prec prec, const double* in_re,
                             const double* in_im, double* out_re, double* out_im);
/* Device variant in complex128: in/out interleaved double2 device vectors of
 * n_idx; stream is a cudaStream_t (NULL = the operator's).  The building block
 * of the solvers whose outer loop runs on the host (pgmresDR, bicgstab). */
vox_status vox_precond_apply_device(vox_precond_t p, const void* in, void* out, void* stream);

/* pgmres(A, b, restart, tol, maxit, L1) / (..., [], [], R1): one precision end to end. */
vox_status vox_pgmres(vox_op_t op, vox_precond_t pc, int side, vox_prec prec, const double* b_re,
                      const double* b_im, int restart, double tol, int maxit, double* x_re,
                      double* x_im, vox_gmres_info* info);

/* complex64 GMRES (matvec, preconditioner, Krylov basis in FP32; inner
 * products, norms and Givens in FP64) inside FP64 iterative refinement:
 * repeat { r = b - A x (FP64); d = GMRES_c64(A, r/|r|, inner_tol); x += |r| d }
 * until ||b - A x|| / ||b|| <= tol.  inner_tol <= 0 aims each inner solve at
 * the remaining target directly, f * tol * ||b|| / ||r||, with f = 0.3 for a
 * left preconditioner (GMRES then sees the preconditioned residual) and 0.9
 * otherwise; a negative inner_tol sets f = -inner_tol (at most 1). */
vox_status vox_solve_refined(vox_op_t op, vox_precond_t pc, int side, const double* b_re,
                             const double* b_im, double tol, int restart, int maxit_inner,
                             double inner_tol, int max_refine, double* x_re, double* x_im,
                             vox_gmres_info* info);

/* Device-resident variants (interleaved double2 device vectors of length n). */
vox_status vox_pgmres_device(vox_op_t op, vox_precond_t pc, int side, vox_prec prec,
                             const void* b, int restart, double tol, int maxit, void* x,
                             vox_gmres_info* info);
vox_status vox_solve_refined_device(vox_op_t op, vox_precond_t pc, int side, const void* b,
                                    double tol, int restart, int maxit_inner, double inner_tol,
                                    int max_refine, void* x, vox_gmres_info* info);

/* vox_solve_refined for `count` (1..members) right-hand sides at once on the
 * members 0..count-1 of a batched operator: b and x hold count vectors of
 * n_idx, member-major; infos holds count records.  The solves advance in
 * lockstep (one launch per kernel for all members; the preconditioner's
 * factors are read once for all of them), and each member's result is
 * identical to solving it alone.  No reference counterpart. */
vox_status vox_solve_refined_batch(vox_op_t op, vox_precond_t pc, int side, int count,
                                   const double* b_re, const double* b_im, double tol,
                                   int restart, int maxit_inner, double inner_tol,
                                   int max_refine, double* x_re, double* x_im,
                                   vox_gmres_info* infos);
/* Device variant: b and x are count interleaved double2 device vectors of n. */
vox_status vox_solve_refined_batch_device(vox_op_t op, vox_precond_t pc, int side, int count,
                                          const void* b, double tol, int restart,
                                          int maxit_inner, double inner_tol, int max_refine,
                                          void* x, vox_gmres_info* infos);

/* Continuous batching on a batched operator (no reference counterpart: the
 * reference solves one system per call).  A lane runs, for each member of the
 * operator, the solve of vox_solve_refined on that member's right-hand side;
 * every restart cycle is one launch per kernel for all members solving, and
 * a member takes a new right-hand side as soon as its previous solve has
 * finished and been collected, without waiting for the other members.  Each
 * result is identical to vox_solve_refined on that member alone.  The lane
 * owns the operator's solve state while members are solving (do not call the
 * other solver entry points on that operator meanwhile); destroying the
 * operator destroys its lanes.  pc must be a handle made or shared for this
 * operator (vox_precond_share), side as for vox_pgmres. */
typedef struct vox_lane_s* vox_lane_t;
vox_status vox_lane_create(vox_op_t op, vox_precond_t pc, int side, double tol, int restart,
                           int maxit_inner, double inner_tol, int max_refine, vox_lane_t* out);
void vox_lane_destroy(vox_lane_t lane);
/* Start a solve on a free member: b and x are interleaved double2 device
 * vectors of n_idx (x receives the solution; both must stay valid until the
 * member is collected). */
vox_status vox_lane_submit_device(vox_lane_t lane, int member, const void* b, void* x);
/* The same from host buffers (split complex, length n_idx); the solution is
 * returned by vox_lane_collect. */
vox_status vox_lane_submit(vox_lane_t lane, int member, const double* b_re, const double* b_im);
/* Advance every solving member, then run the refinement steps of the members
 * whose inner solve ended; the members that finished are written to done
 * (room for `members` entries), their count to *n_done.  For restart + 1 <= 51
 * a call runs VOX_LANE_STEPS (default 2; 0 selects whole cycles) Arnoldi steps
 * with the members' cycles out of phase: each member restarts on its own and
 * a member whose inner solve ends waits only for the rest of this call.  For
 * longer restarts a call runs one restart cycle of every solving member.
 * Either way each member's result equals the single-member solve bit for
 * bit. */
vox_status vox_lane_step(vox_lane_t lane, int* done, int* n_done);
/* Result of a finished member (x_re/x_im: host copy of the solution for host
 * submissions, or NULL), which then becomes free. */
vox_status vox_lane_collect(vox_lane_t lane, int member, double* x_re, double* x_im,
                            vox_gmres_info* info);
/* Per member: 0 free, 1 solving, 2 finished and not yet collected. */
vox_status vox_lane_state(vox_lane_t lane, int* states);

/* Vrhs = Gram * (j omega eo Mc_raw) .* Einc(idx) ./ Mr(idx)  (JVIE-II), with
 * Mc_raw = e_r - 1, Mr = e_r; e_r and Einc column-major (L x M x N, x3 for Einc). */
vox_status vox_jvie_rhs(int L, int M, int N, const double* er_re, const double* er_im,
                        const double* Einc_re, const double* Einc_im, double gram, double freq,
                        const double* idx, long long n_idx, double* out_re, double* out_im);

/* One-call JVIE solve:
 * [Je,flag,relres,iter,resvec,solvert] = JVIE_Solver_const(Einc,e_r,r,freq,fN,tol,
 *     form,solver,precond,max_it,inner_it,outer_it)
 * piecewise_constant/src_vie/src_solver/JVIE_Solver_const.m:1.  Builds the
 * support (|e_r - 1| > 1e-12), the contrast and the right-hand side as the
 * reference does (:133-157), applies the JVIE-II scaling (:243-251), solves
 * with restarted GMRES (inner_it restart, outer_it cycles) and returns the
 * current density on the whole grid (L x M x N x 3, zero outside the
 * scatterer, :521-522).  Implemented: form 2 and solver 'G' (others return
 * VOX_ERR_UNSUPPORTED; the Python mirror routes 'D' and 'B' to its GMRES-DR
 * and BiCGStab drivers).  JVIE-II's own preconditioner is Gram * I, to which
 * GMRES is invariant, so precond 'L' / 'R' give the unpreconditioned
 * iterates.  prec VOX_C128 is the reference's complex128 pgmres;
 * VOX_C64 is complex64 GMRES inside FP64 refinement to the same tol.  The
 * operator is uploaded and freed within the call. */
typedef struct {
  int L, M, N;
  const double* Einc_re;     /* L x M x N x 3, column-major */
  const double* Einc_im;     /* may be NULL */
  const double* er_re;       /* relative permittivity, L x M x N */
  const double* er_im;       /* may be NULL */
  double dx;                 /* voxel edge: Gram = dx^3 (:140-141) */
  double freq;               /* Hz */
  int LfN, MfN, NfN;         /* the N operator fN (as vox_op_desc) ... */
  const double* fN_re;
  const double* fN_im;
  const double* G_re;        /* ... or its Toeplitz tensor: exactly one */
  const double* G_im;
  double tol;                /* outside [1e-15, 1): 1e-3, as the reference */
  int form;                  /* 2 (0 means 2) */
  char solver;               /* 'G' (0 means 'G') */
  char precond;              /* 'L', 'R' or 0 */
  int inner_it;              /* restart length, < 1: 50 */
  int outer_it;              /* restart cycles (refinement: inner cycles), < 1: 200 */
  vox_prec prec;
  int device;
} vox_jvie_desc;
vox_status vox_jvie_solve(const vox_jvie_desc* desc, double* Je_re, double* Je_im,
                          vox_gmres_info* info);

/* Host assembly of the Toeplitz tensor G_mn (L x M x N x 6, column-major),
 * assembly_nop_const(r, ko, dx, 'DEMCEM').  nthreads <= 0 uses all cores. */
vox_status vox_assemble_toeplitz(int L, int M, int N, double ko, double dx, int nthreads,
                                 double* G_re, double* G_im);
/* The same tensor with the regular face-pair cubature on the GPU `device`
 * (one warp per cell and face pair, the host's Gauss rules; the eight near
 * cells' singular corrections on the host): the device half of
 * assembly_nop_const.m:44-92 / cubature_nop_const.cpp:8-125.  Agrees with
 * vox_assemble_toeplitz to rounding; output in the same host arrays. */
vox_status vox_assemble_toeplitz_device(int L, int M, int N, double ko, double dx, int device,
                                        double* G_re, double* G_im);
/* The five singular face-pair integrals (self, edge coplanar/orthogonal,
 * vertex coplanar/orthogonal) of exp(-j ko R)/R over dx-squares: out[10] as
 * re/im pairs in the order ST, EAc, EAo, VAc, VAo. */
vox_status vox_singular_integrals(double ko, double dx, int order, double* out);

#ifdef __cplusplus
}
#endif

#endif /* VOX_H_ */
