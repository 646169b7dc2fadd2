// One-call JVIE solve: JVIE_Solver_const.m (form 2, GMRES) behind the C-ABI.
//
// The reference function takes the incident field, the permittivity, the grid
// and the N operator, builds the support, the contrast and the right-hand
// side itself (JVIE_Solver_const.m:133-157), rescales them for the JVIE-II
// formulation (:243-251), solves with restarted GMRES (:276-343) and returns
// the current density on the whole grid, zero outside the scatterer
// (:521-522).  vox_jvie_solve does the same on the device: the operator is
// created for the call (its fN, contrast and support uploaded once), solved
// with vox_pgmres (complex128, the reference's arithmetic) or
// vox_solve_refined (complex64 GMRES + FP64 refinement), and destroyed.
// Included at the end of api.cu, after lane.cuh.
#pragma once

extern "C" vox_status vox_jvie_solve(const vox_jvie_desc* d, double* Je_re, double* Je_im,
                                     vox_gmres_info* info) {
  using namespace vox;
  cudaGetLastError();
  if (!d || !Je_re || !Je_im || !d->Einc_re || !d->er_re || d->L < 1 || d->M < 1 ||
      d->N < 1 || !(d->dx > 0) || !(d->freq > 0)) {
    set_error("vox_jvie_solve: NULL array or non-positive size, dx or freq");
    return VOX_ERR_BAD_ARG;
  }
  if ((d->fN_re == nullptr) == (d->G_re == nullptr)) {
    set_error("vox_jvie_solve: give exactly one of fN and G");
    return VOX_ERR_BAD_ARG;
  }
  const int form = d->form ? d->form : 2;
  const char solver = d->solver ? d->solver : 'G';
  if (form != 2) {
    set_error("vox_jvie_solve: only the JVIE-II formulation (form 2, the reference's default) "
              "is implemented");
    return VOX_ERR_UNSUPPORTED;
  }
  if (solver != 'G') {
    set_error("vox_jvie_solve: only GMRES ('G') runs behind the C-ABI; GMRES-DR and BiCGStab "
              "are the Python drivers voxphoton_b200.solvers.pgmresDR / bicgstab");
    return VOX_ERR_UNSUPPORTED;
  }
  if (d->precond != 0 && d->precond != 'L' && d->precond != 'R') {
    set_error("vox_jvie_solve: precond is 'L', 'R' or 0");
    return VOX_ERR_BAD_ARG;
  }
  if (d->prec != VOX_C128 && d->prec != VOX_C64) {
    set_error("vox_jvie_solve: prec is VOX_C128 or VOX_C64");
    return VOX_ERR_BAD_ARG;
  }
  // defaults and clamps of JVIE_Solver_const.m:76-106
  const double tol = (d->tol < 1e-15 || d->tol >= 1) ? 1e-3 : d->tol;
  const int inner_it = d->inner_it < 1 ? 50 : d->inner_it;
  const int outer_it = d->outer_it < 1 ? 200 : d->outer_it;
  if (inner_it > kMaxRestart) {
    set_error("vox_jvie_solve: inner_it above the device GMRES maximum of " +
              std::to_string(kMaxRestart));
    return VOX_ERR_BAD_ARG;
  }
  const int L = d->L, M = d->M, N = d->N;
  const long long V = (long long)L * M * N;
  const double gram = d->dx * d->dx * d->dx;  // :140-141
  // support: voxels with |e_r - 1| > 1e-12 (:147-148), 1-based, three components
  std::vector<long long> idxS;
  for (long long c = 0; c < V; c++) {
    const double mr = d->er_re[c] - 1.0, mi = d->er_im ? d->er_im[c] : 0.0;
    if (std::hypot(mr, mi) > 1e-12) idxS.push_back(c + 1);
  }
  const long long nS = (long long)idxS.size();
  const long long n = 3 * nS;
  std::vector<double> idx3(n);
  for (int k = 0; k < 3; k++)
    for (long long i = 0; i < nS; i++) idx3[k * nS + i] = (double)(k * V + idxS[i]);
  auto t0 = std::chrono::steady_clock::now();
  std::fill(Je_re, Je_re + 3 * V, 0.0);
  std::fill(Je_im, Je_im + 3 * V, 0.0);
  vox_gmres_info local{};
  vox_gmres_info* inf = info ? info : &local;
  double* resvec = inf->resvec;
  const long long cap = inf->resvec_cap;
  *inf = vox_gmres_info{};
  inf->resvec = resvec;
  inf->resvec_cap = cap;
  if (n == 0) {  // no scatterer: Je = 0
    inf->flag = 0;
    return VOX_OK;
  }
  // right-hand side Gram * j w eo Mc Einc / Mr at the support (:151-157, :249-250)
  std::vector<double> b_re(n), b_im(n);
  VOX_TRY(vox_jvie_rhs(L, M, N, d->er_re, d->er_im, d->Einc_re, d->Einc_im, gram, d->freq,
                       idx3.data(), n, b_re.data(), b_im.data()));
  // JVIE-II contrast Mc / Mr with Mr = 1 (:243-251)
  std::vector<double> mc_re(V), mc_im(V);
  for (long long c = 0; c < V; c++) {
    const double er = d->er_re[c], ei = d->er_im ? d->er_im[c] : 0.0;
    const double dd = er * er + ei * ei;
    // (e_r - 1) / e_r = 1 - 1/e_r
    mc_re[c] = 1.0 - er / dd;
    mc_im[c] = ei / dd;
  }
  vox_op_desc od{};
  od.L = L;
  od.M = M;
  od.N = N;
  od.LfN = d->LfN;
  od.MfN = d->MfN;
  od.NfN = d->NfN;
  od.fN_re = d->fN_re;
  od.fN_im = d->fN_im;
  od.G_re = d->G_re;
  od.G_im = d->G_im;
  od.Mc_re = mc_re.data();
  od.Mc_im = mc_im.data();
  od.gram = gram;
  od.idx = idx3.data();
  od.n_idx = n;
  od.precisions = d->prec == VOX_C128 ? 1 : 3;
  od.device = d->device;
  vox_op_t op = nullptr;
  VOX_TRY(vox_op_create(&od, &op));
  std::vector<double> x_re(n), x_im(n);
  // JVIE-II's preconditioner fP(J) = mv_AN_const(J, fN, 1./Mr, 1./Mr - 1, Gram) is Gram * J
  // (Mr = 1): a scalar, to which GMRES's iterates are invariant on either side, so
  // the solve runs unpreconditioned for 'L' and 'R' alike.
  vox_status s;
  if (d->prec == VOX_C128)
    s = vox_pgmres(op, nullptr, VOX_PREC_NONE, VOX_C128, b_re.data(), b_im.data(), inner_it, tol,
                   outer_it, x_re.data(), x_im.data(), inf);
  else
    s = vox_solve_refined(op, nullptr, VOX_PREC_NONE, b_re.data(), b_im.data(), tol, inner_it,
                          outer_it, 0.0, 10, x_re.data(), x_im.data(), inf);
  vox_op_destroy(op);
  if (s != VOX_OK) return s;
  // Je(idxS3) = vsol (:521-522)
  for (long long i = 0; i < n; i++) {
    const long long p = (long long)idx3[i] - 1;
    Je_re[p] = x_re[i];
    Je_im[p] = x_im[i];
  }
  inf->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return flag_status(VOX_OK, info != nullptr, *inf);
}
