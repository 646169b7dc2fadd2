// C-ABI shim over the reference's own C++ cubature cores (TEST INFRASTRUCTURE
// ONLY).  The Makefile beside this file compiles the reference sources
//   piecewise_constant/src_vie/src_operators/mexcubatures/cubature_nop_const.cpp
//   piecewise_constant/src_vie/src_operators/mexcubatures/direct_ws_{st,ea,va}_const.cpp
// from where they lie, together with this shim, into oracle/_ref/libvoxref.so.
// The shim only re-packs arguments the way the reference MEX gateways do
// (cubature_nop_const_mex.cpp:36-89, direct_ws_*_const_mex.cpp) so that the
// oracle's restatement of assembly_nop_const.m can call the real cores.
#include <complex>
#include <thread>
#include <vector>

using std::complex;

void cubature_nop(const int Np, const double w[], const double u[], const double v[],
                  const double r_m[3], const double r_n[3], const double R_faces[3][4][6],
                  const double ko, const double dx, complex<double> I_mn[6][6]);
complex<double> direct_ws_st_const(const double r1[], const double r2[], const double r3[],
                                   const double ko, const int Np_1D, const double z[],
                                   const double w[]);
complex<double> direct_ws_ea_const(const double r1[], const double r2[], const double r3[],
                                   const double r4[], const double ko, const int N_theta,
                                   const int N_psi, const double w_theta[], const double z_theta[],
                                   const double w_psi[], const double z_psi[]);
complex<double> direct_ws_va_const(const double r1[], const double r2[], const double r3[],
                                   const double r4[], const double r5[], const double ko,
                                   const int N_theta_p, const int N_theta_q, const int N_psi,
                                   const double w_theta_p[], const double z_theta_p[],
                                   const double w_theta_q[], const double z_theta_q[],
                                   const double w_psi[], const double z_psi[]);

extern "C" {

// R_faces_colmajor: MATLAB 3x4x6 array (cube_faces.m), column-major.
// out_re/out_im: 6x6 column-major, like the MEX output.
void voxref_cubature_nop(int Np, const double* w, const double* u, const double* v,
                         const double* r_m, const double* r_n, const double* R_faces_colmajor,
                         double ko, double dx, double* out_re, double* out_im) {
  double RR[3][4][6];
  for (int k = 0; k < 6; k++)
    for (int j = 0; j < 4; j++)
      for (int i = 0; i < 3; i++) RR[i][j][k] = R_faces_colmajor[i + 3 * j + 12 * k];
  complex<double> I[6][6];
  cubature_nop(Np, w, u, v, r_m, r_n, RR, ko, dx, I);
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      out_re[i + 6 * j] = I[i][j].real();
      out_im[i + 6 * j] = I[i][j].imag();
    }
}

// Gauss nodes z and weights w on [-1,1] (gauss_1d.m order: weight, xtab).
void voxref_direct_ws_st(const double* r1, const double* r2, const double* r3, double ko,
                         int Np, const double* z, const double* w, double* out) {
  complex<double> I = direct_ws_st_const(r1, r2, r3, ko, Np, z, w);
  out[0] = I.real();
  out[1] = I.imag();
}

void voxref_direct_ws_ea(const double* r1, const double* r2, const double* r3, const double* r4,
                         double ko, int Np, const double* z, const double* w, double* out) {
  complex<double> I = direct_ws_ea_const(r1, r2, r3, r4, ko, Np, Np, w, z, w, z);
  out[0] = I.real();
  out[1] = I.imag();
}

void voxref_direct_ws_va(const double* r1, const double* r2, const double* r3, const double* r4,
                         const double* r5, double ko, int Np, const double* z, const double* w,
                         double* out) {
  complex<double> I = direct_ws_va_const(r1, r2, r3, r4, r5, ko, Np, Np, Np, w, z, w, z, w, z);
  out[0] = I.real();
  out[1] = I.imag();
}


// Restatement of the far/medium loops of assembly_nop_const.m:56-66 and :80-92
// in C (the MATLAB parfor body), calling the reference core per cell.
// J_re/J_im: L x M x N x 6 x 6, column-major like the MATLAB J_mn array.
// Cells with mx < nL && my < nM && mz < nN (0-based) are computed; the rest
// are left untouched, so the far pass uses (L, M, N) and the medium pass
// uses (n_mediumL, n_mediumM, n_mediumN).
void voxref_cell_loop(int L, int M, int N, int nL, int nM, int nN, int Np, const double* w,
                      const double* u, const double* v, const double* R_faces_colmajor,
                      double ko, double dx, double* J_re, double* J_im) {
  const long V = (long)L * M * N;
  const long ncell = (long)nL * nM * nN;
  unsigned nth = std::thread::hardware_concurrency();
  if (nth == 0) nth = 1;
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nth; t++) {
    pool.emplace_back([=]() {
      for (long c = t; c < ncell; c += nth) {
        int mx = (int)(c % nL), my = (int)((c / nL) % nM), mz = (int)(c / ((long)nL * nM));
        double r_m[3] = {mx * dx, my * dx, mz * dx};
        double r_n[3] = {0.0, 0.0, 0.0};
        double re[36], im[36];
        voxref_cubature_nop(Np, w, u, v, r_m, r_n, R_faces_colmajor, ko, dx, re, im);
        long cell = mx + (long)L * (my + (long)M * mz);
        for (int k = 0; k < 36; k++) {
          J_re[cell + V * k] = re[k];
          J_im[cell + V * k] = im[k];
        }
      }
    });
  }
  for (auto& th : pool) th.join();
}

}  // extern "C"
