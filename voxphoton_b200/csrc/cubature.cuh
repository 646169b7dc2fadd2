// Device cubature of the Toeplitz Green tensor G_mn (assembly_nop_const.m:44-92,
// cubature_nop_const.cpp:8-125): for every cell m of the L x M x N grid the 21
// face-pair integrals of exp(-j ko R)/R between the voxel at r_m and the voxel
// at the origin with the host assembly's tensor Gauss rules (4 x 4 points per
// face beyond the 5 x 5 x 5 block, 10 x 10 inside it, 20 x 20 for the 2 x 2 x 2
// near block), then the symmetric fill and the projection onto the six tensor
// components.  The eight near cells' singular corrections stay on the host
// (nearby_correct.m), applied to the pair integrals computed here.
#pragma once

#include "vox_common.cuh"

namespace vox {

struct CubGeom {
  double p1[6][3], a[6][3], b[6][3];  // face origin and edge vectors (cube_faces.m)
  int obs[21], src[21];               // the 21 face pairs integrated
  int fill[15][4];                    // I[f0][f1] = I[f2][f3] for the other 15
  double P[6][6][6];                  // (n_ii x e_a).(n_jj x e_b)
};

struct CubRules {
  const double* w[3];  // far, medium, near: np^2 weights and points on [0,1]^2
  const double* u[3];
  const double* v[3];
  int np[3];
};

__device__ __forceinline__ int cub_rule(int mx, int my, int mz, int nL, int nM, int nN) {
  if (mx < 2 && my < 2 && mz < 2) return 2;
  return (mx < nL && my < nM && mz < nN) ? 1 : 0;
}

// One warp per (cell, pair): lanes split the observation points p, each lane
// sums over all source points q; the lanes' sums are added in a fixed tree
// order.  Ipair[cell * 21 + t] = dx^4 * sum_p w_p sum_q w_q exp(-j ko R)/R.
__global__ void __launch_bounds__(256) k_cubature_pairs(int L, int M, int N, int nL, int nM,
                                                        int nN, double ko, double dx, CubGeom g,
                                                        CubRules rr, double2* __restrict__ Ipair) {
  const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const long long V = (long long)L * M * N;
  if (gw >= V * 21) return;  // uniform across the warp
  const long long cell = gw / 21;
  const int t = (int)(gw - cell * 21);
  const int mx = (int)(cell % L);
  const int my = (int)((cell / L) % M);
  const int mz = (int)(cell / ((long long)L * M));
  const int ri = cub_rule(mx, my, mz, nL, nM, nN);
  const int np = rr.np[ri];
  const double* __restrict__ w = rr.w[ri];
  const double* __restrict__ u = rr.u[ri];
  const double* __restrict__ v = rr.v[ri];
  const int Pf = g.obs[t], Qf = g.src[t];
  const double rm0 = mx * dx, rm1 = my * dx, rm2 = mz * dx;
  double sre = 0.0, sim = 0.0;
  for (int p = lane; p < np; p += 32) {
    const double ox = g.p1[Pf][0] + g.a[Pf][0] * u[p] + g.b[Pf][0] * v[p] + rm0;
    const double oy = g.p1[Pf][1] + g.a[Pf][1] * u[p] + g.b[Pf][1] * v[p] + rm1;
    const double oz = g.p1[Pf][2] + g.a[Pf][2] * u[p] + g.b[Pf][2] * v[p] + rm2;
    double are = 0.0, aim = 0.0;
    for (int q = 0; q < np; q++) {
      const double px = g.p1[Qf][0] + g.a[Qf][0] * u[q] + g.b[Qf][0] * v[q];
      const double py = g.p1[Qf][1] + g.a[Qf][1] * u[q] + g.b[Qf][1] * v[q];
      const double pz = g.p1[Qf][2] + g.a[Qf][2] * u[q] + g.b[Qf][2] * v[q];
      const double dxp = px - ox, dyp = py - oy, dzp = pz - oz;
      const double R = sqrt(dxp * dxp + dyp * dyp + dzp * dzp);
      const double wq = w[q] / R;
      double s, c;
      sincos(ko * R, &s, &c);
      are += wq * c;
      aim -= wq * s;
    }
    sre += w[p] * are;
    sim += w[p] * aim;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sre += __shfl_down_sync(0xffffffffu, sre, o);
    sim += __shfl_down_sync(0xffffffffu, sim, o);
  }
  if (lane == 0) {
    const double s4 = dx * dx * dx * dx;
    Ipair[cell * 21 + t] = make_double2(sre * s4, sim * s4);
  }
}

// Per regular cell: fill the 6 x 6 face-pair matrix by symmetry and project it
// onto the six components; G[cell + V k] (the host assembly's layout).  Near
// cells are left to the host.
__global__ void k_cubature_project(int L, int M, int N, CubGeom g,
                                   const double2* __restrict__ Ipair, double2* __restrict__ G) {
  const long long V = (long long)L * M * N;
  const double inv4pi = 1.0 / (4.0 * 3.14159265358979323846);
  for (long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < V;
       cell += (long long)gridDim.x * blockDim.x) {
    const int mx = (int)(cell % L);
    const int my = (int)((cell / L) % M);
    const int mz = (int)(cell / ((long long)L * M));
    if (mx < 2 && my < 2 && mz < 2) continue;
    double2 I[6][6];
    for (int t = 0; t < 21; t++) I[g.obs[t]][g.src[t]] = Ipair[cell * 21 + t];
    for (int f = 0; f < 15; f++) I[g.fill[f][0]][g.fill[f][1]] = I[g.fill[f][2]][g.fill[f][3]];
    for (int k = 0; k < 6; k++) {
      double gr = 0.0, gi = 0.0;
      for (int j = 0; j < 6; j++)
        for (int i = 0; i < 6; i++) {
          gr += I[i][j].x * g.P[i][j][k];
          gi += I[i][j].y * g.P[i][j][k];
        }
      G[cell + V * k] = make_double2(gr * inv4pi, gi * inv4pi);
    }
  }
}

}  // namespace vox
