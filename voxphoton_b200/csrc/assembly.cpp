// Host-side operator setup: Toeplitz Green-tensor assembly of the N operator,
// assembly_nop_const.m:1-174 (DEMCEM branch) of the reference, one time per
// wavelength.
//
// G_mn(m, k) = 1/(4 pi) sum_{ii,jj} J_mn(ii,jj) P(ii,jj,k), where J_mn(ii,jj) is
// the 4-D integral of exp(-j ko R)/R over face ii of the observation voxel m and
// face jj of the source voxel at the origin, and P (vector_projection.m) the
// (n_ii x e_a).(n_jj x e_b) projections of the 6 tensor components.
//
// Regular face pairs use the reference's tensor Gauss rules (4x4 points per face
// beyond the 5x5x5 block, 10x10 inside it, 20x20 for the 2x2x2 near block:
// assembly_nop_const.m:16-19, cubature_nop_const.cpp:8-125), so regular entries
// match the reference to rounding.  The five weakly singular pair integrals
// (touching faces: self, coplanar/orthogonal edge-adjacent, coplanar/orthogonal
// vertex-adjacent) are computed here by a different exact-to-quadrature method
// than the reference's DEMCEM: because the kernel depends only on the
// displacement d = y - x between two axis-aligned squares, the 4-D integral is
// an integral of K(|d|) against the piecewise-linear overlap density of d
// (2-D for coplanar squares, 3-D for orthogonal ones); the cells of that
// density that touch d = 0 are mapped with Duffy transforms (the Jacobian
// cancels 1/R), so tensor Gauss-Legendre converges geometrically.
#include <cmath>
#include <complex>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/vox.h"

namespace vox {
void set_error(const std::string& msg);
}

namespace {

using cd = std::complex<double>;

// Gauss-Legendre nodes/weights on [-1,1] by Newton iteration on P_n.
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; i++) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    double pp = 0;
    for (int it = 0; it < 100; it++) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; j++) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      const double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1e-16) {
        // one more pass for the derivative at the converged node
        p1 = 1.0;
        p2 = 0.0;
        for (int j = 1; j <= n; j++) {
          const double p3 = p2;
          p2 = p1;
          p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
        }
        pp = n * (z * p1 - p2) / (z * z - 1.0);
        break;
      }
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

// 2-D tensor rule on [0,1]^2 in the reference's ordering (gauss_2d.m): I outer,
// J inner, weights scaled by 1/4.
struct Rule2D {
  std::vector<double> w, u, v;
};
Rule2D rule2d(int np) {
  std::vector<double> x, w1;
  gauss_legendre(np, x, w1);
  Rule2D r;
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++) {
      r.w.push_back(w1[i] * w1[j] / 4.0);
      r.u.push_back((x[i] + 1.0) / 2.0);
      r.v.push_back((x[j] + 1.0) / 2.0);
    }
  return r;
}

// Faces of the voxel [0,dx]^3 (cube_faces.m): origin corner, edge vectors a, b.
struct Face {
  double p1[3], a[3], b[3];
};
void cube_faces(double d, Face f[6]) {
  const double c[6][4][3] = {
      {{0, 0, 0}, {0, d, 0}, {0, d, d}, {0, 0, d}},  // -x
      {{d, 0, 0}, {d, d, 0}, {d, d, d}, {d, 0, d}},  // +x
      {{0, 0, 0}, {d, 0, 0}, {d, 0, d}, {0, 0, d}},  // -y
      {{0, d, 0}, {d, d, 0}, {d, d, d}, {0, d, d}},  // +y
      {{0, 0, 0}, {d, 0, 0}, {d, d, 0}, {0, d, 0}},  // -z
      {{0, 0, d}, {d, 0, d}, {d, d, d}, {0, d, d}},  // +z
  };
  for (int k = 0; k < 6; k++)
    for (int j = 0; j < 3; j++) {
      f[k].p1[j] = c[k][0][j];
      f[k].a[j] = c[k][1][j] - c[k][0][j];
      f[k].b[j] = c[k][3][j] - c[k][0][j];
    }
}

// The 21 face pairs evaluated by quadrature; the other 15 entries follow by
// symmetry (cubature_nop_const.cpp:27-30, 95-114).
const int kObs[21] = {0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 4, 4, 5};
const int kSrc[21] = {0, 1, 2, 3, 4, 5, 0, 2, 3, 4, 5, 2, 3, 4, 5, 2, 4, 5, 4, 5, 4};
const int kFill[15][4] = {{1, 1, 0, 0}, {2, 0, 1, 3}, {2, 1, 0, 3}, {3, 0, 1, 2}, {3, 1, 0, 2},
                          {3, 3, 2, 2}, {4, 0, 1, 5}, {4, 1, 0, 5}, {4, 2, 3, 5}, {4, 3, 2, 5},
                          {5, 0, 1, 4}, {5, 1, 0, 4}, {5, 2, 3, 4}, {5, 3, 2, 4}, {5, 5, 4, 4}};

// I[ii][jj] = dx^4 * sum_p sum_q w_p w_q exp(-j ko R)/R, observation voxel at r_m,
// source voxel at the origin.
void face_cubature(const Rule2D& r, const Face F[6], const double rm[3], double ko, double dx,
                   cd I[6][6]) {
  const int np = (int)r.w.size();
  std::vector<double> px(np), py(np), pz(np);
  for (int t = 0; t < 21; t++) {
    const Face& P = F[kObs[t]];
    const Face& Q = F[kSrc[t]];
    double sre = 0.0, sim = 0.0;
    for (int q = 0; q < np; q++) {
      px[q] = Q.p1[0] + Q.a[0] * r.u[q] + Q.b[0] * r.v[q];
      py[q] = Q.p1[1] + Q.a[1] * r.u[q] + Q.b[1] * r.v[q];
      pz[q] = Q.p1[2] + Q.a[2] * r.u[q] + Q.b[2] * r.v[q];
    }
    for (int p = 0; p < np; p++) {
      const double ox = P.p1[0] + P.a[0] * r.u[p] + P.b[0] * r.v[p] + rm[0];
      const double oy = P.p1[1] + P.a[1] * r.u[p] + P.b[1] * r.v[p] + rm[1];
      const double oz = P.p1[2] + P.a[2] * r.u[p] + P.b[2] * r.v[p] + rm[2];
      double are = 0.0, aim = 0.0;
      for (int q = 0; q < np; q++) {
        const double dxp = px[q] - ox, dyp = py[q] - oy, dzp = pz[q] - oz;
        const double R = std::sqrt(dxp * dxp + dyp * dyp + dzp * dzp);
        const double wq = r.w[q] / R;
        are += wq * std::cos(ko * R);
        aim -= wq * std::sin(ko * R);
      }
      sre += r.w[p] * are;
      sim += r.w[p] * aim;
    }
    I[kObs[t]][kSrc[t]] = cd(sre, sim);
  }
  for (const auto& f : kFill) I[f[0]][f[1]] = I[f[2]][f[3]];
  const double s = dx * dx * dx * dx;
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) I[i][j] *= s;
}

// ---------------------------------------------------------- singular terms
struct GL {
  std::vector<double> x, w;  // on [0,1]
};
GL gl01(int n) {
  std::vector<double> x, w;
  gauss_legendre(n, x, w);
  GL g;
  for (int i = 0; i < n; i++) {
    g.x.push_back(0.5 * (x[i] + 1.0));
    g.w.push_back(0.5 * w[i]);
  }
  return g;
}

inline cd kern(double ko, double R) { return std::exp(cd(0.0, -ko * R)) / R; }

// Overlap density of d = y - x for x uniform on [0,h], y uniform on [o, o+h]:
// a triangle of height h centred on o.
inline double tri(double d, double o, double h) {
  const double t = h - std::fabs(d - o);
  return t > 0 ? t : 0.0;
}

// Coplanar squares: I = int K(|d|) g1(d1) g2(d2) dd1 dd2, the source square
// shifted by (o1, o2) in units of h (o in {0,1}).  The density support is
// [o1-1, o1+1] x [o2-1, o2+1] (in h); unit cells that touch d = 0 use Duffy.
cd coplanar(double ko, double h, int o1, int o2, const GL& g) {
  cd tot = 0.0;
  for (int c1 = o1 - 1; c1 <= o1; c1++)
    for (int c2 = o2 - 1; c2 <= o2; c2++) {
      // cell [c1, c1+1] x [c2, c2+1] (units of h)
      const bool sing = (c1 == 0 || c1 == -1) && (c2 == 0 || c2 == -1);
      cd acc = 0.0;
      if (!sing) {
        for (size_t i = 0; i < g.x.size(); i++)
          for (size_t j = 0; j < g.x.size(); j++) {
            const double d1 = h * (c1 + g.x[i]), d2 = h * (c2 + g.x[j]);
            const double R = std::hypot(d1, d2);
            acc += g.w[i] * g.w[j] * kern(ko, R) * tri(d1, o1 * h, h) * tri(d2, o2 * h, h);
          }
        acc *= h * h;
      } else {
        // corner at the origin; direction signs of the cell
        const double s1 = c1 == 0 ? 1.0 : -1.0, s2 = c2 == 0 ? 1.0 : -1.0;
        for (int tri_half = 0; tri_half < 2; tri_half++)
          for (size_t i = 0; i < g.x.size(); i++)
            for (size_t j = 0; j < g.x.size(); j++) {
              const double s = g.x[i], u = g.x[j];
              const double rho = std::sqrt(1.0 + u * u);
              double a = h * s, b = h * s * u;
              if (tri_half) std::swap(a, b);
              const double d1 = s1 * a, d2 = s2 * b;
              // K * Jacobian = exp(-j ko h s rho)/(h s rho) * h^2 s
              const cd kj = std::exp(cd(0.0, -ko * h * s * rho)) * (h / rho);
              acc += g.w[i] * g.w[j] * kj * tri(d1, o1 * h, h) * tri(d2, o2 * h, h);
            }
      }
      tot += acc;
    }
  return tot;
}

// Orthogonal squares: observation square in z=0 ([0,h]^2 in x,y), source
// square in the plane x = h, y in [o2 h, (o2+1) h], z in [0, h].  d1 = h - x1 and
// d3 = z2 are uniform on [0,h]; d2 = y2 - y1 has the triangle density centred
// on o2 h.  The unit cell [0,1]^3 (in h) touching d = 0 uses a 3-D Duffy map.
cd orthogonal(double ko, double h, int o2, const GL& g) {
  cd tot = 0.0;
  const size_t n = g.x.size();
  for (int c2 = o2 - 1; c2 <= o2; c2++) {
    const bool sing = (c2 == 0 || c2 == -1);
    cd acc = 0.0;
    if (!sing) {
      for (size_t i = 0; i < n; i++)
        for (size_t j = 0; j < n; j++)
          for (size_t k = 0; k < n; k++) {
            const double d1 = h * g.x[i], d2 = h * (c2 + g.x[j]), d3 = h * g.x[k];
            const double R = std::sqrt(d1 * d1 + d2 * d2 + d3 * d3);
            acc += g.w[i] * g.w[j] * g.w[k] * kern(ko, R) * tri(d2, o2 * h, h);
          }
      acc *= h * h * h;
    } else {
      const double s2 = c2 == 0 ? 1.0 : -1.0;
      // three pyramids: the largest of (d1, |d2|, d3) is h*s
      for (int pyr = 0; pyr < 3; pyr++)
        for (size_t i = 0; i < n; i++)
          for (size_t j = 0; j < n; j++)
            for (size_t k = 0; k < n; k++) {
              const double s = g.x[i], u = g.x[j], v = g.x[k];
              const double rho = std::sqrt(1.0 + u * u + v * v);
              double q[3];
              q[pyr] = h * s;
              q[(pyr + 1) % 3] = h * s * u;
              q[(pyr + 2) % 3] = h * s * v;
              const double d2 = s2 * q[1];
              // K * Jacobian = exp(-j ko h s rho)/(h s rho) * h^3 s^2
              const cd kj = std::exp(cd(0.0, -ko * h * s * rho)) * (h * h * s / rho);
              acc += g.w[i] * g.w[j] * g.w[k] * kj * tri(d2, o2 * h, h);
            }
    }
    tot += acc;
  }
  return tot;
}

struct Singular {
  cd ST, EAc, EAo, VAc, VAo;
};

Singular singular_terms(double ko, double h, int order) {
  const GL g = gl01(order);
  Singular s;
  s.ST = coplanar(ko, h, 0, 0, g);
  s.EAc = coplanar(ko, h, 1, 0, g);
  s.VAc = coplanar(ko, h, 1, 1, g);
  s.EAo = orthogonal(ko, h, 0, g);
  s.VAo = orthogonal(ko, h, 1, g);
  return s;
}

// nearby_correct.m:73-199.  For each near cell m in {1,2}^3 a 6x6 code table:
// 0 keeps the regular 20x20 cubature, 1..5 take ST, EAc, EAo, VAc, VAo and 6
// is an exact zero (the reference's 0.0 entries where P == 0).
enum { KEEP = 0, ST = 1, EAC = 2, EAO = 3, VAC = 4, VAO = 5, ZERO = 6 };
struct NearTable {
  int m[3];
  int code[6][6];
};
const NearTable kNear[8] = {
    {{1, 1, 1},
     {{ST, KEEP, EAO, EAO, EAO, EAO}, {KEEP, ST, EAO, EAO, EAO, EAO}, {EAO, EAO, ST, KEEP, EAO, EAO},
      {EAO, EAO, KEEP, ST, EAO, EAO}, {EAO, EAO, EAO, EAO, ST, KEEP}, {EAO, EAO, EAO, EAO, KEEP, ST}}},
    {{2, 1, 1},
     {{KEEP, ST, EAO, EAO, EAO, EAO}, {KEEP, KEEP, KEEP, KEEP, KEEP, KEEP},
      {KEEP, EAO, EAC, KEEP, VAO, VAO}, {KEEP, EAO, KEEP, EAC, VAO, VAO},
      {KEEP, EAO, VAO, VAO, EAC, KEEP}, {KEEP, EAO, VAO, VAO, KEEP, EAC}}},
    {{2, 1, 2},
     {{KEEP, EAC, VAO, VAO, KEEP, EAO}, {KEEP, KEEP, KEEP, KEEP, KEEP, KEEP},
      {KEEP, VAO, VAC, KEEP, KEEP, VAO}, {KEEP, VAO, KEEP, VAC, KEEP, VAO},
      {KEEP, EAO, VAO, VAO, KEEP, EAC}, {KEEP, KEEP, KEEP, KEEP, KEEP, KEEP}}},
    {{1, 1, 2},
     {{EAC, KEEP, VAO, VAO, KEEP, EAO}, {KEEP, EAC, VAO, VAO, KEEP, EAO},
      {VAO, VAO, EAC, KEEP, KEEP, EAO}, {VAO, VAO, KEEP, EAC, KEEP, EAO},
      {EAO, EAO, EAO, EAO, KEEP, ST}, {KEEP, KEEP, KEEP, KEEP, KEEP, KEEP}}},
    {{1, 2, 1},
     {{EAC, KEEP, KEEP, EAO, VAO, VAO}, {KEEP, EAC, KEEP, EAO, VAO, VAO},
      {EAO, EAO, KEEP, ST, EAO, EAO}, {KEEP, KEEP, KEEP, KEEP, KEEP, KEEP},
      {VAO, VAO, KEEP, EAO, EAC, KEEP}, {VAO, VAO, KEEP, EAO, KEEP, EAC}}},
    {{2, 2, 1},
     {{KEEP, EAC, KEEP, EAO, VAO, VAO}, {KEEP, KEEP, KEEP, KEEP, KEEP, KEEP},
      {KEEP, EAO, KEEP, EAC, VAO, VAO}, {KEEP, KEEP, KEEP, KEEP, KEEP, KEEP},
      {KEEP, VAO, KEEP, VAO, VAC, KEEP}, {KEEP, VAO, KEEP, VAO, KEEP, VAC}}},
    {{1, 2, 2},
     {{VAC, KEEP, KEEP, VAO, KEEP, VAO}, {KEEP, VAC, KEEP, VAO, KEEP, VAO},
      {VAO, VAO, KEEP, EAC, KEEP, EAO}, {KEEP, KEEP, KEEP, KEEP, KEEP, KEEP},
      {VAO, VAO, KEEP, EAO, KEEP, EAC}, {KEEP, KEEP, KEEP, KEEP, KEEP, KEEP}}},
    {{2, 2, 2},
     {{KEEP, VAC, KEEP, VAO, KEEP, VAO}, {KEEP, KEEP, KEEP, KEEP, KEEP, KEEP},
      {KEEP, VAO, KEEP, VAC, KEEP, VAO}, {KEEP, KEEP, KEEP, KEEP, KEEP, KEEP},
      {KEEP, VAO, KEEP, VAO, KEEP, VAC}, {KEEP, KEEP, KEEP, KEEP, KEEP, KEEP}}},
};

// Which entries of a near table come from the singular values instead of the
// cubature: the reference's P == 0 positions.  Its C tables hold 0.0 at
// some P == 0 positions; ZERO marks those.
const int kNearPzero[8][6][6] = {
    // m = [1,1,1]: P has ones at (1,2),(2,1),(3,4),(4,3),(5,6),(6,5)
    {{1, 0, 1, 1, 1, 1}, {0, 1, 1, 1, 1, 1}, {1, 1, 1, 0, 1, 1},
     {1, 1, 0, 1, 1, 1}, {1, 1, 1, 1, 1, 0}, {1, 1, 1, 1, 0, 1}},
    // m = [2,1,1]
    {{0, 1, 1, 1, 1, 1}, {0, 0, 0, 0, 0, 0}, {0, 1, 1, 0, 1, 1},
     {0, 1, 0, 1, 1, 1}, {0, 1, 1, 1, 1, 0}, {0, 1, 1, 1, 0, 1}},
    // m = [2,1,2]
    {{0, 1, 1, 1, 0, 1}, {0, 0, 0, 0, 0, 0}, {0, 1, 1, 0, 0, 1},
     {0, 1, 0, 1, 0, 1}, {0, 1, 1, 1, 0, 1}, {0, 0, 0, 0, 0, 0}},
    // m = [1,1,2]
    {{1, 0, 1, 1, 0, 1}, {0, 1, 1, 1, 0, 1}, {1, 1, 1, 0, 0, 1},
     {1, 1, 0, 1, 0, 1}, {1, 1, 1, 1, 0, 1}, {0, 0, 0, 0, 0, 0}},
    // m = [1,2,1]
    {{1, 0, 0, 1, 1, 1}, {0, 1, 0, 1, 1, 1}, {1, 1, 0, 1, 1, 1},
     {0, 0, 0, 0, 0, 0}, {1, 1, 0, 1, 1, 0}, {1, 1, 0, 1, 0, 1}},
    // m = [2,2,1]
    {{0, 1, 0, 1, 1, 1}, {0, 0, 0, 0, 0, 0}, {0, 1, 0, 1, 1, 1},
     {0, 0, 0, 0, 0, 0}, {0, 1, 0, 1, 1, 0}, {0, 1, 0, 1, 0, 1}},
    // m = [1,2,2]
    {{1, 0, 0, 1, 0, 1}, {0, 1, 0, 1, 0, 1}, {1, 1, 0, 1, 0, 1},
     {0, 0, 0, 0, 0, 0}, {1, 1, 0, 1, 0, 1}, {0, 0, 0, 0, 0, 0}},
    // m = [2,2,2]
    {{0, 1, 0, 1, 0, 1}, {0, 0, 0, 0, 0, 0}, {0, 1, 0, 1, 0, 1},
     {0, 0, 0, 0, 0, 0}, {0, 1, 0, 1, 0, 1}, {0, 0, 0, 0, 0, 0}},
};

// P(ii, jj, comp) = (n_ii x e_a).(n_jj x e_b) for comp in xx,xy,xz,yy,yz,zz.
void projection(double P[6][6][6]) {
  const double n[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
  const int ab[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  auto cross = [](const double* u, const double* v, double* o) {
    o[0] = u[1] * v[2] - u[2] * v[1];
    o[1] = u[2] * v[0] - u[0] * v[2];
    o[2] = u[0] * v[1] - u[1] * v[0];
  };
  const double e[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++)
      for (int c = 0; c < 6; c++) {
        double u[3], v[3];
        cross(n[i], e[ab[c][0]], u);
        cross(n[j], e[ab[c][1]], v);
        P[i][j][c] = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
      }
}

}  // namespace

// Host parts shared with the device cubature (vox_assemble_toeplitz_device):
// the quadrature rules, the face geometry and projections, and the near-cell
// correction, all exactly as the host assembly below uses them.
namespace vox {

// 2-D rule of np x np points on [0,1]^2 (gauss_2d.m ordering): w, u, v.
void asm_rule(int np, std::vector<double>& w, std::vector<double>& u, std::vector<double>& v) {
  const Rule2D r = rule2d(np);
  w = r.w;
  u = r.u;
  v = r.v;
}

// Face origins and edge vectors of the voxel [0,dx]^3, and P(ii, jj, comp).
void asm_tables(double dx, double p1[6][3], double a[6][3], double b[6][3], double P[6][6][6],
                int obs[21], int src[21], int fill[15][4]) {
  Face F[6];
  cube_faces(dx, F);
  for (int k = 0; k < 6; k++)
    for (int j = 0; j < 3; j++) {
      p1[k][j] = F[k].p1[j];
      a[k][j] = F[k].a[j];
      b[k][j] = F[k].b[j];
    }
  projection(P);
  for (int t = 0; t < 21; t++) {
    obs[t] = kObs[t];
    src[t] = kSrc[t];
  }
  std::memcpy(fill, kFill, sizeof(kFill));
}

// G(m) of a near cell (mx, my, mz < 2) from its 21 regular pair integrals
// (20 x 20 rule, already scaled by dx^4): fill by symmetry, replace the
// singular entries (nearby_correct.m), project.  G[k] = re/im of component k.
void asm_near_cell(int mx, int my, int mz, const double Ipair[21][2], double ko, double dx,
                   double G[6][2]) {
  const Singular sg = singular_terms(ko, dx, 32);
  const cd sv[6] = {0.0, sg.ST, sg.EAc, sg.EAo, sg.VAc, sg.VAo};
  cd I[6][6];
  for (int t = 0; t < 21; t++) I[kObs[t]][kSrc[t]] = cd(Ipair[t][0], Ipair[t][1]);
  for (const auto& f : kFill) I[f[0]][f[1]] = I[f[2]][f[3]];
  int ti = -1;
  for (int t = 0; t < 8; t++)
    if (kNear[t].m[0] == mx + 1 && kNear[t].m[1] == my + 1 && kNear[t].m[2] == mz + 1) ti = t;
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++)
      if (kNearPzero[ti][i][j]) {
        const int c = kNear[ti].code[i][j];
        I[i][j] = (c == KEEP || c == ZERO) ? cd(0.0) : sv[c];
      }
  double P[6][6][6];
  projection(P);
  const double inv4pi = 1.0 / (4.0 * M_PI);
  for (int k = 0; k < 6; k++) {
    cd g = 0.0;
    for (int j = 0; j < 6; j++)
      for (int i = 0; i < 6; i++) g += I[i][j] * P[i][j][k];
    g *= inv4pi;
    G[k][0] = g.real();
    G[k][1] = g.imag();
  }
}

}  // namespace vox

extern "C" {

vox_status vox_singular_integrals(double ko, double dx, int order, double* out) {
  if (!out || dx <= 0 || order < 2) {
    vox::set_error("vox_singular_integrals: bad argument");
    return VOX_ERR_BAD_ARG;
  }
  const Singular s = singular_terms(ko, dx, order);
  const cd v[5] = {s.ST, s.EAc, s.EAo, s.VAc, s.VAo};
  for (int i = 0; i < 5; i++) {
    out[2 * i] = v[i].real();
    out[2 * i + 1] = v[i].imag();
  }
  return VOX_OK;
}

vox_status vox_assemble_toeplitz(int L, int M, int N, double ko, double dx, int nthreads,
                                 double* G_re, double* G_im) {
  if (L < 2 || M < 2 || N < 2 || !G_re || !G_im || dx <= 0) {
    vox::set_error("vox_assemble_toeplitz: needs L, M, N >= 2 and output buffers");
    return VOX_ERR_BAD_ARG;
  }
  const long long V = (long long)L * M * N;
  Face F[6];
  cube_faces(dx, F);
  double P[6][6][6];
  projection(P);
  const Rule2D far = rule2d(4), medium = rule2d(10), nearr = rule2d(20);
  const int nL = std::min(5, L), nM = std::min(5, M), nN = std::min(5, N);
  const Singular sg = singular_terms(ko, dx, 32);
  const cd sv[6] = {0.0, sg.ST, sg.EAc, sg.EAo, sg.VAc, sg.VAo};
  unsigned nth = nthreads > 0 ? (unsigned)nthreads : std::thread::hardware_concurrency();
  if (nth == 0) nth = 1;
  const double inv4pi = 1.0 / (4.0 * M_PI);
  auto cell_G = [&](int mx, int my, int mz) {
    cd I[6][6];
    const double rm[3] = {mx * dx, my * dx, mz * dx};
    const bool near = mx < 2 && my < 2 && mz < 2;
    const bool med = mx < nL && my < nM && mz < nN;
    if (near) {
      face_cubature(nearr, F, rm, ko, dx, I);
      int ti = -1;
      for (int t = 0; t < 8; t++)
        if (kNear[t].m[0] == mx + 1 && kNear[t].m[1] == my + 1 && kNear[t].m[2] == mz + 1) ti = t;
      for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++)
          if (kNearPzero[ti][i][j]) {
            const int c = kNear[ti].code[i][j];
            I[i][j] = (c == KEEP || c == ZERO) ? cd(0.0) : sv[c];
          }
    } else {
      face_cubature(med ? medium : far, F, rm, ko, dx, I);
    }
    const long long cell = mx + (long long)L * (my + (long long)M * mz);
    for (int k = 0; k < 6; k++) {
      cd g = 0.0;
      for (int j = 0; j < 6; j++)
        for (int i = 0; i < 6; i++) g += I[i][j] * P[i][j][k];
      g *= inv4pi;
      G_re[cell + V * k] = g.real();
      G_im[cell + V * k] = g.imag();
    }
  };
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nth; t++) {
    pool.emplace_back([&, t]() {
      for (long long c = t; c < V; c += nth) {
        const int mx = (int)(c % L), my = (int)((c / L) % M), mz = (int)(c / ((long long)L * M));
        cell_G(mx, my, mz);
      }
    });
  }
  for (auto& th : pool) th.join();
  return VOX_OK;
}

}  // extern "C"
