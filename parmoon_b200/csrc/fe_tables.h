// Reference-element tables (host side): Lagrange bases of the hexahedral and
// tetrahedral elements and the quadrature rules the reference selects.
//
//   Q1/Q2 hexahedra: tensor Lagrange on [-1,1]^3, local index i + n (j + n k)
//     (x fastest), as include/FE3D/BF_C_H_Q1_3D.h and BF_C_H_Q2_3D.h order them.
//   P1/P2 tetrahedra on the unit simplex; P2 nodes are the lattice points
//     (i,j,k)/2 with i+j+k <= 2, k slowest then j then i
//     (include/FE3D/BF_C_T_P2_3D.h).
//   Gauss2 / Gauss3 hexahedral rules with point index 9i+3j+k, x <- k
//     (src/QuadFormulas/QuadFormulaHexa.C:67-114); Keast tetrahedral rules with
//     4 and 11 points (src/QuadFormulas/QuadFormulaTetra.C:75-150) and the
//     Keast 5-point rule (degree 3), which the reference does not have.
#pragma once
#include <cmath>
#include <vector>

namespace pmg {

enum { RULE_GAUSS2 = 2, RULE_GAUSS3 = 3, RULE_GAUSS4 = 4, RULE_KEAST4 = 104, RULE_KEAST5 = 105, RULE_KEAST11 = 111 };

struct QuadRule {
  int n = 0;
  std::vector<double> w, x, y, z;
};

inline QuadRule make_rule(int rule) {
  QuadRule q;
  auto push = [&](double w, double x, double y, double z) {
    q.w.push_back(w); q.x.push_back(x); q.y.push_back(y); q.z.push_back(z); q.n++;
  };
  if (rule == RULE_GAUSS2 || rule == RULE_GAUSS3 || rule == RULE_GAUSS4) {
    int n = rule;
    double gw[4], gx[4];
    if (n == 2) { gw[0] = gw[1] = 1.0; gx[0] = -1.0 / std::sqrt(3.0); gx[1] = 1.0 / std::sqrt(3.0); }
    else if (n == 3) { gw[0] = gw[2] = 5.0 / 9.0; gw[1] = 8.0 / 9.0; gx[0] = -std::sqrt(0.6); gx[1] = 0; gx[2] = std::sqrt(0.6); }
    else {
      // 4-point Gauss-Legendre: nodes +-sqrt(3/7 -+ 2/7 sqrt(6/5)), weights (18 +- sqrt(30))/36
      double a = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(1.2)), b = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(1.2));
      double wa = (18.0 + std::sqrt(30.0)) / 36.0, wb = (18.0 - std::sqrt(30.0)) / 36.0;
      gx[0] = -b; gx[1] = -a; gx[2] = a; gx[3] = b;
      gw[0] = wb; gw[1] = wa; gw[2] = wa; gw[3] = wb;
    }
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++)
        for (int k = 0; k < n; k++) push(gw[i] * gw[j] * gw[k], gx[k], gx[j], gx[i]);
  } else if (rule == RULE_KEAST4) {
    double a = (5.0 - std::sqrt(5.0)) / 20.0, b = (5.0 + 3.0 * std::sqrt(5.0)) / 20.0;
    push(1.0 / 24, a, a, a); push(1.0 / 24, a, a, b); push(1.0 / 24, a, b, a); push(1.0 / 24, b, a, a);
  } else if (rule == RULE_KEAST5) {
    push(-2.0 / 15.0, .25, .25, .25);
    double a = 1.0 / 6.0, b = 0.5;
    push(3.0 / 40, a, a, a); push(3.0 / 40, a, a, b); push(3.0 / 40, a, b, a); push(3.0 / 40, b, a, a);
  } else if (rule == RULE_KEAST11) {
    double s = std::sqrt(5.0 / 14.0), a = (1 + s) / 4, b = (1 - s) / 4, c = 1.0 / 14.0, d = 11.0 / 14.0;
    double w0 = -74.0 / 5625.0, w1 = 343.0 / 45000.0, w2 = 56.0 / 2250.0;
    push(w0, .25, .25, .25);
    push(w1, c, c, c); push(w1, d, c, c); push(w1, c, d, c); push(w1, c, c, d);
    push(w2, a, a, b); push(w2, a, b, a); push(w2, b, a, a); push(w2, b, b, a); push(w2, b, a, b); push(w2, a, b, b);
  }
  return q;
}

inline int elem_nloc(int e) {
  return e == PMG_ELEM_Q1_HEX ? 8 : e == PMG_ELEM_Q2_HEX ? 27 : e == PMG_ELEM_NQ1_HEX ? 6 : e == PMG_ELEM_P1_TET ? 4 : 10;
}
inline bool elem_is_hex(int e) { return e == PMG_ELEM_Q1_HEX || e == PMG_ELEM_Q2_HEX || e == PMG_ELEM_NQ1_HEX; }
// polynomial degree the quadrature rule is chosen from (GetOrig: N_terms x degree);
// N_Q1's basis holds xi^2 terms, so its rules are Q2's
inline int elem_degree(int e) { return (e == PMG_ELEM_Q2_HEX || e == PMG_ELEM_P2_TET || e == PMG_ELEM_NQ1_HEX) ? 2 : 1; }

// N_Q1 on [-1,1]^3: local dof f sits at the midpoint of face f, faces in the
// order zeta = -1, eta = -1, xi = +1, eta = +1, xi = -1, zeta = +1
// (NF_N_H_Q1_3D.h).  phi_f = 1/6 + s_f t_f / 2 + (t_f^2 - (u^2 + v^2) / 2) / 3
// with t_f the coordinate normal to face f, s_f = +-1 its side and u, v the
// other two coordinates: 1 at its own face midpoint, 0 at the other five.
constexpr int NQ1_AXIS[6] = {2, 1, 0, 1, 0, 2};
constexpr double NQ1_SIDE[6] = {-1, -1, 1, 1, -1, 1};

// value and reference gradient of every local basis function at (x,y,z):
// out[l*4 + 0..2] = d/dxi, d/deta, d/dzeta ; out[l*4 + 3] = value
inline void basis_eval(int e, double x, double y, double z, double *out) {
  if (e == PMG_ELEM_NQ1_HEX) {
    const double c[3] = {x, y, z};
    for (int f = 0; f < 6; f++) {
      const int a = NQ1_AXIS[f];
      const double s = NQ1_SIDE[f], t = c[a];
      double others = 0.0;
      for (int d = 0; d < 3; d++)
        if (d != a) others += c[d] * c[d];
      out[f * 4 + 3] = 1.0 / 6.0 + 0.5 * s * t + (t * t - 0.5 * others) / 3.0;
      for (int d = 0; d < 3; d++)
        out[f * 4 + d] = d == a ? 0.5 * s + 2.0 * t / 3.0 : -c[d] / 3.0;
    }
    return;
  }
  if (elem_is_hex(e)) {
    int p = elem_degree(e), n = p + 1;
    auto lag = [p](double s, double *v, double *d) {
      if (p == 1) { v[0] = 0.5 * (1 - s); d[0] = -0.5; v[1] = 0.5 * (1 + s); d[1] = 0.5; }
      else {
        v[0] = 0.5 * s * (s - 1); d[0] = s - 0.5;
        v[1] = 1 - s * s; d[1] = -2 * s;
        v[2] = 0.5 * s * (s + 1); d[2] = s + 0.5;
      }
    };
    double vx[3], dx[3], vy[3], dy[3], vz[3], dz[3];
    lag(x, vx, dx); lag(y, vy, dy); lag(z, vz, dz);
    for (int k = 0; k < n; k++)
      for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
          int l = i + n * (j + n * k);
          out[l * 4 + 0] = dx[i] * vy[j] * vz[k];
          out[l * 4 + 1] = vx[i] * dy[j] * vz[k];
          out[l * 4 + 2] = vx[i] * vy[j] * dz[k];
          out[l * 4 + 3] = vx[i] * vy[j] * vz[k];
        }
    return;
  }
  double L0 = 1 - x - y - z;
  auto set = [out](int l, double v, double gx, double gy, double gz) {
    out[l * 4 + 0] = gx; out[l * 4 + 1] = gy; out[l * 4 + 2] = gz; out[l * 4 + 3] = v;
  };
  if (e == PMG_ELEM_P1_TET) {
    set(0, L0, -1, -1, -1); set(1, x, 1, 0, 0); set(2, y, 0, 1, 0); set(3, z, 0, 0, 1);
    return;
  }
  // barycentric form: vertex L(2L-1), edge 4 La Lb
  double g0 = -(4 * L0 - 1);
  set(0, L0 * (2 * L0 - 1), g0, g0, g0);
  set(1, 4 * L0 * x, 4 * (L0 - x), -4 * x, -4 * x);
  set(2, x * (2 * x - 1), 4 * x - 1, 0, 0);
  set(3, 4 * L0 * y, -4 * y, 4 * (L0 - y), -4 * y);
  set(4, 4 * x * y, 4 * y, 4 * x, 0);
  set(5, y * (2 * y - 1), 0, 4 * y - 1, 0);
  set(6, 4 * L0 * z, -4 * z, -4 * z, 4 * (L0 - z));
  set(7, 4 * x * z, 4 * z, 0, 4 * x);
  set(8, 4 * y * z, 0, 4 * z, 4 * y);
  set(9, z * (2 * z - 1), 0, 0, 4 * z - 1);
}

}  // namespace pmg
