// Finite-element assembly on the device (sm_100a).
//
// Replaces TAssembleMat3D::Reset + Assemble3D (src/System/AssembleMat3D.C:261-535)
// with its local forms (src/FE/ConvDiff3D.C:87-214, src/FE/TCD3D.C:37-266) and
// the scatter AddLocalSqMatToGlobal / AddLocalRhsToGlobal (:751-857, :913-1096).
//
// Layout and schedule:
//   * elements are stored in colour order; the elements of one colour share
//     no degree of freedom, so one launch per colour scatters without atomics;
//   * a group of NLOC lanes handles one element (Q2: 27 lanes = one element
//     per warp; Q1: 4 elements per warp; P2: 3; P1: 8);
//   * the reference-element table u_l(q) = (d/dxi, d/deta, d/dzeta, value) of
//     every basis function at every quadrature point lives in shared memory;
//   * per quadrature point the form is a 4x4 matrix D_q acting on u
//     (A_ij = sum_q u_i(q)^T D_q u_j(q)); lane j owns column j of the local
//     matrix and accumulates all NLOC rows in registers;
//   * the element -> CSR slot map (precomputed once per mesh by binary search
//     in the sorted rows, replacing the linear search of AssembleMat3D.C:795-817)
//     turns the scatter into plain loads/stores.
#include "pmg_internal.h"
#include "fe_tables.h"
#include <cstdio>

namespace pmg {

// ----------------------------------------------------------------- coefficients
// Device stand-in for the CoeffFct3D callback; c[0..6] = eps, b1, b2, b3, c, f, |b|.
struct CoefDev {
  int kind;
  double eps, b[3], c, f, t;
  int n_modes;
  const double *modes;
};

__device__ __forceinline__ void coeff_eval(const CoefDev &C, double x, double y, double z, double *c) {
  const double PI = 3.14159265358979323846;
  c[0] = C.eps; c[1] = C.b[0]; c[2] = C.b[1]; c[3] = C.b[2]; c[4] = C.c; c[5] = C.f;
  switch (C.kind) {
    case PMG_COEF_SINE_RHS:
      c[5] = 3 * PI * PI * C.eps * sin(PI * x) * sin(PI * y) * sin(PI * z);
      break;
    case PMG_COEF_LOGNORMAL: {
      double g = 0;
      for (int m = 0; m < C.n_modes; m++) {
        const double *M = C.modes + 8 * m;
        g += M[3] * cos(2 * PI * (M[0] * x + M[1] * y + M[2] * z) + M[4]);
      }
      c[0] = C.eps * exp(g);
      break;
    }
    case PMG_COEF_CURL_FOURIER: {
      double bx = 0, by = 0, bz = 0;
      for (int m = 0; m < C.n_modes; m++) {
        const double *M = C.modes + 8 * m;
        double arg = 2 * PI * (M[0] * x + M[1] * y + M[2] * z) + M[4];
        double s = -M[3] * sin(arg) * 2 * PI;
        double gx = s * M[0], gy = s * M[1], gz = s * M[2];
        bx += gy * M[7] - gz * M[6];
        by += gz * M[5] - gx * M[7];
        bz += gx * M[6] - gy * M[5];
      }
      c[1] = C.b[0] * bx; c[2] = C.b[0] * by; c[3] = C.b[0] * bz;
      break;
    }
    case PMG_COEF_ROTATING:
      c[1] = -(y - 0.5); c[2] = x - 0.5; c[3] = 0.2 * sin(2 * PI * C.t);
      break;
    case PMG_COEF_AMC:
      c[0] = 1.0; c[1] = c[2] = c[3] = 0; c[4] = 0;
      c[5] = (3. * PI * PI - 0.1) * exp(-0.1 * C.t) * sin(PI * x) * cos(PI * y) * cos(PI * z);
      break;
    default:
      break;
  }
  c[6] = sqrt(c[1] * c[1] + c[2] * c[2] + c[3] * c[3]);
}

// coefficients at quadrature point q of element e: analytic kinds, or the
// host-evaluated table (PMG_COEF_TABLE, 6 values per point)
__device__ __forceinline__ void coeff_at(const CoefDev &C, const double *ctab, int nq, int e, int q, double x,
                                         double y, double z, double *c) {
  if (C.kind == PMG_COEF_TABLE) {
    const double *v = ctab + ((size_t)e * nq + q) * 6;
#pragma unroll
    for (int k = 0; k < 6; k++) c[k] = v[k];
    c[6] = sqrt(c[1] * c[1] + c[2] * c[2] + c[3] * c[3]);
  } else {
    coeff_eval(C, x, y, z, c);
  }
}

// SDFEM_TYPE 2 (src/FE/ConvDiff.C:591-611)
__device__ __forceinline__ double sdfem_delta(double h, double eps, double b1, double b2, double b3, int poly,
                                              double delta0) {
  if (fabs(eps) < 1e-20) eps = 1e-20;
  double nb = sqrt(b1 * b1 + b2 * b2 + b3 * b3);
  if (!(nb > 0)) return 0.0;
  double nu = 1.0 / poly;
  double alpha = nu * nb * h / (2 * eps);
  return delta0 * nu * h * (1 / tanh(alpha) - 1 / alpha) / (2 * nb);
}

// Mesh size in convection direction (src/FE/ConvDiff.C:373-470):
// 2|b| / sum_i |b . grad phi_i(barycentre)| over the vertex basis.
// Tetrahedra: phi_i are the barycentric coordinates (gradients from J^{-1}).
// Axis-aligned bricks: phi_i trilinear, gradient at the centre (+-1/(4hx), ..).
// Other hexahedra: the physical-coordinate trilinear interpolant is solved for.
__device__ double hk_convection(bool hex, bool brick, const double *cv, const double *Ji, double b1, double b2,
                                double b3) {
  double nb = sqrt(b1 * b1 + b2 * b2 + b3 * b3), den = 0;
  if (!hex) {
    double g[4][3];
    for (int a = 0; a < 3; a++) {
      g[a + 1][0] = Ji[a * 3 + 0]; g[a + 1][1] = Ji[a * 3 + 1]; g[a + 1][2] = Ji[a * 3 + 2];
    }
    for (int d = 0; d < 3; d++) g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
    for (int i = 0; i < 4; i++) den += fabs(b1 * g[i][0] + b2 * g[i][1] + b3 * g[i][2]);
  } else if (brick) {
    // edge lengths from the bounding box (any vertex order of an axis-aligned cell)
    double lo[3] = {cv[0], cv[1], cv[2]}, hi[3] = {cv[0], cv[1], cv[2]};
    for (int v = 1; v < 8; v++)
      for (int d = 0; d < 3; d++) {
        lo[d] = fmin(lo[d], cv[3 * v + d]);
        hi[d] = fmax(hi[d], cv[3 * v + d]);
      }
    double px = b1 / (hi[0] - lo[0]), py = b2 / (hi[1] - lo[1]), pz = b3 / (hi[2] - lo[2]);
    den = 0.5 * (fabs(px + py + pz) + fabs(px + py - pz) + fabs(px - py + pz) + fabs(px - py - pz));
  } else {
    // general hexahedron: invert the 8x8 monomial matrix (1,x,y,z,xy,xz,yz,xyz)
    double A[8][16], sx = 0, sy = 0, sz = 0;
    for (int v = 0; v < 8; v++) {
      double x = cv[3 * v], y = cv[3 * v + 1], z = cv[3 * v + 2];
      sx += x; sy += y; sz += z;
      double m[8] = {1, x, y, z, x * y, x * z, y * z, x * y * z};
      for (int k = 0; k < 8; k++) { A[v][k] = m[k]; A[v][8 + k] = (k == v) ? 1.0 : 0.0; }
    }
    sx *= 0.125; sy *= 0.125; sz *= 0.125;
    for (int k = 0; k < 8; k++) {
      int p = k;
      for (int i = k + 1; i < 8; i++) if (fabs(A[i][k]) > fabs(A[p][k])) p = i;
      if (p != k) for (int j = 0; j < 16; j++) { double t = A[k][j]; A[k][j] = A[p][j]; A[p][j] = t; }
      double inv = 1.0 / A[k][k];
      for (int j = 0; j < 16; j++) A[k][j] *= inv;
      for (int i = 0; i < 8; i++)
        if (i != k) {
          double f = A[i][k];
          for (int j = 0; j < 16; j++) A[i][j] -= f * A[k][j];
        }
    }
    for (int i = 0; i < 8; i++) {
      double c1 = A[1][8 + i], c2 = A[2][8 + i], c3 = A[3][8 + i], c4 = A[4][8 + i], c5 = A[5][8 + i],
             c6 = A[6][8 + i], c7 = A[7][8 + i];
      double val = b1 * (c1 + c4 * sy + c5 * sz + c7 * sy * sz);
      val += b2 * (c2 + c4 * sx + c6 * sz + c7 * sx * sz);
      val += b3 * (c3 + c5 * sx + c6 * sy + c7 * sx * sy);
      den += fabs(val);
    }
  }
  if (den < 1e-10) {
    // fall back to the cell diameter (CELL_MEASURE default branch)
    int nv = hex ? 8 : 4;
    double hK = 0;
    for (int a = 0; a < nv; a++)
      for (int b = a + 1; b < nv; b++) {
        double dx = cv[3 * a] - cv[3 * b], dy = cv[3 * a + 1] - cv[3 * b + 1], dz = cv[3 * a + 2] - cv[3 * b + 2];
        hK = fmax(hK, sqrt(dx * dx + dy * dy + dz * dz));
      }
    return hK;
  }
  return 2 * nb / den;
}

// ----------------------------------------------------------------- kernel
template <int E> struct ET;
template <> struct ET<PMG_ELEM_Q1_HEX> { static constexpr int NLOC = 8, NV = 8; static constexpr bool HEX = true; };
template <> struct ET<PMG_ELEM_Q2_HEX> { static constexpr int NLOC = 27, NV = 8; static constexpr bool HEX = true; };
template <> struct ET<PMG_ELEM_P1_TET> { static constexpr int NLOC = 4, NV = 4; static constexpr bool HEX = false; };
template <> struct ET<PMG_ELEM_P2_TET> { static constexpr int NLOC = 10, NV = 4; static constexpr bool HEX = false; };

constexpr int ASM_WARPS = 8;

struct AsmArgs {
  int n_elems;              // elements of this colour
  const int *elem_dof;      // colour-sorted, n x NLOC (already offset to the colour)
  const double *cell_vert;  // n x NV x 3
  const int *slot;          // n x NLOC x NLOC
  int Na;
  double *entries, *rhs;
  int form, poly, brick;
  double delta0;
  CoefDev coef;
  const double *ctab;  // n x NQ x 6 (PMG_COEF_TABLE), already offset to the colour
  const double *utab;  // NQ x NLOC x 4
  const double *qtab;  // NQ x 4 : weight, xi, eta, zeta
  int *flags;
};

// affine map of a cell (HexaAffin on vertices 0, 1, 3, 4 over [-1,1]^3;
// TetraAffin on vertices 0..3 over the unit simplex): x = x0 + J xi, its
// inverse Ji, |det J| and K = Ji Ji^T (diffusion in reference gradients)
template <bool HEX>
__device__ __forceinline__ void cell_map(const double *cv, double *J, double *x0, double *Ji, double &adet,
                                         double *K) {
  if (HEX) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      J[d * 3 + 0] = (cv[3 + d] - cv[d]) * 0.5;
      J[d * 3 + 1] = (cv[9 + d] - cv[d]) * 0.5;
      J[d * 3 + 2] = (cv[12 + d] - cv[d]) * 0.5;
      x0[d] = (cv[3 + d] + cv[9 + d] + cv[12 + d] - cv[d]) * 0.5;
    }
  } else {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      J[d * 3 + 0] = cv[3 + d] - cv[d];
      J[d * 3 + 1] = cv[6 + d] - cv[d];
      J[d * 3 + 2] = cv[9 + d] - cv[d];
      x0[d] = cv[d];
    }
  }
  double det = J[0] * J[4] * J[8] + J[1] * J[5] * J[6] + J[2] * J[3] * J[7] - J[2] * J[4] * J[6] -
               J[1] * J[3] * J[8] - J[0] * J[5] * J[7];
  double rd = 1.0 / det;
  Ji[0] = (J[4] * J[8] - J[5] * J[7]) * rd;
  Ji[1] = (J[2] * J[7] - J[1] * J[8]) * rd;
  Ji[2] = (J[1] * J[5] - J[2] * J[4]) * rd;
  Ji[3] = (J[5] * J[6] - J[3] * J[8]) * rd;
  Ji[4] = (J[0] * J[8] - J[2] * J[6]) * rd;
  Ji[5] = (J[2] * J[3] - J[0] * J[5]) * rd;
  Ji[6] = (J[3] * J[7] - J[4] * J[6]) * rd;
  Ji[7] = (J[1] * J[6] - J[0] * J[7]) * rd;
  Ji[8] = (J[0] * J[4] - J[1] * J[3]) * rd;
  adet = fabs(det);
#pragma unroll
  for (int p = 0; p < 3; p++)
#pragma unroll
    for (int q = 0; q < 3; q++)
      K[p * 3 + q] = Ji[p * 3 + 0] * Ji[q * 3 + 0] + Ji[p * 3 + 1] * Ji[q * 3 + 1] + Ji[p * 3 + 2] * Ji[q * 3 + 2];
}

// the 4x4 matrix D of one form at one point, in reference gradients:
// A_ij = sum_q w_q |det J| sum_{a,b} u_ia(q) D_ab u_jb(q), u = (d/dxi, d/deta,
// d/dzeta, value) of the test (i) and trial (j) basis functions
// (BilinearAssemble / _SD, ConvDiff3D.C:87-214; MatrixMRhsAssemble(_SUPG),
// TCD3D.C:37-266).  bh = Ji b.
__device__ __forceinline__ void form_matrix(int form, bool supg, const double *c, const double *K,
                                            const double *bh, double delta, double *D) {
#pragma unroll
  for (int k = 0; k < 16; k++) D[k] = 0.0;
  if (form == PMG_FORM_MASS || form == PMG_FORM_MASS_SUPG) {
    D[15] = 1.0;
    if (form == PMG_FORM_MASS_SUPG)
#pragma unroll
      for (int p = 0; p < 3; p++) D[p * 4 + 3] = delta * bh[p];
  } else {
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int r = 0; r < 3; r++) D[p * 4 + r] = c[0] * K[p * 3 + r] + (supg ? delta * bh[p] * bh[r] : 0.0);
#pragma unroll
    for (int r = 0; r < 3; r++) D[12 + r] = bh[r];
    D[15] = c[4];
    if (supg)
#pragma unroll
      for (int p = 0; p < 3; p++) D[p * 4 + 3] = delta * c[4] * bh[p];
  }
}

template <int E, int NQ>
__global__ void __launch_bounds__(ASM_WARPS * 32, 2) k_assemble(AsmArgs a) {
  constexpr int NLOC = ET<E>::NLOC, NV = ET<E>::NV, GPW = 32 / NLOC;
  constexpr bool HEX = ET<E>::HEX;
  constexpr int GS = NQ * 20;  // per-element scratch: D_q (16) + F_q (4)
  extern __shared__ double sm[];
  double *sU = sm;
  double *sQ = sU + NQ * NLOC * 4;
  double *sG = sQ + NQ * 4;
  for (int k = threadIdx.x; k < NQ * NLOC * 4; k += blockDim.x) sU[k] = a.utab[k];
  for (int k = threadIdx.x; k < NQ * 4; k += blockDim.x) sQ[k] = a.qtab[k];
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = lane / NLOC, t = lane - grp * NLOC;
  const bool lane_used = grp < GPW;
  double *G = sG + (size_t)(warp * GPW + (lane_used ? grp : 0)) * GS;
  const bool supg = (a.form == PMG_FORM_SUPG || a.form == PMG_FORM_MASS_SUPG || a.form == PMG_FORM_STIFF_SUPG);

  for (int base = (blockIdx.x * ASM_WARPS + warp) * GPW; base < a.n_elems; base += gridDim.x * ASM_WARPS * GPW) {
    const int e = base + grp;
    const bool valid = lane_used && e < a.n_elems;
    if (valid) {
      const double *cv = a.cell_vert + (size_t)e * NV * 3;
      double J[9], x0[3], Ji[9], K[9], adet;
      cell_map<HEX>(cv, J, x0, Ji, adet, K);
      double hconv = 0;
      if (supg) {
        // the reference caches the convection-direction size from the first
        // quadrature point's b for the whole cell (ConvDiff.C:376-383)
        double X = x0[0] + J[0] * sQ[1] + J[1] * sQ[2] + J[2] * sQ[3];
        double Y = x0[1] + J[3] * sQ[1] + J[4] * sQ[2] + J[5] * sQ[3];
        double Z = x0[2] + J[6] * sQ[1] + J[7] * sQ[2] + J[8] * sQ[3];
        double c[7];
        coeff_at(a.coef, a.ctab, NQ, e, 0, X, Y, Z, c);
        hconv = hk_convection(HEX, a.brick != 0, cv, Ji, c[1], c[2], c[3]);
      }
      for (int q = t; q < NQ; q += NLOC) {
        const double xi = sQ[q * 4 + 1], eta = sQ[q * 4 + 2], zeta = sQ[q * 4 + 3];
        double X = x0[0] + J[0] * xi + J[1] * eta + J[2] * zeta;
        double Y = x0[1] + J[3] * xi + J[4] * eta + J[5] * zeta;
        double Z = x0[2] + J[6] * xi + J[7] * eta + J[8] * zeta;
        double c[7];
        coeff_at(a.coef, a.ctab, NQ, e, q, X, Y, Z, c);
        const double mult = sQ[q * 4] * adet;
        double delta = supg ? sdfem_delta(hconv, c[0], c[1], c[2], c[3], a.poly, a.delta0) : 0.0;
        double bh[3];  // b in reference gradients: b . (Ji^T g^) = (Ji b) . g^
#pragma unroll
        for (int p = 0; p < 3; p++) bh[p] = Ji[p * 3 + 0] * c[1] + Ji[p * 3 + 1] * c[2] + Ji[p * 3 + 2] * c[3];
        double D[16];
        form_matrix(a.form, supg, c, K, bh, delta, D);
        double *Gq = G + q * 20;
#pragma unroll
        for (int k = 0; k < 16; k++) Gq[k] = D[k] * mult;
        const double fm = mult * c[5];
        const bool supg_rhs = supg;
        Gq[16] = supg_rhs ? fm * delta * bh[0] : 0.0;
        Gq[17] = supg_rhs ? fm * delta * bh[1] : 0.0;
        Gq[18] = supg_rhs ? fm * delta * bh[2] : 0.0;
        Gq[19] = fm;
      }
    }
    __syncwarp();
    if (valid) {
      double acc[NLOC];
#pragma unroll
      for (int i = 0; i < NLOC; i++) acc[i] = 0.0;
      double racc = 0.0;
      for (int q = 0; q < NQ; q++) {
        const double *uj = sU + (q * NLOC + t) * 4;
        const double *Dq = G + q * 20;
        const double u0 = uj[0], u1 = uj[1], u2 = uj[2], u3 = uj[3];
        const double T0 = Dq[0] * u0 + Dq[1] * u1 + Dq[2] * u2 + Dq[3] * u3;
        const double T1 = Dq[4] * u0 + Dq[5] * u1 + Dq[6] * u2 + Dq[7] * u3;
        const double T2 = Dq[8] * u0 + Dq[9] * u1 + Dq[10] * u2 + Dq[11] * u3;
        const double T3 = Dq[12] * u0 + Dq[13] * u1 + Dq[14] * u2 + Dq[15] * u3;
        racc += Dq[16] * u0 + Dq[17] * u1 + Dq[18] * u2 + Dq[19] * u3;
        const double *ui = sU + q * NLOC * 4;
#pragma unroll
        for (int i = 0; i < NLOC; i++) {
          const double2 p01 = *reinterpret_cast<const double2 *>(ui + i * 4);
          const double2 p23 = *reinterpret_cast<const double2 *>(ui + i * 4 + 2);
          acc[i] += p01.x * T0 + p01.y * T1 + p23.x * T2 + p23.y * T3;
        }
      }
      // scatter through the slot map (no two elements of a colour share a row)
      const int *dof = a.elem_dof + (size_t)e * NLOC;
      const int *sl = a.slot + (size_t)e * NLOC * NLOC;
      int bad = 0;
#pragma unroll
      for (int i = 0; i < NLOC; i++) {
        const int di = __ldg(dof + i);
        const int s = __ldg(sl + i * NLOC + t);
        if (di < a.Na) {
          if (s >= 0) a.entries[s] += acc[i];
          else bad = 1;
        } else if (i == t && s >= 0) {
          a.entries[s] = 1.0;  // Dirichlet row: unit diagonal (AssembleMat3D.C:840-848)
        }
      }
      if (a.rhs) {
        const int dt = __ldg(dof + t);
        if (dt < a.Na) a.rhs[dt] += racc;
      }
      if (bad) atomicOr(a.flags, 1);
    }
    __syncwarp();
  }
}

// ------------------------------------------------- constant-coefficient kernel
// When eps, b and c do not vary in space (PMG_COEF_CONST, SINE_RHS, AMC) and
// the cell map is affine, D is the same at every quadrature point of a cell,
// so the local matrix is a 16-term combination of reference matrices:
//   A_ij = |det J| sum_{a,b} D_ab S_ab[i][j],  S_ab[i][j] = sum_q w_q u_ia(q) u_jb(q)
// (S from the element's basis and quadrature rule, computed once on the host).
// That is n_loc^2 x 16 FMA per cell instead of n_q x n_loc^2 x 4, which moves
// the Q2 kernel from FP64-bound to HBM-bound (slot map + entry read-modify-
// write).  The result equals the per-point sum up to rounding order.
// A warp takes P cells at a time; S sits in shared memory ([ab][i*n_loc+j],
// conflict-free across lanes) and each value read serves P cells.
constexpr int ASMC_WARPS = 8, ASMC_P = 2;

template <int E, int NQ>
__global__ void __launch_bounds__(ASMC_WARPS * 32, 2) k_assemble_cc(AsmArgs a, const double *__restrict__ stab) {
  constexpr int NLOC = ET<E>::NLOC, NV = ET<E>::NV, NN = NLOC * NLOC, P = ASMC_P;
  constexpr bool HEX = ET<E>::HEX;
  constexpr int WE = 33 + NQ;  // per-cell scratch: D|det| (16), bh (3), delta, J (9), x0 (3), |det|, w_q |det| f(x_q) (NQ)
  extern __shared__ double sm[];
  double *sS = sm;
  double *sW = sS + 16 * NN;
  for (int k = threadIdx.x; k < 16 * NN; k += blockDim.x) sS[k] = stab[k];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *W = sW + warp * P * WE;
  const bool supg = (a.form == PMG_FORM_SUPG || a.form == PMG_FORM_MASS_SUPG || a.form == PMG_FORM_STIFF_SUPG);

  for (int base = (blockIdx.x * ASMC_WARPS + warp) * P; base < a.n_elems; base += gridDim.x * ASMC_WARPS * P) {
    // cell set-up: lane p handles cell base + p
    if (lane < P && base + lane < a.n_elems) {
      const int e = base + lane;
      const double *cv = a.cell_vert + (size_t)e * NV * 3;
      double J[9], x0[3], Ji[9], K[9], adet;
      cell_map<HEX>(cv, J, x0, Ji, adet, K);
      const double *q0 = a.qtab;
      double c[7];
      coeff_eval(a.coef, x0[0] + J[0] * q0[1] + J[1] * q0[2] + J[2] * q0[3],
                 x0[1] + J[3] * q0[1] + J[4] * q0[2] + J[5] * q0[3], x0[2] + J[6] * q0[1] + J[7] * q0[2] + J[8] * q0[3],
                 c);
      double hconv = supg ? hk_convection(HEX, a.brick != 0, cv, Ji, c[1], c[2], c[3]) : 0.0;
      double delta = supg ? sdfem_delta(hconv, c[0], c[1], c[2], c[3], a.poly, a.delta0) : 0.0;
      double bh[3];
#pragma unroll
      for (int p = 0; p < 3; p++) bh[p] = Ji[p * 3 + 0] * c[1] + Ji[p * 3 + 1] * c[2] + Ji[p * 3 + 2] * c[3];
      double D[16];
      form_matrix(a.form, supg, c, K, bh, delta, D);
      double *w = W + lane * WE;
#pragma unroll
      for (int k = 0; k < 16; k++) w[k] = D[k] * adet;
      w[16] = bh[0]; w[17] = bh[1]; w[18] = bh[2];
      w[19] = supg ? delta : 0.0;
#pragma unroll
      for (int k = 0; k < 9; k++) w[20 + k] = J[k];
      w[29] = x0[0]; w[30] = x0[1]; w[31] = x0[2];
      w[32] = adet;
    }
    __syncwarp();
    // w_q |det J| f(x_q) at every quadrature point of every cell
#pragma unroll
    for (int p = 0; p < P; p++) {
      double *w = W + p * WE;
      const double adet = w[32];
      if (base + p < a.n_elems)
        for (int q = lane; q < NQ; q += 32) {
          const double *qq = a.qtab + q * 4;
          const double X = w[29] + w[20] * qq[1] + w[21] * qq[2] + w[22] * qq[3];
          const double Y = w[30] + w[23] * qq[1] + w[24] * qq[2] + w[25] * qq[3];
          const double Z = w[31] + w[26] * qq[1] + w[27] * qq[2] + w[28] * qq[3];
          double c[7];
          coeff_eval(a.coef, X, Y, Z, c);
          w[33 + q] = qq[0] * adet * c[5];
        }
      __syncwarp();
    }
    double Dr[P][16];
#pragma unroll
    for (int p = 0; p < P; p++)
#pragma unroll
      for (int k = 0; k < 16; k++) Dr[p][k] = W[p * WE + k];
    int bad = 0;
    // MB entries per lane per batch: all slot and entry loads of a batch are
    // issued before any arithmetic, so each lane keeps 2 MB P reads in flight
    constexpr int MB = 4;
    const int ne = min(P, a.n_elems - base);
    for (int m0 = lane; m0 < NN; m0 += 32 * MB) {
      int sl[MB][P];
      double old[MB][P];
#pragma unroll
      for (int b = 0; b < MB; b++) {
        const int m = m0 + 32 * b;
#pragma unroll
        for (int p = 0; p < P; p++) {
          sl[b][p] = -2;  // no entry
          if (m < NN && p < ne) {
            const int e = base + p;
            const int i = m / NLOC;
            const int di = __ldg(a.elem_dof + (size_t)e * NLOC + i);
            const int s = __ldg(a.slot + (size_t)e * NN + m);
            if (di < a.Na) {
              if (s >= 0) sl[b][p] = s;
              else bad = 1;
            } else if (i == m - i * NLOC && s >= 0) {
              sl[b][p] = -3 - s;  // Dirichlet diagonal
            }
          }
        }
      }
#pragma unroll
      for (int b = 0; b < MB; b++)
#pragma unroll
        for (int p = 0; p < P; p++) old[b][p] = sl[b][p] >= 0 ? a.entries[sl[b][p]] : 0.0;
#pragma unroll
      for (int b = 0; b < MB; b++) {
        const int m = m0 + 32 * b;
        if (m >= NN) break;
        double acc[P];
#pragma unroll
        for (int p = 0; p < P; p++) acc[p] = 0.0;
#pragma unroll
        for (int ab = 0; ab < 16; ab++) {
          const double sv = sS[ab * NN + m];
#pragma unroll
          for (int p = 0; p < P; p++) acc[p] += Dr[p][ab] * sv;
        }
#pragma unroll
        for (int p = 0; p < P; p++) {
          const int q = sl[b][p];
          if (q >= 0) a.entries[q] = old[b][p] + acc[p];
          else if (q <= -3) a.entries[-3 - q] = 1.0;  // Dirichlet row: unit diagonal (AssembleMat3D.C:840-848)
        }
      }
    }
    // rhs: f_i = sum_q w_q |det J| f(x_q) (u_i3(q) + delta bh . u_i(q))
    if (a.rhs)
#pragma unroll
      for (int p = 0; p < P; p++) {
        const int e = base + p;
        if (e >= a.n_elems) break;
        const double *w = W + p * WE;
        for (int i = lane; i < NLOC; i += 32) {
          const int di = __ldg(a.elem_dof + (size_t)e * NLOC + i);
          if (di >= a.Na) continue;
          double r = 0.0;
          for (int q = 0; q < NQ; q++) {
            const double *u = a.utab + ((size_t)q * NLOC + i) * 4;
            r += w[33 + q] * (__ldg(u + 3) + w[19] * (w[16] * __ldg(u) + w[17] * __ldg(u + 1) + w[18] * __ldg(u + 2)));
          }
          a.rhs[di] += r;
        }
      }
    if (bad) atomicOr(a.flags, 1);
    __syncwarp();
  }
}

// ----------------------------------------------------------------- slot map
// slot[e][i][j] = position of column dof_j in the sorted CSR row dof_i
// (-1 where the row is a Dirichlet row and j != i, or the pair is missing).
__global__ void k_slot_map(int n_cells, int nloc, int Na, const int *__restrict__ elem_dof,
                           const int *__restrict__ rowptr, const int *__restrict__ kcol, int *__restrict__ slot,
                           int *flags) {
  size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t total = (size_t)n_cells * nloc * nloc;
  if (tid >= total) return;
  int e = (int)(tid / (nloc * nloc));
  int r = (int)(tid % (nloc * nloc));
  int i = r / nloc, j = r % nloc;
  int row = elem_dof[(size_t)e * nloc + i], col = elem_dof[(size_t)e * nloc + j];
  int lo = rowptr[row], hi = rowptr[row + 1] - 1, pos = -1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1, v = kcol[mid];
    if (v == col) { pos = mid; break; }
    if (v < col) lo = mid + 1; else hi = mid - 1;
  }
  if (pos < 0 && row < Na) atomicOr(flags, 2);
  slot[tid] = pos;
}

int build_slot_map(Handle &h, Level &L) {
  size_t total = (size_t)L.n_cells * L.nloc * L.nloc;
  PMG_TRY(L.slot.alloc(total));
  PMG_CUDA(cudaMemsetAsync(h.d_flags.p, 0, sizeof(int) * 4, h.stream));
  int bs = 256;
  size_t nb = (total + bs - 1) / bs;
  k_slot_map<<<(unsigned)nb, bs, 0, h.stream>>>(L.n_cells, L.nloc, L.Na, L.elem_dof.p, L.rowptr.p, L.kcol.p,
                                                   L.slot.p, h.d_flags.p); count_launches(1);
  PMG_CUDA(cudaGetLastError());
  int flags[4];
  PMG_CUDA(cudaMemcpyAsync(flags, h.d_flags.p, sizeof(flags), cudaMemcpyDeviceToHost, h.stream));
  PMG_CUDA(cudaStreamSynchronize(h.stream));
  if (flags[0] & 2) {
    set_error("element coupling missing from the CSR pattern (AssembleMat3D.C:811-816 case)");
    return PMG_ERR_SLOT;
  }
  return PMG_OK;
}

// ----------------------------------------------------------------- tables cache
struct TableCache {
  int elem = -1, rule = -1;
  DBuf<double> utab, qtab;
  DBuf<double> stab;  // 16 x n_loc^2: S_ab[i][j] = sum_q w_q u_ia(q) u_jb(q)
  int nq = 0;
};
static TableCache g_tab[4];

// quadrature rule of the reference (TFEDatabase3D::GetOrig, FEDatabase3D.C:1203-1309):
// degree N_terms * polynomial degree with N_terms = 2 (INTERNAL_PROBLEM_LINEAR) or 3
static int rule_for(int elem, int problem_linear) {
  switch (elem) {
    case PMG_ELEM_Q1_HEX: return problem_linear ? RULE_GAUSS2 : RULE_GAUSS3;
    case PMG_ELEM_Q2_HEX: return problem_linear ? RULE_GAUSS3 : RULE_GAUSS4;
    case PMG_ELEM_P1_TET: return problem_linear ? RULE_KEAST4 : RULE_KEAST11;
    default: return problem_linear ? RULE_KEAST11 : -1;  // P5Tetra (degree 6) is not built
  }
}

static int get_tables(int elem, int rule, TableCache *&out) {
  int slot = elem == PMG_ELEM_Q1_HEX ? 0 : elem == PMG_ELEM_Q2_HEX ? 1 : elem == PMG_ELEM_P1_TET ? 2 : 3;
  TableCache &T = g_tab[slot];
  if (T.elem != elem || T.rule != rule) {
    QuadRule q = make_rule(rule);
    int nl = elem_nloc(elem);
    std::vector<double> u((size_t)q.n * nl * 4), qt((size_t)q.n * 4);
    for (int k = 0; k < q.n; k++) {
      basis_eval(elem, q.x[k], q.y[k], q.z[k], &u[(size_t)k * nl * 4]);
      qt[k * 4] = q.w[k]; qt[k * 4 + 1] = q.x[k]; qt[k * 4 + 2] = q.y[k]; qt[k * 4 + 3] = q.z[k];
    }
    const size_t nn = (size_t)nl * nl;
    std::vector<double> st(16 * nn, 0.0);
    for (int ab = 0; ab < 16; ab++)
      for (int i = 0; i < nl; i++)
        for (int j = 0; j < nl; j++) {
          double acc = 0.0;
          for (int k = 0; k < q.n; k++)
            acc += q.w[k] * u[((size_t)k * nl + i) * 4 + ab / 4] * u[((size_t)k * nl + j) * 4 + ab % 4];
          st[ab * nn + (size_t)i * nl + j] = acc;
        }
    PMG_TRY(T.utab.upload(u.data(), u.size(), 0));
    PMG_TRY(T.qtab.upload(qt.data(), qt.size(), 0));
    PMG_TRY(T.stab.upload(st.data(), st.size(), 0));
    PMG_CUDA(cudaDeviceSynchronize());
    T.elem = elem; T.rule = rule; T.nq = q.n;
  }
  out = &T;
  return PMG_OK;
}

template <int E, int NQ>
static int launch_assemble(Handle &h, Level &L, AsmArgs a) {
  constexpr int NLOC = ET<E>::NLOC, GPW = 32 / NLOC;
  size_t smem = sizeof(double) * ((size_t)NQ * NLOC * 4 + NQ * 4 + (size_t)ASM_WARPS * GPW * NQ * 20);
  static bool attr_set = false;
  if (!attr_set) {
    PMG_CUDA(cudaFuncSetAttribute(k_assemble<E, NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set = true;
  }
  int per_block = ASM_WARPS * GPW;
  const int *ed0 = a.elem_dof;
  const double *cv0 = a.cell_vert;
  const int *sl0 = a.slot;
  for (size_t c = 0; c + 1 < L.ecolor_ptr.size(); c++) {
    int beg = L.ecolor_ptr[c], n = L.ecolor_ptr[c + 1] - beg;
    if (n <= 0) continue;
    AsmArgs b = a;
    b.n_elems = n;
    b.elem_dof = ed0 + (size_t)beg * NLOC;
    b.cell_vert = cv0 + (size_t)beg * ET<E>::NV * 3;
    b.slot = sl0 + (size_t)beg * NLOC * NLOC;
    b.ctab = a.ctab ? a.ctab + (size_t)beg * NQ * 6 : nullptr;
    int blocks = (n + per_block - 1) / per_block;
    int cap = h.num_sms * 8;
    if (blocks > cap) blocks = cap;
    k_assemble<E, NQ><<<blocks, ASM_WARPS * 32, smem, h.stream>>>(b); count_launches(1);
    PMG_CUDA(cudaGetLastError());
  }
  return PMG_OK;
}

template <int E, int NQ>
static int launch_assemble_cc(Handle &h, Level &L, AsmArgs a, const double *stab) {
  constexpr int NLOC = ET<E>::NLOC;
  const size_t smem = sizeof(double) * (16 * (size_t)NLOC * NLOC + (size_t)ASMC_WARPS * ASMC_P * (33 + NQ));
  static bool attr_set = false;
  if (!attr_set) {
    PMG_CUDA(cudaFuncSetAttribute(k_assemble_cc<E, NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    PMG_CUDA(cudaFuncSetAttribute(k_assemble_cc<E, NQ>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    attr_set = true;
  }
  const int per_block = ASMC_WARPS * ASMC_P;
  const int *ed0 = a.elem_dof;
  const double *cv0 = a.cell_vert;
  const int *sl0 = a.slot;
  for (size_t c = 0; c + 1 < L.ecolor_ptr.size(); c++) {
    int beg = L.ecolor_ptr[c], n = L.ecolor_ptr[c + 1] - beg;
    if (n <= 0) continue;
    AsmArgs b = a;
    b.n_elems = n;
    b.elem_dof = ed0 + (size_t)beg * NLOC;
    b.cell_vert = cv0 + (size_t)beg * ET<E>::NV * 3;
    b.slot = sl0 + (size_t)beg * NLOC * NLOC;
    int blocks = std::min((n + per_block - 1) / per_block, h.num_sms * 2);
    k_assemble_cc<E, NQ><<<blocks, ASMC_WARPS * 32, smem, h.stream>>>(b, stab); count_launches(1);
    PMG_CUDA(cudaGetLastError());
  }
  return PMG_OK;
}

// coefficient kinds whose eps, b and c are constant in space
static bool constant_matrix_coefficients(int kind) {
  return kind == PMG_COEF_CONST || kind == PMG_COEF_SINE_RHS || kind == PMG_COEF_AMC;
}

// Assemble one level into `target` (A or M) and rhs_target (may be NULL).
int assemble_level(Handle &h, Level &L, int form, double *target, bool zero_rhs, double *rhs_target) {
  if (!L.has_mesh || !L.has_csr) {
    set_error("assemble: level needs pmg_set_level_mesh and pmg_set_level_csr first");
    return PMG_ERR_STATE;
  }
  if (form < PMG_FORM_GALERKIN || form > PMG_FORM_STIFF_SUPG) {
    set_error("assemble: unknown form");
    return PMG_ERR_ARG;
  }
  if ((form == PMG_FORM_SUPG || form == PMG_FORM_MASS_SUPG || form == PMG_FORM_STIFF_SUPG) &&
      h.prm.sdfem_type != 2) {
    set_error("assemble: only SDFEM_TYPE 2 is built");
    return PMG_ERR_UNSUPPORTED;
  }
  if (!L.slot.p) PMG_TRY(build_slot_map(h, L));
  TableCache *T = nullptr;
  const int rule = rule_for(L.elem, h.prm.problem_linear);
  if (rule < 0) {
    set_error("assemble: the degree-6 tetrahedral rule (P2 with INTERNAL_PROBLEM_LINEAR = 0) is not built");
    return PMG_ERR_UNSUPPORTED;
  }
  PMG_TRY(get_tables(L.elem, rule, T));
  if (h.coeff.kind == PMG_COEF_TABLE && (!L.ctab.p || L.ctab_nq != T->nq)) {
    set_error("assemble: PMG_COEF_TABLE needs pmg_set_coefficient_table for this level and quadrature rule");
    return PMG_ERR_STATE;
  }
  PMG_CUDA(cudaMemsetAsync(target, 0, sizeof(double) * L.nnz, h.stream));
  if (rhs_target && zero_rhs) PMG_CUDA(cudaMemsetAsync(rhs_target, 0, sizeof(double) * L.N, h.stream));
  PMG_CUDA(cudaMemsetAsync(h.d_flags.p, 0, sizeof(int) * 4, h.stream));
  AsmArgs a{};
  a.elem_dof = L.elem_dof.p;
  a.cell_vert = L.cell_vert.p;
  a.slot = L.slot.p;
  a.Na = L.Na;
  a.entries = target;
  a.rhs = rhs_target;
  a.form = form;
  a.poly = h.prm.poly_degree > 0 ? h.prm.poly_degree : (L.elem == PMG_ELEM_Q2_HEX || L.elem == PMG_ELEM_P2_TET ? 2 : 1);
  a.brick = L.brick;
  a.delta0 = h.prm.delta0;
  a.coef.kind = h.coeff.kind;
  a.coef.eps = h.coeff.eps;
  for (int k = 0; k < 3; k++) a.coef.b[k] = h.coeff.b[k];
  a.coef.c = h.coeff.c;
  a.coef.f = h.coeff.f;
  a.coef.t = h.coeff.t;
  a.coef.n_modes = h.coeff.n_modes;
  a.coef.modes = h.d_modes.p;
  a.ctab = h.coeff.kind == PMG_COEF_TABLE ? L.ctab.p : nullptr;
  a.utab = T->utab.p;
  a.qtab = T->qtab.p;
  a.flags = h.d_flags.p;
  if (constant_matrix_coefficients(h.coeff.kind) && h.prm.assembly_kernel != 1) {
    const double *st = T->stab.p;
    switch (L.elem * 1000 + T->nq) {
      case PMG_ELEM_Q1_HEX * 1000 + 8: return launch_assemble_cc<PMG_ELEM_Q1_HEX, 8>(h, L, a, st);
      case PMG_ELEM_Q1_HEX * 1000 + 27: return launch_assemble_cc<PMG_ELEM_Q1_HEX, 27>(h, L, a, st);
      case PMG_ELEM_Q2_HEX * 1000 + 27: return launch_assemble_cc<PMG_ELEM_Q2_HEX, 27>(h, L, a, st);
      case PMG_ELEM_Q2_HEX * 1000 + 64: return launch_assemble_cc<PMG_ELEM_Q2_HEX, 64>(h, L, a, st);
      case PMG_ELEM_P1_TET * 1000 + 4: return launch_assemble_cc<PMG_ELEM_P1_TET, 4>(h, L, a, st);
      case PMG_ELEM_P1_TET * 1000 + 11: return launch_assemble_cc<PMG_ELEM_P1_TET, 11>(h, L, a, st);
      case PMG_ELEM_P2_TET * 1000 + 11: return launch_assemble_cc<PMG_ELEM_P2_TET, 11>(h, L, a, st);
      default: break;
    }
  }
  switch (L.elem * 1000 + T->nq) {
    case PMG_ELEM_Q1_HEX * 1000 + 8: PMG_TRY((launch_assemble<PMG_ELEM_Q1_HEX, 8>(h, L, a))); break;
    case PMG_ELEM_Q1_HEX * 1000 + 27: PMG_TRY((launch_assemble<PMG_ELEM_Q1_HEX, 27>(h, L, a))); break;
    case PMG_ELEM_Q2_HEX * 1000 + 27: PMG_TRY((launch_assemble<PMG_ELEM_Q2_HEX, 27>(h, L, a))); break;
    case PMG_ELEM_Q2_HEX * 1000 + 64: PMG_TRY((launch_assemble<PMG_ELEM_Q2_HEX, 64>(h, L, a))); break;
    case PMG_ELEM_P1_TET * 1000 + 4: PMG_TRY((launch_assemble<PMG_ELEM_P1_TET, 4>(h, L, a))); break;
    case PMG_ELEM_P1_TET * 1000 + 11: PMG_TRY((launch_assemble<PMG_ELEM_P1_TET, 11>(h, L, a))); break;
    case PMG_ELEM_P2_TET * 1000 + 11: PMG_TRY((launch_assemble<PMG_ELEM_P2_TET, 11>(h, L, a))); break;
    default: set_error("assemble: no kernel for this element / quadrature rule"); return PMG_ERR_UNSUPPORTED;
  }
  return PMG_OK;
}

// rhs of Dirichlet rows = nodal boundary values (AssembleMat3D.C:1031-1081)
__global__ void k_dirichlet_rhs(int Na, int N, const double *__restrict__ dv, double *__restrict__ rhs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + Na;
  if (i < N) rhs[i] = dv ? dv[i - Na] : 0.0;
}

int set_dirichlet_rows(Handle &h, Level &L, double *target, double *rhs_target) {
  (void)target;
  int n = L.N - L.Na;
  if (n > 0 && rhs_target) {
    k_dirichlet_rhs<<<(n + 255) / 256, 256, 0, h.stream>>>(L.Na, L.N, L.dirval.p, rhs_target); count_launches(1);
    PMG_CUDA(cudaGetLastError());
  }
  return PMG_OK;
}

}  // namespace pmg

using namespace pmg;

// quadrature points of one level in the caller's cell order, mapped like the
// kernel maps them (HexaAffin: vertices 0, 1, 3, 4; TetraAffin: 0, 1, 2, 3)
extern "C" int pmg_quad_points(pmg_handle hh, int level, int *nq, double *xyz) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || level < 0 || level >= (int)h->lv.size() || !nq) {
    set_error("pmg_quad_points: bad arguments");
    return PMG_ERR_ARG;
  }
  Level &L = h->lv[level];
  if (!L.has_mesh) {
    set_error("pmg_quad_points: call pmg_set_level_mesh first");
    return PMG_ERR_STATE;
  }
  const int rule = rule_for(L.elem, h->prm.problem_linear);
  if (rule < 0) {
    set_error("pmg_quad_points: the degree-6 tetrahedral rule is not built");
    return PMG_ERR_UNSUPPORTED;
  }
  QuadRule q = make_rule(rule);
  *nq = q.n;
  if (!xyz) return PMG_OK;
  const int nv = L.nvert;
  std::vector<double> cv((size_t)L.n_cells * nv * 3);
  PMG_CUDA(cudaMemcpyAsync(cv.data(), L.cell_vert.p, sizeof(double) * cv.size(), cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  const bool hex = nv == 8;
  for (int k = 0; k < L.n_cells; k++) {
    const double *v = &cv[(size_t)k * nv * 3];
    double J[9], x0[3];
    for (int d = 0; d < 3; d++) {
      if (hex) {
        J[d * 3 + 0] = (v[3 + d] - v[d]) * 0.5;
        J[d * 3 + 1] = (v[9 + d] - v[d]) * 0.5;
        J[d * 3 + 2] = (v[12 + d] - v[d]) * 0.5;
        x0[d] = (v[3 + d] + v[9 + d] + v[12 + d] - v[d]) * 0.5;
      } else {
        J[d * 3 + 0] = v[3 + d] - v[d];
        J[d * 3 + 1] = v[6 + d] - v[d];
        J[d * 3 + 2] = v[9 + d] - v[d];
        x0[d] = v[d];
      }
    }
    double *o = xyz + (size_t)L.cell_order[k] * q.n * 3;
    for (int p = 0; p < q.n; p++)
      for (int d = 0; d < 3; d++)
        o[p * 3 + d] = x0[d] + J[d * 3 + 0] * q.x[p] + J[d * 3 + 1] * q.y[p] + J[d * 3 + 2] * q.z[p];
  }
  return PMG_OK;
}

extern "C" int pmg_set_coefficient_table(pmg_handle hh, int level, const double *values) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || level < 0 || level >= (int)h->lv.size() || !values) {
    set_error("pmg_set_coefficient_table: bad arguments");
    return PMG_ERR_ARG;
  }
  Level &L = h->lv[level];
  int nq = 0;
  PMG_TRY(pmg_quad_points(hh, level, &nq, nullptr));
  const size_t per = (size_t)nq * 6;
  std::vector<double> t((size_t)L.n_cells * per);
  for (int k = 0; k < L.n_cells; k++) {
    const double *src = values + (size_t)L.cell_order[k] * per;
    for (size_t j = 0; j < per; j++)
      if (!std::isfinite(src[j])) {
        set_error("pmg_set_coefficient_table: non-finite value");
        return PMG_ERR_NONFINITE;
      }
    std::copy(src, src + per, &t[(size_t)k * per]);
  }
  PMG_TRY(L.ctab.upload(t.data(), t.size(), h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  L.ctab_nq = nq;
  return PMG_OK;
}
