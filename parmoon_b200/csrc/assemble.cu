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
//     turns the scatter into plain loads/stores;
//   * or, the row gather: the local matrices of all cells in one launch, then
//     one pass over the CSR rows, each summed from its cells' local rows in
//     colour order (the scatter's order: the same bits) and written once.
#include "pmg_internal.h"
#include "fe_tables.h"
#include <cstdio>
#include <functional>
#include <cstdlib>

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
      // cos(2 pi k.x + phi) as cospi(2 k.x + phi / pi): the reduction of an
      // argument in units of pi is exact, so no general range reduction.
      // Four partial sums keep four independent cospi chains in flight (the
      // FP64 pipe is latency-bound with one); g = (g0 + g1) + (g2 + g3).
      double g0 = 0, g1 = 0, g2 = 0, g3 = 0;
      auto term = [&](int m) {
        const double *M = C.modes + 8 * m;
        return M[3] * cospi(2.0 * (M[0] * x + M[1] * y + M[2] * z) + M[4] * (1.0 / PI));
      };
      int m = 0;
      for (; m + 4 <= C.n_modes; m += 4) {
        g0 += term(m);
        g1 += term(m + 1);
        g2 += term(m + 2);
        g3 += term(m + 3);
      }
      for (; m < C.n_modes; m++) g0 += term(m);
      c[0] = C.eps * exp((g0 + g1) + (g2 + g3));
      break;
    }
    case PMG_COEF_CURL_FOURIER: {
      double bx = 0, by = 0, bz = 0;
      for (int m = 0; m < C.n_modes; m++) {
        const double *M = C.modes + 8 * m;
        double s = -M[3] * sinpi(2.0 * (M[0] * x + M[1] * y + M[2] * z) + M[4] * (1.0 / PI)) * 2 * PI;
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
template <> struct ET<PMG_ELEM_NQ1_HEX> { static constexpr int NLOC = 6, NV = 8; static constexpr bool HEX = true; };
template <> struct ET<PMG_ELEM_P1_TET> { static constexpr int NLOC = 4, NV = 4; static constexpr bool HEX = false; };
template <> struct ET<PMG_ELEM_P2_TET> { static constexpr int NLOC = 10, NV = 4; static constexpr bool HEX = false; };

constexpr int ASM_WARPS = 8;

// Add v into the entry of slot s (>= 0) as an L2 reduction: no value comes
// back, so the scatter carries no load latency.  The cells of one launch share
// no row, so no two adds of a launch meet, and the order of the adds into an
// entry is the colour order, the same on every run.  (Storing instead of
// adding at an entry's first touch, to drop the zeroing, was measured slower:
// 8-byte stores into sectors not in L2 cost more than the zeroing.)
__device__ __forceinline__ void scatter_entry(double *entries, int s, double v) { atomicAdd(entries + s, v); }

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
  int item_chunk;  // k_assemble_tc16: consecutive work items per warp
  // local-matrix mode (row gather): the kernels store each cell's local
  // matrix (ae, n x NLOC^2, row i of the test function, column j) and local
  // rhs (rloc, n x NLOC) instead of adding them into the matrix
  double *ae, *rloc;
  int add_rhs;  // row gather: add the rhs to the existing values instead of storing it
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

  const int nw = blockDim.x >> 5;  // ASM_WARPS, or fewer when the per-element scratch is large
  for (int base = (blockIdx.x * nw + warp) * GPW; base < a.n_elems; base += gridDim.x * nw * GPW) {
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
      if (a.ae) {  // local-matrix mode
#pragma unroll
        for (int i = 0; i < NLOC; i++) a.ae[(size_t)e * NLOC * NLOC + i * NLOC + t] = acc[i];
        a.rloc[(size_t)e * NLOC + t] = racc;
      } else {
        // scatter through the slot map (no two elements of a colour share a row)
        const int *dof = a.elem_dof + (size_t)e * NLOC;
        const int *sl = a.slot + (size_t)e * NLOC * NLOC;
#pragma unroll
        for (int i = 0; i < NLOC; i++) {
          const int s = __ldg(sl + i * NLOC + t);
          if (s >= 0) scatter_entry(a.entries, s, acc[i]);
          else if (s <= -3) a.entries[-3 - s] = 1.0;  // Dirichlet row: unit diagonal (AssembleMat3D.C:840-848)
        }
        if (a.rhs) {
          const int dt = __ldg(dof + t);
          if (dt < a.Na) a.rhs[dt] += racc;
        }
      }
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
          sl[b][p] = (m < NN && p < ne) ? __ldg(a.slot + (size_t)(base + p) * NN + m) : -1;
        }
      }
#pragma unroll
      for (int b = 0; b < MB; b++)
#pragma unroll
        for (int p = 0; p < P; p++)
          old[b][p] = sl[b][p] >= 0 ? a.entries[sl[b][p]] : 0.0;
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
    __syncwarp();
  }
}

// ------------------------------------------- tensor-core contraction kernel
// The local matrix as a product of a fixed reference table and per-cell
// coefficients, on the FP64 tensor cores (mma.sync.m8n8k4 .f64, DMMA):
//   A_cell[m] = sum_k T[m][k] d_cell[k],   m = i * n_loc + j
// CONST (eps, b, c constant in space, affine cells; the form of
//   BilinearAssemble / _SD, ConvDiff3D.C:87-214, and the TCD forms):
//   k = ab (16), d = |det J| D_ab (D as form_matrix), T[m][ab] = S_ab[i][j]
//   = sum_q w_q u_ia(q) u_jb(q), the reference-element integrals.
// DIFF (pure diffusion, eps varying in space: b = 0, c = 0): k = (q, p) with p
//   over the 6 entries of the symmetric K = Ji Ji^T, d = w_q |det J| eps(x_q) K_p,
//   T[m][(q,p)] = u_ia u_ja (p = aa) or u_ia u_jb + u_ib u_ja (p = ab, a < b).
// d is computed per cell beforehand (k_tc_setup, k_tc_setup_diff).  A warp
// takes 8 cells.  Per 8 x 8 output block (8 entries x 8 cells) the mma chain
// runs over the k steps of 4: the A operand (8 entries x 4 k) comes from T in
// shared memory, stored per (entry block, k step) as the 32 lane values of the
// fragment; the B operand (4 k x 8 cells) from the cells' d.  Lane l ends with
// entries m = 8t + l/4 of cells 2(l%4), 2(l%4)+1 and adds them into the CSR
// through the slot map with L2 reductions (cells of one colour share no row,
// so no two adds of a launch meet).  Slot loads of the next batch go out
// before the current batch's mma chains.  The sums equal the per-point ones
// up to rounding order.

__device__ __forceinline__ void dmma_8x8x4(double &c0, double &c1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

// --- space-constant coefficients: per-cell set-up, then the contraction ----
// k_tc_setup (one thread per cell, all cells of the level in one launch):
// d_e = |det J| D_ab (16 values) and the cell's local rhs
//   r_i = sum_q w_q |det J| f(x_q) (u_i3(q) + delta bh . u_i(q))
// into per-cell buffers.  k_assemble_tc16 (per colour) then only contracts and
// scatters: per 8 cells a warp loads its B fragments straight from d (8 cells
// x 4 consecutive k per load), runs the 4-step mma chain per 8-entry block, and
// adds the local rhs of its cells.  Shared memory holds the table alone
// (94 KB for Q2).
template <int E, int NQ>
__global__ void __launch_bounds__(128) k_tc_setup(AsmArgs a, double *__restrict__ dbuf, double *__restrict__ rbuf,
                                                  const double *__restrict__ rtab) {
  constexpr int NLOC = ET<E>::NLOC, NV = ET<E>::NV;
  constexpr bool HEX = ET<E>::HEX;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.n_elems) return;
  const bool supg = a.form == PMG_FORM_SUPG || a.form == PMG_FORM_MASS_SUPG || a.form == PMG_FORM_STIFF_SUPG;
  const double *cv = a.cell_vert + (size_t)e * NV * 3;
  double J[9], x0[3], Ji[9], K[9], adet;
  cell_map<HEX>(cv, J, x0, Ji, adet, K);
  const double *q0 = a.qtab;
  double c[7];
  coeff_eval(a.coef, x0[0] + J[0] * q0[1] + J[1] * q0[2] + J[2] * q0[3], x0[1] + J[3] * q0[1] + J[4] * q0[2] + J[5] * q0[3],
             x0[2] + J[6] * q0[1] + J[7] * q0[2] + J[8] * q0[3], c);
  const double hconv = supg ? hk_convection(HEX, a.brick != 0, cv, Ji, c[1], c[2], c[3]) : 0.0;
  const double delta = supg ? sdfem_delta(hconv, c[0], c[1], c[2], c[3], a.poly, a.delta0) : 0.0;
  double bh[3];
#pragma unroll
  for (int p = 0; p < 3; p++) bh[p] = Ji[p * 3 + 0] * c[1] + Ji[p * 3 + 1] * c[2] + Ji[p * 3 + 2] * c[3];
  double D[16];
  form_matrix(a.form, supg, c, K, bh, delta, D);
  double *d = dbuf + (size_t)e * 16;
#pragma unroll
  for (int k = 0; k < 16; k++) d[k] = D[k] * adet;
  if (!rbuf) return;
  double *r = rbuf + (size_t)e * NLOC;
  if (a.coef.kind == PMG_COEF_CONST) {
    // f constant: r_i = |det J| f (R_3[i] + delta bh . R[i]), R_a[i] = sum_q w_q u_ia(q)
    const double af = adet * c[5];
    for (int i = 0; i < NLOC; i++)
      r[i] = af * (__ldg(rtab + 3 * NLOC + i) +
                   delta * (bh[0] * __ldg(rtab + i) + bh[1] * __ldg(rtab + NLOC + i) + bh[2] * __ldg(rtab + 2 * NLOC + i)));
    return;
  }
  double fw[NQ];
  for (int q = 0; q < NQ; q++) {
    const double *qq = a.qtab + q * 4;
    double cq[7];
    coeff_eval(a.coef, x0[0] + J[0] * qq[1] + J[1] * qq[2] + J[2] * qq[3], x0[1] + J[3] * qq[1] + J[4] * qq[2] + J[5] * qq[3],
               x0[2] + J[6] * qq[1] + J[7] * qq[2] + J[8] * qq[3], cq);
    fw[q] = qq[0] * adet * cq[5];
  }
  for (int i = 0; i < NLOC; i++) {
    double acc = 0.0;
    for (int q = 0; q < NQ; q++) {
      const double *u = a.utab + ((size_t)q * NLOC + i) * 4;
      acc += fw[q] * (__ldg(u + 3) + delta * (bh[0] * __ldg(u) + bh[1] * __ldg(u + 1) + bh[2] * __ldg(u + 2)));
    }
    r[i] = acc;
  }
}

// Pure diffusion with a coefficient eps(x) (b = 0, c = 0): one thread per
// quadrature point (a block holds CB = 128 / NQ whole cells) evaluates eps and
// f there (the Fourier modes of the field read through the cache) and stores
// d[(q, p)] = w_q |det J| eps(x_q) K_p (K = Ji Ji^T, p over 00 11 22 01 02 12,
// zero-padded to 4 KS); then the block's threads form the cells' local rhs
// r_i = sum_q w_q |det J| f(x_q) u_i(q) from the point weights in shared
// memory.  k_assemble_tc16<E, KS> contracts d with the per-point table on DMMA.
// A thread per point keeps one point's mode chain per thread: the coarse
// levels' few cells finish in one chain of n_modes terms instead of NQ.
template <int E, int NQ>
__global__ void __launch_bounds__(128) k_tc_setup_diff(AsmArgs a, double *__restrict__ dbuf, double *__restrict__ rbuf) {
  constexpr int NLOC = ET<E>::NLOC, NV = ET<E>::NV, KD = 6 * NQ, KP = 4 * ((KD + 3) / 4), CB = 128 / NQ;
  constexpr bool HEX = ET<E>::HEX;
  __shared__ double sfw[CB * NQ];
  const int e0 = blockIdx.x * CB, t = threadIdx.x;
  const int lc = t / NQ, q = t - lc * NQ, e = e0 + lc;
  if (t < CB * NQ && e < a.n_elems) {
    const double *cv = a.cell_vert + (size_t)e * NV * 3;
    double J[9], x0[3], Ji[9], K[9], adet;
    cell_map<HEX>(cv, J, x0, Ji, adet, K);
    const double Kp[6] = {K[0], K[4], K[8], K[1], K[2], K[5]};
    double *d = dbuf + (size_t)e * KP;
    const double *qq = a.qtab + q * 4;
    double cf[7];
    coeff_eval(a.coef, x0[0] + J[0] * qq[1] + J[1] * qq[2] + J[2] * qq[3], x0[1] + J[3] * qq[1] + J[4] * qq[2] + J[5] * qq[3],
               x0[2] + J[6] * qq[1] + J[7] * qq[2] + J[8] * qq[3], cf);
    const double w = qq[0] * adet, ew = w * cf[0];
    sfw[t] = w * cf[5];
#pragma unroll
    for (int p = 0; p < 6; p++) d[q * 6 + p] = ew * Kp[p];
    if (q == 0)
      for (int k = KD; k < KP; k++) d[k] = 0.0;
  }
  if (!rbuf) return;
  __syncthreads();
  const int nc = min(CB, a.n_elems - e0);
  for (int idx = t; idx < nc * NLOC; idx += blockDim.x) {
    const int c = idx / NLOC, i = idx - c * NLOC;
    double acc = 0.0;
#pragma unroll
    for (int p = 0; p < NQ; p++) acc += sfw[c * NQ + p] * __ldg(a.utab + ((size_t)p * NLOC + i) * 4 + 3);
    rbuf[(size_t)e0 * NLOC + idx] = acc;
  }
}

// Work items are (group of 8 cells, batch of MB = 8 entry blocks), NB = MT / MB
// items per group; warp gw takes items [gw per, (gw + 1) per) with per at most
// NB, so a coarse level's short launch spreads one group's batches over
// several warps (a chain of ~3 items instead of NB).  The slot loads (and, for
// KS = 4, the B fragments) of a warp's next item are in flight while the
// current one contracts and scatters; one 512-thread block per SM, up to 128
// registers.  The cells of one launch share no row, so every slot is hit
// at most once per launch whatever warp handles it: the result is the same
// for any item order.
// KS k-steps of 4: KS = 4 for space-constant coefficients (d = the 16
// coefficients of D), KS = ceil(6 NQ / 4) for pure diffusion (d = the 6
// entries of w_q |det J| eps(x_q) K per quadrature point, zero-padded)
template <int E, int KS>
__global__ void __launch_bounds__(512, 1) k_assemble_tc16(AsmArgs a, const double *__restrict__ tfrag,
                                                          const double *__restrict__ dbuf,
                                                          const double *__restrict__ rbuf) {
  constexpr int NLOC = ET<E>::NLOC, NN = NLOC * NLOC, MT = (NN + 7) / 8, MB = 8, NB = (MT + MB - 1) / MB, KP = 4 * KS;
  // B fragments d[cell row][4 s + lane % 4]: held in registers for KS = 4,
  // re-read through L1 per entry block for the longer diffusion rows
  constexpr bool REG = KS <= 4;
  constexpr int NBF = REG ? KS : 1;
  extern __shared__ double sT[];
  for (int k = threadIdx.x; k < MT * KS * 32; k += blockDim.x) sT[k] = tfrag[k];
  __syncthreads();
  const int lane = threadIdx.x & 31, row = lane >> 2, c0 = 2 * (lane & 3);
  const int n_items = ((a.n_elems + 7) >> 3) * NB, per = a.item_chunk;  // items [gw per, (gw + 1) per)
  const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int item_end = min(n_items, (gw + 1) * per);
  auto load = [&](int it, int (&sl)[MB][2], double (&bf)[NBF]) {
    const int base = (it / NB) * 8, t0 = (it % NB) * MB, ne = min(8, a.n_elems - base);
#pragma unroll
    for (int b = 0; b < MB; b++) {
      const int m = 8 * (t0 + b) + row;
#pragma unroll
      for (int u = 0; u < 2; u++)
        sl[b][u] = (!a.ae && t0 + b < MT && m < NN && c0 + u < ne) ? __ldg(a.slot + (size_t)(base + c0 + u) * NN + m)
                                                                     : -1;
    }
    if (REG) {
      const double *drow = dbuf + (size_t)(base + (row < ne ? row : 0)) * KP + (lane & 3);
#pragma unroll
      for (int s = 0; s < NBF; s++) bf[s] = row < ne ? __ldg(drow + 4 * s) : 0.0;
    }
  };
  int slc[MB][2], sln[MB][2];
  double bfc[NBF], bfn[NBF];
  int item = gw * per;
  if (item < item_end) load(item, slc, bfc);
  for (; item < item_end; item++) {
    if (item + 1 < item_end) load(item + 1, sln, bfn);
    const int base = (item / NB) * 8, t0 = (item % NB) * MB, ne = min(8, a.n_elems - base);
    const double *drow = dbuf + (size_t)(base + (row < ne ? row : 0)) * KP + (lane & 3);
    double acc[MB][2];
#pragma unroll
    for (int b = 0; b < MB; b++) {
      acc[b][0] = 0.0;
      acc[b][1] = 0.0;
      if (t0 + b < MT) {
        const double *tb = sT + (size_t)(t0 + b) * KS * 32 + lane;
#pragma unroll
        for (int s = 0; s < KS; s++)
          dmma_8x8x4(acc[b][0], acc[b][1], tb[s * 32], REG ? bfc[REG ? s : 0] : (row < ne ? __ldg(drow + 4 * s) : 0.0));
      }
    }
    if (a.ae) {
      // local-matrix mode: entry m = 8 (t0 + b) + row of cells base + c0 + u
#pragma unroll
      for (int b = 0; b < MB; b++) {
        const int m = 8 * (t0 + b) + row;
#pragma unroll
        for (int u = 0; u < 2; u++)
          if (t0 + b < MT && m < NN && c0 + u < ne) a.ae[(size_t)(base + c0 + u) * NN + m] = acc[b][u];
      }
    } else {
      // L2 reductions (no value returned)
#pragma unroll
      for (int b = 0; b < MB; b++)
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const int q = slc[b][u];
          if (q >= 0) scatter_entry(a.entries, q, acc[b][u]);
          else if (q <= -3) a.entries[-3 - q] = 1.0;  // Dirichlet row: unit diagonal (AssembleMat3D.C:840-848)
        }
    }
    // the cells' local rhs (active rows), once per group
    if (a.rhs && !a.ae && t0 == 0)
      for (int ci = lane; ci < ne * NLOC; ci += 32) {
        const int di = __ldg(a.elem_dof + (size_t)base * NLOC + ci);
        if (di < a.Na) atomicAdd(a.rhs + di, __ldg(rbuf + (size_t)base * NLOC + ci));
      }
#pragma unroll
    for (int b = 0; b < MB; b++) {
      slc[b][0] = sln[b][0];
      slc[b][1] = sln[b][1];
    }
#pragma unroll
    for (int s = 0; s < NBF; s++) bfc[s] = bfn[s];
  }
}

// ----------------------------------------------------------------- slot map
// slot[e][i][j] = position of column dof_j in the sorted CSR row dof_i when
// dof_i is an active row; for a Dirichlet row -3 - (position of the diagonal)
// when j = i (the kernels set that entry to 1) and -1 otherwise.  A coupling
// of an active row missing from the pattern fails the build (flag 2), so the
// kernels need neither the dofs nor a check to scatter.
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
  if (row >= Na) pos = (col == row && pos >= 0) ? -3 - pos : -1;
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

// ----------------------------------------------------------------- row gather
// Incidence of the row gather: for each dof the flat indices e * nloc + li of
// the cells holding it (li = its local index there), sorted, so in cell order;
// the cells are stored colour by colour, so this is the colour order in which
// the scatter adds them.
__global__ void k_inc_count(size_t total, const int *__restrict__ ed, int *__restrict__ cnt) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < total) atomicAdd(cnt + ed[k], 1);
}
__global__ void k_inc_fill(size_t total, const int *__restrict__ ed, int *__restrict__ cursor, int *__restrict__ inc) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < total) inc[atomicAdd(cursor + ed[k], 1)] = (int)k;
}
// insertion sort of each dof's list (a few to a few dozen cells)
__global__ void k_inc_sort(int N, const int *__restrict__ ptr, int *__restrict__ inc) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  const int b = ptr[r], e = ptr[r + 1];
  for (int i = b + 1; i < e; i++) {
    const int v = inc[i];
    int j = i - 1;
    while (j >= b && inc[j] > v) {
      inc[j + 1] = inc[j];
      j--;
    }
    inc[j + 1] = v;
  }
}

__global__ void k_slot_gather_order(size_t total, int nloc, const int *__restrict__ inc, const int *__restrict__ slot,
                                    int *__restrict__ slot_g) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= total) return;
  const size_t p = k / nloc, j = k - p * nloc;
  slot_g[k] = slot[(size_t)inc[p] * nloc + j];
}

int build_row_gather(Handle &h, Level &L) {
  const size_t total = (size_t)L.n_cells * L.nloc;
  if (total >= (size_t)INT32_MAX) {
    set_error("assemble: too many cell-dof pairs for the row gather");
    return PMG_ERR_UNSUPPORTED;
  }
  DBuf<int> cnt, cursor;
  PMG_TRY(cnt.alloc(L.N));
  PMG_TRY(cursor.alloc(L.N + 1));
  PMG_TRY(L.inc_ptr.alloc(L.N + 1));
  PMG_TRY(L.inc.alloc(total));
  PMG_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * L.N, h.stream));
  const unsigned nb = (unsigned)((total + 255) / 256);
  k_inc_count<<<nb, 256, 0, h.stream>>>(total, L.elem_dof.p, cnt.p); count_launches(1);
  PMG_CUDA(cudaGetLastError());
  PMG_TRY(scan_exclusive(h.stream, L.N, cnt.p, L.inc_ptr.p));
  PMG_CUDA(cudaMemcpyAsync(cursor.p, L.inc_ptr.p, sizeof(int) * (L.N + 1), cudaMemcpyDeviceToDevice, h.stream));
  k_inc_fill<<<nb, 256, 0, h.stream>>>(total, L.elem_dof.p, cursor.p, L.inc.p); count_launches(1);
  k_inc_sort<<<(L.N + 255) / 256, 256, 0, h.stream>>>(L.N, L.inc_ptr.p, L.inc.p); count_launches(1);
  PMG_CUDA(cudaGetLastError());
  PMG_TRY(L.slot_g.alloc(total * L.nloc));
  const size_t tg = total * L.nloc;
  k_slot_gather_order<<<(unsigned)((tg + 255) / 256), 256, 0, h.stream>>>(tg, L.nloc, L.inc.p, L.slot.p, L.slot_g.p);
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  int rmax = 0;
  for (size_t r = 0; r + 1 < L.h_rowptr.size(); r++) rmax = std::max(rmax, L.h_rowptr[r + 1] - L.h_rowptr[r]);
  L.rmax = rmax;
  PMG_CUDA(cudaStreamSynchronize(h.stream));  // cnt and cursor are freed on return
  return PMG_OK;
}

// Row gather (local-matrix mode, second pass): a group of NLOC lanes builds
// CSR row r in shared memory from row li of the local matrix of every cell
// holding r, in cell order: entry += value at the slot map's position
// (Dirichlet row: the diagonal set to 1, AssembleMat3D.C:840-848), then writes
// the row and the active row's rhs once.  Every entry is a sum from zero over
// the cells in colour order, the order of the colour-by-colour scatter, so the
// two agree bitwise; the matrix needs no zeroing and no entry is read back.
// The slot map is kept a second time in list order (slot_g), so a row's
// slots are one contiguous run; the local rows stay in cell order (the first
// pass writes them in order; storing them in list order instead made that
// pass scatter and was measured slower: Q2 64^3 finest level 2.57 against
// 2.06 ms, P2 lognormal 4.72 against 4.45 ms).
// The values of a chunk of CH cells are loaded together (one latency per
// chunk), then added in order with the group in step.
template <int NLOC>
__global__ void __launch_bounds__(256, (NLOC == 8 || NLOC == 10) ? 3 : 4) k_gather_rows(int N, int Na, int rmax, const int *__restrict__ rowptr,
                                                        const int *__restrict__ inc_ptr, const int *__restrict__ inc,
                                                        const double *__restrict__ ae, const int *__restrict__ slot,
                                                        const double *__restrict__ rloc, double *__restrict__ entries,
                                                        double *__restrict__ rhs, int add_rhs) {
  constexpr int GPW = 32 / NLOC, CH = NLOC < 8 ? NLOC : 8;
  extern __shared__ double srow[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int grp = lane / NLOC, t = lane - grp * NLOC;
  const bool used = grp < GPW;
  const int src = (used ? grp : 0) * NLOC;  // lane 0 of the group
  double *buf = srow + ((size_t)warp * GPW + (used ? grp : 0)) * rmax;
  const int stride = gridDim.x * nw * GPW;
  // a row's pointers and its first CH cells: loaded one row ahead, so a row
  // waits for one round trip (its cells' local rows and slots)
  struct Meta { int rp, len, c0, nc, fl; };
  auto meta = [&](int r, Meta &m) {
    m.rp = m.len = m.c0 = m.nc = m.fl = 0;
    if (used && r < N) {
      m.rp = __ldg(rowptr + r);
      m.len = __ldg(rowptr + r + 1) - m.rp;
      m.c0 = __ldg(inc_ptr + r);
      m.nc = __ldg(inc_ptr + r + 1) - m.c0;
      if (t < CH && t < m.nc) m.fl = __ldg(inc + m.c0 + t);
    }
  };
  int r0 = (blockIdx.x * nw + warp) * GPW;
  Meta cur, nxt;
  meta(r0 + grp, cur);
  for (; r0 < N; r0 += stride) {
    meta(r0 + stride + grp, nxt);
    const int r = r0 + grp;
    const bool valid = used && r < N;
    for (int k = t; k < cur.len; k += NLOC) buf[k] = 0.0;
    int ncmax = cur.nc;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ncmax = max(ncmax, __shfl_xor_sync(0xffffffffu, ncmax, o));
    double racc = 0.0;
    for (int k0 = 0; k0 < ncmax; k0 += CH) {
      const int fl = k0 == 0 ? cur.fl : ((valid && t < CH && k0 + t < cur.nc) ? __ldg(inc + cur.c0 + k0 + t) : 0);
      // lane t < CH of the group also loads the local rhs of cell k0 + t
      const double rl = (valid && rloc && t < CH && k0 + t < cur.nc) ? __ldcs(rloc + fl) : 0.0;
      // local row li of cell e (list entry f = e NLOC + li) and its slots,
      // stored contiguously in list order (positions c0 + k)
      double v[CH];
      int sl[CH];
#pragma unroll
      for (int j = 0; j < CH; j++) {
        const bool on = valid && k0 + j < cur.nc;
        const size_t q = (size_t)(cur.c0 + k0 + j) * NLOC + t;
        const int f = __shfl_sync(0xffffffffu, fl, src + j);
        v[j] = on ? __ldcs(ae + (size_t)f * NLOC + t) : 0.0;
        sl[j] = on ? __ldg(slot + q) : -1;
      }
#pragma unroll
      for (int j = 0; j < CH; j++) {
        __syncwarp();
        if (sl[j] >= 0) buf[sl[j] - cur.rp] += v[j];
        else if (sl[j] <= -3) buf[-3 - sl[j] - cur.rp] = 1.0;
        racc += __shfl_sync(0xffffffffu, rl, src + j);  // cell order
      }
    }
    __syncwarp();
    if (valid) {
      for (int k = t; k < cur.len; k += NLOC) entries[cur.rp + k] = buf[k];
      if (t == 0 && rhs && r < Na) rhs[r] = add_rhs ? rhs[r] + racc : racc;
    }
    __syncwarp();
    cur = nxt;
  }
}

template <int NLOC>
static int launch_gather(Handle &h, Level &L, double *entries, double *rhs, const double *rloc, int add_rhs) {
  constexpr int GPW = 32 / NLOC, WARPS = 8;
  const size_t smem = sizeof(double) * (size_t)WARPS * GPW * L.rmax;
  const int nb = (int)std::min<long>((L.N + WARPS * GPW - 1) / (WARPS * GPW), (long)h.num_sms * 8);
  k_gather_rows<NLOC><<<nb, WARPS * 32, smem, h.stream>>>(L.N, L.Na, L.rmax, L.rowptr.p, L.inc_ptr.p, L.inc.p,
                                                          h.asm_ae.p, L.slot_g.p, rloc, entries, rhs, add_rhs);
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}

// whether the row gather can take this level: the row buffer of a block's
// groups fits in 48 KB of shared memory
static bool gather_fits(const Level &L) {
  const int gpw = 32 / L.nloc;
  return L.rmax > 0 && (size_t)8 * gpw * L.rmax * sizeof(double) <= 48 * 1024;
}

static int run_gather(Handle &h, Level &L, double *entries, double *rhs, const double *rloc, int add_rhs) {
  switch (L.nloc) {
    case 4: return launch_gather<4>(h, L, entries, rhs, rloc, add_rhs);
    case 6: return launch_gather<6>(h, L, entries, rhs, rloc, add_rhs);
    case 8: return launch_gather<8>(h, L, entries, rhs, rloc, add_rhs);
    case 10: return launch_gather<10>(h, L, entries, rhs, rloc, add_rhs);
    case 27: return launch_gather<27>(h, L, entries, rhs, rloc, add_rhs);
    default: set_error("assemble: no row gather for this element"); return PMG_ERR_UNSUPPORTED;
  }
}

// ----------------------------------------------------------------- tables cache
struct TableCache {
  int elem = -1, rule = -1;
  DBuf<double> utab, qtab;
  DBuf<double> stab;  // 16 x n_loc^2: S_ab[i][j] = sum_q w_q u_ia(q) u_jb(q)
  // the tensor-core kernel's tables in mma A-fragment order (see k_assemble_tc):
  // [entry block t][k step s][lane l] = T[8t + l/4][4s + l%4]
  DBuf<double> tc_const, tc_diff;
  DBuf<double> rtab;  // 4 x n_loc: R_a[i] = sum_q w_q u_ia(q)
  int nq = 0;
};

// T[m][k] of k_assemble_tc in A-fragment order; tk(m, k) gives the entry
static std::vector<double> tc_fragments(int nn, int kd, const std::function<double(int, int)> &tk) {
  const int mt = (nn + 7) / 8, ks = (kd + 3) / 4;
  std::vector<double> f((size_t)mt * ks * 32, 0.0);
  for (int t = 0; t < mt; t++)
    for (int sk = 0; sk < ks; sk++)
      for (int l = 0; l < 32; l++) {
        const int m = 8 * t + (l >> 2), k = 4 * sk + (l & 3);
        f[((size_t)t * ks + sk) * 32 + l] = (m < nn && k < kd) ? tk(m, k) : 0.0;
      }
  return f;
}
static TableCache g_tab[5];

// quadrature rule of the reference (TFEDatabase3D::GetOrig, FEDatabase3D.C:1203-1309):
// degree N_terms * polynomial degree with N_terms = 2 (INTERNAL_PROBLEM_LINEAR) or 3
static int rule_for(int elem, int problem_linear, int quad_rule = PMG_QUAD_AUTO) {
  if (quad_rule != PMG_QUAD_AUTO) {
    const bool hex_rule = quad_rule < 100;
    return hex_rule == elem_is_hex(elem) ? quad_rule : -2;
  }
  switch (elem) {
    case PMG_ELEM_Q1_HEX: return problem_linear ? RULE_GAUSS2 : RULE_GAUSS3;
    case PMG_ELEM_Q2_HEX:
    case PMG_ELEM_NQ1_HEX: return problem_linear ? RULE_GAUSS3 : RULE_GAUSS4;
    case PMG_ELEM_P1_TET: return problem_linear ? RULE_KEAST4 : RULE_KEAST11;
    default: return problem_linear ? RULE_KEAST11 : -1;  // P5Tetra (degree 6) is not built
  }
}

static int get_tables(int elem, int rule, TableCache *&out) {
  int slot = elem == PMG_ELEM_Q1_HEX ? 0 : elem == PMG_ELEM_Q2_HEX ? 1 : elem == PMG_ELEM_P1_TET ? 2
           : elem == PMG_ELEM_P2_TET ? 3 : 4;
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
    // CONST: T[m][ab] = S_ab[m]
    std::vector<double> fc = tc_fragments((int)nn, 16, [&](int m, int k) { return st[(size_t)k * nn + m]; });
    PMG_TRY(T.tc_const.upload(fc.data(), fc.size(), 0));
    // DIFF: T[m][(q, p)], p over (00, 11, 22, 01, 02, 12) of the reference gradients
    static const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
    std::vector<double> fd = tc_fragments((int)nn, 6 * q.n, [&](int m, int k) {
      const int i = m / nl, j = m % nl, qq = k / 6, pp = k % 6;
      const double *ui = &u[((size_t)qq * nl + i) * 4], *uj = &u[((size_t)qq * nl + j) * 4];
      const int x = pa[pp], y = pb[pp];
      return x == y ? ui[x] * uj[x] : ui[x] * uj[y] + ui[y] * uj[x];
    });
    PMG_TRY(T.tc_diff.upload(fd.data(), fd.size(), 0));
    std::vector<double> rt((size_t)4 * nl, 0.0);
    for (int a4 = 0; a4 < 4; a4++)
      for (int i = 0; i < nl; i++)
        for (int k = 0; k < q.n; k++) rt[(size_t)a4 * nl + i] += q.w[k] * u[((size_t)k * nl + i) * 4 + a4];
    PMG_TRY(T.rtab.upload(rt.data(), rt.size(), 0));
    PMG_CUDA(cudaDeviceSynchronize());
    T.elem = elem; T.rule = rule; T.nq = q.n;
  }
  out = &T;
  return PMG_OK;
}

template <int E, int NQ>
static int launch_assemble(Handle &h, Level &L, AsmArgs a) {
  constexpr int NLOC = ET<E>::NLOC, GPW = 32 / NLOC;
  // warps per block: ASM_WARPS, fewer when the per-element scratch (NQ x 20
  // doubles per element) would not fit the 227 KB of shared memory (N_Q1 with
  // Gauss4: 5 elements per warp x 64 points)
  const size_t fixed = (size_t)NQ * NLOC * 4 + NQ * 4, per_warp = (size_t)GPW * NQ * 20;
  const int warps = (int)std::min<size_t>(ASM_WARPS, (227 * 1024 / sizeof(double) - fixed) / per_warp);
  if (warps < 1) {
    set_error("assemble: the quadrature rule does not fit the per-point kernel's shared memory");
    return PMG_ERR_UNSUPPORTED;
  }
  size_t smem = sizeof(double) * (fixed + (size_t)warps * per_warp);
  static bool attr_set = false;
  if (!attr_set) {
    PMG_CUDA(cudaFuncSetAttribute(k_assemble<E, NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    attr_set = true;
  }
  h.asm_path = 3;
  int per_block = warps * GPW;
  const int *ed0 = a.elem_dof;
  const double *cv0 = a.cell_vert;
  const int *sl0 = a.slot;
  const size_t ncol = a.ae ? 2 : L.ecolor_ptr.size();  // local-matrix mode: all cells in one launch
  for (size_t c = 0; c + 1 < ncol; c++) {
    int beg = a.ae ? 0 : L.ecolor_ptr[c], n = a.ae ? L.n_cells : L.ecolor_ptr[c + 1] - beg;
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
    k_assemble<E, NQ><<<blocks, warps * 32, smem, h.stream>>>(b); count_launches(1);
    PMG_CUDA(cudaGetLastError());
  }
  if (a.ae) return run_gather(h, L, a.entries, a.rhs, a.rhs ? a.rloc : nullptr, a.add_rhs);
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
  h.asm_path = 2;
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

// the per-colour contraction launches over the per-cell data in h.tc_dbuf / h.tc_rbuf
template <int E, int KS>
static int launch_contract(Handle &h, Level &L, AsmArgs a, const double *tfrag) {
  constexpr int NLOC = ET<E>::NLOC, NN = NLOC * NLOC, MT = (NN + 7) / 8, NB = (MT + 7) / 8, WARPS = 16;
  const size_t smem = sizeof(double) * (size_t)MT * KS * 32;
  static int per_sm = 0;  // resident blocks per SM: the grid never exceeds one wave
  if (!per_sm) {
    PMG_CUDA(cudaFuncSetAttribute(k_assemble_tc16<E, KS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    PMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_assemble_tc16<E, KS>, WARPS * 32, smem));
    if (per_sm < 1) per_sm = 1;
  }
  const size_t ncol = a.ae ? 2 : L.ecolor_ptr.size();  // local-matrix mode: all cells in one launch
  for (size_t c = 0; c + 1 < ncol; c++) {
    const int beg = a.ae ? 0 : L.ecolor_ptr[c], n = a.ae ? L.n_cells : L.ecolor_ptr[c + 1] - beg;
    if (n <= 0) continue;
    AsmArgs b = a;
    b.n_elems = n;
    b.elem_dof = a.elem_dof + (size_t)beg * NLOC;
    b.slot = a.slot + (size_t)beg * NN;
    // items per warp: spread a short colour over all resident warps, but give
    // a warp at most one group's NB items (a long colour runs in several
    // waves of one group per warp: measured 1.651 ms on the 64^3 Q2 finest
    // level, against 1.701 ms with one wave of ~21 items per warp)
    const int items = (n + 7) / 8 * NB;
    const int rw = per_sm * h.num_sms * WARPS;
    const int per = std::min((items + rw - 1) / rw, NB);
    b.item_chunk = per;
    const int blocks = ((items + per - 1) / per + WARPS - 1) / WARPS;
    k_assemble_tc16<E, KS><<<blocks, WARPS * 32, smem, h.stream>>>(b, tfrag, h.tc_dbuf.p + (size_t)beg * 4 * KS,
                                                                   h.tc_rbuf.p + (size_t)beg * NLOC);
    count_launches(1);
    PMG_CUDA(cudaGetLastError());
  }
  if (a.ae) return run_gather(h, L, a.entries, a.rhs, a.rhs ? h.tc_rbuf.p : nullptr, a.add_rhs);
  return PMG_OK;
}

// space-constant coefficients: d = |det J| D (16 per cell), then the contraction
template <int E, int NQ>
static int launch_assemble_tc16(Handle &h, Level &L, AsmArgs a, const double *tfrag, const double *rtab) {
  constexpr int NLOC = ET<E>::NLOC;
  h.asm_path = 0;
  h.asm_kd = 16;
  PMG_TRY(h.tc_dbuf.reserve((size_t)L.n_cells * 16));
  PMG_TRY(h.tc_rbuf.reserve((size_t)L.n_cells * NLOC));
  AsmArgs all = a;
  all.n_elems = L.n_cells;
  k_tc_setup<E, NQ><<<(L.n_cells + 127) / 128, 128, 0, h.stream>>>(all, h.tc_dbuf.p, a.rhs ? h.tc_rbuf.p : nullptr,
                                                                     rtab);
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  return launch_contract<E, 4>(h, L, a, tfrag);
}

// pure diffusion with eps(x): per-point coefficients per cell, then the contraction
template <int E, int NQ>
static int launch_assemble_diff(Handle &h, Level &L, AsmArgs a, const double *tfrag) {
  constexpr int NLOC = ET<E>::NLOC, KS = (6 * NQ + 3) / 4;
  h.asm_path = 1;
  h.asm_kd = 6 * NQ;
  PMG_TRY(h.tc_dbuf.reserve((size_t)L.n_cells * 4 * KS));
  PMG_TRY(h.tc_rbuf.reserve((size_t)L.n_cells * NLOC));
  AsmArgs all = a;
  all.n_elems = L.n_cells;
  constexpr int CB = 128 / NQ;
  k_tc_setup_diff<E, NQ><<<(L.n_cells + CB - 1) / CB, 128, 0, h.stream>>>(all, h.tc_dbuf.p, a.rhs ? h.tc_rbuf.p : nullptr);
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  return launch_contract<E, KS>(h, L, a, tfrag);
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
  const int rule = rule_for(L.elem, h.prm.problem_linear, h.prm.quad_rule);
  if (rule == -2) {
    set_error("assemble: quad_rule does not fit the element's shape");
    return PMG_ERR_UNSUPPORTED;
  }
  if (rule < 0) {
    set_error("assemble: the degree-6 tetrahedral rule (P2 with INTERNAL_PROBLEM_LINEAR = 0) is not built");
    return PMG_ERR_UNSUPPORTED;
  }
  PMG_TRY(get_tables(L.elem, rule, T));
  if (h.coeff.kind == PMG_COEF_TABLE && (!L.ctab.p || L.ctab_nq != T->nq)) {
    set_error("assemble: PMG_COEF_TABLE needs pmg_set_coefficient_table for this level and quadrature rule");
    return PMG_ERR_STATE;
  }
  // row gather (local matrices, then one pass over the rows) or the
  // colour-by-colour scatter; the reference-matrix kernel only scatters.
  // Automatic: the gather for the short rows of Q1 / N_Q1 / P1 / P2, whose
  // colour launches each read and write back most of the matrix's sectors;
  // the scatter for Q2.  Measured on one B200 (scatter -> gather, all
  // levels): P2 lognormal 64^3 (31 colours per level) 5.63 -> 4.88 ms; Q1
  // SUPG 128^3 mass + stiffness on the per-point kernel 7.09 -> 6.71 ms; Q1
  // Poisson 32^3 0.33 -> 0.14 ms; but Q2 SUPG 64^3, finest level, 1.67 ->
  // 2.06 ms (the DMMA contraction scatters 729 entries per cell at 0.37 of
  // HBM; the gather's reads of the local rows are scattered).
  bool gather = (h.prm.assembly_scatter == 2 || (h.prm.assembly_scatter == 0 && L.elem != PMG_ELEM_Q2_HEX)) &&
                h.prm.assembly_kernel != 2;
  if (gather && !L.inc.p) PMG_TRY(build_row_gather(h, L));
  gather = gather && gather_fits(L);
  if (gather) {
    PMG_TRY(h.asm_ae.reserve((size_t)L.n_cells * L.nloc * L.nloc));
    PMG_TRY(h.asm_rloc.reserve((size_t)L.n_cells * L.nloc));
  } else {
    PMG_CUDA(cudaMemsetAsync(target, 0, sizeof(double) * L.nnz, h.stream));  // TAssembleMat3D::Reset
  }
  if (rhs_target && zero_rhs) PMG_CUDA(cudaMemsetAsync(rhs_target, 0, sizeof(double) * L.N, h.stream));
  AsmArgs a{};
  a.ae = gather ? h.asm_ae.p : nullptr;
  a.rloc = gather ? h.asm_rloc.p : nullptr;
  a.add_rhs = zero_rhs ? 0 : 1;
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
  // tensor-core kernel: space-constant coefficients (any element), or pure
  // diffusion with a varying eps on Q1 / P1 / P2 (per-cell coefficients at the
  // quadrature points, then the same contraction)
  const bool pure_diffusion = h.coeff.kind == PMG_COEF_LOGNORMAL && h.coeff.b[0] == 0.0 && h.coeff.b[1] == 0.0 &&
                              h.coeff.b[2] == 0.0 && h.coeff.c == 0.0 && form != PMG_FORM_MASS &&
                              form != PMG_FORM_MASS_SUPG;
  if (h.prm.assembly_kernel == 0 && constant_matrix_coefficients(h.coeff.kind)) {
    const double *tf = T->tc_const.p;
    switch (L.elem * 1000 + T->nq) {
      case PMG_ELEM_Q1_HEX * 1000 + 8: return launch_assemble_tc16<PMG_ELEM_Q1_HEX, 8>(h, L, a, tf, T->rtab.p);
      case PMG_ELEM_Q1_HEX * 1000 + 27: return launch_assemble_tc16<PMG_ELEM_Q1_HEX, 27>(h, L, a, tf, T->rtab.p);
      case PMG_ELEM_Q2_HEX * 1000 + 27: return launch_assemble_tc16<PMG_ELEM_Q2_HEX, 27>(h, L, a, tf, T->rtab.p);
      case PMG_ELEM_Q2_HEX * 1000 + 64: return launch_assemble_tc16<PMG_ELEM_Q2_HEX, 64>(h, L, a, tf, T->rtab.p);
      case PMG_ELEM_NQ1_HEX * 1000 + 8: return launch_assemble_tc16<PMG_ELEM_NQ1_HEX, 8>(h, L, a, tf, T->rtab.p);
      case PMG_ELEM_NQ1_HEX * 1000 + 27: return launch_assemble_tc16<PMG_ELEM_NQ1_HEX, 27>(h, L, a, tf, T->rtab.p);
      case PMG_ELEM_NQ1_HEX * 1000 + 64: return launch_assemble_tc16<PMG_ELEM_NQ1_HEX, 64>(h, L, a, tf, T->rtab.p);
      case PMG_ELEM_P1_TET * 1000 + 4: return launch_assemble_tc16<PMG_ELEM_P1_TET, 4>(h, L, a, tf, T->rtab.p);
      case PMG_ELEM_P1_TET * 1000 + 5: return launch_assemble_tc16<PMG_ELEM_P1_TET, 5>(h, L, a, tf, T->rtab.p);
      case PMG_ELEM_P1_TET * 1000 + 11: return launch_assemble_tc16<PMG_ELEM_P1_TET, 11>(h, L, a, tf, T->rtab.p);
      case PMG_ELEM_P2_TET * 1000 + 4: return launch_assemble_tc16<PMG_ELEM_P2_TET, 4>(h, L, a, tf, T->rtab.p);
      case PMG_ELEM_P2_TET * 1000 + 5: return launch_assemble_tc16<PMG_ELEM_P2_TET, 5>(h, L, a, tf, T->rtab.p);
      case PMG_ELEM_P2_TET * 1000 + 11: return launch_assemble_tc16<PMG_ELEM_P2_TET, 11>(h, L, a, tf, T->rtab.p);
      default: break;
    }
  }
  if (h.prm.assembly_kernel == 0 && pure_diffusion) {
    const double *tf = T->tc_diff.p;
    switch (L.elem * 1000 + T->nq) {
      case PMG_ELEM_Q1_HEX * 1000 + 8: return launch_assemble_diff<PMG_ELEM_Q1_HEX, 8>(h, L, a, tf);
      case PMG_ELEM_Q1_HEX * 1000 + 27: return launch_assemble_diff<PMG_ELEM_Q1_HEX, 27>(h, L, a, tf);
      case PMG_ELEM_P1_TET * 1000 + 4: return launch_assemble_diff<PMG_ELEM_P1_TET, 4>(h, L, a, tf);
      case PMG_ELEM_P1_TET * 1000 + 5: return launch_assemble_diff<PMG_ELEM_P1_TET, 5>(h, L, a, tf);
      case PMG_ELEM_P1_TET * 1000 + 11: return launch_assemble_diff<PMG_ELEM_P1_TET, 11>(h, L, a, tf);
      case PMG_ELEM_P2_TET * 1000 + 4: return launch_assemble_diff<PMG_ELEM_P2_TET, 4>(h, L, a, tf);
      case PMG_ELEM_P2_TET * 1000 + 5: return launch_assemble_diff<PMG_ELEM_P2_TET, 5>(h, L, a, tf);
      case PMG_ELEM_P2_TET * 1000 + 11: return launch_assemble_diff<PMG_ELEM_P2_TET, 11>(h, L, a, tf);
      default: break;
    }
  }
  if (h.prm.assembly_kernel == 2 && constant_matrix_coefficients(h.coeff.kind)) {
    const double *st = T->stab.p;
    switch (L.elem * 1000 + T->nq) {
      case PMG_ELEM_Q1_HEX * 1000 + 8: return launch_assemble_cc<PMG_ELEM_Q1_HEX, 8>(h, L, a, st);
      case PMG_ELEM_Q1_HEX * 1000 + 27: return launch_assemble_cc<PMG_ELEM_Q1_HEX, 27>(h, L, a, st);
      case PMG_ELEM_Q2_HEX * 1000 + 27: return launch_assemble_cc<PMG_ELEM_Q2_HEX, 27>(h, L, a, st);
      case PMG_ELEM_Q2_HEX * 1000 + 64: return launch_assemble_cc<PMG_ELEM_Q2_HEX, 64>(h, L, a, st);
      case PMG_ELEM_NQ1_HEX * 1000 + 8: return launch_assemble_cc<PMG_ELEM_NQ1_HEX, 8>(h, L, a, st);
      case PMG_ELEM_NQ1_HEX * 1000 + 27: return launch_assemble_cc<PMG_ELEM_NQ1_HEX, 27>(h, L, a, st);
      case PMG_ELEM_NQ1_HEX * 1000 + 64: return launch_assemble_cc<PMG_ELEM_NQ1_HEX, 64>(h, L, a, st);
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
    case PMG_ELEM_NQ1_HEX * 1000 + 8: PMG_TRY((launch_assemble<PMG_ELEM_NQ1_HEX, 8>(h, L, a))); break;
    case PMG_ELEM_NQ1_HEX * 1000 + 27: PMG_TRY((launch_assemble<PMG_ELEM_NQ1_HEX, 27>(h, L, a))); break;
    case PMG_ELEM_NQ1_HEX * 1000 + 64: PMG_TRY((launch_assemble<PMG_ELEM_NQ1_HEX, 64>(h, L, a))); break;
    case PMG_ELEM_P1_TET * 1000 + 4: PMG_TRY((launch_assemble<PMG_ELEM_P1_TET, 4>(h, L, a))); break;
    case PMG_ELEM_P1_TET * 1000 + 5: PMG_TRY((launch_assemble<PMG_ELEM_P1_TET, 5>(h, L, a))); break;
    case PMG_ELEM_P1_TET * 1000 + 11: PMG_TRY((launch_assemble<PMG_ELEM_P1_TET, 11>(h, L, a))); break;
    case PMG_ELEM_P2_TET * 1000 + 4: PMG_TRY((launch_assemble<PMG_ELEM_P2_TET, 4>(h, L, a))); break;
    case PMG_ELEM_P2_TET * 1000 + 5: PMG_TRY((launch_assemble<PMG_ELEM_P2_TET, 5>(h, L, a))); break;
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
  const int rule = rule_for(L.elem, h->prm.problem_linear, h->prm.quad_rule);
  if (rule < 0) {
    set_error(rule == -2 ? "pmg_quad_points: quad_rule does not fit the element's shape"
                         : "pmg_quad_points: the degree-6 tetrahedral rule is not built");
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
