// Host-side set-up of structured unit-cube levels (see include/pmg_mesh.h).
// Stands in for what the ParMooN host computes once per mesh with TDomain,
// TFESpace3D, TSquareStructure3D and GetProlongationMatrix3D, so that the
// device path can be driven without the reference's mesh machinery.
#include "../../include/pmg_b200.h"
#include "../../include/pmg_mesh.h"
#include "fe_tables.h"
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

int degree_of(int e) { return (e == PMG_ELEM_Q2_HEX || e == PMG_ELEM_P2_TET) ? 2 : 1; }
bool is_hex(int e) { return e == PMG_ELEM_Q1_HEX || e == PMG_ELEM_Q2_HEX || e == PMG_ELEM_NQ1_HEX; }
int nloc_of(int e) { return pmg::elem_nloc(e); }
bool valid_elem(int e) {
  return e == PMG_ELEM_Q1_HEX || e == PMG_ELEM_Q2_HEX || e == PMG_ELEM_NQ1_HEX || e == PMG_ELEM_P1_TET ||
         e == PMG_ELEM_P2_TET;
}

// N_Q1 on the n^3 cube: one dof per face.  Faces normal to x are (i, j+1/2,
// k+1/2) with i = 0..n (id i + (n+1)(j + n k)), then the y faces
// (i+1/2, j, k+1/2) and the z faces (i+1/2, j+1/2, k) in the same pattern;
// interior faces are numbered first (in id order), the boundary faces after.
// Cell (i, j, k) takes its faces in N_Q1's local order: z = k (zeta = -1),
// y = j, x = i+1, y = j+1, x = i, z = k+1.
int build_nq1(int n, int *elem_dof, double *cell_vert, double *dof_xyz, int *face_id, int *active_bound) {
  const long nf1 = (long)(n + 1) * n * n, N = 3 * nf1;
  auto fx = [&](int i, int j, int k) { return (long)i + (n + 1) * ((long)j + (long)n * k); };
  auto fy = [&](int i, int j, int k) { return nf1 + i + (long)n * ((long)j + (long)(n + 1) * k); };
  auto fz = [&](int i, int j, int k) { return 2 * nf1 + i + (long)n * ((long)j + (long)n * k); };
  auto boundary = [&](long f) {
    const int dir = (int)(f / nf1);
    const long r = f % nf1;
    // the coordinate along the face normal runs 0..n
    const long t = dir == 0 ? r % (n + 1) : dir == 1 ? (r / n) % (n + 1) : r / ((long)n * n);
    return t == 0 || t == n;
  };
  std::vector<int> num(N);
  int a = 0;
  for (long f = 0; f < N; f++)
    if (!boundary(f)) num[f] = a++;
  *active_bound = a;
  int b = a;
  for (long f = 0; f < N; f++)
    if (boundary(f)) num[f] = b++;
  const double h = 1.0 / n;
  for (long f = 0; f < N; f++) {
    const int dir = (int)(f / nf1);
    const long r = f % nf1;
    double x, y, z;
    if (dir == 0) { x = (r % (n + 1)) * h; y = ((r / (n + 1)) % n + 0.5) * h; z = (r / ((long)(n + 1) * n) + 0.5) * h; }
    else if (dir == 1) { x = (r % n + 0.5) * h; y = ((r / n) % (n + 1)) * h; z = (r / ((long)n * (n + 1)) + 0.5) * h; }
    else { x = (r % n + 0.5) * h; y = ((r / n) % n + 0.5) * h; z = (r / ((long)n * n)) * h; }
    const int d = num[f];
    face_id[d] = (int)f;
    dof_xyz[3 * (size_t)d] = x; dof_xyz[3 * (size_t)d + 1] = y; dof_xyz[3 * (size_t)d + 2] = z;
  }
  static const int hoff[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  size_t c = 0;
  for (int k = 0; k < n; k++)
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++, c++) {
        double *cv = cell_vert + c * 24;
        for (int v = 0; v < 8; v++) {
          cv[3 * v] = (i + hoff[v][0]) * h; cv[3 * v + 1] = (j + hoff[v][1]) * h; cv[3 * v + 2] = (k + hoff[v][2]) * h;
        }
        const long f[6] = {fz(i, j, k), fy(i, j, k), fx(i + 1, j, k), fy(i, j + 1, k), fx(i, j, k), fz(i, j, k + 1)};
        for (int l = 0; l < 6; l++) elem_dof[c * 6 + l] = num[f[l]];
      }
  return PMG_OK;
}

// reference coordinates of the local nodes, in units of the element's lattice
// step (hexahedra: 0..p per axis; tetrahedra: barycentric lattice / p)
void local_node(int e, int l, int *ijk) {
  if (is_hex(e)) {
    int n = degree_of(e) + 1;
    ijk[0] = l % n; ijk[1] = (l / n) % n; ijk[2] = l / (n * n);
    return;
  }
  static const int p1[4][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  static const int p2[10][3] = {{0, 0, 0}, {1, 0, 0}, {2, 0, 0}, {0, 1, 0}, {1, 1, 0},
                                {0, 2, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}};
  const int *q = e == PMG_ELEM_P1_TET ? p1[l] : p2[l];
  ijk[0] = q[0]; ijk[1] = q[1]; ijk[2] = q[2];
}

// the six Kuhn tetrahedra of the unit cube: vertex t of tet k is the corner
// reached after t unit steps along the axis order perm[k]
const int kPerm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
void kuhn_vertices(int k, int v[4][3]) {
  int cur[3] = {0, 0, 0};
  for (int d = 0; d < 3; d++) v[0][d] = 0;
  for (int s = 0; s < 3; s++) {
    cur[kPerm[k][s]] = 1;
    for (int d = 0; d < 3; d++) v[s + 1][d] = cur[d];
  }
}

struct SplitMix {
  uint64_t s;
  double next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  }
};

}  // namespace

extern "C" {

int pmg_struct_sizes(int e, int n, int *n_cells, int *n_dofs, int *nloc) {
  if (!valid_elem(e) || n < 1 || !n_cells || !n_dofs || !nloc) return PMG_ERR_ARG;
  if (e == PMG_ELEM_NQ1_HEX) {
    *n_cells = n * n * n;
    *n_dofs = 3 * n * n * (n + 1);
    *nloc = 6;
    return PMG_OK;
  }
  long n1 = (long)degree_of(e) * n + 1;
  *n_cells = is_hex(e) ? n * n * n : 6 * n * n * n;
  *n_dofs = (int)(n1 * n1 * n1);
  *nloc = nloc_of(e);
  return PMG_OK;
}

int pmg_struct_build(int e, int n, double jitter, unsigned long long seed, int *elem_dof, double *cell_vert,
                     double *dof_xyz, int *dof_lat, int *active_bound) {
  if (!valid_elem(e) || n < 1 || !elem_dof || !cell_vert || !dof_xyz || !dof_lat || !active_bound) return PMG_ERR_ARG;
  if (e == PMG_ELEM_NQ1_HEX) {
    if (jitter != 0.0) return PMG_ERR_UNSUPPORTED;  // affine bricks only
    return build_nq1(n, elem_dof, cell_vert, dof_xyz, dof_lat, active_bound);
  }
  const int p = degree_of(e), n1 = p * n + 1, nv1 = n + 1;
  const long N = (long)n1 * n1 * n1;
  std::vector<int> num(N);
  int a = 0;
  for (int k = 0; k < n1; k++)
    for (int j = 0; j < n1; j++)
      for (int i = 0; i < n1; i++) {
        long L = i + (long)n1 * (j + (long)n1 * k);
        bool bd = i == 0 || j == 0 || k == 0 || i == n1 - 1 || j == n1 - 1 || k == n1 - 1;
        num[L] = bd ? -1 : a++;
      }
  *active_bound = a;
  int b = a;
  for (long L = 0; L < N; L++)
    if (num[L] < 0) num[L] = b++;
  // vertices
  const double h = 1.0 / n;
  std::vector<double> V((size_t)3 * nv1 * nv1 * nv1);
  SplitMix rng{seed * 0x2545F4914F6CDD1DULL + 7};
  for (int k = 0; k < nv1; k++)
    for (int j = 0; j < nv1; j++)
      for (int i = 0; i < nv1; i++) {
        size_t v = i + (size_t)nv1 * (j + (size_t)nv1 * k);
        V[3 * v] = i * h; V[3 * v + 1] = j * h; V[3 * v + 2] = k * h;
        bool interior = i > 0 && j > 0 && k > 0 && i < n && j < n && k < n;
        if (jitter > 0 && interior)
          for (int d = 0; d < 3; d++) V[3 * v + d] += (2 * rng.next() - 1) * jitter * h;
      }
  auto vid = [&](int i, int j, int k) { return (size_t)i + (size_t)nv1 * (j + (size_t)nv1 * k); };
  // dof positions: the node is the midpoint of the segment between the two
  // lattice vertices that bracket it (vertex, edge, face-diagonal or
  // body-diagonal midpoint); on hexahedra the average of the bracketing
  // vertices, which coincides for affine cells
  for (long L = 0; L < N; L++) {
    int i = (int)(L % n1), j = (int)((L / n1) % n1), k = (int)(L / ((long)n1 * n1));
    int d = num[L];
    dof_lat[d] = (int)L;
    int i0 = i / p, j0 = j / p, k0 = k / p, ri = i % p, rj = j % p, rk = k % p;
    double x = 0, y = 0, z = 0;
    if (is_hex(e)) {
      int cnt = 0;
      for (int di = 0; di <= ri; di++)
        for (int dj = 0; dj <= rj; dj++)
          for (int dk = 0; dk <= rk; dk++) {
            size_t v = vid(i0 + di, j0 + dj, k0 + dk);
            x += V[3 * v]; y += V[3 * v + 1]; z += V[3 * v + 2]; cnt++;
          }
      x /= cnt; y /= cnt; z /= cnt;
    } else {
      size_t v0 = vid(i0, j0, k0), v1 = vid(i0 + ri, j0 + rj, k0 + rk);
      x = 0.5 * (V[3 * v0] + V[3 * v1]); y = 0.5 * (V[3 * v0 + 1] + V[3 * v1 + 1]); z = 0.5 * (V[3 * v0 + 2] + V[3 * v1 + 2]);
    }
    dof_xyz[3 * (size_t)d] = x; dof_xyz[3 * (size_t)d + 1] = y; dof_xyz[3 * (size_t)d + 2] = z;
  }
  const int nl = nloc_of(e);
  size_t c = 0;
  static const int hoff[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  for (int kz = 0; kz < n; kz++)
    for (int jy = 0; jy < n; jy++)
      for (int ix = 0; ix < n; ix++) {
        int ntet = is_hex(e) ? 1 : 6;
        for (int t = 0; t < ntet; t++, c++) {
          double *cv = cell_vert + c * 24;
          std::memset(cv, 0, sizeof(double) * 24);
          int tv[4][3];
          if (is_hex(e)) {
            for (int v = 0; v < 8; v++) {
              size_t g = vid(ix + hoff[v][0], jy + hoff[v][1], kz + hoff[v][2]);
              for (int d = 0; d < 3; d++) cv[3 * v + d] = V[3 * g + d];
            }
          } else {
            kuhn_vertices(t, tv);
            for (int v = 0; v < 4; v++) {
              size_t g = vid(ix + tv[v][0], jy + tv[v][1], kz + tv[v][2]);
              for (int d = 0; d < 3; d++) cv[3 * v + d] = V[3 * g + d];
            }
          }
          for (int l = 0; l < nl; l++) {
            int r[3], li, lj, lk;
            local_node(e, l, r);
            if (is_hex(e)) {
              li = r[0]; lj = r[1]; lk = r[2];
            } else {
              // lattice offset = sum_t r_t (v_{t} - v_0) with r in units of 1/p
              li = r[0] * tv[1][0] + r[1] * tv[2][0] + r[2] * tv[3][0];
              lj = r[0] * tv[1][1] + r[1] * tv[2][1] + r[2] * tv[3][1];
              lk = r[0] * tv[1][2] + r[1] * tv[2][2] + r[2] * tv[3][2];
            }
            long L = (p * ix + li) + (long)n1 * ((p * jy + lj) + (long)n1 * (p * kz + lk));
            elem_dof[c * nl + l] = num[L];
          }
        }
      }
  return PMG_OK;
}

int pmg_struct_csr(int n_cells, int nloc, const int *ed, int N, int Na, int *rp, int *kc) {
  if (n_cells < 1 || nloc < 1 || !ed || N < 1 || !rp) return PMG_ERR_ARG;
  std::vector<int> cnt(N + 1, 0);
  for (size_t k = 0; k < (size_t)n_cells * nloc; k++) {
    if (ed[k] < 0 || ed[k] >= N) return PMG_ERR_ARG;
    cnt[ed[k] + 1]++;
  }
  for (int i = 0; i < N; i++) cnt[i + 1] += cnt[i];
  std::vector<int> cells(cnt[N]), fp(cnt.begin(), cnt.end() - 1);
  for (int e = 0; e < n_cells; e++)
    for (int l = 0; l < nloc; l++) cells[fp[ed[(size_t)e * nloc + l]]++] = e;
  // row lengths, then fill (rows processed in parallel chunks)
  std::vector<int> len(N);
  auto row_cols = [&](int r, std::vector<int> &buf) {
    buf.clear();
    if (r >= Na) { buf.push_back(r); return; }
    for (int t = cnt[r]; t < cnt[r + 1]; t++) {
      const int *d = ed + (size_t)cells[t] * nloc;
      buf.insert(buf.end(), d, d + nloc);
    }
    std::sort(buf.begin(), buf.end());
    buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
  };
#pragma omp parallel
  {
    std::vector<int> buf;
#pragma omp for schedule(dynamic, 4096)
    for (int r = 0; r < N; r++) {
      row_cols(r, buf);
      len[r] = (int)buf.size();
    }
  }
  rp[0] = 0;
  for (int r = 0; r < N; r++) {
    long next = (long)rp[r] + len[r];
    if (next > 2147483647L) return PMG_ERR_ARG;
    rp[r + 1] = (int)next;
  }
  if (!kc) return PMG_OK;
#pragma omp parallel
  {
    std::vector<int> buf;
#pragma omp for schedule(dynamic, 4096)
    for (int r = 0; r < N; r++) {
      row_cols(r, buf);
      std::memcpy(kc + rp[r], buf.data(), sizeof(int) * buf.size());
    }
  }
  return PMG_OK;
}

int pmg_struct_prolongation(int e, int nc, const int *lat_c, int Nc, const int *lat_f, int Nf, int *prp, int *pcol,
                            double *pval) {
  if (!valid_elem(e) || nc < 1 || !lat_c || !lat_f || !prp) return PMG_ERR_ARG;
  if (e == PMG_ELEM_NQ1_HEX) return PMG_ERR_UNSUPPORTED;  // no node lattice: pmg_cell_prolongation
  const int p = degree_of(e), n1c = p * nc + 1, n1f = 2 * p * nc + 1;
  std::vector<int> inv((size_t)n1c * n1c * n1c, -1);
  for (int d = 0; d < Nc; d++) inv[lat_c[d]] = d;
  prp[0] = 0;
  for (int r = 0; r < Nf; r++) {
    int L = lat_f[r];
    int fi = L % n1f, fj = (L / n1f) % n1f, fk = L / (n1f * n1f);
    int f[3] = {fi, fj, fk}, c0[3];
    double s[3];
    for (int d = 0; d < 3; d++) {
      // fine node in coarse-cell units: f / (2p)
      c0[d] = std::min(f[d] / (2 * p), nc - 1);
      s[d] = f[d] / (2.0 * p) - c0[d];
    }
    int cols[32], m = 0;
    double vals[32];
    if (is_hex(e)) {
      double bx[3][3];
      for (int d = 0; d < 3; d++) {
        // 1D Lagrange values on {-1,1} / {-1,0,1}
        double t = 2 * s[d] - 1;
        if (p == 1) { bx[d][0] = 0.5 * (1 - t); bx[d][1] = 0.5 * (1 + t); }
        else { bx[d][0] = 0.5 * t * (t - 1); bx[d][1] = 1 - t * t; bx[d][2] = 0.5 * t * (t + 1); }
      }
      for (int lk = 0; lk <= p; lk++)
        for (int lj = 0; lj <= p; lj++)
          for (int li = 0; li <= p; li++) {
            double w = bx[0][li] * bx[1][lj] * bx[2][lk];
            if (w == 0.0) continue;
            int Lc = (p * c0[0] + li) + n1c * ((p * c0[1] + lj) + n1c * (p * c0[2] + lk));
            cols[m] = inv[Lc]; vals[m] = w; m++;
          }
    } else {
      // Kuhn simplex of the coarse cube containing s: coordinates sorted decreasing
      int ord[3] = {0, 1, 2};
      std::sort(ord, ord + 3, [&](int x, int y) { return s[x] > s[y] || (s[x] == s[y] && x < y); });
      int tv[4][3] = {{0, 0, 0}}, cur[3] = {0, 0, 0};
      for (int t = 0; t < 3; t++) {
        cur[ord[t]] = 1;
        for (int d = 0; d < 3; d++) tv[t + 1][d] = cur[d];
      }
      double xi = s[ord[0]] - s[ord[1]], eta = s[ord[1]] - s[ord[2]], zeta = s[ord[2]];
      double tab[40];
      pmg::basis_eval(e, xi, eta, zeta, tab);
      for (int l = 0; l < nloc_of(e); l++) {
        double w = tab[l * 4 + 3];
        if (std::fabs(w) < 1e-14) continue;
        int r3[3];
        local_node(e, l, r3);
        int li = r3[0] * tv[1][0] + r3[1] * tv[2][0] + r3[2] * tv[3][0];
        int lj = r3[0] * tv[1][1] + r3[1] * tv[2][1] + r3[2] * tv[3][1];
        int lk = r3[0] * tv[1][2] + r3[1] * tv[2][2] + r3[2] * tv[3][2];
        int Lc = (p * c0[0] + li) + n1c * ((p * c0[1] + lj) + n1c * (p * c0[2] + lk));
        cols[m] = inv[Lc]; vals[m] = w; m++;
      }
    }
    for (int x = 1; x < m; x++) {
      int cc = cols[x]; double vv = vals[x]; int y = x - 1;
      while (y >= 0 && cols[y] > cc) { cols[y + 1] = cols[y]; vals[y + 1] = vals[y]; y--; }
      cols[y + 1] = cc; vals[y + 1] = vv;
    }
    if (pcol) {
      std::memcpy(pcol + prp[r], cols, sizeof(int) * m);
      std::memcpy(pval + prp[r], vals, sizeof(double) * m);
    }
    prp[r + 1] = prp[r] + m;
  }
  return PMG_OK;
}

// Interpolation from a coarse level onto the dof nodes of a nested fine
// level, for any mesh the reference refines (GetProlongationMatrix3D composes
// the same values from the reference-element tables, FEDatabase3D.C:1656-1815):
// row r holds the coarse basis functions of the coarse cell f_dof_cell[r]
// evaluated at the fine node.  For conforming nested spaces the value does not
// depend on which containing coarse cell is named.
int pmg_nested_prolongation(int e, int n_coarse_cells, const int *c_elem_dof, const double *c_cell_vert, int Nc,
                            int Nf, const double *f_dof_xyz, const int *f_dof_cell, int *prp, int *pcol,
                            double *pval) {
  if (!valid_elem(e) || n_coarse_cells < 1 || !c_elem_dof || !c_cell_vert || !f_dof_xyz || !f_dof_cell || !prp)
    return PMG_ERR_ARG;
  const int nl = nloc_of(e);
  const bool hex = is_hex(e);
  prp[0] = 0;
  for (int r = 0; r < Nf; r++) {
    const int c = f_dof_cell[r];
    if (c < 0 || c >= n_coarse_cells) return PMG_ERR_ARG;
    const double *v = c_cell_vert + (size_t)c * 24;
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
    const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                       J[2] * (J[3] * J[7] - J[4] * J[6]);
    if (!(std::fabs(det) > 0)) return PMG_ERR_ARG;
    double Ji[9];
    Ji[0] = (J[4] * J[8] - J[5] * J[7]) / det; Ji[1] = (J[2] * J[7] - J[1] * J[8]) / det;
    Ji[2] = (J[1] * J[5] - J[2] * J[4]) / det; Ji[3] = (J[5] * J[6] - J[3] * J[8]) / det;
    Ji[4] = (J[0] * J[8] - J[2] * J[6]) / det; Ji[5] = (J[2] * J[3] - J[0] * J[5]) / det;
    Ji[6] = (J[3] * J[7] - J[4] * J[6]) / det; Ji[7] = (J[1] * J[6] - J[0] * J[7]) / det;
    Ji[8] = (J[0] * J[4] - J[1] * J[3]) / det;
    const double dx[3] = {f_dof_xyz[3 * (size_t)r] - x0[0], f_dof_xyz[3 * (size_t)r + 1] - x0[1],
                          f_dof_xyz[3 * (size_t)r + 2] - x0[2]};
    double ref[3];
    for (int d = 0; d < 3; d++) ref[d] = Ji[d * 3] * dx[0] + Ji[d * 3 + 1] * dx[1] + Ji[d * 3 + 2] * dx[2];
    double tab[27 * 4];
    pmg::basis_eval(e, ref[0], ref[1], ref[2], tab);
    int cols[27], m = 0;
    double vals[27];
    for (int l = 0; l < nl; l++) {
      const double w = tab[l * 4 + 3];
      if (std::fabs(w) < 1e-12) continue;
      const int col = c_elem_dof[(size_t)c * nl + l];
      if (col < 0 || col >= Nc) return PMG_ERR_ARG;
      cols[m] = col; vals[m] = w; m++;
    }
    for (int x = 1; x < m; x++) {
      int cc = cols[x]; double vv = vals[x]; int y = x - 1;
      while (y >= 0 && cols[y] > cc) { cols[y + 1] = cols[y]; vals[y + 1] = vals[y]; y--; }
      cols[y + 1] = cc; vals[y + 1] = vv;
    }
    if (pcol) {
      std::memcpy(pcol + prp[r], cols, sizeof(int) * m);
      std::memcpy(pval + prp[r], vals, sizeof(double) * m);
    }
    prp[r + 1] = prp[r] + m;
  }
  return PMG_OK;
}

int pmg_cell_prolongation(int ce, int n_coarse_cells, const int *c_elem_dof, const double *c_cell_vert, int Nc,
                          int fe, int n_fine_cells, const int *f_elem_dof, const double *f_cell_vert,
                          const int *f_parent, int Nf, int *prp, int *pcol, double *pval) {
  if (!valid_elem(ce) || !valid_elem(fe) || is_hex(ce) != is_hex(fe) || n_coarse_cells < 1 || n_fine_cells < 1 ||
      !c_elem_dof || !c_cell_vert || !f_elem_dof || !f_cell_vert || !f_parent || Nc < 1 || Nf < 1 || !prp)
    return PMG_ERR_ARG;
  const bool hex = is_hex(ce);
  const int nlc = nloc_of(ce), nlf = nloc_of(fe);
  // the fine element's nodal points on its reference cell
  std::vector<double> fnode((size_t)nlf * 3);
  for (int k = 0; k < nlf; k++) {
    double *q = &fnode[(size_t)k * 3];
    if (fe == PMG_ELEM_NQ1_HEX) {
      q[0] = q[1] = q[2] = 0.0;
      q[pmg::NQ1_AXIS[k]] = pmg::NQ1_SIDE[k];
    } else {
      int r[3];
      local_node(fe, k, r);
      const int p = degree_of(fe);
      for (int d = 0; d < 3; d++) q[d] = hex ? -1.0 + 2.0 * r[d] / p : (double)r[d] / p;
    }
  }
  // affine map of a cell (8 vertex slots) and its inverse
  auto map_of = [&](const double *v, double *J, double *x0) {
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
  };
  std::vector<std::vector<std::pair<int, double>>> rows(Nf);
  std::vector<int> count(Nf, 0);
  double tab[27 * 4];
  for (int K = 0; K < n_fine_cells; K++) {
    const int c = f_parent[K];
    if (c < 0 || c >= n_coarse_cells) return PMG_ERR_ARG;
    double Jf[9], xf[3], Jc[9], xc[3], Ji[9];
    map_of(f_cell_vert + (size_t)K * 24, Jf, xf);
    map_of(c_cell_vert + (size_t)c * 24, Jc, xc);
    const double det = Jc[0] * (Jc[4] * Jc[8] - Jc[5] * Jc[7]) - Jc[1] * (Jc[3] * Jc[8] - Jc[5] * Jc[6]) +
                       Jc[2] * (Jc[3] * Jc[7] - Jc[4] * Jc[6]);
    if (!(std::fabs(det) > 0)) return PMG_ERR_ARG;
    Ji[0] = (Jc[4] * Jc[8] - Jc[5] * Jc[7]) / det; Ji[1] = (Jc[2] * Jc[7] - Jc[1] * Jc[8]) / det;
    Ji[2] = (Jc[1] * Jc[5] - Jc[2] * Jc[4]) / det; Ji[3] = (Jc[5] * Jc[6] - Jc[3] * Jc[8]) / det;
    Ji[4] = (Jc[0] * Jc[8] - Jc[2] * Jc[6]) / det; Ji[5] = (Jc[2] * Jc[3] - Jc[0] * Jc[5]) / det;
    Ji[6] = (Jc[3] * Jc[7] - Jc[4] * Jc[6]) / det; Ji[7] = (Jc[1] * Jc[6] - Jc[0] * Jc[7]) / det;
    Ji[8] = (Jc[0] * Jc[4] - Jc[1] * Jc[3]) / det;
    for (int k = 0; k < nlf; k++) {
      const int d = f_elem_dof[(size_t)K * nlf + k];
      if (d < 0 || d >= Nf) return PMG_ERR_ARG;
      const double *q = &fnode[(size_t)k * 3];
      double x[3], ref[3];
      for (int t = 0; t < 3; t++) x[t] = xf[t] + Jf[t * 3] * q[0] + Jf[t * 3 + 1] * q[1] + Jf[t * 3 + 2] * q[2] - xc[t];
      for (int t = 0; t < 3; t++) ref[t] = Ji[t * 3] * x[0] + Ji[t * 3 + 1] * x[1] + Ji[t * 3 + 2] * x[2];
      pmg::basis_eval(ce, ref[0], ref[1], ref[2], tab);
      count[d]++;
      for (int l = 0; l < nlc; l++) {
        const double w = tab[l * 4 + 3];
        if (std::fabs(w) < 1e-12) continue;
        const int col = c_elem_dof[(size_t)c * nlc + l];
        if (col < 0 || col >= Nc) return PMG_ERR_ARG;
        rows[d].push_back({col, w});
      }
    }
  }
  prp[0] = 0;
  for (int r = 0; r < Nf; r++) {
    auto &v = rows[r];
    std::sort(v.begin(), v.end(), [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
      return a.first < b.first;
    });
    int m = 0;
    for (size_t t = 0; t < v.size();) {
      const int col = v[t].first;
      double sum = 0.0;
      for (; t < v.size() && v[t].first == col; t++) sum += v[t].second;
      sum /= count[r] > 0 ? count[r] : 1;
      if (std::fabs(sum) <= 1e-15) continue;
      if (pcol) {
        pcol[prp[r] + m] = col;
        pval[prp[r] + m] = sum;
      }
      m++;
    }
    prp[r + 1] = prp[r] + m;
  }
  return PMG_OK;
}

int pmg_struct_row_colors(int e, int n, int N, const int *lat, int *colors, int *n_colors) {
  if (!valid_elem(e) || !lat || !colors || !n_colors) return PMG_ERR_ARG;
  if (e == PMG_ELEM_NQ1_HEX) return PMG_ERR_UNSUPPORTED;  // no node lattice: greedy row colours
  const int p = degree_of(e), n1 = p * n + 1, m = p + 1;
  for (int d = 0; d < N; d++) {
    int L = lat[d], i = L % n1, j = (L / n1) % n1, k = L / (n1 * n1);
    colors[d] = (i % m) + m * ((j % m) + m * (k % m));
  }
  *n_colors = m * m * m;
  return PMG_OK;
}

}  // extern "C"
