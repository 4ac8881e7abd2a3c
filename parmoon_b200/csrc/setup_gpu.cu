// Level set-up on the device: the CSR pattern of TSquareStructure3D + Sort
// (src/FE/SquareStructure3D.C:58-527, src/FE/SquareStructure.C:91-110) and the
// nested prolongation of GetProlongationMatrix3D + Prolongate
// (src/FE/FEDatabase3D.C:1656-1815, src/FE/MGComponents3D.C:208-488) for
// conforming nested spaces, built from the element -> dof map instead of on
// the host.
//
// CSR pattern.  Row r of an active dof couples to every dof of every cell that
// holds r; a Dirichlet row (r >= active_bound) holds its diagonal alone; the
// columns of a row are sorted ascending.  On the device:
//   1. the dof -> cell incidence (counts, exclusive scan, fill);
//   2. one warp per row gathers the incident cells' dofs into shared memory,
//      sorts them (bitonic, up to 1024 candidates per row) and drops the
//      repeats; the first pass only counts, the scan of the counts gives the
//      row pointers, the second pass writes the columns.
// Prolongation.  Fine dof r lies in the coarse cell f_dof_cell[r]; its row of
// P holds the coarse basis of that cell evaluated at the dof (inverse affine
// map, HexaAffin / TetraAffin), entries below 1e-12 dropped, columns sorted
// (the host builder pmg_nested_prolongation does the same on the CPU).  The
// restriction R = P^T is formed on the device too (counts, scan, fill, rows
// sorted so the summation order does not depend on the fill order).
#include "pmg_internal.h"
#include "fe_tables.h"
#include <chrono>
#include <cstdio>

namespace pmg {

// ------------------------------------------------------------ exclusive scan
// out[i] = sum_{k<i} in[i] for i <= n (out has n + 1 entries); block sums
// scanned recursively
constexpr int SCAN_B = 1024;

__global__ void __launch_bounds__(SCAN_B) k_scan_block(int n, const int *__restrict__ in, int *__restrict__ out,
                                                       int *__restrict__ block_sums) {
  __shared__ int sh[SCAN_B];
  const int i = blockIdx.x * SCAN_B + threadIdx.x;
  const int v = i < n ? in[i] : 0;
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < SCAN_B; o <<= 1) {
    const int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = sh[threadIdx.x] - v;  // exclusive
  if (threadIdx.x == SCAN_B - 1) block_sums[blockIdx.x] = sh[SCAN_B - 1];
}
__global__ void k_scan_add(int n, int *__restrict__ out, const int *__restrict__ block_off) {
  const int i = blockIdx.x * SCAN_B + threadIdx.x;
  if (i < n) out[i] += block_off[blockIdx.x];
}

// exclusive scan of in[0..n) into out[0..n], out[n] = total; scratch: the
// block sums (allocated here)
int scan_exclusive(cudaStream_t s, int n, const int *in, int *out) {
  const int nb = (n + SCAN_B - 1) / SCAN_B;
  DBuf<int> sums, offs;
  PMG_TRY(sums.alloc(nb + 1));
  PMG_TRY(offs.alloc(nb + 1));
  k_scan_block<<<nb, SCAN_B, 0, s>>>(n, in, out, sums.p);
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  if (nb > 1) {
    PMG_TRY(scan_exclusive(s, nb, sums.p, offs.p));
    k_scan_add<<<nb, SCAN_B, 0, s>>>(n, out, offs.p);
    count_launches(1);
    // total = offs[nb]
    PMG_CUDA(cudaMemcpyAsync(out + n, offs.p + nb, sizeof(int), cudaMemcpyDeviceToDevice, s));
  } else {
    PMG_CUDA(cudaMemcpyAsync(out + n, sums.p, sizeof(int), cudaMemcpyDeviceToDevice, s));
  }
  PMG_CUDA(cudaGetLastError());
  // the recursion's buffers are freed on return: finish before that
  PMG_CUDA(cudaStreamSynchronize(s));
  return PMG_OK;
}

// ------------------------------------------------------------ CSR pattern
__global__ void k_count_dof_cells(size_t total, const int *__restrict__ ed, int *__restrict__ cnt) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < total) atomicAdd(cnt + ed[k], 1);
}
// incidence in cell order per dof (each dof's cells sorted afterwards by the row kernel's sort, so the
// fill order does not matter)
__global__ void k_fill_dof_cells(size_t total, int nloc, const int *__restrict__ ed, int *__restrict__ cursor,
                                 int *__restrict__ cells) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < total) cells[atomicAdd(cursor + ed[k], 1)] = (int)(k / nloc);
}

constexpr int ROW_WARPS = 8, ROW_MAX = 1024;

// one warp per row: sorted distinct columns; kcol == NULL: count into len
__global__ void __launch_bounds__(ROW_WARPS * 32) k_csr_rows(int N, int Na, int nloc, const int *__restrict__ ed,
                                                            const int *__restrict__ dc_ptr,
                                                            const int *__restrict__ dc_cells,
                                                            const int *__restrict__ rp, int *__restrict__ len,
                                                            int *__restrict__ kcol, int *__restrict__ flags) {
  __shared__ int buf[ROW_WARPS][ROW_MAX];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int *b = buf[warp];
  for (int r = blockIdx.x * ROW_WARPS + warp; r < N; r += gridDim.x * ROW_WARPS) {
    if (r >= Na) {  // Dirichlet row: the diagonal alone
      if (lane == 0) {
        if (kcol) kcol[rp[r]] = r;
        else len[r] = 1;
      }
      continue;
    }
    const int c0 = dc_ptr[r], nc = dc_ptr[r + 1] - c0;
    const int m = nc * nloc;
    if (m > ROW_MAX) {
      if (lane == 0) {
        atomicOr(flags, 4);
        if (!kcol) len[r] = 0;
      }
      continue;
    }
    int P = 32;
    while (P < m) P <<= 1;
    for (int t = lane; t < P; t += 32) b[t] = t < m ? ed[(size_t)dc_cells[c0 + t / nloc] * nloc + t % nloc] : 0x7fffffff;
    __syncwarp();
    // bitonic sort of b[0..P)
    for (int k = 2; k <= P; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int t = lane; t < P; t += 32) {
          const int u = t ^ j;
          if (u > t) {
            const bool up = (t & k) == 0;
            const int x = b[t], y = b[u];
            if ((x > y) == up) { b[t] = y; b[u] = x; }
          }
        }
        __syncwarp();
      }
    // distinct values (the first of each run), written in order
    int base = 0;
    for (int t0 = 0; t0 < m; t0 += 32) {
      const int t = t0 + lane;
      const bool first = t < m && (t == 0 || b[t] != b[t - 1]);
      const unsigned ball = __ballot_sync(0xffffffffu, first);
      if (first && kcol) kcol[rp[r] + base + __popc(ball & ((1u << lane) - 1))] = b[t];
      base += __popc(ball);
    }
    if (!kcol && lane == 0) len[r] = base;
    __syncwarp();
  }
}

int build_csr_device(cudaStream_t s, int N, int Na, int n_cells, int nloc, const int *ed_dev, DBuf<int> &rowptr,
                     DBuf<int> &kcol) {
  const size_t total = (size_t)n_cells * nloc;
  DBuf<int> cnt, dc_ptr, cursor, dc_cells, len, flags;
  PMG_TRY(cnt.alloc(N + 1));
  PMG_TRY(dc_ptr.alloc(N + 1));
  PMG_TRY(dc_cells.alloc(total));
  PMG_TRY(len.alloc(N + 1));
  PMG_TRY(flags.alloc(1));
  PMG_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * (N + 1), s));
  PMG_CUDA(cudaMemsetAsync(flags.p, 0, sizeof(int), s));
  const unsigned nb = (unsigned)((total + 255) / 256);
  k_count_dof_cells<<<nb, 256, 0, s>>>(total, ed_dev, cnt.p);
  count_launches(1);
  PMG_TRY(scan_exclusive(s, N, cnt.p, dc_ptr.p));
  PMG_TRY(cursor.alloc(N));
  PMG_CUDA(cudaMemcpyAsync(cursor.p, dc_ptr.p, sizeof(int) * N, cudaMemcpyDeviceToDevice, s));
  k_fill_dof_cells<<<nb, 256, 0, s>>>(total, nloc, ed_dev, cursor.p, dc_cells.p);
  count_launches(1);
  const int rb = std::min((N + ROW_WARPS - 1) / ROW_WARPS, 148 * 16);
  k_csr_rows<<<rb, ROW_WARPS * 32, 0, s>>>(N, Na, nloc, ed_dev, dc_ptr.p, dc_cells.p, nullptr, len.p, nullptr,
                                          flags.p);
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  PMG_TRY(rowptr.alloc(N + 1));
  PMG_TRY(scan_exclusive(s, N, len.p, rowptr.p));
  int nnz = 0, fl = 0;
  PMG_CUDA(cudaMemcpyAsync(&nnz, rowptr.p + N, sizeof(int), cudaMemcpyDeviceToHost, s));
  PMG_CUDA(cudaMemcpyAsync(&fl, flags.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  PMG_CUDA(cudaStreamSynchronize(s));
  if (fl & 4) {
    set_error("pmg_build_level_csr: a row gathers more than 1024 candidate columns (cells x local dofs)");
    return PMG_ERR_UNSUPPORTED;
  }
  if (nnz < 0) {
    set_error("pmg_build_level_csr: more than 2^31 - 1 couplings");
    return PMG_ERR_UNSUPPORTED;
  }
  PMG_TRY(kcol.alloc(std::max(nnz, 1)));
  k_csr_rows<<<rb, ROW_WARPS * 32, 0, s>>>(N, Na, nloc, ed_dev, dc_ptr.p, dc_cells.p, rowptr.p, nullptr, kcol.p,
                                          flags.p);
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  PMG_CUDA(cudaStreamSynchronize(s));
  return PMG_OK;
}

// ------------------------------------------------------------ prolongation
// Lagrange bases of the four elements (values only), as basis_eval
template <int E>
__device__ void basis_values(double x, double y, double z, double *v) {
  if (E == PMG_ELEM_Q1_HEX || E == PMG_ELEM_Q2_HEX) {
    constexpr int n = E == PMG_ELEM_Q1_HEX ? 2 : 3;
    double vx[3], vy[3], vz[3];
    auto lag = [](double s, double *w) {
      if (n == 2) { w[0] = 0.5 * (1 - s); w[1] = 0.5 * (1 + s); }
      else { w[0] = 0.5 * s * (s - 1); w[1] = 1 - s * s; w[2] = 0.5 * s * (s + 1); }
    };
    lag(x, vx); lag(y, vy); lag(z, vz);
    for (int k = 0; k < n; k++)
      for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) v[i + n * (j + n * k)] = vx[i] * vy[j] * vz[k];
    return;
  }
  const double L0 = 1 - x - y - z;
  if (E == PMG_ELEM_P1_TET) { v[0] = L0; v[1] = x; v[2] = y; v[3] = z; return; }
  v[0] = L0 * (2 * L0 - 1); v[1] = 4 * L0 * x; v[2] = x * (2 * x - 1); v[3] = 4 * L0 * y; v[4] = 4 * x * y;
  v[5] = y * (2 * y - 1); v[6] = 4 * L0 * z; v[7] = 4 * x * z; v[8] = 4 * y * z; v[9] = z * (2 * z - 1);
}

// row r of P: cols / vals of the coarse basis functions of cell (colour
// position) cpos[r] above 1e-12 at the fine dof, sorted by column; prp == NULL:
// count into len
template <int E>
__global__ void k_prolong_rows(int Nf, const double *__restrict__ fxyz, const int *__restrict__ cpos,
                               const int *__restrict__ c_ed, const double *__restrict__ c_cv,
                               const int *__restrict__ prp, int *__restrict__ len, int *__restrict__ pcol,
                               double *__restrict__ pval, int *__restrict__ flags) {
  constexpr int NL = E == PMG_ELEM_Q1_HEX ? 8 : E == PMG_ELEM_Q2_HEX ? 27 : E == PMG_ELEM_P1_TET ? 4 : 10;
  constexpr bool HEX = E == PMG_ELEM_Q1_HEX || E == PMG_ELEM_Q2_HEX;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= Nf) return;
  const int c = cpos[r];
  const double *v = c_cv + (size_t)c * (HEX ? 24 : 12);
  double J[9], x0[3];
  for (int d = 0; d < 3; d++) {
    if (HEX) {
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
  if (!(fabs(det) > 0)) {
    atomicOr(flags, 8);
    if (len) len[r] = 0;
    return;
  }
  double Ji[9];
  Ji[0] = (J[4] * J[8] - J[5] * J[7]) / det; Ji[1] = (J[2] * J[7] - J[1] * J[8]) / det;
  Ji[2] = (J[1] * J[5] - J[2] * J[4]) / det; Ji[3] = (J[5] * J[6] - J[3] * J[8]) / det;
  Ji[4] = (J[0] * J[8] - J[2] * J[6]) / det; Ji[5] = (J[2] * J[3] - J[0] * J[5]) / det;
  Ji[6] = (J[3] * J[7] - J[4] * J[6]) / det; Ji[7] = (J[1] * J[6] - J[0] * J[7]) / det;
  Ji[8] = (J[0] * J[4] - J[1] * J[3]) / det;
  const double dx[3] = {fxyz[3 * (size_t)r] - x0[0], fxyz[3 * (size_t)r + 1] - x0[1], fxyz[3 * (size_t)r + 2] - x0[2]};
  double ref[3];
  for (int d = 0; d < 3; d++) ref[d] = Ji[d * 3] * dx[0] + Ji[d * 3 + 1] * dx[1] + Ji[d * 3 + 2] * dx[2];
  double w[NL];
  basis_values<E>(ref[0], ref[1], ref[2], w);
  int cols[NL];
  double vals[NL];
  int m = 0;
  for (int l = 0; l < NL; l++) {
    if (fabs(w[l]) < 1e-12) continue;
    const int col = c_ed[(size_t)c * NL + l];
    int y = m - 1;
    while (y >= 0 && cols[y] > col) { cols[y + 1] = cols[y]; vals[y + 1] = vals[y]; y--; }
    cols[y + 1] = col;
    vals[y + 1] = w[l];
    m++;
  }
  if (!prp) { len[r] = m; return; }
  for (int k = 0; k < m; k++) { pcol[prp[r] + k] = cols[k]; pval[prp[r] + k] = vals[k]; }
}

// R = P^T: counts per coarse row, scan, fill, then each row sorted by fine index
__global__ void k_count_cols(int nnz, const int *__restrict__ pcol, int *__restrict__ cnt) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nnz) atomicAdd(cnt + pcol[k], 1);
}
__global__ void k_fill_transpose(int Nf, const int *__restrict__ prp, const int *__restrict__ pcol,
                                 const double *__restrict__ pval, int *__restrict__ cursor, int *__restrict__ rcol,
                                 double *__restrict__ rval) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= Nf) return;
  for (int k = prp[r]; k < prp[r + 1]; k++) {
    const int q = atomicAdd(cursor + pcol[k], 1);
    rcol[q] = r;
    rval[q] = pval[k];
  }
}
__global__ void k_sort_rows(int n, const int *__restrict__ rp, int *__restrict__ col, double *__restrict__ val) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  for (int a = rp[r] + 1; a < rp[r + 1]; a++) {  // insertion sort (rows of a few dozen entries)
    const int c = col[a];
    const double v = val[a];
    int b = a - 1;
    while (b >= rp[r] && col[b] > c) { col[b + 1] = col[b]; val[b + 1] = val[b]; b--; }
    col[b + 1] = c;
    val[b + 1] = v;
  }
}

}  // namespace pmg

using namespace pmg;

extern "C" int pmg_build_level_csr(pmg_handle hh, int level, int n_rows, int active_bound, int n_cells, int nloc,
                                   const int *elem_dof, int *nnz_out) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || level < 0 || level >= (int)h->lv.size() || n_rows <= 0 || active_bound < 0 || active_bound > n_rows ||
      n_cells <= 0 || nloc <= 0 || nloc > 27 || !elem_dof) {
    set_error("pmg_build_level_csr: bad arguments");
    return PMG_ERR_ARG;
  }
  const size_t total = (size_t)n_cells * nloc;
  for (size_t k = 0; k < total; k++)
    if (elem_dof[k] < 0 || elem_dof[k] >= n_rows) {
      set_error("pmg_build_level_csr: dof index out of range");
      return PMG_ERR_ARG;
    }
  DBuf<int> ed, rp, kc;
  const auto t0 = std::chrono::steady_clock::now();
  PMG_TRY(ed.upload(elem_dof, total, h->stream));
  PMG_TRY(build_csr_device(h->stream, n_rows, active_bound, n_cells, nloc, ed.p, rp, kc));
  const auto t1 = std::chrono::steady_clock::now();
  // install as the level's pattern through the same path as a host pattern
  // (validation, colouring and the host mirror the solve set-up uses)
  std::vector<int> hrp(n_rows + 1);
  PMG_CUDA(cudaMemcpy(hrp.data(), rp.p, sizeof(int) * (n_rows + 1), cudaMemcpyDeviceToHost));
  std::vector<int> hkc(std::max(hrp[n_rows], 1));
  PMG_CUDA(cudaMemcpy(hkc.data(), kc.p, sizeof(int) * hrp[n_rows], cudaMemcpyDeviceToHost));
  if (nnz_out) *nnz_out = hrp[n_rows];
  const int rc = pmg_set_level_csr(hh, level, n_rows, active_bound, hrp.data(), hkc.data());
  h->t_setup_csr_device = std::chrono::duration<double>(t1 - t0).count();
  h->t_setup_csr_install = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
  return rc;
}

extern "C" int pmg_setup_timings(pmg_handle hh, double *csr_device_s, double *csr_install_s) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h) return PMG_ERR_ARG;
  if (csr_device_s) *csr_device_s = h->t_setup_csr_device;
  if (csr_install_s) *csr_install_s = h->t_setup_csr_install;
  return PMG_OK;
}

extern "C" int pmg_get_level_csr(pmg_handle hh, int level, int *row_ptr, int *kcol) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || level < 0 || level >= (int)h->lv.size() || !row_ptr) {
    set_error("pmg_get_level_csr: bad arguments");
    return PMG_ERR_ARG;
  }
  Level &L = h->lv[level];
  if (!L.has_csr) {
    set_error("pmg_get_level_csr: the level has no pattern");
    return PMG_ERR_STATE;
  }
  PMG_CUDA(cudaMemcpy(row_ptr, L.rowptr.p, sizeof(int) * (L.N + 1), cudaMemcpyDeviceToHost));
  if (kcol) PMG_CUDA(cudaMemcpy(kcol, L.kcol.p, sizeof(int) * L.nnz, cudaMemcpyDeviceToHost));
  return PMG_OK;
}

extern "C" int pmg_build_transfer(pmg_handle hh, int level, int n_fine, const double *f_dof_xyz,
                                  const int *f_dof_cell) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || level < 1 || level >= (int)h->lv.size() || !f_dof_xyz || !f_dof_cell) {
    set_error("pmg_build_transfer: bad arguments");
    return PMG_ERR_ARG;
  }
  Level &L = h->lv[level], &C = h->lv[level - 1];
  if (!L.has_csr || !C.has_csr || !C.has_mesh || n_fine != L.N) {
    set_error("pmg_build_transfer: needs the fine level's pattern and the coarse level's pattern and mesh");
    return PMG_ERR_STATE;
  }
  if (C.elem == PMG_ELEM_NQ1_HEX || L.elem == PMG_ELEM_NQ1_HEX) {
    set_error("pmg_build_transfer: conforming nested spaces only (N_Q1 levels: pmg_cell_prolongation)");
    return PMG_ERR_UNSUPPORTED;
  }
  // the coarse cells sit on the device in colour order: caller index -> position
  std::vector<int> pos(C.n_cells), cpos(n_fine);
  for (int k = 0; k < C.n_cells; k++) pos[C.cell_order[k]] = k;
  for (int r = 0; r < n_fine; r++) {
    if (f_dof_cell[r] < 0 || f_dof_cell[r] >= C.n_cells) {
      set_error("pmg_build_transfer: coarse cell index out of range");
      return PMG_ERR_ARG;
    }
    cpos[r] = pos[f_dof_cell[r]];
  }
  cudaStream_t s = h->stream;
  DBuf<double> fxyz;
  DBuf<int> dcpos, len, flags, prp, pcol, cnt, rrp, cursor, rcol;
  DBuf<double> pval, rval;
  PMG_TRY(fxyz.upload(f_dof_xyz, (size_t)n_fine * 3, s));
  PMG_TRY(dcpos.upload(cpos.data(), n_fine, s));
  PMG_TRY(len.alloc(n_fine + 1));
  PMG_TRY(flags.alloc(1));
  PMG_CUDA(cudaMemsetAsync(flags.p, 0, sizeof(int), s));
  const int nb = (n_fine + 255) / 256;
  auto rows = [&](const int *p, int *l, int *pc, double *pv) -> int {
    switch (C.elem) {
      case PMG_ELEM_Q1_HEX: k_prolong_rows<PMG_ELEM_Q1_HEX><<<nb, 256, 0, s>>>(n_fine, fxyz.p, dcpos.p, C.elem_dof.p, C.cell_vert.p, p, l, pc, pv, flags.p); break;
      case PMG_ELEM_Q2_HEX: k_prolong_rows<PMG_ELEM_Q2_HEX><<<nb, 256, 0, s>>>(n_fine, fxyz.p, dcpos.p, C.elem_dof.p, C.cell_vert.p, p, l, pc, pv, flags.p); break;
      case PMG_ELEM_P1_TET: k_prolong_rows<PMG_ELEM_P1_TET><<<nb, 256, 0, s>>>(n_fine, fxyz.p, dcpos.p, C.elem_dof.p, C.cell_vert.p, p, l, pc, pv, flags.p); break;
      default: k_prolong_rows<PMG_ELEM_P2_TET><<<nb, 256, 0, s>>>(n_fine, fxyz.p, dcpos.p, C.elem_dof.p, C.cell_vert.p, p, l, pc, pv, flags.p); break;
    }
    count_launches(1);
    PMG_CUDA(cudaGetLastError());
    return PMG_OK;
  };
  PMG_TRY(rows(nullptr, len.p, nullptr, nullptr));
  PMG_TRY(prp.alloc(n_fine + 1));
  PMG_TRY(scan_exclusive(s, n_fine, len.p, prp.p));
  int nnz = 0, fl = 0;
  PMG_CUDA(cudaMemcpyAsync(&nnz, prp.p + n_fine, sizeof(int), cudaMemcpyDeviceToHost, s));
  PMG_CUDA(cudaMemcpyAsync(&fl, flags.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  PMG_CUDA(cudaStreamSynchronize(s));
  if (fl & 8) {
    set_error("pmg_build_transfer: a coarse cell with zero volume");
    return PMG_ERR_ARG;
  }
  PMG_TRY(pcol.alloc(std::max(nnz, 1)));
  PMG_TRY(pval.alloc(std::max(nnz, 1)));
  PMG_TRY(rows(prp.p, nullptr, pcol.p, pval.p));
  // R = P^T
  const int Nc = C.N;
  PMG_TRY(cnt.alloc(Nc + 1));
  PMG_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * (Nc + 1), s));
  k_count_cols<<<(nnz + 255) / 256, 256, 0, s>>>(nnz, pcol.p, cnt.p);
  count_launches(1);
  PMG_TRY(rrp.alloc(Nc + 1));
  PMG_TRY(scan_exclusive(s, Nc, cnt.p, rrp.p));
  PMG_TRY(cursor.alloc(Nc));
  PMG_CUDA(cudaMemcpyAsync(cursor.p, rrp.p, sizeof(int) * Nc, cudaMemcpyDeviceToDevice, s));
  PMG_TRY(rcol.alloc(std::max(nnz, 1)));
  PMG_TRY(rval.alloc(std::max(nnz, 1)));
  k_fill_transpose<<<nb, 256, 0, s>>>(n_fine, prp.p, pcol.p, pval.p, cursor.p, rcol.p, rval.p);
  k_sort_rows<<<(Nc + 255) / 256, 256, 0, s>>>(Nc, rrp.p, rcol.p, rval.p);
  count_launches(2);
  PMG_CUDA(cudaGetLastError());
  PMG_CUDA(cudaStreamSynchronize(s));
  // install (the level keeps these buffers)
  std::swap(L.prp.p, prp.p); std::swap(L.prp.n, prp.n);
  std::swap(L.pcol.p, pcol.p); std::swap(L.pcol.n, pcol.n);
  std::swap(L.pval.p, pval.p); std::swap(L.pval.n, pval.n);
  std::swap(L.rrp.p, rrp.p); std::swap(L.rrp.n, rrp.n);
  std::swap(L.rcol.p, rcol.p); std::swap(L.rcol.n, rcol.n);
  std::swap(L.rval.p, rval.p); std::swap(L.rval.n, rval.n);
  L.pval32.release();
  L.rval32.release();
  L.Nc = Nc;
  L.has_P = true;
  invalidate_graphs(h);
  return PMG_OK;
}

extern "C" int pmg_get_transfer(pmg_handle hh, int level, int *p_row_ptr, int *p_col, double *p_val) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || level < 1 || level >= (int)h->lv.size() || !p_row_ptr) {
    set_error("pmg_get_transfer: bad arguments");
    return PMG_ERR_ARG;
  }
  Level &L = h->lv[level];
  if (!L.has_P) {
    set_error("pmg_get_transfer: the level has no transfer");
    return PMG_ERR_STATE;
  }
  PMG_CUDA(cudaMemcpy(p_row_ptr, L.prp.p, sizeof(int) * (L.N + 1), cudaMemcpyDeviceToHost));
  int nnz = 0;
  PMG_CUDA(cudaMemcpy(&nnz, L.prp.p + L.N, sizeof(int), cudaMemcpyDeviceToHost));
  if (p_col) PMG_CUDA(cudaMemcpy(p_col, L.pcol.p, sizeof(int) * nnz, cudaMemcpyDeviceToHost));
  if (p_val) PMG_CUDA(cudaMemcpy(p_val, L.pval.p, sizeof(double) * nnz, cudaMemcpyDeviceToHost));
  return PMG_OK;
}
