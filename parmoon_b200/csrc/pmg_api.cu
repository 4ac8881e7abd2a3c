// extern "C" entry points of libpmg_b200 (declared in include/pmg_b200.h).
//
// Host-side set-up kept here: element colouring (greedy over shared degrees
// of freedom), multicolour row ordering for the parallel SSOR, transposition
// of the prolongation, and the validation of every array handed in (the
// reference exits on bad input; this library returns PMG_ERR_*).
#include "pmg_internal.h"
#include "fe_tables.h"
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <numeric>

namespace pmg {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }

static std::atomic<unsigned long long> g_launches{0};
void count_launches(unsigned long long n) { g_launches += n; }
unsigned long long launches_so_far() { return g_launches.load(); }

int level_invdiag(cudaStream_t s, Level &L, int *flags);

static Handle *H(pmg_handle h) { return reinterpret_cast<Handle *>(h); }

// PMG_TRACE=1 prints the progress of the set-up calls (diagnostics)
static bool tracing() {
  static int t = -1;
  if (t < 0) { const char *e = getenv("PMG_TRACE"); t = (e && e[0] == '1') ? 1 : 0; }
  return t == 1;
}
#define PMG_TRACE_AT(tag) do { if (tracing()) { fprintf(stderr, "[pmg] %s:%d %s\n", __func__, __LINE__, tag); fflush(stderr); } } while (0)

void invalidate_graphs(Handle *h) {
  if (h->vgraph) { cudaGraphExecDestroy(h->vgraph); h->vgraph = nullptr; }
  if (h->vgraph_ssor) { cudaGraphExecDestroy(h->vgraph_ssor); h->vgraph_ssor = nullptr; }
}

static int check_level(Handle *h, int level) {
  if (!h) { set_error("null handle"); return PMG_ERR_ARG; }
  if (level < 0 || level >= (int)h->lv.size()) { set_error("level out of range"); return PMG_ERR_ARG; }
  return PMG_OK;
}

int check_matrix(Handle *h, int level, const char *who) {
  PMG_TRY(check_level(h, level));
  const Level &L = h->lv[level];
  if (!L.has_csr || !L.assembled) {
    set_error(std::string(who) + ": the level has no matrix values yet (pmg_assemble or pmg_set_matrix first)");
    return PMG_ERR_STATE;
  }
  return PMG_OK;
}

// The parameter sets this library builds (the reference exits or falls back
// to SOR on unknown smoother codes, MultiGrid3D.C:210-213; here they are
// rejected).
static int validate_params(const pmg_params *p) {
  auto bad = [](const char *m) { set_error(std::string("params: ") + m); return PMG_ERR_ARG; };
  const int sm = p->smoother;
  if (sm != PMG_SMOOTHER_JACOBI && sm != PMG_SMOOTHER_SOR && sm != PMG_SMOOTHER_SSOR && sm != PMG_SMOOTHER_LEARNED)
    return bad("smoother must be PMG_SMOOTHER_JACOBI, _SOR, _SSOR or _LEARNED");
  const int cs = p->coarse_smoother;
  if (cs != PMG_COARSE_JACOBI && cs != PMG_COARSE_SOR && cs != PMG_COARSE_SSOR && cs != PMG_COARSE_DIRECT)
    return bad("coarse_smoother must be PMG_COARSE_JACOBI, _SOR, _SSOR or _DIRECT");
  if (p->pre_smooth < 0 || p->pre_smooth > 64 || p->post_smooth < 0 || p->post_smooth > 64)
    return bad("pre_smooth / post_smooth must be in [0, 64]");
  if (p->coarse_maxit < 1 || p->coarse_maxit > 100000) return bad("coarse_maxit must be in [1, 100000]");
  if (p->restart < 1 || p->restart > 60) return bad("restart must be in [1,60]");
  if (p->lin_maxit < 1) return bad("lin_maxit must be >= 1");
  if (p->precision != PMG_PREC_FP64 && p->precision != PMG_PREC_FP32) return bad("precision must be PMG_PREC_FP64 or _FP32");
  if (p->assembly_kernel < 0 || p->assembly_kernel > 2) return bad("assembly_kernel must be 0, 1 or 2");
  if (p->problem_linear != 0 && p->problem_linear != 1) return bad("problem_linear must be 0 or 1");
  if (p->reference_restart_rule != 0 && p->reference_restart_rule != 1) return bad("reference_restart_rule must be 0 or 1");
  if ((p->slc_all != 0 && p->slc_all != 1) || (p->slc_fine != 0 && p->slc_fine != 1)) return bad("slc_all / slc_fine must be 0 or 1");
  if (p->learned_steps < 0 || p->learned_steps > 64) return bad("learned_steps must be in [0, 64]");
  if (p->learned_guard_off != 0 && p->learned_guard_off != 1) return bad("learned_guard_off must be 0 or 1");
  if (p->assembly_scatter < 0 || p->assembly_scatter > 2) return bad("assembly_scatter must be 0, 1 or 2");
  if (p->quad_rule != PMG_QUAD_AUTO && p->quad_rule != PMG_QUAD_GAUSS2 && p->quad_rule != PMG_QUAD_GAUSS3 &&
      p->quad_rule != PMG_QUAD_GAUSS4 && p->quad_rule != PMG_QUAD_KEAST4 && p->quad_rule != PMG_QUAD_KEAST5 &&
      p->quad_rule != PMG_QUAD_KEAST11)
    return bad("quad_rule must be 0 or one of PMG_QUAD_*");
  if (p->poly_degree < 0) return bad("poly_degree must be >= 0");
  const double pos[] = {p->smooth_omega, p->div_factor};
  for (double v : pos)
    if (!std::isfinite(v) || v <= 0.0) return bad("smooth_omega and div_factor must be finite and positive");
  const double nonneg[] = {p->coarse_red, p->lin_red, p->lin_res_min, p->delta0};
  for (double v : nonneg)
    if (!std::isfinite(v) || v < 0.0) return bad("coarse_red, lin_red, lin_res_min and delta0 must be finite and >= 0");
  if (!std::isfinite(p->gmg_damp)) return bad("gmg_damp must be finite");
  return PMG_OK;
}

// greedy colouring of the cells so that no two cells of one colour share a dof
static std::vector<int> color_cells(int n_cells, int nloc, const int *ed, int N, int &ncolors) {
  std::vector<int> cnt(N + 1, 0);
  for (size_t k = 0; k < (size_t)n_cells * nloc; k++) cnt[ed[k] + 1]++;
  for (int i = 0; i < N; i++) cnt[i + 1] += cnt[i];
  std::vector<int> cells(cnt[N]), fillp(cnt.begin(), cnt.end() - 1);
  for (int e = 0; e < n_cells; e++)
    for (int l = 0; l < nloc; l++) cells[fillp[ed[(size_t)e * nloc + l]]++] = e;
  std::vector<int> color(n_cells, -1);
  std::vector<int> mark(256, -1);
  ncolors = 0;
  for (int e = 0; e < n_cells; e++) {
    for (int l = 0; l < nloc; l++) {
      int d = ed[(size_t)e * nloc + l];
      for (int t = cnt[d]; t < cnt[d + 1]; t++) {
        int c = color[cells[t]];
        if (c >= 0) mark[c] = e;
      }
    }
    int c = 0;
    while (c < 256 && mark[c] == e) c++;
    color[e] = c;
    ncolors = std::max(ncolors, c + 1);
  }
  return color;
}

// greedy distance-1 colouring of the active rows of a CSR pattern
static std::vector<int> color_rows(int N, int Na, const int *rp, const int *kc, int &ncolors) {
  std::vector<int> color(N, -1), mark(1024, -1);
  ncolors = 0;
  for (int r = 0; r < Na; r++) {
    for (int k = rp[r]; k < rp[r + 1]; k++) {
      int c = kc[k] < N ? color[kc[k]] : -1;
      if (c >= 0) mark[c] = r;
    }
    int c = 0;
    while (c < 1024 && mark[c] == r) c++;
    color[r] = c;
    ncolors = std::max(ncolors, c + 1);
  }
  return color;
}

static int upload_row_colors(Handle *h, Level &L, int ncolors, const std::vector<int> &color) {
  std::vector<int> ptr(ncolors + 1, 0), list(L.Na);
  for (int r = 0; r < L.Na; r++) ptr[color[r] + 1]++;
  for (int c = 0; c < ncolors; c++) ptr[c + 1] += ptr[c];
  std::vector<int> fp(ptr.begin(), ptr.end() - 1);
  for (int r = 0; r < L.Na; r++) list[fp[color[r]]++] = r;
  PMG_TRY(L.row_list.upload(list.data(), list.size(), h->stream));
  L.rcolor_ptr = ptr;
  L.h_row_list = list;
  L.sell_ready = false;
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  return PMG_OK;
}

}  // namespace pmg

using namespace pmg;

extern "C" {

const char *pmg_last_error(void) { return g_err.c_str(); }

int pmg_device_count(int *n) {
  if (!n) return PMG_ERR_ARG;
  PMG_CUDA(cudaGetDeviceCount(n));
  return PMG_OK;
}

int pmg_params_size(void) { return (int)sizeof(pmg_params); }

void pmg_default_params(pmg_params *p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->smoother = PMG_SMOOTHER_SSOR;       // SC_SMOOTHER_SCALAR = 3 (Database.C:672)
  p->pre_smooth = 2;
  p->post_smooth = 2;
  p->coarse_smoother = PMG_COARSE_DIRECT;
  p->coarse_maxit = 10;                  // SC_COARSE_MAXIT_SCALAR
  p->coarse_red = 0.1;                   // SC_COARSE_RED_FACTOR_SCALAR
  p->smooth_omega = 1.0;                 // SC_SMOOTH_DAMP_FACTOR_SCALAR
  p->gmg_damp = 1.0;                     // SC_GMG_DAMP_FACTOR_SCALAR
  p->lin_red = 1e-10;
  p->lin_res_min = 0.0;
  p->lin_maxit = 1000;
  p->restart = 20;
  p->div_factor = 1e10;                  // SC_DIV_FACTOR (Database.C:770)
  p->precision = PMG_PREC_FP64;
  p->sdfem_type = 2;                     // SDFEM_TYPE (Database.C:483)
  p->poly_degree = 0;                    // 0: element degree
  p->delta0 = 1.0;                       // DELTA0 (Database.C:480)
  p->reference_restart_rule = 0;
  p->problem_linear = 1;                 // the configs' quadrature (Gauss2 for Q1, Gauss3 for Q2)
}

int pmg_create(pmg_handle *out, int n_levels, const pmg_params *p) {
  if (!out || n_levels < 1 || n_levels > 16) { set_error("pmg_create: bad arguments"); return PMG_ERR_ARG; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("pmg_create: no CUDA device");
    return PMG_ERR_CUDA;
  }
  pmg_params prm;
  if (p) prm = *p; else pmg_default_params(&prm);
  PMG_TRY(validate_params(&prm));
  Handle *h = new Handle();
  h->prm = prm;
  h->lv.resize(n_levels);
  cudaGetDevice(&h->device);
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    set_error("pmg_create: stream creation failed");
    return PMG_ERR_CUDA;
  }
  for (int k = 0; k < 10; k++) cudaEventCreate(&h->ev[k]);
  int rc = h->d_flags.alloc(4);
  if (rc == PMG_OK && cudaStreamCreateWithFlags(&h->aux, cudaStreamNonBlocking) != cudaSuccess) rc = PMG_ERR_CUDA;
  for (int k = 0; k < 2 && rc == PMG_OK; k++)
    if (cudaEventCreateWithFlags(&h->aux_ev[k], cudaEventDisableTiming) != cudaSuccess) rc = PMG_ERR_CUDA;
  if (rc == PMG_OK) rc = h->coarse_flags.alloc(4);
  if (rc == PMG_OK && cudaMallocHost(&h->h_coarse_flags, sizeof(int) * 4) != cudaSuccess) rc = PMG_ERR_CUDA;
  if (rc == PMG_OK) rc = h->red_partial.alloc(1024);
  if (rc == PMG_OK) rc = h->red_counter.alloc(1);
  if (rc == PMG_OK && cudaMemset(h->red_counter.p, 0, sizeof(unsigned)) != cudaSuccess) rc = PMG_ERR_CUDA;
  if (rc == PMG_OK && cudaMallocHost(&h->h_H, sizeof(double) * 256) != cudaSuccess) rc = PMG_ERR_CUDA;
  if (rc != PMG_OK) { pmg_destroy(reinterpret_cast<pmg_handle>(h)); return rc; }
  {
    const char *ng = getenv("PMG_NO_GRAPH");
    h->use_graph = !(ng && ng[0] == '1');
  }
  h->coeff.kind = PMG_COEF_CONST;
  h->coeff.eps = 1.0;
  h->coeff.f = 1.0;
  *out = reinterpret_cast<pmg_handle>(h);
  return PMG_OK;
}

int pmg_destroy(pmg_handle hh) {
  Handle *h = H(hh);
  if (!h) return PMG_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->aux) cudaStreamSynchronize(h->aux);
  if (h->vgraph) cudaGraphExecDestroy(h->vgraph);
  if (h->vgraph_ssor) cudaGraphExecDestroy(h->vgraph_ssor);
  for (int k = 0; k < 10; k++) if (h->ev[k]) cudaEventDestroy(h->ev[k]);
  if (h->h_H) cudaFreeHost(h->h_H);
  if (h->h_coarse_flags) cudaFreeHost(h->h_coarse_flags);
  for (int k = 0; k < 2; k++) if (h->aux_ev[k]) cudaEventDestroy(h->aux_ev[k]);
  h->lv.clear();
  if (h->aux) cudaStreamDestroy(h->aux);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return PMG_OK;
}

int pmg_set_params(pmg_handle hh, const pmg_params *p) {
  Handle *h = H(hh);
  if (!h || !p) return PMG_ERR_ARG;
  PMG_TRY(validate_params(p));
  bool graph_shape = p->precision != h->prm.precision || p->pre_smooth != h->prm.pre_smooth ||
                     p->post_smooth != h->prm.post_smooth || p->coarse_smoother != h->prm.coarse_smoother ||
                     p->smooth_omega != h->prm.smooth_omega || p->gmg_damp != h->prm.gmg_damp ||
                     p->coarse_maxit != h->prm.coarse_maxit || p->smoother != h->prm.smoother ||
                     p->learned_steps != h->prm.learned_steps || p->slc_all != h->prm.slc_all ||
                     p->slc_fine != h->prm.slc_fine;
  h->prm = *p;
  if (graph_shape) invalidate_graphs(h);
  return PMG_OK;
}

int pmg_set_level_mesh(pmg_handle hh, int level, int elem_type, int n_cells, const int *elem_dof,
                       const double *cell_vert, int brick) {
  Handle *h = H(hh);
  PMG_TRY(check_level(h, level));
  Level &L = h->lv[level];
  if (elem_type != PMG_ELEM_Q1_HEX && elem_type != PMG_ELEM_Q2_HEX && elem_type != PMG_ELEM_NQ1_HEX &&
      elem_type != PMG_ELEM_P1_TET && elem_type != PMG_ELEM_P2_TET) {
    set_error("pmg_set_level_mesh: unknown element type");
    return PMG_ERR_ARG;
  }
  if (n_cells <= 0 || !elem_dof || !cell_vert) { set_error("pmg_set_level_mesh: empty mesh"); return PMG_ERR_ARG; }
  const int nloc = elem_nloc(elem_type), nv = elem_is_hex(elem_type) ? 8 : 4;
  if (!L.has_csr) { set_error("pmg_set_level_mesh: call pmg_set_level_csr first"); return PMG_ERR_STATE; }
  for (size_t k = 0; k < (size_t)n_cells * nloc; k++)
    if (elem_dof[k] < 0 || elem_dof[k] >= L.N) { set_error("pmg_set_level_mesh: dof index out of range"); return PMG_ERR_ARG; }
  if (nv == 8) {
    // the kernels map hexahedra affinely (HexaAffin): every cell must be a
    // parallelepiped, v2 = v1 + v3 - v0, v5 = v1 + v4 - v0, v7 = v3 + v4 - v0,
    // v6 = v1 + v3 + v4 - 2 v0 (the trilinear map of HexaTrilinear is not built)
    for (int e = 0; e < n_cells; e++) {
      const double *v = cell_vert + (size_t)e * 24;
      double diam = 0.0, dev = 0.0;
      for (int d = 0; d < 3; d++) {
        const double a = v[3 + d] - v[d], b = v[9 + d] - v[d], c = v[12 + d] - v[d];
        diam = std::max(diam, std::fabs(a) + std::fabs(b) + std::fabs(c));
        dev = std::max(dev, std::fabs(v[6 + d] - (v[3 + d] + v[9 + d] - v[d])));
        dev = std::max(dev, std::fabs(v[15 + d] - (v[3 + d] + v[12 + d] - v[d])));
        dev = std::max(dev, std::fabs(v[21 + d] - (v[9 + d] + v[12 + d] - v[d])));
        dev = std::max(dev, std::fabs(v[18 + d] - (v[3 + d] + v[9 + d] + v[12 + d] - 2 * v[d])));
      }
      if (!(dev <= 1e-10 * diam)) {
        set_error("pmg_set_level_mesh: cell " + std::to_string(e) +
                  " is a hexahedron that is not a parallelepiped (the trilinear map, HexaTrilinear, is not built)");
        return PMG_ERR_UNSUPPORTED;
      }
    }
  }
  int ncol = 0;
  std::vector<int> color = color_cells(n_cells, nloc, elem_dof, L.N, ncol);
  // colour-sorted copies
  std::vector<int> ptr(ncol + 1, 0);
  for (int e = 0; e < n_cells; e++) ptr[color[e] + 1]++;
  for (int c = 0; c < ncol; c++) ptr[c + 1] += ptr[c];
  std::vector<int> fp(ptr.begin(), ptr.end() - 1), order(n_cells);
  for (int e = 0; e < n_cells; e++) order[fp[color[e]]++] = e;
  std::vector<int> ed((size_t)n_cells * nloc);
  std::vector<double> cv((size_t)n_cells * nv * 3);
  for (int k = 0; k < n_cells; k++) {
    int e = order[k];
    memcpy(&ed[(size_t)k * nloc], elem_dof + (size_t)e * nloc, sizeof(int) * nloc);
    // input cells carry 8 vertex slots (hexahedra) or 8 slots with 4 used (tetrahedra)
    memcpy(&cv[(size_t)k * nv * 3], cell_vert + (size_t)e * 24, sizeof(double) * nv * 3);
  }
  L.elem = elem_type;
  L.nloc = nloc;
  L.nvert = nv;
  L.n_cells = n_cells;
  L.brick = brick;
  L.ecolor_ptr = ptr;
  L.cell_order = order;
  L.ctab.release();
  L.ctab_nq = 0;
  PMG_TRY(L.elem_dof.upload(ed.data(), ed.size(), h->stream));
  PMG_TRY(L.cell_vert.upload(cv.data(), cv.size(), h->stream));
  L.slot.release();
  L.inc.release();
  L.inc_ptr.release();
  L.slot_g.release();
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  L.has_mesh = true;
  L.assembled = false;
  return build_slot_map(*h, L);
}

int pmg_set_level_csr(pmg_handle hh, int level, int n_rows, int active_bound, const int *row_ptr, const int *kcol) {
  Handle *h = H(hh);
  PMG_TRACE_AT("enter");
  PMG_TRY(check_level(h, level));
  if (n_rows <= 0 || active_bound < 0 || active_bound > n_rows || !row_ptr || !kcol) {
    set_error("pmg_set_level_csr: bad sizes");
    return PMG_ERR_ARG;
  }
  if (row_ptr[0] != 0) { set_error("pmg_set_level_csr: row_ptr[0] != 0"); return PMG_ERR_ARG; }
  int nnz = row_ptr[n_rows];
  std::vector<int> dpos(n_rows, -1);
  for (int r = 0; r < n_rows; r++) {
    if (row_ptr[r + 1] < row_ptr[r]) { set_error("pmg_set_level_csr: row_ptr not monotone"); return PMG_ERR_ARG; }
    for (int k = row_ptr[r]; k < row_ptr[r + 1]; k++) {
      if (kcol[k] < 0 || kcol[k] >= n_rows) { set_error("pmg_set_level_csr: column out of range"); return PMG_ERR_ARG; }
      if (k > row_ptr[r] && kcol[k] <= kcol[k - 1]) {
        set_error("pmg_set_level_csr: columns must be sorted ascending (TSquareStructure3D::Sort)");
        return PMG_ERR_ARG;
      }
      if (kcol[k] == r) dpos[r] = k;
    }
    if (dpos[r] < 0) { set_error("pmg_set_level_csr: missing diagonal entry"); return PMG_ERR_ARG; }
  }
  PMG_TRACE_AT("validated");
  Level &L = h->lv[level];
  L.N = n_rows;
  L.Na = active_bound;
  L.nnz = nnz;
  L.avg_row = (int)(nnz / std::max(1, n_rows));
  PMG_TRY(L.rowptr.upload(row_ptr, n_rows + 1, h->stream));
  PMG_TRY(L.kcol.upload(kcol, nnz, h->stream));
  PMG_TRY(L.diagpos.upload(dpos.data(), n_rows, h->stream));
  PMG_TRY(L.A.alloc(nnz));
  PMG_TRY(L.rhs.alloc(n_rows));
  PMG_TRACE_AT("uploaded");
  PMG_CUDA(cudaMemsetAsync(L.A.p, 0, sizeof(double) * nnz, h->stream));
  PMG_CUDA(cudaMemsetAsync(L.rhs.p, 0, sizeof(double) * n_rows, h->stream));
  int ncol = 0;
  std::vector<int> color = color_rows(n_rows, active_bound, row_ptr, kcol, ncol);
  PMG_TRACE_AT("coloured");
  PMG_TRY(upload_row_colors(h, L, ncol, color));
  PMG_TRACE_AT("colours uploaded");
  L.h_rowptr.assign(row_ptr, row_ptr + n_rows + 1);
  L.h_kcol.assign(kcol, kcol + nnz);
  PMG_TRACE_AT("host copies");
  L.sell_ready = false;
  L.has_csr = true;
  L.has_mesh = false;
  L.slot.release();
  L.inc.release();
  L.inc_ptr.release();
  L.slot_g.release();
  L.assembled = false;
  h->coarse_ready = false;
  invalidate_graphs(h);
  PMG_TRACE_AT("done");
  return PMG_OK;
}

int pmg_set_level_row_colors(pmg_handle hh, int level, int n_colors, const int *colors) {
  Handle *h = H(hh);
  PMG_TRY(check_level(h, level));
  Level &L = h->lv[level];
  if (!L.has_csr || !colors || n_colors < 1) { set_error("pmg_set_level_row_colors: bad state/arguments"); return PMG_ERR_ARG; }
  // verify: no two coupled active rows share a colour
  const std::vector<int> &rp = L.h_rowptr, &kc = L.h_kcol;
  std::vector<int> c(colors, colors + L.N);
  for (int r = 0; r < L.Na; r++) {
    if (c[r] < 0 || c[r] >= n_colors) { set_error("pmg_set_level_row_colors: colour out of range"); return PMG_ERR_ARG; }
    for (int k = rp[r]; k < rp[r + 1]; k++)
      if (kc[k] != r && kc[k] < L.Na && c[kc[k]] == c[r]) {
        set_error("pmg_set_level_row_colors: coupled rows share a colour");
        return PMG_ERR_ARG;
      }
  }
  PMG_TRY(upload_row_colors(h, L, n_colors, c));
  invalidate_graphs(h);
  return PMG_OK;
}

int pmg_set_transfer(pmg_handle hh, int level, int n_fine, int n_coarse, const int *p_row_ptr, const int *p_col,
                     const double *p_val) {
  Handle *h = H(hh);
  PMG_TRY(check_level(h, level));
  if (level == 0) { set_error("pmg_set_transfer: level 0 has no coarser level"); return PMG_ERR_ARG; }
  Level &L = h->lv[level], &C = h->lv[level - 1];
  if (!L.has_csr || !C.has_csr || n_fine != L.N || n_coarse != C.N || !p_row_ptr || !p_col || !p_val) {
    set_error("pmg_set_transfer: sizes do not match the levels' CSR");
    return PMG_ERR_ARG;
  }
  int nnz = p_row_ptr[n_fine];
  for (int k = 0; k < nnz; k++)
    if (p_col[k] < 0 || p_col[k] >= n_coarse) { set_error("pmg_set_transfer: column out of range"); return PMG_ERR_ARG; }
  // R = P^T in CSR
  std::vector<int> rrp(n_coarse + 1, 0), rcol(nnz);
  std::vector<double> rval(nnz);
  for (int k = 0; k < nnz; k++) rrp[p_col[k] + 1]++;
  for (int c = 0; c < n_coarse; c++) rrp[c + 1] += rrp[c];
  std::vector<int> fp(rrp.begin(), rrp.end() - 1);
  for (int r = 0; r < n_fine; r++)
    for (int k = p_row_ptr[r]; k < p_row_ptr[r + 1]; k++) {
      int pos = fp[p_col[k]]++;
      rcol[pos] = r;
      rval[pos] = p_val[k];
    }
  PMG_TRY(L.prp.upload(p_row_ptr, n_fine + 1, h->stream));
  PMG_TRY(L.pcol.upload(p_col, nnz, h->stream));
  PMG_TRY(L.pval.upload(p_val, nnz, h->stream));
  PMG_TRY(L.rrp.upload(rrp.data(), n_coarse + 1, h->stream));
  PMG_TRY(L.rcol.upload(rcol.data(), nnz, h->stream));
  PMG_TRY(L.rval.upload(rval.data(), nnz, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  L.Nc = n_coarse;
  L.has_P = true;
  invalidate_graphs(h);
  return PMG_OK;
}

int pmg_set_dirichlet_values(pmg_handle hh, int level, const double *values) {
  Handle *h = H(hh);
  PMG_TRY(check_level(h, level));
  Level &L = h->lv[level];
  if (!L.has_csr) { set_error("pmg_set_dirichlet_values: set the CSR first"); return PMG_ERR_STATE; }
  int n = L.N - L.Na;
  if (n > 0) {
    if (!values) { set_error("pmg_set_dirichlet_values: null values"); return PMG_ERR_ARG; }
    for (int k = 0; k < n; k++)
      if (!std::isfinite(values[k])) { set_error("pmg_set_dirichlet_values: non-finite value"); return PMG_ERR_NONFINITE; }
    PMG_TRY(L.dirval.upload(values, n, h->stream));
    PMG_CUDA(cudaStreamSynchronize(h->stream));
  }
  return PMG_OK;
}

int pmg_set_coefficients(pmg_handle hh, const pmg_coeff_desc *c) {
  Handle *h = H(hh);
  if (!h || !c) return PMG_ERR_ARG;
  if (c->kind < PMG_COEF_CONST || c->kind > PMG_COEF_TABLE) { set_error("unknown coefficient kind"); return PMG_ERR_ARG; }
  double vals[7] = {c->eps, c->b[0], c->b[1], c->b[2], c->c, c->f, c->t};
  for (double v : vals)
    if (!std::isfinite(v)) { set_error("pmg_set_coefficients: non-finite coefficient"); return PMG_ERR_NONFINITE; }
  h->coeff = *c;
  if ((c->kind == PMG_COEF_LOGNORMAL || c->kind == PMG_COEF_CURL_FOURIER)) {
    if (c->n_modes <= 0 || !c->modes) { set_error("Fourier coefficient kinds need modes"); return PMG_ERR_ARG; }
    h->modes.assign(c->modes, c->modes + (size_t)8 * c->n_modes);
    for (double v : h->modes)
      if (!std::isfinite(v)) { set_error("pmg_set_coefficients: non-finite mode"); return PMG_ERR_NONFINITE; }
    PMG_TRY(h->d_modes.upload(h->modes.data(), h->modes.size(), h->stream));
    PMG_CUDA(cudaStreamSynchronize(h->stream));
  } else {
    h->coeff.n_modes = 0;
  }
  h->coeff.modes = nullptr;
  return PMG_OK;
}

static int assemble_one(Handle *h, int level, int form, double *entries_out, double *rhs_out) {
  Level &L = h->lv[level];
  bool mass = (form == PMG_FORM_MASS || form == PMG_FORM_MASS_SUPG);
  double *target;
  if (mass) {
    PMG_TRY(L.M.alloc(L.nnz));
    target = L.M.p;
  } else {
    target = L.A.p;
  }
  PMG_TRY(assemble_level(*h, L, form, target, true, L.rhs.p));
  PMG_TRY(set_dirichlet_rows(*h, L, target, L.rhs.p));
  if (mass && level == (int)h->lv.size() - 1) {
    // f(t_0) of the mass assembly is the first f_old of the theta scheme (AssembleMRhs)
    PMG_TRY(h->tcd_fold.alloc(L.N));
    PMG_CUDA(cudaMemcpyAsync(h->tcd_fold.p, L.rhs.p, sizeof(double) * L.N, cudaMemcpyDeviceToDevice, h->stream));
  }
  if (!mass) {
    L.assembled = true;
    L.sell_val_fresh32 = L.sell_val_fresh64 = false;
    L.lw_fresh = false;
    if (level == 0) h->coarse_ready = false;
  }
  if (entries_out) PMG_CUDA(cudaMemcpyAsync(entries_out, target, sizeof(double) * L.nnz, cudaMemcpyDeviceToHost, h->stream));
  if (rhs_out) PMG_CUDA(cudaMemcpyAsync(rhs_out, L.rhs.p, sizeof(double) * L.N, cudaMemcpyDeviceToHost, h->stream));
  return PMG_OK;  // pmg_assemble waits for the stream once, after every level
}

int pmg_assemble(pmg_handle hh, int level, int form, double *entries_out, double *rhs_out) {
  Handle *h = H(hh);
  if (!h) return PMG_ERR_ARG;
  if (level < -1 || level >= (int)h->lv.size()) { set_error("pmg_assemble: level out of range"); return PMG_ERR_ARG; }
  PMG_CUDA(cudaEventRecord(h->ev[0], h->stream));
  if (level >= 0) {
    PMG_TRY(assemble_one(h, level, form, entries_out, rhs_out));
  } else {
    for (int l = 0; l < (int)h->lv.size(); l++) PMG_TRY(assemble_one(h, l, form, nullptr, nullptr));
  }
  PMG_CUDA(cudaEventRecord(h->ev[1], h->stream));
  PMG_CUDA(cudaEventSynchronize(h->ev[1]));
  float ms = 0;
  PMG_CUDA(cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
  h->t_assemble = ms * 1e-3;
  return PMG_OK;
}

int pmg_get_matrix(pmg_handle hh, int level, int which, double *out) {
  Handle *h = H(hh);
  PMG_TRY(check_level(h, level));
  Level &L = h->lv[level];
  const double *src = which == 1 ? L.M.p : L.A.p;
  if (!src || !out) { set_error("pmg_get_matrix: nothing assembled"); return PMG_ERR_STATE; }
  PMG_CUDA(cudaMemcpyAsync(out, src, sizeof(double) * L.nnz, cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  return PMG_OK;
}

int pmg_set_matrix(pmg_handle hh, int level, int which, const double *in) {
  Handle *h = H(hh);
  PMG_TRY(check_level(h, level));
  Level &L = h->lv[level];
  if (!in || !L.has_csr) { set_error("pmg_set_matrix: bad state"); return PMG_ERR_ARG; }
  if (which == 1) { PMG_TRY(L.M.upload(in, L.nnz, h->stream)); }
  else {
    PMG_TRY(L.A.upload(in, L.nnz, h->stream));
    L.assembled = true;
    L.sell_val_fresh32 = L.sell_val_fresh64 = false;
    L.lw_fresh = false;
    if (level == 0) h->coarse_ready = false;
  }
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  return PMG_OK;
}

int pmg_get_rhs(pmg_handle hh, int level, double *out) {
  Handle *h = H(hh);
  PMG_TRY(check_level(h, level));
  if (!out) return PMG_ERR_ARG;
  Level &L = h->lv[level];
  PMG_CUDA(cudaMemcpyAsync(out, L.rhs.p, sizeof(double) * L.N, cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  return PMG_OK;
}

// ------------------------------------------------------------ host-array kernels
int pmg_matvec(pmg_handle hh, int level, const double *x, double *y) {
  Handle *h = H(hh);
  PMG_TRY(check_matrix(h, level, "pmg_matvec"));
  if (!x || !y) return PMG_ERR_ARG;
  Level &L = h->lv[level];
  DBuf<double> dx, dy;
  PMG_TRY(dx.upload(x, L.N, h->stream));
  PMG_TRY(dy.alloc(L.N));
  PMG_TRY(spmv<double>(h->stream, L, L.A.p, dx.p, dy.p));
  PMG_CUDA(cudaMemcpyAsync(y, dy.p, sizeof(double) * L.N, cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  return PMG_OK;
}

int pmg_defect(pmg_handle hh, int level, const double *x, const double *b, double *r, double *norm) {
  Handle *h = H(hh);
  PMG_TRY(check_matrix(h, level, "pmg_defect"));
  if (!x || !b || !r) return PMG_ERR_ARG;
  Level &L = h->lv[level];
  DBuf<double> dx, db, dr, dn;
  PMG_TRY(dx.upload(x, L.N, h->stream));
  PMG_TRY(db.upload(b, L.N, h->stream));
  PMG_TRY(dr.alloc(L.N));
  PMG_TRY(dn.alloc(1));
  PMG_TRY(defect<double>(h->stream, L, L.A.p, dx.p, db.p, dr.p));
  PMG_TRY(dot(*h, dr.p, dr.p, L.N, dn.p));
  double n2 = 0;
  PMG_CUDA(cudaMemcpyAsync(r, dr.p, sizeof(double) * L.N, cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaMemcpyAsync(&n2, dn.p, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  if (norm) *norm = sqrt(n2);
  return PMG_OK;
}

int pmg_ssor(pmg_handle hh, int level, const double *rhs, double *sol, int n_sweeps) {
  Handle *h = H(hh);
  PMG_TRY(check_matrix(h, level, "pmg_ssor"));
  if (!rhs || !sol || n_sweeps < 0) return PMG_ERR_ARG;
  Level &L = h->lv[level];
  PMG_TRY(level_invdiag(h->stream, L, h->d_flags.p));
  DBuf<double> df, dx;
  PMG_TRY(df.upload(rhs, L.N, h->stream));
  PMG_TRY(dx.upload(sol, L.N, h->stream));
  for (int k = 0; k < n_sweeps; k++)
    PMG_TRY(ssor_sweep<double>(h->stream, L, L.A.p, L.invdiag.p, df.p, dx.p, h->prm.smooth_omega));
  PMG_CUDA(cudaMemcpyAsync(sol, dx.p, sizeof(double) * L.N, cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  return PMG_OK;
}

int pmg_prolongate(pmg_handle hh, int level, const double *coarse, double *fine) {
  Handle *h = H(hh);
  PMG_TRY(check_level(h, level));
  Level &L = h->lv[level];
  if (!L.has_P || !coarse || !fine) { set_error("pmg_prolongate: no transfer"); return PMG_ERR_STATE; }
  // plain P c on every fine row (CorrectNodes is applied inside the V-cycle only)
  DBuf<double> dc, df;
  PMG_TRY(dc.upload(coarse, L.Nc, h->stream));
  PMG_TRY(df.alloc(L.N));
  PMG_CUDA(cudaMemsetAsync(df.p, 0, sizeof(double) * L.N, h->stream));
  Level tmp;  // view with Na = N so that every row is prolongated
  tmp.Na = L.N;
  tmp.prp.p = L.prp.p; tmp.pcol.p = L.pcol.p;
  int rc = prolongate_add<double>(h->stream, tmp, L.pval.p, dc.p, df.p, 1.0);
  tmp.prp.p = nullptr; tmp.pcol.p = nullptr;
  PMG_TRY(rc);
  PMG_CUDA(cudaMemcpyAsync(fine, df.p, sizeof(double) * L.N, cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  return PMG_OK;
}

int pmg_restrict(pmg_handle hh, int level, const double *fine, double *coarse) {
  Handle *h = H(hh);
  PMG_TRY(check_level(h, level));
  Level &L = h->lv[level];
  if (!L.has_P || !coarse || !fine) { set_error("pmg_restrict: no transfer"); return PMG_ERR_STATE; }
  DBuf<double> dfine, dc;
  PMG_TRY(dfine.upload(fine, L.N, h->stream));
  PMG_TRY(dc.alloc(L.Nc));
  Level tmpc;  // P^T d on every coarse row (CorrectDefect is applied inside the V-cycle only)
  tmpc.N = L.Nc;
  tmpc.Na = L.Nc;
  PMG_TRY(restrict_defect<double>(h->stream, L, tmpc, L.rval.p, dfine.p, dc.p));
  PMG_CUDA(cudaMemcpyAsync(coarse, dc.p, sizeof(double) * L.Nc, cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  return PMG_OK;
}

int pmg_solve(pmg_handle hh, double *sol, const double *rhs, pmg_solve_stats *stats) {
  Handle *h = H(hh);
  if (!h) return PMG_ERR_ARG;
  return pmg::solve(*h, sol, rhs, stats);
}

int pmg_get_solution(pmg_handle hh, double *out) {
  Handle *h = H(hh);
  if (!h || !out || !h->sol.p) return PMG_ERR_STATE;
  PMG_CUDA(cudaMemcpyAsync(out, h->sol.p, sizeof(double) * h->krylov_n, cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  return PMG_OK;
}

int pmg_last_timings(pmg_handle hh, double *assemble_s, double *solve_s, double *assemble_kernel_s) {
  Handle *h = H(hh);
  if (!h) return PMG_ERR_ARG;
  if (assemble_s) *assemble_s = h->t_assemble;
  if (solve_s) *solve_s = h->t_solve;
  if (assemble_kernel_s) *assemble_kernel_s = h->t_assemble_kernel;
  return PMG_OK;
}

int pmg_launch_count(unsigned long long *n) {
  if (!n) return PMG_ERR_ARG;
  *n = launches_so_far();
  return PMG_OK;
}

int pmg_time_kernel(pmg_handle hh, int kernel, int level, int form, int reps, double *sec, double *bytes,
                    double *flops) {
  Handle *h = H(hh);
  PMG_TRY(check_level(h, level));
  Level &L = h->lv[level];
  if (reps < 1 || !sec) return PMG_ERR_ARG;
  if (!L.assembled && kernel != PMG_KERNEL_ASSEMBLE) { set_error("pmg_time_kernel: assemble first"); return PMG_ERR_STATE; }
  const double N = L.N, nnz = L.nnz;
  // the solve copy's stored entries: 2-byte column deltas, 4-byte columns in
  // the slices whose deltas do not fit (known once the copy is built)
  double by = 0, fl = 0;
  DBuf<double> x64, y64;
  DBuf<float> x32, y32;
  cudaStream_t s = h->stream;
  auto run = [&]() -> int {
    switch (kernel) {
      case PMG_KERNEL_SPMV64: return sell_spmv<double>(s, L, x64.p, nullptr, y64.p, 0, h->num_sms);
      case PMG_KERNEL_SPMV32: return sell_spmv<float>(s, L, x32.p, nullptr, y32.p, 0, h->num_sms);
      case PMG_KERNEL_SSOR64: return sell_ssor<double>(s, L, y64.p, x64.p, 1.0, h->num_sms);
      case PMG_KERNEL_SSOR32: return sell_ssor<float>(s, L, y32.p, x32.p, 1.0, h->num_sms);
      case PMG_KERNEL_CSR_SPMV64: return spmv<double>(s, L, L.A.p, x64.p, y64.p);
      case PMG_KERNEL_ASSEMBLE: return assemble_level(*h, L, form, L.A.p, true, L.rhs.p);
      case PMG_KERNEL_COARSE_FACTOR: return coarse_factor(*h);
      case PMG_KERNEL_LEARNED_FWD: return learned_forward(*h, L);
      default: set_error("pmg_time_kernel: unknown kernel"); return PMG_ERR_ARG;
    }
  };
  if (kernel == PMG_KERNEL_SPMV64 || kernel == PMG_KERNEL_SSOR64 || kernel == PMG_KERNEL_CSR_SPMV64) {
    PMG_TRY(x64.alloc(L.N)); PMG_TRY(y64.alloc(L.N));
    PMG_TRY(fill(s, x64.p, 1.0, L.N)); PMG_TRY(fill(s, y64.p, 1.0, L.N));
    double spmv_b = 12 * nnz + 4 * (N + 1) + 16 * N;  // CSR: values + columns + row pointers + x once + y
    if (kernel != PMG_KERNEL_CSR_SPMV64) {
      PMG_TRY(sell_values<double>(*h, L));
      // SELL: values + column deltas / columns + slice pointers + row of each lane + x once + y
      spmv_b = 8.0 * (L.sell_nnz_narrow + L.sell_nnz_wide) + 2.0 * L.sell_nnz_narrow + 4.0 * L.sell_nnz_wide +
               4.0 * (L.sell_nslices + 1) + 4 * N + 16 * N;
    }
    by = kernel == PMG_KERNEL_SSOR64 ? 2 * spmv_b + 16 * N : spmv_b;
    fl = kernel == PMG_KERNEL_SSOR64 ? 4 * nnz : 2 * nnz;
  } else if (kernel == PMG_KERNEL_SPMV32 || kernel == PMG_KERNEL_SSOR32) {
    PMG_TRY(sell_values<float>(*h, L));
    PMG_TRY(x32.alloc(L.N)); PMG_TRY(y32.alloc(L.N));
    PMG_CUDA(cudaMemsetAsync(x32.p, 0, sizeof(float) * L.N, s));
    PMG_CUDA(cudaMemsetAsync(y32.p, 0, sizeof(float) * L.N, s));
    double spmv_b = 4.0 * (L.sell_nnz_narrow + L.sell_nnz_wide) + 2.0 * L.sell_nnz_narrow + 4.0 * L.sell_nnz_wide +
                    4.0 * (L.sell_nslices + 1) + 4 * N + 8 * N;
    by = kernel == PMG_KERNEL_SPMV32 ? spmv_b : 2 * spmv_b + 8 * N;
    fl = kernel == PMG_KERNEL_SPMV32 ? 2 * nnz : 4 * nnz;
  } else if (kernel == PMG_KERNEL_COARSE_FACTOR) {
    if (level != 0) { set_error("pmg_time_kernel: the coarse factorisation is of level 0"); return PMG_ERR_ARG; }
    // LU (2/3 n^3) and inverse (4/3 n^3) flops; the dense matrix is read and written
    by = 2.0 * 8.0 * N * N;
    fl = 2.0 * N * N * N;
  } else if (kernel == PMG_KERNEL_LEARNED_FWD) {
    if (!h->has_learned || L.lat_n[0] <= 0) {
      set_error("pmg_time_kernel: the learned forward needs weights and the level's lattice");
      return PMG_ERR_STATE;
    }
    // per lattice node: the CSR row (12 B per entry), three BF16 layer inputs and
    // outputs (64 B each way), the FP32 stencil (27 x 4 B)
    const double NL = (double)L.lat_n[0] * L.lat_n[0] * L.lat_n[0];
    by = 12.0 * nnz + NL * (3 * 128.0 + 108.0);
    fl = 2.0 * 27 * (27 * 32 + 32 * 32 + 32 * 27) * NL;
  } else {
    // coloured scatter per element: n_loc^2 (4 slot + 8 read + 8 write) + n_loc (4 dof + 16 rhs) + vertices
    const double nl = L.nloc, nv = L.nvert;
    by = L.n_cells * (nl * nl * 20 + nl * 20 + nv * 4 + nv * 24);
    const double nq = L.elem == PMG_ELEM_Q1_HEX ? 8 : (L.elem == PMG_ELEM_Q2_HEX || L.elem == PMG_ELEM_NQ1_HEX) ? 27
                    : L.elem == PMG_ELEM_P1_TET ? 4 : 11;
    fl = L.n_cells * (nq * nl * nl * 8 + nq * nl * 32);  // 4 FMA per (q,i,j) + D_q u_j (16 FMA per q,j)
  }
  PMG_TRY(run());  // warm-up
  if (kernel == PMG_KERNEL_ASSEMBLE) {
    // flops of the contraction the chosen kernel does
    const double nn = (double)L.nloc * L.nloc;
    if (h->asm_path <= 1) fl = L.n_cells * nn * 2.0 * h->asm_kd;
    else if (h->asm_path == 2) fl = L.n_cells * nn * 2.0 * 16;
  }
  PMG_CUDA(cudaEventRecord(h->ev[4], s));
  for (int r = 0; r < reps; r++) PMG_TRY(run());
  PMG_CUDA(cudaEventRecord(h->ev[5], s));
  PMG_CUDA(cudaEventSynchronize(h->ev[5]));
  float ms = 0;
  PMG_CUDA(cudaEventElapsedTime(&ms, h->ev[4], h->ev[5]));
  *sec = ms * 1e-3 / reps;
  if (bytes) *bytes = by;
  if (flops) *flops = fl;
  if (kernel == PMG_KERNEL_ASSEMBLE) {
    L.sell_val_fresh32 = L.sell_val_fresh64 = false;
    L.lw_fresh = false;
    PMG_TRY(set_dirichlet_rows(*h, L, L.A.p, L.rhs.p));
    PMG_CUDA(cudaStreamSynchronize(s));
  }
  return PMG_OK;
}

}  // extern "C"
