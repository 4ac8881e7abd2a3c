// Internal declarations of the B200 ParMooN CD3D library (not part of the ABI).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/pmg_b200.h"

namespace pmg {

// ------------------------------------------------------------- errors
void set_error(const std::string &msg);
// kernel-launch accounting (pmg_launch_count)
void count_launches(unsigned long long n);
unsigned long long launches_so_far();
#define PMG_CUDA(call)                                                            \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      pmg::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));         \
      return PMG_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)
#define PMG_TRY(call)                                                             \
  do {                                                                            \
    int r_ = (call);                                                              \
    if (r_ != PMG_OK) return r_;                                                  \
  } while (0)

// ------------------------------------------------------------- programmatic dependent launch
// Kernels of the solve are launched with programmatic stream serialization:
// a kernel may be scheduled while its predecessor drains and waits in
// pdl_wait() (griddepcontrol.wait, sm_90+) until the predecessor has completed
// and its writes are visible, so nothing is read or written before that.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_wait() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}
__device__ __forceinline__ void pdl_trigger() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}
template <typename... KArgs, typename... Args>
static inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                     Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}
#endif

// ------------------------------------------------------------- device buffers
template <typename T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  int alloc(size_t count) {
    if (count == n && p) return PMG_OK;
    release();
    if (count == 0) return PMG_OK;
    PMG_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
    return PMG_OK;
  }
  // grow only: keep the buffer when it already holds count elements
  int reserve(size_t count) {
    if (p && n >= count) return PMG_OK;
    return alloc(count);
  }
  int upload(const T *h, size_t count, cudaStream_t s) {
    PMG_TRY(alloc(count));
    if (count) PMG_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    return PMG_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { release(); }
};

// element descriptors
struct ElemInfo {
  int nloc, nvert, quad_default;
};
ElemInfo elem_info(int elem_type);

// one multigrid level
struct Level {
  // sizes
  int N = 0, Na = 0, nnz = 0, n_cells = 0, elem = 0, nloc = 0, nvert = 0, brick = 0;
  bool has_mesh = false, has_csr = false, has_P = false, assembled = false;
  // CSR pattern (rows sorted)
  DBuf<int> rowptr, kcol, diagpos;
  // matrices: A (system), M (mass, time-dependent), A32 (FP32 copy for the V-cycle)
  DBuf<double> A, M, Astash;
  DBuf<float> A32;
  DBuf<double> invdiag;
  DBuf<float> invdiag32;
  // rhs / Dirichlet values
  DBuf<double> rhs, dirval;
  // mesh in element-colour order
  DBuf<int> elem_dof;       // n_cells x nloc
  DBuf<double> cell_vert;   // n_cells x nvert x 3
  DBuf<int> slot;           // n_cells x nloc x nloc
  // row gather: the cells holding each dof, as e * nloc + (local index), in
  // cell (= colour) order; inc_ptr has N + 1 entries; slot_g[p][j] = the slot
  // map's row li of cell e at list position p; rmax = longest CSR row
  DBuf<int> inc_ptr, inc, slot_g;
  int rmax = 0;
  std::vector<int> ecolor_ptr;  // element colour classes [ecolor_ptr[c], ecolor_ptr[c+1])
  std::vector<int> cell_order;  // colour-sorted position -> caller's cell index
  // tabulated coefficients (PMG_COEF_TABLE): n_cells x ctab_nq x 6, colour order
  DBuf<double> ctab;
  int ctab_nq = 0;
  // multicolour SSOR row lists (active rows only), grouped by colour
  DBuf<int> row_list;
  std::vector<int> rcolor_ptr;
  // transfer from level-1: P (N x Nc), R = P^T (Nc x N)
  int Nc = 0;
  DBuf<int> prp, pcol, rrp, rcol;
  DBuf<double> pval, rval;
  DBuf<float> pval32, rval32;
  // work vectors of the V-cycle (FP64 and FP32)
  DBuf<double> x64, f64, d64;
  DBuf<float> x32, f32, d32;
  // step-length control (old iterate, old defect, A times the update) and the
  // Jacobi step's new iterate
  DBuf<double> slc64[3], jac64;
  DBuf<float> slc32[3], jac32;
  // lattice and stencil of the learned smoother (learned.cu)
  int lat_n[3] = {0, 0, 0};
  DBuf<int> dof_ijk, lat_dof, tpos;
  DBuf<float> lw_stencil;
  bool lw_fresh = false;
  // average row length (SpMV launch shape)
  int avg_row = 0;
  // host copies of the pattern and of the colour row lists (SELL set-up)
  std::vector<int> h_rowptr, h_kcol, h_row_list;
  // SELL-32 copy for the solve (see sell.cu)
  bool sell_ready = false, sell_val_fresh32 = false, sell_val_fresh64 = false;
  int sell_nslices = 0;
  long sell_nnz = 0;
  std::vector<int> sell_group;  // slice range of each colour group (+ Dirichlet group)
  DBuf<int> sell_perm, sell_ptr, sell_col;
  // solve copy of an active row = its columns < Na (a prefix: columns are
  // sorted); the Dirichlet columns are applied separately (dd_row / dd_beg)
  DBuf<short> sell_c16;          // column - the lane's row, for slices whose deltas fit 16 bits
  DBuf<unsigned char> sell_wide; // 1: the slice keeps 32-bit columns (sell_col)
  DBuf<int> sell_alen;           // entries of each row in the solve copy
  DBuf<int> dd_row, dd_beg;      // active rows with Dirichlet columns, first such CSR position
  int n_dd = 0;
  long sell_nnz_narrow = 0, sell_nnz_wide = 0;  // stored entries with 16-bit / 32-bit columns
  DBuf<float> sell_val32, sell_invd32;
  DBuf<double> sell_val64, sell_invd64;
};

// Activations of the stencil network.  The tensor-core forward reads and
// writes node-major BF16 (32 channels = 64 bytes per lattice node, two
// ping-pong buffers); training also keeps FP32 channel-major copies of every
// layer's input (the BF16-rounded values) and pre-activations for the
// backward kernels.
struct NetScratch {
  DBuf<uint16_t> xa, xb, wpk;
  DBuf<float> feat, a1, z1, a2, z2, dscale;
  // grow-only: the levels of a hierarchy share the buffers of the largest
  int alloc(int nl, int c0, int c1, int c2, bool train) {
    PMG_TRY(xa.reserve((size_t)32 * nl));
    PMG_TRY(xb.reserve((size_t)32 * nl));
    PMG_TRY(dscale.reserve(nl));
    PMG_TRY(wpk.reserve((size_t)3 * 27 * 32 * 32));
    if (train) {
      PMG_TRY(feat.reserve((size_t)c0 * nl));
      PMG_TRY(a1.reserve((size_t)c1 * nl));
      PMG_TRY(z1.reserve((size_t)c1 * nl));
      PMG_TRY(a2.reserve((size_t)c2 * nl));
      PMG_TRY(z2.reserve((size_t)c2 * nl));
    }
    return PMG_OK;
  }
};

struct Handle {
  pmg_params prm;
  pmg_coeff_desc coeff{};
  std::vector<double> modes;
  DBuf<double> d_modes;
  std::vector<Level> lv;
  cudaStream_t stream = nullptr;
  // auxiliary stream: the coarsest-level factorisation overlaps the per-solve set-up
  cudaStream_t aux = nullptr;
  cudaEvent_t aux_ev[2] = {nullptr, nullptr};
  DBuf<int> coarse_flags;
  int *h_coarse_flags = nullptr;  // page-locked, 4 ints
  int device = 0;
  int num_sms = 148;
  // coarsest-level dense inverse (FP64)
  DBuf<double> coarse_lu, coarse_inv, coarse_t;  // active block: LU, inverse; reduced rhs
  DBuf<int> coarse_piv, coarse_perm;
  DBuf<int> coarse_cptr;  // colour pointers of the coarsest level's rows (iterative coarse solve)
  bool coarse_ready = false;
  // FGMRES workspace
  int krylov_n = 0, krylov_restart = 0;
  DBuf<double> V, Z, w, sol, rhs, H, scal;
  DBuf<double> red_partial;
  DBuf<double> slc_part;  // step-length control: block partials of (d0, y), (y, y) and alpha
  DBuf<unsigned int> red_counter;
  double *h_H = nullptr;  // pinned mirror of one Hessenberg column
  // error flags written by kernels (slot lookups, non-finite values)
  DBuf<int> d_flags;
  // timing
  cudaEvent_t ev[10];
  double t_assemble = 0, t_solve = 0, t_assemble_kernel = 0;
  // kernel of the last assemble_level: 0 tensor-core (space-constant
  // coefficients), 1 tensor-core (pure diffusion), 2 reference matrices on
  // CUDA cores, 3 per quadrature point; asm_kd: contraction length of 0 / 1
  int asm_path = 3, asm_kd = 0;
  // wall times of the last pmg_build_level_csr: pattern on the device (upload
  // included), install (checks, colouring, host mirror)
  double t_setup_csr_device = 0, t_setup_csr_install = 0;
  // per-cell coefficients (16) and local rhs of the space-constant tensor-core assembly
  DBuf<double> tc_dbuf, tc_rbuf;
  DBuf<double> asm_ae, asm_rloc;  // local matrices / rhs of the row-gather assembly
  // V-cycle graph
  cudaGraphExec_t vgraph = nullptr;
  int vgraph_prec = -1;
  unsigned long long vgraph_kernels = 0;
  bool use_graph = true;  // PMG_NO_GRAPH=1 launches the V-cycle kernels directly (profilers)
  int cc_top = 0;         // levels 0..cc_top run as one launch (0: none)
  DBuf<int> cc_err;      // set by the one-launch coarse cycle when a bounded wait gives up
  int cc_ctas = 0;        // CTAs of that launch (1, or a cluster of up to 16)
  // learned smoother: BF16 weights used by the kernels, FP32 master copy, Adam state
  DBuf<uint16_t> lw_bf16;
  DBuf<float> lw_master, lw_grad, lw_m, lw_v;
  bool has_learned = false;
  long adam_t = 0;
  NetScratch net_scratch;
  // learned-smoother guard: V-cycle graph with SSOR, active choice
  cudaGraphExec_t vgraph_ssor = nullptr;
  unsigned long long vgraph_ssor_kernels = 0;
  // halo of a subdomain (solve_dd): owned dofs packed for the neighbours, ghost rows
  // filled from them; the packing buffers belong to the caller's transport
  bool halo_set = false;
  int halo_nsend = 0, halo_nrecv = 0;
  DBuf<int> halo_send_idx, halo_recv_idx;
  double *halo_send_buf = nullptr, *halo_recv_buf = nullptr;
  // time-dependent state (tcd.cu): previous rhs, start vector preset, system assembled
  DBuf<double> tcd_fold;
  bool sol_preset = false, tcd_active = false;
};

// the level exists and its system matrix holds values (assembled or set)
int check_matrix(Handle *h, int level, const char *who);

// ------------------------------------------------------------- kernels (assemble.cu)
int build_slot_map(Handle &h, Level &L);
int scan_exclusive(cudaStream_t s, int n, const int *in, int *out);
int assemble_level(Handle &h, Level &L, int form, double *target, bool zero_rhs, double *rhs_target);
int set_dirichlet_rows(Handle &h, Level &L, double *target, double *rhs_target);

// ------------------------------------------------------------- kernels (sparse.cu)
template <typename T>
int spmv(cudaStream_t s, const Level &L, const T *A, const T *x, T *y);
template <typename T>
int defect(cudaStream_t s, const Level &L, const T *A, const T *x, const T *f, T *d);
template <typename T>
int ssor_sweep(cudaStream_t s, const Level &L, const T *A, const T *invdiag, const T *f, T *x, double omega);
template <typename T>
int restrict_defect(cudaStream_t s, const Level &Lf, const Level &Lc, const T *rval, const T *d, T *fc, T *xc = nullptr);
template <typename T>
int prolongate_add(cudaStream_t s, const Level &Lf, const T *pval, const T *xc, T *xf, double damp);
int convert_f64_f32(cudaStream_t s, const double *a, float *b, size_t n);
int copy_dirichlet(cudaStream_t s, int Na, int N, const double *f, double *x);
int dot(Handle &h, const double *a, const double *b, size_t n, double *result_dev);
// w -= (*hk_dev) vk, then *h_next = w . u (u = w: the squared norm)
int mgs_step(Handle &h, size_t n, const double *hk_dev, const double *vk, const double *u, double *w, double *h_next);
int scale_by_inv_sqrt(cudaStream_t s, size_t n, const double *nrm2_dev, const double *x, double *y);
int fill(cudaStream_t s, double *x, double v, size_t n);
template <typename T>
int zero(cudaStream_t s, T *x, size_t n);
int check_finite(cudaStream_t s, const double *x, size_t n, int *flag);

// ------------------------------------------------------------- SELL-32 (sell.cu)
int build_sell(Handle &h, Level &L);
template <typename T>
int sell_values(Handle &h, Level &L);
template <typename T>
int sell_spmv(cudaStream_t s, const Level &L, const T *x, const T *f, T *y, int mode, int num_sms);
template <typename T>
int sell_ssor(cudaStream_t s, const Level &L, const T *f, T *x, double omega, int num_sms, bool dirichlet = true,
              bool after_ssor = false, bool skip_repeats = false, bool forward_only = false);
// one damped Jacobi step; tmp: a level-sized work vector other than x and f
template <typename T>
int sell_jacobi(cudaStream_t s, const Level &L, const T *f, T *x, T *tmp, double omega, int num_sms, bool dirichlet);
// y_a -= A_aD v_D (add: y_a += A_aD v_D) over the active rows' Dirichlet
// columns (the part of A the solve copy leaves out)
template <typename T>
int dirichlet_cols(cudaStream_t s, const Level &L, const T *v, T *y, bool add = false);

// ------------------------------------------------------------- solver (solver.cu)
int coarse_factor(Handle &h);
int solve(Handle &h, double *sol_host, const double *rhs_host, pmg_solve_stats *st);

// ------------------------------------------------------------- learned smoother (learned.cu)
int learned_num_params();
int learned_prepare(Handle &h);
// the network's forward on one level (stencil into L.lw_stencil)
int learned_forward(Handle &h, Level &L);
template <typename T>
int learned_smooth(cudaStream_t s, const Level &L, const T *r, T *x, double omega);

// drop the captured V-cycle graphs (their shape changed)
void invalidate_graphs(Handle *h);

// the coarse end of the V-cycle in one thread-block-cluster launch (coarse_cycle.cu)
int coarse_cycle_top(Handle &h);
// PMG_ERR_STATE (and the flag cleared) when a wait of the one-launch coarse cycle gave up
int coarse_cycle_check(Handle &h);
template <typename T>
int coarse_cycle(Handle &h, int top);

}  // namespace pmg
