// Geometric multigrid V-cycle and flexible GMRES on the device.
//
//   vcycle          TMultiGrid3D::Cycle (src/FE/MultiGrid3D.C:449-695) with
//                   step-length control off; FP64 or FP32 storage/compute
//   coarse solve    SolveExact (src/FE/MGLevel3D.C:865-906): dense LU with
//                   partial pivoting of the coarsest matrix, turned into an
//                   explicit inverse so each V-cycle applies one dense GEMV
//   preconditioner  TMultiGridScaIte::Iterate (src/FE/MultiGridScaIte.C:89-130)
//   fgmres          TFgmresIte::Iterate, flexible branch (src/FE/FgmresIte.C:245-624):
//                   right preconditioning, modified Gram-Schmidt, Givens rotations.
//                   Dots, axpys and normalisation run on the device with the
//                   Hessenberg entries kept in device memory; the host reads one
//                   column per iteration for the rotations and the stop test.
//
// The V-cycle is captured once per solve into a CUDA graph and replayed for
// every preconditioner application (hundreds of small colour launches).
#include "pmg_internal.h"
#include <algorithm>
#include <cmath>
#include <vector>

namespace pmg {

int level_invdiag(cudaStream_t s, Level &L, int *flags);

// ----------------------------------------------------------------- coarse LU
// Blocked right-looking LU with partial pivoting (panel width LU_NB), row-major
// n x n in global memory:
//   k_lu_panel   one block factors the (n-k0) x nb panel held in shared memory
//   k_lu_swap    applies the panel's row interchanges to the other columns
//   k_lu_trsm    U12 = L11^{-1} A12 (one thread per column)
//   k_lu_gemm    A22 -= L21 U12 (32 x 32 output tiles)
// then the inverse is formed in one launch (k_lu_inverse_slab, below).
constexpr int LU_NB = 32;
constexpr int LU_MAX_N = 832;  // panel (n x 33 doubles) must fit in 227 KB of shared memory

__global__ void __launch_bounds__(1024) k_lu_panel(int n, int k0, int nb, double *A, int *piv, int *flags) {
  extern __shared__ double S[];  // m x nb, row-major with stride nb + 1 (column reads hit distinct banks)
  __shared__ double sval[32];
  __shared__ int sidx[32];
  __shared__ int spiv;
  const int m = n - k0, tid = threadIdx.x, nt = blockDim.x, ld = nb + 1;
  for (int t = tid; t < m * nb; t += nt) S[(t / nb) * ld + t % nb] = A[(size_t)(k0 + t / nb) * n + k0 + t % nb];
  __syncthreads();
  for (int j = 0; j < nb; j++) {
    double best = -1.0;
    int bi = j;
    for (int i = j + tid; i < m; i += nt) {
      double v = fabs(S[i * ld + j]);
      if (v > best) { best = v; bi = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_xor_sync(0xffffffffu, best, o);
      int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
    }
    if ((tid & 31) == 0) { sval[tid >> 5] = best; sidx[tid >> 5] = bi; }
    __syncthreads();
    if (tid < 32) {
      double b = tid < (nt >> 5) ? sval[tid] : -1.0;
      int p = tid < (nt >> 5) ? sidx[tid] : j;
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, b, o);
        const int op = __shfl_xor_sync(0xffffffffu, p, o);
        if (ob > b || (ob == b && op < p)) { b = ob; p = op; }
      }
      if (tid == 0) {
        spiv = p;
        piv[k0 + j] = k0 + p;
        if (!(b > 0.0)) atomicOr(flags, 16);
      }
    }
    __syncthreads();
    const int p = spiv;
    if (p != j && tid < nb) {
      double t = S[j * ld + tid];
      S[j * ld + tid] = S[p * ld + tid];
      S[p * ld + tid] = t;
    }
    __syncthreads();
    const double d = S[j * ld + j];
    const double inv = d != 0.0 ? 1.0 / d : 0.0;
    for (int i = j + 1 + tid; i < m; i += nt) S[i * ld + j] *= inv;
    __syncthreads();
    // rank-1 update of the panel: lane = column to the right, warp = row group
    const int w = nb - j - 1, cc = tid & 31, rg = tid >> 5, ng = nt >> 5;
    if (cc < w) {
      const double u = S[j * ld + j + 1 + cc];
      for (int i = j + 1 + rg; i < m; i += ng) S[i * ld + j + 1 + cc] -= S[i * ld + j] * u;
    }
    __syncthreads();
  }
  for (int t = tid; t < m * nb; t += nt) A[(size_t)(k0 + t / nb) * n + k0 + t % nb] = S[(t / nb) * ld + t % nb];
}

// row interchanges of panel k0 on the columns outside the panel
__global__ void k_lu_swap(int n, int k0, int nb, double *A, const int *__restrict__ piv) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n || (c >= k0 && c < k0 + nb)) return;
  for (int j = 0; j < nb; j++) {
    const int p = piv[k0 + j];
    if (p != k0 + j) {
      double t = A[(size_t)(k0 + j) * n + c];
      A[(size_t)(k0 + j) * n + c] = A[(size_t)p * n + c];
      A[(size_t)p * n + c] = t;
    }
  }
}

// U12 = L11^{-1} A12 for the columns right of the panel
__global__ void k_lu_trsm(int n, int k0, int nb, double *A) {
  __shared__ double L11[LU_NB][LU_NB];
  for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) L11[t / nb][t % nb] = A[(size_t)(k0 + t / nb) * n + k0 + t % nb];
  __syncthreads();
  const int c = k0 + nb + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double y[LU_NB];
#pragma unroll
  for (int i = 0; i < LU_NB; i++) y[i] = i < nb ? A[(size_t)(k0 + i) * n + c] : 0.0;
#pragma unroll
  for (int i = 1; i < LU_NB; i++)
#pragma unroll
    for (int j = 0; j < LU_NB; j++)
      if (j < i && i < nb) y[i] -= L11[i][j] * y[j];
#pragma unroll
  for (int i = 0; i < LU_NB; i++)
    if (i < nb) A[(size_t)(k0 + i) * n + c] = y[i];
}

// A22 -= L21 U12 on 32 x 32 tiles (k0+nb <= row, col < n)
__global__ void __launch_bounds__(256) k_lu_gemm(int n, int k0, int nb, double *A) {
  __shared__ double Ls[32][LU_NB + 1], Us[LU_NB][33];
  const int r0 = k0 + nb + blockIdx.y * 32, c0 = k0 + nb + blockIdx.x * 32;
  for (int t = threadIdx.x; t < 32 * LU_NB; t += blockDim.x) {
    const int a = t / LU_NB, b = t % LU_NB;
    Ls[a][b] = (r0 + a < n && b < nb) ? A[(size_t)(r0 + a) * n + k0 + b] : 0.0;
    const int u = t / 32, v = t % 32;
    Us[u][v] = (u < nb && c0 + v < n) ? A[(size_t)(k0 + u) * n + c0 + v] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;  // 8 rows per pass
  for (int a = ty; a < 32; a += 8) {
    const int r = r0 + a, c = c0 + tx;
    if (r >= n || c >= n) continue;
    double s = 0.0;
#pragma unroll 8
    for (int k = 0; k < LU_NB; k++) s += Ls[a][k] * Us[k][tx];
    A[(size_t)r * n + c] -= s;
  }
}

// Inverse from the factors, X = U^{-1} L^{-1} P: block b of the grid owns
// the 32 columns [32 b, 32 b + 32) of X and keeps that n x 32 slab in shared
// memory through both substitutions (left-looking: row i of the slab is
// finished from the rows already final, L / U streamed from L2), so the whole
// inverse is one launch; lane = column, warps take rows.
__global__ void k_lu_perm_identity(int n, const int *__restrict__ piv, int *perm) {
  // perm[i] = original row that the interchanges bring to position i
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int i = 0; i < n; i++) perm[i] = i;
    for (int k = 0; k < n; k++) {
      const int p = piv[k];
      if (p != k) { int t = perm[k]; perm[k] = perm[p]; perm[p] = t; }
    }
  }
}

constexpr int INV_COLS = 16, INV_THREADS = 256, INV_ROWS = INV_THREADS / INV_COLS;
__global__ void __launch_bounds__(INV_THREADS) k_lu_inverse_slab(int n, const double *__restrict__ LU,
                                                                const int *__restrict__ perm, double *Inv) {
  extern __shared__ double sm[];
  double *Xs = sm;           // n x INV_COLS, the block's columns of X
  double *Rb = sm + (size_t)n * INV_COLS;  // INV_ROWS rows of L or U, staged
  const int tid = threadIdx.x, rr = tid / INV_COLS, col = tid % INV_COLS;
  const int warp = tid >> 5, lane = tid & 31, nwarps = INV_THREADS / 32;
  const int c = blockIdx.x * INV_COLS + col;
  for (int i = rr; i < n; i += INV_ROWS) Xs[i * INV_COLS + col] = (c < n && __ldg(perm + i) == c) ? 1.0 : 0.0;
  // forward with the unit lower factor, INV_ROWS rows per group
  for (int i0 = 0; i0 < n; i0 += INV_ROWS) {
    const int rows = min(INV_ROWS, n - i0), width = i0 + rows;
    __syncthreads();
    for (int r = warp; r < rows; r += nwarps)
      for (int k = lane; k < width; k += 32) Rb[r * width + k] = __ldg(LU + (size_t)(i0 + r) * n + k);
    __syncthreads();
    double s = 0.0;
    if (rr < rows) {
      const double *Lr = Rb + rr * width;
      double s1 = 0.0;
      int k = 0;
      for (; k + 2 <= i0; k += 2) {
        s += Lr[k] * Xs[k * INV_COLS + col];
        s1 += Lr[k + 1] * Xs[(k + 1) * INV_COLS + col];
      }
      if (k < i0) s += Lr[k] * Xs[k * INV_COLS + col];
      s += s1;
    }
    for (int r = 0; r < rows; r++) {
      if (rr == r) {
        const double *Lr = Rb + r * width;
        double t = Xs[(i0 + r) * INV_COLS + col] - s;
        for (int k = i0; k < i0 + r; k++) t -= Lr[k] * Xs[k * INV_COLS + col];
        Xs[(i0 + r) * INV_COLS + col] = t;
      }
      __syncthreads();
    }
  }
  // backward with the upper factor, from the last rows
  for (int i1 = n; i1 > 0; i1 -= INV_ROWS) {
    const int lo = max(0, i1 - INV_ROWS), rows = i1 - lo, width = n - lo;
    __syncthreads();
    for (int r = warp; r < rows; r += nwarps)
      for (int k = lane; k < width; k += 32) Rb[r * width + k] = __ldg(LU + (size_t)(lo + r) * n + lo + k);
    __syncthreads();
    const int i = i1 - 1 - rr;  // the row this thread sums for
    double s = 0.0;
    if (rr < rows) {
      const double *Ur = Rb + (i - lo) * width - lo;  // Ur[k] = U[i][k] for k >= lo
      double s1 = 0.0;
      int k = i1;
      for (; k + 2 <= n; k += 2) {
        s += Ur[k] * Xs[k * INV_COLS + col];
        s1 += Ur[k + 1] * Xs[(k + 1) * INV_COLS + col];
      }
      if (k < n) s += Ur[k] * Xs[k * INV_COLS + col];
      s += s1;
    }
    for (int r = 0; r < rows; r++) {
      const int row = i1 - 1 - r;
      if (rr == r) {
        const double *Ur = Rb + (row - lo) * width - lo;
        double t = Xs[row * INV_COLS + col] - s;
        for (int k = row + 1; k < i1; k++) t -= Ur[k] * Xs[k * INV_COLS + col];
        Xs[row * INV_COLS + col] = t / Ur[row];
      }
      __syncthreads();
    }
  }
  if (c < n)
    for (int i = rr; i < n; i += INV_ROWS) Inv[(size_t)i * n + c] = Xs[i * INV_COLS + col];
}

// the coarsest level's rhs reduced to its active rows: t = f_a - A_ad f_d
// (rows >= Na are Dirichlet: x_d = f_d); one warp per row
template <typename T>
__global__ void __launch_bounds__(256) k_coarse_rhs(int n, int na, const int *__restrict__ rp, const int *__restrict__ kc,
                                                    const double *__restrict__ a, const T *__restrict__ f, double *t,
                                                    T *x) {
  pdl_wait();
  pdl_trigger();
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  if (warp >= na) {
    if (lane == 0) x[warp] = f[warp];
    return;
  }
  double s = 0.0;
  for (int k = rp[warp] + lane; k < rp[warp + 1]; k += 32) {
    const int j = kc[k];
    if (j >= na) s += a[k] * (double)f[j];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) t[warp] = (double)f[warp] - s;
}

// x_a = Inv t (dense GEMV in FP64 over the active rows; x in T)
template <typename T>
__global__ void __launch_bounds__(256) k_dense_apply(int na, const double *__restrict__ Inv, const double *__restrict__ t,
                                                     T *x) {
  pdl_wait();
  pdl_trigger();
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= na) return;
  double s = 0;
  for (int j = lane; j < na; j += 32) s += Inv[(size_t)warp * na + j] * t[j];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) x[warp] = (T)s;
}

// dense active block of the coarsest matrix (rows and columns < na)
__global__ void k_csr_to_dense_active(int na, const int *__restrict__ rp, const int *__restrict__ kc,
                                      const double *__restrict__ a, double *D) {
  int i = blockIdx.x;
  if (i >= na) return;
  for (int j = threadIdx.x; j < na; j += blockDim.x) D[(size_t)i * na + j] = 0.0;
  __syncthreads();
  for (int k = rp[i] + threadIdx.x; k < rp[i + 1]; k += blockDim.x)
    if (kc[k] < na) D[(size_t)i * na + kc[k]] = a[k];
}

// the launches of the factorisation on stream s; the pivot flags are copied
// to h.h_coarse_flags (page-locked) on s, read by coarse_factor_finish
static int coarse_factor_launch(Handle &h, cudaStream_t s) {
  Level &L = h.lv[0];
  // Dirichlet rows are identity rows, so only the active block is factored:
  // x_a = A_aa^{-1} (f_a - A_ad f_d), x_d = f_d
  const int n = L.Na;
  if (n > LU_MAX_N) {
    set_error("coarsest level has too many active rows for the dense direct solve (> 832); use the SSOR coarse smoother");
    return PMG_ERR_UNSUPPORTED;
  }
  PMG_TRY(h.coarse_t.alloc(std::max(n, 1)));
  if (n == 0) {
    h.h_coarse_flags[0] = 0;
    return PMG_OK;
  }
  PMG_TRY(h.coarse_lu.alloc((size_t)n * n));
  PMG_TRY(h.coarse_inv.alloc((size_t)n * n));
  PMG_TRY(h.coarse_piv.alloc(n));
  PMG_CUDA(cudaMemsetAsync(h.coarse_flags.p, 0, sizeof(int) * 4, s));
  k_csr_to_dense_active<<<n, 256, 0, s>>>(n, L.rowptr.p, L.kcol.p, L.A.p, h.coarse_lu.p); count_launches(1);
  static bool attr = false;
  if (!attr) {
    PMG_CUDA(cudaFuncSetAttribute(k_lu_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, LU_MAX_N * (LU_NB + 1) * 8));
    PMG_CUDA(cudaFuncSetAttribute(k_lu_inverse_slab, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  LU_MAX_N * 2 * INV_COLS * 8));
    attr = true;
  }
  for (int k0 = 0; k0 < n; k0 += LU_NB) {
    const int nb = std::min(LU_NB, n - k0);
    k_lu_panel<<<1, 1024, (size_t)(n - k0) * (nb + 1) * 8, s>>>(n, k0, nb, h.coarse_lu.p, h.coarse_piv.p, h.coarse_flags.p);
    k_lu_swap<<<(n + 255) / 256, 256, 0, s>>>(n, k0, nb, h.coarse_lu.p, h.coarse_piv.p);
    count_launches(2);
    const int rest = n - k0 - nb;
    if (rest > 0) {
      k_lu_trsm<<<(rest + 127) / 128, 128, 0, s>>>(n, k0, nb, h.coarse_lu.p);
      dim3 g((rest + 31) / 32, (rest + 31) / 32);
      k_lu_gemm<<<g, 256, 0, s>>>(n, k0, nb, h.coarse_lu.p);
      count_launches(2);
    }
  }
  PMG_TRY(h.coarse_perm.alloc(n));
  k_lu_perm_identity<<<1, 32, 0, s>>>(n, h.coarse_piv.p, h.coarse_perm.p);
  k_lu_inverse_slab<<<(n + INV_COLS - 1) / INV_COLS, INV_THREADS, (size_t)n * 2 * INV_COLS * 8, s>>>(
      n, h.coarse_lu.p, h.coarse_perm.p, h.coarse_inv.p);
  count_launches(2);
  PMG_CUDA(cudaGetLastError());
  PMG_CUDA(cudaMemcpyAsync(h.h_coarse_flags, h.coarse_flags.p, sizeof(int) * 4, cudaMemcpyDeviceToHost, s));
  return PMG_OK;
}

// after the launches completed (the caller synchronised s): the pivot check
static int coarse_factor_finish(Handle &h) {
  if (h.lv[0].Na > 0 && (h.h_coarse_flags[0] & 16)) {
    set_error("zero pivot in the coarsest-level factorisation");
    return PMG_ERR_SINGULAR;
  }
  h.coarse_ready = true;
  return PMG_OK;
}

int coarse_factor(Handle &h) {
  PMG_TRY(coarse_factor_launch(h, h.stream));
  PMG_CUDA(cudaStreamSynchronize(h.stream));
  return coarse_factor_finish(h);
}

// ----------------------------------------------------------------- V-cycle
template <typename T> struct Prec;
template <> struct Prec<double> {
  static const double *A(const Level &L) { return L.A.p; }
  static const double *invd(const Level &L) { return L.invdiag.p; }
  static double *x(Level &L) { return L.x64.p; }
  static double *f(Level &L) { return L.f64.p; }
  static double *d(Level &L) { return L.d64.p; }
  static const double *P(const Level &L) { return L.pval.p; }
  static const double *R(const Level &L) { return L.rval.p; }
  static double *slc(Level &L, int k) { return L.slc64[k].p; }
  static double *jac(Level &L) { return L.jac64.p; }
};
template <> struct Prec<float> {
  static const float *A(const Level &L) { return L.A32.p; }
  static const float *invd(const Level &L) { return L.invdiag32.p; }
  static float *x(Level &L) { return L.x32.p; }
  static float *f(Level &L) { return L.f32.p; }
  static float *d(Level &L) { return L.d32.p; }
  static const float *P(const Level &L) { return L.pval32.p; }
  static const float *R(const Level &L) { return L.rval32.p; }
  static float *slc(Level &L, int k) { return L.slc32[k].p; }
  static float *jac(Level &L) { return L.jac32.p; }
};

// one pre/post smoothing step (TMultiGrid3D::Smooth, MultiGrid3D.C:117-446):
// Jacobi, SOR or SSOR in colour order (kind = PMG_SMOOTHER_*), or
// x += omega W (f - A x) with the learned stencil
template <typename T>
static int smooth_step(Handle &h, Level &L, bool learned, bool first, bool after_ssor, int kind) {
  using PT = Prec<T>;
  if (learned) {
    PMG_TRY(sell_spmv<T>(h.stream, L, PT::x(L), PT::f(L), PT::d(L), 1, h.num_sms));
    return learned_smooth<T>(h.stream, L, PT::d(L), PT::x(L), h.prm.smooth_omega);
  }
  if (kind == PMG_SMOOTHER_JACOBI)
    return sell_jacobi<T>(h.stream, L, PT::f(L), PT::x(L), PT::jac(L), h.prm.smooth_omega, h.num_sms, first);
  if (kind == PMG_SMOOTHER_SOR)
    return sell_ssor<T>(h.stream, L, PT::f(L), PT::x(L), h.prm.smooth_omega, h.num_sms, first, false, false, true);
  return sell_ssor<T>(h.stream, L, PT::f(L), PT::x(L), h.prm.smooth_omega, h.num_sms, first, after_ssor, true);
}

// Step-length control (TMGLevel3D::StepLengthControl, MGLevel3D.C:908-961,
// applied by TMultiGrid3D::Cycle, MultiGrid3D.C:655-663): with u0 and d0 the
// iterate and defect before the pre-smoothing and y = A (u - u0),
// alpha = (d0, y) / (y, y) -- the omega parameter when (y, y) = 0 or
// |alpha| < 0.1 -- and u := u0 + alpha (u - u0).  Computed on the device
// (block partials in a fixed order, one block for alpha), so the cycle stays
// one captured graph.
template <typename T>
__global__ void k_slc_diff(int n, const T *__restrict__ x, const T *__restrict__ x0, T *__restrict__ dx) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dx[i] = x[i] - x0[i];
}
constexpr int SLC_BLOCKS = 592;
template <typename T>
__global__ void __launch_bounds__(256) k_slc_partials(int n, const T *__restrict__ d0, const T *__restrict__ y,
                                                      double *__restrict__ part) {
  pdl_wait();
  pdl_trigger();
  __shared__ double sa[256], sb[256];
  double a = 0, b = 0;
  for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
    const double yi = (double)y[i];
    a += (double)d0[i] * yi;
    b += yi * yi;
  }
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) { sa[threadIdx.x] += sa[threadIdx.x + o]; sb[threadIdx.x] += sb[threadIdx.x + o]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = sa[0]; part[2 * blockIdx.x + 1] = sb[0]; }
}
__global__ void __launch_bounds__(256) k_slc_alpha(int nb, const double *__restrict__ part, double omega,
                                                   double *__restrict__ alpha) {
  pdl_wait();
  pdl_trigger();
  __shared__ double sa[256], sb[256];
  double a = 0, b = 0;
  for (int k = threadIdx.x; k < nb; k += 256) { a += part[2 * k]; b += part[2 * k + 1]; }
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) { sa[threadIdx.x] += sa[threadIdx.x + o]; sb[threadIdx.x] += sb[threadIdx.x + o]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double al = sb[0] > 0 ? sa[0] / sb[0] : omega;
    if (fabs(al) < 0.1) al = omega;
    *alpha = al;
  }
}
template <typename T>
__global__ void k_slc_apply(int n, const double *__restrict__ alpha, const T *__restrict__ x0, T *__restrict__ x) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const double a = *alpha;
    x[i] = (T)((double)x0[i] + a * ((double)x[i] - (double)x0[i]));
  }
}

template <typename T>
static int slc_begin(Handle &h, Level &L) {
  using PT = Prec<T>;
  PMG_TRY(sell_spmv<T>(h.stream, L, PT::x(L), PT::f(L), PT::slc(L, 1), 1, h.num_sms));
  PMG_CUDA(cudaMemcpyAsync(PT::slc(L, 0), PT::x(L), sizeof(T) * L.N, cudaMemcpyDeviceToDevice, h.stream));
  return PMG_OK;
}

template <typename T>
static int slc_end(Handle &h, Level &L) {
  using PT = Prec<T>;
  cudaStream_t s = h.stream;
  const int nb = (L.N + 255) / 256, np = std::min(SLC_BLOCKS, nb);
  PMG_CUDA(launch_pdl(k_slc_diff<T>, dim3(nb), dim3(256), 0, s, L.N, (const T *)PT::x(L), (const T *)PT::slc(L, 0),
                      PT::d(L)));
  PMG_TRY(sell_spmv<T>(s, L, PT::d(L), PT::f(L), PT::slc(L, 2), 0, h.num_sms));
  PMG_CUDA(launch_pdl(k_slc_partials<T>, dim3(np), dim3(256), 0, s, L.N, (const T *)PT::slc(L, 1),
                      (const T *)PT::slc(L, 2), h.slc_part.p));
  PMG_CUDA(launch_pdl(k_slc_alpha, dim3(1), dim3(256), 0, s, np, (const double *)h.slc_part.p, h.prm.smooth_omega,
                      h.slc_part.p + 2 * SLC_BLOCKS));
  PMG_CUDA(launch_pdl(k_slc_apply<T>, dim3(nb), dim3(256), 0, s, L.N, (const double *)(h.slc_part.p + 2 * SLC_BLOCKS),
                      (const T *)PT::slc(L, 0), PT::x(L)));
  count_launches(4);
  return PMG_OK;
}

// Iterative coarsest-level solve, the CoarseSmooth branch of
// TMultiGrid3D::Smooth (MultiGrid3D.C:262-330): res = |f - A x|; while
// res > coarse_red * res_0 and it < coarse_maxit: one Jacobi / SOR / SSOR step
// (rows in colour order), res = |f - A x|.  The coarsest level is small
// (hundreds to a few thousand rows), so one block runs the whole loop --
// colour by colour with block barriers, the residual by a block reduction --
// on the FP64 CSR values, and the loop's exit test stays on the device.
__device__ __forceinline__ double cc_block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  for (int k = 0; k < nw; k++) t += sh[k];
  return t;
}

template <typename T>
__device__ __forceinline__ double coarse_row_sum(int i, const int *__restrict__ rp, const int *__restrict__ kc,
                                                 const double *__restrict__ a, const T *x, double &diag) {
  double s = 0;
  diag = 1.0;
  for (int k = rp[i]; k < rp[i + 1]; k++) {
    const int c = kc[k];
    if (c == i) diag = a[k];
    else s += a[k] * (double)x[c];
  }
  return s;
}

template <typename T>
__global__ void __launch_bounds__(1024) k_coarse_iterate(int N, int Na, const int *__restrict__ rp,
                                                         const int *__restrict__ kc, const double *__restrict__ a,
                                                         const int *__restrict__ rows, const int *__restrict__ cptr,
                                                         int nc, int kind, double omega, double red, int maxit,
                                                         const T *__restrict__ f, T *x, double *tmp) {
  pdl_wait();
  pdl_trigger();
  __shared__ double sh[32];
  auto residual = [&]() {
    double r2 = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      double dg;
      const double s = coarse_row_sum<T>(i, rp, kc, a, x, dg);
      const double d = (double)f[i] - s - dg * (double)x[i];
      r2 += d * d;
    }
    return sqrt(cc_block_sum(r2, sh));
  };
  auto relax_colour = [&](int c) {
    for (int t = cptr[c] + threadIdx.x; t < cptr[c + 1]; t += blockDim.x) {
      const int i = rows[t];
      double dg;
      const double s = (double)f[i] - coarse_row_sum<T>(i, rp, kc, a, x, dg);
      const double xi = (double)x[i];
      x[i] = (T)(omega * (s / dg - xi) + xi);
    }
    __syncthreads();
  };
  double res = residual();
  const double target = red * res;
  for (int it = 0; it < maxit && res > target; it++) {
    for (int i = Na + threadIdx.x; i < N; i += blockDim.x) x[i] = f[i];  // Dirichlet rows from the rhs
    __syncthreads();
    if (kind == PMG_SMOOTHER_JACOBI) {
      for (int i = threadIdx.x; i < Na; i += blockDim.x) {
        double dg;
        const double s = (double)f[i] - coarse_row_sum<T>(i, rp, kc, a, x, dg);
        tmp[i] = (1.0 - omega) * (double)x[i] + omega * s / dg;
      }
      __syncthreads();
      for (int i = threadIdx.x; i < Na; i += blockDim.x) x[i] = (T)tmp[i];
      __syncthreads();
    } else {
      for (int c = 0; c < nc; c++) relax_colour(c);
      if (kind == PMG_SMOOTHER_SSOR)
        for (int c = nc - 1; c >= 0; c--) relax_colour(c);
    }
    res = residual();
  }
}

template <typename T>
static int vcycle(Handle &h, int i, bool learned) {
  cudaStream_t s = h.stream;
  Level &L = h.lv[i];
  using PT = Prec<T>;
  if (!learned && i >= 1 && i == h.cc_top) return coarse_cycle<T>(h, i);
  // The solve copy of the matrix leaves out the active rows' Dirichlet
  // columns.  The cycle's input has f_D = 0 (an FGMRES vector is exactly 0 on
  // the Dirichlet rows; pmg_vcycle folds A_aD v_D into the active rows first
  // and passes f_D = 0 on), so those columns contribute nothing, and the
  // smoothers keep x_D = f_D = 0.  Coarser levels: the restriction writes 0
  // into their Dirichlet rows.  The coarsest-level solves (dense or iterative)
  // read the full CSR rows themselves.
  if (i == 0) {
    if (h.prm.coarse_smoother == PMG_COARSE_DIRECT) {
      PMG_CUDA(launch_pdl(k_coarse_rhs<T>, dim3((L.N * 32 + 255) / 256), dim3(256), 0, s, L.N, L.Na,
                          (const int *)L.rowptr.p, (const int *)L.kcol.p, (const double *)L.A.p, (const T *)PT::f(L),
                          h.coarse_t.p, PT::x(L)));
      count_launches(1);
      if (L.Na > 0) {
        PMG_CUDA(launch_pdl(k_dense_apply<T>, dim3((L.Na * 32 + 255) / 256), dim3(256), 0, s, L.Na,
                            (const double *)h.coarse_inv.p, (const double *)h.coarse_t.p, PT::x(L)));
        count_launches(1);
      }
      PMG_CUDA(cudaGetLastError());
    } else {
      const int nc = (int)L.rcolor_ptr.size() - 1;
      PMG_CUDA(launch_pdl(k_coarse_iterate<T>, dim3(1), dim3(1024), 0, s, L.N, L.Na, (const int *)L.rowptr.p,
                          (const int *)L.kcol.p, (const double *)L.A.p, (const int *)L.row_list.p,
                          (const int *)h.coarse_cptr.p, nc, h.prm.coarse_smoother, h.prm.smooth_omega,
                          h.prm.coarse_red, h.prm.coarse_maxit, (const T *)PT::f(L), PT::x(L), h.coarse_t.p));
      count_launches(1);
    }
    return PMG_OK;
  }
  Level &C = h.lv[i - 1];
  const int pre = (learned && h.prm.learned_steps > 0) ? h.prm.learned_steps : h.prm.pre_smooth;
  const int post = (learned && h.prm.learned_steps > 0) ? h.prm.learned_steps : h.prm.post_smooth;
  const bool slc = h.prm.slc_all || (h.prm.slc_fine && i == (int)h.lv.size() - 1);
  if (slc) PMG_TRY(slc_begin<T>(h, L));
  for (int k = 0; k < pre; k++) PMG_TRY(smooth_step<T>(h, L, learned, k == 0, k > 0, h.prm.smoother));
  PMG_TRY(sell_spmv<T>(s, L, PT::x(L), PT::f(L), PT::d(L), 1, h.num_sms));
  PMG_TRY(restrict_defect<T>(s, L, C, PT::R(L), PT::d(L), PT::f(C), PT::x(C)));  // also x_C := 0
  PMG_TRY(vcycle<T>(h, i - 1, learned));
  PMG_TRY(prolongate_add<T>(s, L, PT::P(L), PT::x(C), PT::x(L), h.prm.gmg_damp));
  for (int k = 0; k < post; k++)
    PMG_TRY(smooth_step<T>(h, L, learned, pre == 0 && k == 0, k > 0, h.prm.smoother));
  if (slc) PMG_TRY(slc_end<T>(h, L));
  return PMG_OK;
}

// fine-level input/output conversions around the captured V-cycle
__global__ void k_prec_in64(int Na, int N, const double *__restrict__ v, double *f, double *x) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double t = v[i];
  f[i] = t;
  x[i] = i < Na ? 0.0 : t;  // zero start + SetDirichletNodes
}
__global__ void k_prec_in32(int Na, int N, const double *__restrict__ v, float *f, float *x) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  float t = (float)v[i];
  f[i] = t;
  x[i] = i < Na ? 0.0f : t;
}
__global__ void k_prec_out32(int N, const float *__restrict__ x, double *z) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) z[i] = (double)x[i];
}

static int prepare_levels(Handle &h) {
  bool fp32 = h.prm.precision == PMG_PREC_FP32;
  // the coarsest level's LU and inverse run on the auxiliary stream while the
  // level loop below converts the SELL values on the main stream; every path
  // out of here joins the two streams first
  const bool factor = h.prm.coarse_smoother == PMG_COARSE_DIRECT && !h.coarse_ready && h.lv[0].assembled;
  int frc = PMG_OK;
  if (factor) {
    PMG_CUDA(cudaEventRecord(h.aux_ev[0], h.stream));
    PMG_CUDA(cudaStreamWaitEvent(h.aux, h.aux_ev[0], 0));
    frc = coarse_factor_launch(h, h.aux);
    PMG_CUDA(cudaEventRecord(h.aux_ev[1], h.aux));
  }
  auto body = [&]() -> int {
    PMG_TRY(frc);
    for (size_t i = 0; i < h.lv.size(); i++) {
      Level &L = h.lv[i];
      if (!L.assembled) {
        set_error("solve: every level must be assembled (pmg_assemble) first");
        return PMG_ERR_STATE;
      }
      if (i > 0 && !L.has_P) {
        set_error("solve: missing transfer (pmg_set_transfer) for a level");
        return PMG_ERR_STATE;
      }
      PMG_TRY(L.x64.alloc(L.N)); PMG_TRY(L.f64.alloc(L.N)); PMG_TRY(L.d64.alloc(L.N));
      const bool slc = i > 0 && (h.prm.slc_all || (h.prm.slc_fine && i + 1 == h.lv.size()));
      const bool jac = h.prm.smoother == PMG_SMOOTHER_JACOBI || (i == 0 && h.prm.coarse_smoother == PMG_COARSE_JACOBI);
      for (int k = 0; k < 3 && slc; k++) PMG_TRY(fp32 ? L.slc32[k].alloc(L.N) : L.slc64[k].alloc(L.N));
      if (jac) PMG_TRY(fp32 ? L.jac32.alloc(L.N) : L.jac64.alloc(L.N));
      if (fp32) {
        PMG_TRY(sell_values<float>(h, L));
        PMG_TRY(L.x32.alloc(L.N)); PMG_TRY(L.f32.alloc(L.N)); PMG_TRY(L.d32.alloc(L.N));
        if (i > 0 && !L.pval32.p) {
          PMG_TRY(L.pval32.alloc(L.pval.n));
          PMG_TRY(convert_f64_f32(h.stream, L.pval.p, L.pval32.p, L.pval.n));
          PMG_TRY(L.rval32.alloc(L.rval.n));
          PMG_TRY(convert_f64_f32(h.stream, L.rval.p, L.rval32.p, L.rval.n));
        }
      } else {
        PMG_TRY(sell_values<double>(h, L));
      }
    }
    // the outer Krylov method multiplies with the FP64 finest matrix
    PMG_TRY(sell_values<double>(h, h.lv.back()));
    if (h.prm.slc_all || h.prm.slc_fine) PMG_TRY(h.slc_part.alloc(2 * SLC_BLOCKS + 1));
    if (h.prm.coarse_smoother != PMG_COARSE_DIRECT) {
      // colour pointers of the coarsest level's row list, and the Jacobi scratch
      const Level &C = h.lv[0];
      PMG_TRY(h.coarse_cptr.upload(C.rcolor_ptr.data(), C.rcolor_ptr.size(), h.stream));
      PMG_TRY(h.coarse_t.alloc(std::max(C.N, 1)));
    }
    if (h.prm.smoother == PMG_SMOOTHER_LEARNED) PMG_TRY(learned_prepare(h));
    return PMG_OK;
  };
  int rc = body();
  if (factor) {
    PMG_CUDA(cudaStreamWaitEvent(h.stream, h.aux_ev[1], 0));
    PMG_CUDA(cudaEventSynchronize(h.aux_ev[1]));
    if (rc == PMG_OK) rc = coarse_factor_finish(h);
  }
  PMG_TRY(rc);
  if (h.prm.coarse_smoother == PMG_COARSE_DIRECT && !h.coarse_ready) PMG_TRY(coarse_factor(h));
  const int cc = coarse_cycle_top(h);
  if (cc != h.cc_top) {
    h.cc_top = cc;
    invalidate_graphs(&h);
  }
  return PMG_OK;
}

static int capture_one(Handle &h, bool learned, cudaGraphExec_t &exec, unsigned long long &kernels) {
  if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
  cudaGraph_t g;
  const unsigned long long before = launches_so_far();
  PMG_CUDA(cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal));
  int top = (int)h.lv.size() - 1;
  int rc = h.prm.precision == PMG_PREC_FP32 ? vcycle<float>(h, top, learned) : vcycle<double>(h, top, learned);
  cudaGraph_t g_end = nullptr;
  cudaError_t e = cudaStreamEndCapture(h.stream, &g_end);
  g = g_end;
  if (rc != PMG_OK || e != cudaSuccess) {
    // the captured launches never ran: take them off the count, free the graph
    count_launches(0ULL - (launches_so_far() - before));
    if (e == cudaSuccess && g) cudaGraphDestroy(g);
    if (rc != PMG_OK) return rc;
    PMG_CUDA(e);
  }
  cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  PMG_CUDA(ei);
  // kernels recorded during capture run at each replay, not now
  kernels = launches_so_far() - before;
  count_launches(0ULL - kernels);
  return PMG_OK;
}

static int capture_vcycle(Handle &h) {
  if (!h.use_graph) return PMG_OK;
  const bool learned = h.prm.smoother == PMG_SMOOTHER_LEARNED;
  if (h.vgraph && h.vgraph_prec == h.prm.precision) return PMG_OK;
  PMG_TRY(capture_one(h, learned, h.vgraph, h.vgraph_kernels));
  if (learned) PMG_TRY(capture_one(h, false, h.vgraph_ssor, h.vgraph_ssor_kernels));
  h.vgraph_prec = h.prm.precision;
  return PMG_OK;
}

// z = MG(v): one V-cycle with zero start (MultiGridScaIte.C:89-130)
static int precondition(Handle &h, const double *v, double *z, bool learned) {
  Level &F = h.lv.back();
  cudaGraphExec_t graph = learned ? h.vgraph : (h.prm.smoother == PMG_SMOOTHER_LEARNED ? h.vgraph_ssor : h.vgraph);
  const unsigned long long nk = learned ? h.vgraph_kernels
                                        : (h.prm.smoother == PMG_SMOOTHER_LEARNED ? h.vgraph_ssor_kernels : h.vgraph_kernels);
  int nb = (F.N + 255) / 256;
  const int top = (int)h.lv.size() - 1;
  if (h.prm.precision == PMG_PREC_FP32) {
    k_prec_in32<<<nb, 256, 0, h.stream>>>(F.Na, F.N, v, F.f32.p, F.x32.p); count_launches(1);
    if (h.use_graph) {
      PMG_CUDA(cudaGraphLaunch(graph, h.stream));
      count_launches(nk);
    } else {
      PMG_TRY(vcycle<float>(h, top, learned));
    }
    k_prec_out32<<<nb, 256, 0, h.stream>>>(F.N, F.x32.p, z); count_launches(1);
  } else {
    k_prec_in64<<<nb, 256, 0, h.stream>>>(F.Na, F.N, v, F.f64.p, F.x64.p); count_launches(1);
    if (h.use_graph) {
      PMG_CUDA(cudaGraphLaunch(graph, h.stream));
      count_launches(nk);
    } else {
      PMG_TRY(vcycle<double>(h, top, learned));
    }
    PMG_CUDA(cudaMemcpyAsync(z, F.x64.p, sizeof(double) * F.N, cudaMemcpyDeviceToDevice, h.stream));
  }
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}

// sol += sum_k y_k Z_k  (y in device memory, m terms)
__global__ void k_lincomb(size_t n, int m, const double *__restrict__ y, const double *__restrict__ Z, size_t ldz,
                          double *__restrict__ sol) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double s = sol[i];
    for (int k = 0; k < m; k++) s += y[k] * Z[(size_t)k * ldz + i];
    sol[i] = s;
  }
}

static void givens(double &dx, double &dy, double &cs, double &sn) {
  if (dy == 0.0) { cs = 1.0; sn = 0.0; }
  else if (fabs(dy) > fabs(dx)) { double t = dx / dy; sn = 1.0 / sqrt(1.0 + t * t); cs = t * sn; }
  else { double t = dy / dx; cs = 1.0 / sqrt(1.0 + t * t); sn = t * cs; }
}

int solve(Handle &h, double *sol_host, const double *rhs_host, pmg_solve_stats *st) {
  if (h.lv.empty()) { set_error("solve: no levels"); return PMG_ERR_STATE; }
  // the solve's device time covers everything below: per-solve set-up (SELL
  // values, coarsest factorisation), the iteration and the final true residual
  PMG_CUDA(cudaEventRecord(h.ev[2], h.stream));
  PMG_TRY(prepare_levels(h));
  PMG_TRY(capture_vcycle(h));
  PMG_CUDA(cudaEventRecord(h.ev[6], h.stream));  // end of the per-solve set-up
  bool vc_timed = false;
  Level &F = h.lv.back();
  const size_t N = F.N;
  const int m = h.prm.restart > 0 ? h.prm.restart : 10;
  if (m > 60) { set_error("solve: restart must be <= 60"); return PMG_ERR_ARG; }
  if (h.krylov_n != (int)N || h.krylov_restart != m) {
    PMG_TRY(h.V.alloc(N * (m + 1)));
    PMG_TRY(h.Z.alloc(N * m));
    PMG_TRY(h.w.alloc(N));
    PMG_TRY(h.sol.alloc(N));
    PMG_TRY(h.rhs.alloc(N));
    PMG_TRY(h.H.alloc((size_t)(m + 1) * (m + 1) + 64));
    h.krylov_n = (int)N;
    h.krylov_restart = m;
  }
  cudaStream_t s = h.stream;
  if (rhs_host) PMG_CUDA(cudaMemcpyAsync(h.rhs.p, rhs_host, sizeof(double) * N, cudaMemcpyHostToDevice, s));
  else PMG_CUDA(cudaMemcpyAsync(h.rhs.p, F.rhs.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  if (sol_host) PMG_CUDA(cudaMemcpyAsync(h.sol.p, sol_host, sizeof(double) * N, cudaMemcpyHostToDevice, s));
  else if (!h.sol_preset) PMG_TRY(zero<double>(s, h.sol.p, N));  // (pmg_tcd_system presets u_old)
  h.sol_preset = false;
  // Dirichlet part of the start vector = rhs (TSystemCD3D::Assemble copies it, SystemCD3D.C:361)
  PMG_TRY(copy_dirichlet(s, F.Na, F.N, h.rhs.p, h.sol.p));

  double *V = h.V.p, *Z = h.Z.p, *w = h.w.p;
  double *Hd = h.H.p;  // column i at Hd + i*(m+1); scratch scalars after (m+1)^2
  double *sc = Hd + (size_t)(m + 1) * (m + 1);
  std::vector<double> H((size_t)(m + 1) * m, 0.0), sv(m + 1), cs(m), sn(m), y(m);
  double *hcol = h.h_H;

  auto residual = [&](double *out_vec, double &nrm) -> int {
    PMG_TRY(sell_spmv<double>(s, F, h.sol.p, h.rhs.p, out_vec, 1, h.num_sms));
    PMG_TRY(dirichlet_cols<double>(s, F, h.sol.p, out_vec));  // - A_aD x_D
    PMG_TRY(dot(h, out_vec, out_vec, N, sc));
    PMG_CUDA(cudaMemcpyAsync(hcol, sc, sizeof(double), cudaMemcpyDeviceToHost, s));
    PMG_CUDA(cudaStreamSynchronize(s));
    nrm = sqrt(hcol[0]);
    return PMG_OK;
  };

  // learned smoother guard: 0 = calibrating with SSOR, 1 = learned, 2 = SSOR took over
  // (without the guard the learned smoother runs from the first cycle on)
  const bool learned = h.prm.smoother == PMG_SMOOTHER_LEARNED;
  const bool guarded = learned && !h.prm.learned_guard_off;
  const int kCalib = 2;
  int guard_phase = learned ? (guarded ? 0 : 1) : 2, learned_start = 0, learned_cycles = 0;
  double rho_plain = 0.0, rho_learned = 0.0;
  std::vector<double> res_hist;
  double beta;
  PMG_TRY(residual(V, beta));
  const double res0 = beta;
  res_hist.push_back(beta);
  double r0 = beta, res = beta;
  int j = 1, status = PMG_ERR_NOT_CONVERGED, iters = 0;
  const double red = h.prm.lin_red, rmin = h.prm.lin_res_min;
  const int maxit = h.prm.lin_maxit;
  if (!std::isfinite(beta)) { set_error("solve: non-finite initial residual"); return PMG_ERR_NONFINITE; }
  if (beta <= rmin || beta < 1e-300) status = PMG_OK;
  while (status == PMG_ERR_NOT_CONVERGED && j <= maxit) {
    PMG_TRY(scale_by_inv_sqrt(s, N, sc, V, V));  // v0 = r / beta  (sc holds beta^2)
    std::fill(sv.begin(), sv.end(), 0.0);
    sv[0] = beta;
    int i;
    bool done = false;
    for (i = 0; i < m && j <= maxit; i++, j++) {
      double *vi = V + (size_t)i * N, *zi = Z + (size_t)i * N;
      if (!vc_timed) PMG_CUDA(cudaEventRecord(h.ev[7], s));
      PMG_TRY(precondition(h, vi, zi, guard_phase == 1));
      if (guard_phase == 1) learned_cycles++;
      if (!vc_timed) {
        PMG_CUDA(cudaEventRecord(h.ev[8], s));
        vc_timed = true;
      }
      // w = A z_i.  The solve copy holds no Dirichlet columns, and none are
      // needed: the start vector carries the Dirichlet values (copied above),
      // so the residual and every Krylov vector are exactly 0 on the
      // Dirichlet rows (identity rows), and every smoother copies f_D = 0
      // into x_D, so z_i is exactly 0 there too and A_aD z_D adds nothing
      PMG_TRY(sell_spmv<double>(s, F, zi, nullptr, w, 0, h.num_sms));
      double *Hc = Hd + (size_t)i * (m + 1);
      // modified Gram-Schmidt (FgmresIte.C): h_k = w.v_k, w -= h_k v_k for
      // k = 0..i, then h_{i+1}^2 = w.w; each update fused with the next product
      PMG_TRY(dot(h, w, V, N, Hc));
      for (int k = 0; k <= i; k++)
        PMG_TRY(mgs_step(h, N, Hc + k, V + (size_t)k * N, k < i ? V + (size_t)(k + 1) * N : w, w, Hc + k + 1));
      PMG_TRY(scale_by_inv_sqrt(s, N, Hc + i + 1, w, V + (size_t)(i + 1) * N));
      PMG_CUDA(cudaMemcpyAsync(hcol, Hc, sizeof(double) * (i + 2), cudaMemcpyDeviceToHost, s));
      PMG_CUDA(cudaStreamSynchronize(s));
      for (int k = 0; k <= i; k++) H[(size_t)k * m + i] = hcol[k];
      H[(size_t)(i + 1) * m + i] = sqrt(hcol[i + 1]);
      for (int k = 0; k < i; k++) {
        double t = cs[k] * H[(size_t)k * m + i] + sn[k] * H[(size_t)(k + 1) * m + i];
        H[(size_t)(k + 1) * m + i] = -sn[k] * H[(size_t)k * m + i] + cs[k] * H[(size_t)(k + 1) * m + i];
        H[(size_t)k * m + i] = t;
      }
      givens(H[(size_t)i * m + i], H[(size_t)(i + 1) * m + i], cs[i], sn[i]);
      {
        double t = cs[i] * H[(size_t)i * m + i] + sn[i] * H[(size_t)(i + 1) * m + i];
        H[(size_t)(i + 1) * m + i] = 0.0;
        H[(size_t)i * m + i] = t;
        t = cs[i] * sv[i] + sn[i] * sv[i + 1];
        sv[i + 1] = -sn[i] * sv[i] + cs[i] * sv[i + 1];
        sv[i] = t;
      }
      res = fabs(sv[i + 1]);
      iters = j;
      res_hist.push_back(res);
      if (guard_phase == 0 && j == kCalib) {
        // per-cycle contraction of the plain SSOR V-cycle over the first cycles
        rho_plain = pow(res / res_hist[0], 1.0 / kCalib);
        guard_phase = 1;
        learned_start = j;
      } else if (guard_phase == 1 && j - learned_start >= 2) {
        const int nl = j - learned_start;
        rho_learned = pow(res / res_hist[learned_start], 1.0 / nl);
        if (guarded && rho_learned > rho_plain) guard_phase = 2;  // the plain SSOR smoother takes over
      }
      if (!std::isfinite(res)) { status = PMG_ERR_NONFINITE; set_error("solve: non-finite residual estimate"); done = true; i++; break; }
      double ref = h.prm.reference_restart_rule ? r0 : res0;
      if (res < rmin || res < red * ref) { status = PMG_OK; done = true; i++; break; }
      if (res > h.prm.div_factor * res0) { status = PMG_ERR_DIVERGED; set_error("solve: diverged"); done = true; i++; break; }
    }
    // x += Z y with y from the triangular system of the i columns built
    int mm = i;
    for (int k = mm - 1; k >= 0; k--) {
      double t = sv[k];
      for (int l = k + 1; l < mm; l++) t -= H[(size_t)k * m + l] * y[l];
      y[k] = t / H[(size_t)k * m + k];
    }
    if (mm > 0) {
      for (int k = 0; k < mm; k++) hcol[k] = y[k];
      PMG_CUDA(cudaMemcpyAsync(sc + 1, hcol, sizeof(double) * mm, cudaMemcpyHostToDevice, s));
      size_t nb = (N + 255) / 256;
      k_lincomb<<<(unsigned)(nb < 148 * 16 ? nb : 148 * 16), 256, 0, s>>>(N, mm, sc + 1, Z, N, h.sol.p); count_launches(1);
      PMG_CUDA(cudaGetLastError());
      PMG_CUDA(cudaStreamSynchronize(s));  // hcol is reused below
    }
    if (done || j > maxit) break;
    PMG_TRY(residual(V, beta));  // restart
    r0 = beta;
  }
  double res_final;
  PMG_TRY(residual(w, res_final));
  PMG_CUDA(cudaEventRecord(h.ev[3], s));
  PMG_CUDA(cudaEventSynchronize(h.ev[3]));
  float ms = 0;
  PMG_CUDA(cudaEventElapsedTime(&ms, h.ev[2], h.ev[3]));
  h.t_solve = ms * 1e-3;
  if (sol_host) PMG_CUDA(cudaMemcpyAsync(sol_host, h.sol.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
  PMG_CUDA(cudaStreamSynchronize(s));
  PMG_TRY(coarse_cycle_check(h));
  if (st) {
    st->iterations = iters;
    st->res0 = res0;
    st->res_final = res_final;
    st->rel_res = res0 > 0 ? res_final / res0 : 0.0;
    st->mean_contraction = (iters > 0 && res0 > 0 && res_final > 0) ? pow(res_final / res0, 1.0 / iters) : 0.0;
    st->smoother_used = learned ? (guard_phase == 1 ? PMG_SMOOTHER_LEARNED : PMG_SMOOTHER_SSOR) : h.prm.smoother;
    st->rho_plain = rho_plain;
    st->rho_learned = rho_learned;
    st->learned_cycles = learned_cycles;
    st->seconds = h.t_solve;
    float a = 0, b = 0;
    st->setup_seconds = cudaEventElapsedTime(&a, h.ev[2], h.ev[6]) == cudaSuccess ? a * 1e-3 : 0.0;
    st->vcycle_seconds = (vc_timed && cudaEventElapsedTime(&b, h.ev[7], h.ev[8]) == cudaSuccess) ? b * 1e-3 : 0.0;
    cudaGetLastError();
  }
  if (status == PMG_ERR_NOT_CONVERGED)
    set_error("solve: the iteration limit (lin_maxit) was reached before |r| <= max(lin_res_min, lin_red |r0|)");
  return status;
}

// ------------------------------------------------------- domain decomposition
// FGMRES over a domain-decomposed finest level (the parallel path of the
// reference: TParFECommunicator3D::CommUpdate before each product and an
// all-reduce of every inner product, src/Parallel/ParFECommunicator3D.C:218-346,
// src/FE/MGLevel3D.C:220-272).  Each rank's handle holds its subdomain: the
// rows it owns (active rows, and its Dirichlet rows) plus ghost rows -- the
// dofs of a layer of neighbouring cells -- stored as Dirichlet rows of the
// local problem.  Per iteration:
//   * the preconditioner is the rank's own V-cycle with the ghost rows held at
//     zero (overlapping additive Schwarz, one subdomain per rank, multigrid
//     inside each);
//   * the product w = A z takes the ghost values of z from the neighbours
//     (halo exchange) and drops the ghost rows of w;
//   * every inner product is summed over the ranks before it is used
//     (modified Gram-Schmidt: one sum per step, as the reference's Ddot);
//   * the residual takes the ghost values of x from the neighbours.
// The transport is the caller's: pmg_comm's callbacks move the packed halo
// buffers and sum host doubles (NCCL, MPI, gloo ...).
__global__ void k_halo_gather(int n, const int *__restrict__ idx, const double *__restrict__ x, double *__restrict__ buf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) buf[i] = x[idx[i]];
}
__global__ void k_halo_scatter(int n, const int *__restrict__ idx, const double *__restrict__ buf, double *__restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[idx[i]] = buf[i];
}
__global__ void k_zero_rows(int n, const int *__restrict__ idx, double *__restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[idx[i]] = 0.0;
}

static int halo_exchange(Handle &h, const pmg_comm *comm, double *x) {
  cudaStream_t s = h.stream;
  if (h.halo_nsend > 0) {
    k_halo_gather<<<(h.halo_nsend + 255) / 256, 256, 0, s>>>(h.halo_nsend, h.halo_send_idx.p, x, h.halo_send_buf);
    count_launches(1);
    PMG_CUDA(cudaGetLastError());
  }
  PMG_CUDA(cudaStreamSynchronize(s));
  if (comm->exchange(comm->ctx, h.halo_send_buf, h.halo_nsend, h.halo_recv_buf, h.halo_nrecv) != 0) {
    set_error("solve_dd: the halo exchange callback failed");
    return PMG_ERR_STATE;
  }
  if (h.halo_nrecv > 0) {
    k_halo_scatter<<<(h.halo_nrecv + 255) / 256, 256, 0, s>>>(h.halo_nrecv, h.halo_recv_idx.p, h.halo_recv_buf, x);
    count_launches(1);
    PMG_CUDA(cudaGetLastError());
  }
  return PMG_OK;
}

static int zero_ghosts(Handle &h, double *x) {
  if (h.halo_nrecv > 0) {
    k_zero_rows<<<(h.halo_nrecv + 255) / 256, 256, 0, h.stream>>>(h.halo_nrecv, h.halo_recv_idx.p, x);
    count_launches(1);
    PMG_CUDA(cudaGetLastError());
  }
  return PMG_OK;
}

// the device scalar *d summed over the ranks, in place (host round trip)
static int sum_over_ranks(Handle &h, const pmg_comm *comm, double *d, int n) {
  double *hv = h.h_H + 128;  // the pinned scratch (256 doubles; FGMRES uses at most 62)
  PMG_CUDA(cudaMemcpyAsync(hv, d, sizeof(double) * n, cudaMemcpyDeviceToHost, h.stream));
  PMG_CUDA(cudaStreamSynchronize(h.stream));
  if (comm->allreduce_sum(comm->ctx, hv, n) != 0) {
    set_error("solve_dd: the all-reduce callback failed");
    return PMG_ERR_STATE;
  }
  PMG_CUDA(cudaMemcpyAsync(d, hv, sizeof(double) * n, cudaMemcpyHostToDevice, h.stream));
  return PMG_OK;
}

int solve_dd(Handle &h, const pmg_comm *comm, double *sol_host, const double *rhs_host, pmg_solve_stats *st) {
  if (h.lv.empty()) { set_error("solve_dd: no levels"); return PMG_ERR_STATE; }
  if (!comm || !comm->allreduce_sum || !comm->exchange) { set_error("solve_dd: incomplete communicator"); return PMG_ERR_ARG; }
  if (!h.halo_set) { set_error("solve_dd: pmg_set_halo first"); return PMG_ERR_STATE; }
  if (h.prm.smoother == PMG_SMOOTHER_LEARNED) { set_error("solve_dd: the learned smoother is not built for subdomains"); return PMG_ERR_UNSUPPORTED; }
  PMG_CUDA(cudaEventRecord(h.ev[2], h.stream));
  PMG_TRY(prepare_levels(h));
  PMG_TRY(capture_vcycle(h));
  Level &F = h.lv.back();
  const size_t N = F.N;
  const int m = h.prm.restart;
  if (h.krylov_n != (int)N || h.krylov_restart != m) {
    PMG_TRY(h.V.alloc(N * (m + 1)));
    PMG_TRY(h.Z.alloc(N * m));
    PMG_TRY(h.w.alloc(N));
    PMG_TRY(h.sol.alloc(N));
    PMG_TRY(h.rhs.alloc(N));
    PMG_TRY(h.H.alloc((size_t)(m + 1) * (m + 1) + 64));
    h.krylov_n = (int)N;
    h.krylov_restart = m;
  }
  cudaStream_t s = h.stream;
  if (rhs_host) PMG_CUDA(cudaMemcpyAsync(h.rhs.p, rhs_host, sizeof(double) * N, cudaMemcpyHostToDevice, s));
  else PMG_CUDA(cudaMemcpyAsync(h.rhs.p, F.rhs.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  if (sol_host) PMG_CUDA(cudaMemcpyAsync(h.sol.p, sol_host, sizeof(double) * N, cudaMemcpyHostToDevice, s));
  else PMG_TRY(zero<double>(s, h.sol.p, N));
  PMG_TRY(copy_dirichlet(s, F.Na, F.N, h.rhs.p, h.sol.p));
  double *V = h.V.p, *Z = h.Z.p, *w = h.w.p;
  double *Hd = h.H.p, *sc = Hd + (size_t)(m + 1) * (m + 1);
  std::vector<double> H((size_t)(m + 1) * m, 0.0), sv(m + 1), cs(m), sn(m), y(m);
  double *hcol = h.h_H;

  auto residual = [&](double *out_vec, double &nrm) -> int {
    PMG_TRY(halo_exchange(h, comm, h.sol.p));
    PMG_TRY(sell_spmv<double>(s, F, h.sol.p, h.rhs.p, out_vec, 1, h.num_sms));
    PMG_TRY(dirichlet_cols<double>(s, F, h.sol.p, out_vec));
    PMG_TRY(zero_ghosts(h, out_vec));
    PMG_TRY(dot(h, out_vec, out_vec, N, sc));
    PMG_TRY(sum_over_ranks(h, comm, sc, 1));
    PMG_CUDA(cudaMemcpyAsync(hcol, sc, sizeof(double), cudaMemcpyDeviceToHost, s));
    PMG_CUDA(cudaStreamSynchronize(s));
    nrm = sqrt(hcol[0]);
    return PMG_OK;
  };

  double beta;
  PMG_TRY(residual(V, beta));
  const double res0 = beta;
  double r0 = beta, res = beta;
  int j = 1, status = PMG_ERR_NOT_CONVERGED, iters = 0;
  const double red = h.prm.lin_red, rmin = h.prm.lin_res_min;
  const int maxit = h.prm.lin_maxit;
  if (!std::isfinite(beta)) { set_error("solve_dd: non-finite initial residual"); return PMG_ERR_NONFINITE; }
  if (beta <= rmin || beta < 1e-300) status = PMG_OK;
  while (status == PMG_ERR_NOT_CONVERGED && j <= maxit) {
    PMG_TRY(scale_by_inv_sqrt(s, N, sc, V, V));
    std::fill(sv.begin(), sv.end(), 0.0);
    sv[0] = beta;
    int i;
    bool done = false;
    for (i = 0; i < m && j <= maxit; i++, j++) {
      double *vi = V + (size_t)i * N, *zi = Z + (size_t)i * N;
      PMG_TRY(precondition(h, vi, zi, false));
      PMG_TRY(halo_exchange(h, comm, zi));
      PMG_TRY(sell_spmv<double>(s, F, zi, nullptr, w, 0, h.num_sms));
      PMG_TRY(dirichlet_cols<double>(s, F, zi, w, true));  // + A_aG z_G: the neighbours' values of z
      PMG_TRY(zero_ghosts(h, w));
      double *Hc = Hd + (size_t)i * (m + 1);
      PMG_TRY(dot(h, w, V, N, Hc));
      PMG_TRY(sum_over_ranks(h, comm, Hc, 1));
      for (int k = 0; k <= i; k++) {
        PMG_TRY(mgs_step(h, N, Hc + k, V + (size_t)k * N, k < i ? V + (size_t)(k + 1) * N : w, w, Hc + k + 1));
        PMG_TRY(sum_over_ranks(h, comm, Hc + k + 1, 1));
      }
      PMG_TRY(scale_by_inv_sqrt(s, N, Hc + i + 1, w, V + (size_t)(i + 1) * N));
      PMG_CUDA(cudaMemcpyAsync(hcol, Hc, sizeof(double) * (i + 2), cudaMemcpyDeviceToHost, s));
      PMG_CUDA(cudaStreamSynchronize(s));
      for (int k = 0; k <= i; k++) H[(size_t)k * m + i] = hcol[k];
      H[(size_t)(i + 1) * m + i] = sqrt(hcol[i + 1]);
      for (int k = 0; k < i; k++) {
        double t = cs[k] * H[(size_t)k * m + i] + sn[k] * H[(size_t)(k + 1) * m + i];
        H[(size_t)(k + 1) * m + i] = -sn[k] * H[(size_t)k * m + i] + cs[k] * H[(size_t)(k + 1) * m + i];
        H[(size_t)k * m + i] = t;
      }
      givens(H[(size_t)i * m + i], H[(size_t)(i + 1) * m + i], cs[i], sn[i]);
      {
        double t = cs[i] * H[(size_t)i * m + i] + sn[i] * H[(size_t)(i + 1) * m + i];
        H[(size_t)(i + 1) * m + i] = 0.0;
        H[(size_t)i * m + i] = t;
        t = cs[i] * sv[i] + sn[i] * sv[i + 1];
        sv[i + 1] = -sn[i] * sv[i] + cs[i] * sv[i + 1];
        sv[i] = t;
      }
      res = fabs(sv[i + 1]);
      iters = j;
      if (!std::isfinite(res)) { status = PMG_ERR_NONFINITE; set_error("solve_dd: non-finite residual estimate"); done = true; i++; break; }
      const double ref = h.prm.reference_restart_rule ? r0 : res0;
      if (res < rmin || res < red * ref) { status = PMG_OK; done = true; i++; break; }
      if (res > h.prm.div_factor * res0) { status = PMG_ERR_DIVERGED; set_error("solve_dd: diverged"); done = true; i++; break; }
    }
    int mm = i;
    for (int k = mm - 1; k >= 0; k--) {
      double t = sv[k];
      for (int l = k + 1; l < mm; l++) t -= H[(size_t)k * m + l] * y[l];
      y[k] = t / H[(size_t)k * m + k];
    }
    if (mm > 0) {
      for (int k = 0; k < mm; k++) hcol[k] = y[k];
      PMG_CUDA(cudaMemcpyAsync(sc + 1, hcol, sizeof(double) * mm, cudaMemcpyHostToDevice, s));
      size_t nb = (N + 255) / 256;
      k_lincomb<<<(unsigned)(nb < 148 * 16 ? nb : 148 * 16), 256, 0, s>>>(N, mm, sc + 1, Z, N, h.sol.p); count_launches(1);
      PMG_CUDA(cudaGetLastError());
      PMG_CUDA(cudaStreamSynchronize(s));
    }
    if (done || j > maxit) break;
    PMG_TRY(residual(V, beta));
    r0 = beta;
  }
  double res_final;
  PMG_TRY(residual(w, res_final));  // also refreshes the ghost values of x
  PMG_CUDA(cudaEventRecord(h.ev[3], s));
  PMG_CUDA(cudaEventSynchronize(h.ev[3]));
  float ms = 0;
  PMG_CUDA(cudaEventElapsedTime(&ms, h.ev[2], h.ev[3]));
  h.t_solve = ms * 1e-3;
  if (sol_host) PMG_CUDA(cudaMemcpyAsync(sol_host, h.sol.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
  PMG_CUDA(cudaStreamSynchronize(s));
  PMG_TRY(coarse_cycle_check(h));
  if (st) {
    st->iterations = iters;
    st->res0 = res0;
    st->res_final = res_final;
    st->rel_res = res0 > 0 ? res_final / res0 : 0.0;
    st->mean_contraction = (iters > 0 && res0 > 0 && res_final > 0) ? pow(res_final / res0, 1.0 / iters) : 0.0;
    st->smoother_used = h.prm.smoother;
    st->seconds = h.t_solve;
    st->setup_seconds = 0.0;
    st->vcycle_seconds = 0.0;
    st->rho_plain = st->rho_learned = 0.0;
    st->learned_cycles = 0;
  }
  if (status == PMG_ERR_NOT_CONVERGED)
    set_error("solve_dd: the iteration limit (lin_maxit) was reached before |r| <= max(lin_res_min, lin_red |r0|)");
  return status;
}

}  // namespace pmg

extern "C" int pmg_set_halo(pmg_handle hh, int n_send, const int *send_idx, int n_recv, const int *recv_idx,
                            double *send_buf_dev, double *recv_buf_dev) {
  pmg::Handle *h = reinterpret_cast<pmg::Handle *>(hh);
  if (!h || h->lv.empty() || n_send < 0 || n_recv < 0 || (n_send && (!send_idx || !send_buf_dev)) ||
      (n_recv && (!recv_idx || !recv_buf_dev))) {
    pmg::set_error("pmg_set_halo: bad arguments");
    return PMG_ERR_ARG;
  }
  pmg::Level &F = h->lv.back();
  if (!F.has_csr) { pmg::set_error("pmg_set_halo: set the finest level's pattern first"); return PMG_ERR_STATE; }
  for (int k = 0; k < n_send; k++)
    if (send_idx[k] < 0 || send_idx[k] >= F.N) { pmg::set_error("pmg_set_halo: send index out of range"); return PMG_ERR_ARG; }
  for (int k = 0; k < n_recv; k++)
    if (recv_idx[k] < F.Na || recv_idx[k] >= F.N) {
      pmg::set_error("pmg_set_halo: ghost rows must be rows of the local problem past active_bound");
      return PMG_ERR_ARG;
    }
  PMG_TRY(h->halo_send_idx.upload(send_idx, n_send, h->stream));
  PMG_TRY(h->halo_recv_idx.upload(recv_idx, n_recv, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  h->halo_nsend = n_send;
  h->halo_nrecv = n_recv;
  h->halo_send_buf = send_buf_dev;
  h->halo_recv_buf = recv_buf_dev;
  h->halo_set = true;
  return PMG_OK;
}

extern "C" int pmg_solve_dd(pmg_handle hh, const pmg_comm *comm, double *sol, const double *rhs,
                            pmg_solve_stats *stats) {
  pmg::Handle *h = reinterpret_cast<pmg::Handle *>(hh);
  if (!h) return PMG_ERR_ARG;
  return pmg::solve_dd(*h, comm, sol, rhs, stats);
}

extern "C" int pmg_vcycle(pmg_handle hh, const double *v_dev, double *z_dev) {
  pmg::Handle *h = reinterpret_cast<pmg::Handle *>(hh);
  if (!h || !v_dev || !z_dev) return PMG_ERR_ARG;
  PMG_TRY(pmg::prepare_levels(*h));
  PMG_TRY(pmg::capture_vcycle(*h));
  // the cycle takes f_D = 0: fold the Dirichlet part of v into the active
  // rows in FP64 (f_a = v_a - A_aD v_D, f_D = 0), the cycle then keeps
  // z_D = v_D as the smoothers' x_D = f_D did
  pmg::Level &F = h->lv.back();
  PMG_TRY(h->w.alloc(std::max<size_t>(h->w.n, (size_t)F.N)));
  double *f = h->w.p;
  PMG_CUDA(cudaMemcpyAsync(f, v_dev, sizeof(double) * F.N, cudaMemcpyDeviceToDevice, h->stream));
  PMG_TRY(pmg::dirichlet_cols<double>(h->stream, F, v_dev, f, false));
  PMG_CUDA(cudaMemsetAsync(f + F.Na, 0, sizeof(double) * (F.N - F.Na), h->stream));
  PMG_TRY(pmg::precondition(*h, f, z_dev, h->prm.smoother == PMG_SMOOTHER_LEARNED));
  PMG_TRY(pmg::copy_dirichlet(h->stream, F.Na, F.N, v_dev, z_dev));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  return pmg::coarse_cycle_check(*h);
}
