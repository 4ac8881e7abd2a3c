// Sparse and vector kernels of the solve (sm_100a).
//
//   spmv / defect       MatVect, ScalarDefect (src/FE/Blas2.C:37-126)
//   ssor_sweep          TMGLevel3D::SSOR (src/FE/MGLevel3D.C:363-467) in
//                       multicolour order: forward over colours, then backward
//   restrict_defect     DefectRestriction + CorrectDefect (src/FE/MGComponents3D.C:732,
//                       src/FE/MGLevel3D.C CorrectDefect): f_c = P^T d, Dirichlet rows 0
//   prolongate_add      Prolongate + CorrectNodes + Update (MGComponents3D.C:208,
//                       MGLevel3D.C:565-638): x_f += damp * (P x_c) on active rows
//   dot / axpy / scale  Ddot / Daxpy / Dscal (src/FE/Blas1.C:40-157), the dot
//                       reduced in a fixed order (bitwise reproducible)
//
// All matrix kernels are HBM-bandwidth bound: a group of W lanes owns one row
// (W = 8 / 16 / 32 from the mean row length), streams the row's values and
// column indices with coalesced loads, gathers x through L2 and reduces with
// warp shuffles.
#include "pmg_internal.h"

namespace pmg {

template <typename T>
__device__ __forceinline__ T ldg(const T *p) { return __ldg(p); }

// first row of this warp and rows covered by the whole grid, for W-lane row groups
template <int W>
__device__ __forceinline__ int warp_first_row() { return ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * (32 / W); }
template <int W>
__device__ __forceinline__ int rows_per_grid() { return (gridDim.x * blockDim.x >> 5) * (32 / W); }

template <int W, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, W);
  return v;
}

// y = A x  (mode 0) ;  d = f - A x (mode 1)
template <int W, typename T, int MODE>
__global__ void __launch_bounds__(256) k_csr(int N, const int *__restrict__ rp, const int *__restrict__ kc,
                                             const T *__restrict__ a, const T *__restrict__ x,
                                             const T *__restrict__ f, T *__restrict__ y) {
  // the row loop is warp-uniform so every lane reaches the shuffles
  const int lane = threadIdx.x & (W - 1);
  for (int base = warp_first_row<W>(); base < N; base += rows_per_grid<W>()) {
    const int row = base + (threadIdx.x & 31) / W;
    T s = 0;
    if (row < N) {
      const int beg = ldg(rp + row), end = ldg(rp + row + 1);
      for (int k = beg + lane; k < end; k += W) s += ldg(a + k) * ldg(x + ldg(kc + k));
    }
    s = group_sum<W>(s);
    if (lane == 0 && row < N) y[row] = MODE ? ldg(f + row) - s : s;
  }
}

static int pick_width(const Level &L) { return L.avg_row >= 48 ? 32 : (L.avg_row >= 16 ? 16 : 8); }

static int grid_for(int rows, int W, int num_sms) {
  long blocks = ((long)rows * W + 255) / 256;
  long cap = (long)num_sms * 16;
  return (int)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

template <typename T, int MODE>
static int launch_csr(cudaStream_t s, const Level &L, const T *A, const T *x, const T *f, T *y) {
  int W = pick_width(L);
  int g = grid_for(L.N, W, 148);
  if (W == 32) { k_csr<32, T, MODE><<<g, 256, 0, s>>>(L.N, L.rowptr.p, L.kcol.p, A, x, f, y); count_launches(1); }
  else if (W == 16) { k_csr<16, T, MODE><<<g, 256, 0, s>>>(L.N, L.rowptr.p, L.kcol.p, A, x, f, y); count_launches(1); }
  else { k_csr<8, T, MODE><<<g, 256, 0, s>>>(L.N, L.rowptr.p, L.kcol.p, A, x, f, y); count_launches(1); }
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}

template <typename T>
int spmv(cudaStream_t s, const Level &L, const T *A, const T *x, T *y) {
  return launch_csr<T, 0>(s, L, A, x, nullptr, y);
}
template <typename T>
int defect(cudaStream_t s, const Level &L, const T *A, const T *x, const T *f, T *d) {
  return launch_csr<T, 1>(s, L, A, x, f, d);
}
template int spmv<double>(cudaStream_t, const Level &, const double *, const double *, double *);
template int spmv<float>(cudaStream_t, const Level &, const float *, const float *, float *);
template int defect<double>(cudaStream_t, const Level &, const double *, const double *, const double *, double *);
template int defect<float>(cudaStream_t, const Level &, const float *, const float *, const float *, float *);

// ----------------------------------------------------------------- SSOR
// One colour of a Gauss-Seidel sweep: rows of the colour are independent.
// x_r += omega * (f_r - (A x)_r) / a_rr   (== omega (s/diag - x_r) of MGLevel3D.C:398)
template <int W, typename T>
__global__ void __launch_bounds__(256) k_gs_color(int nrows, const int *__restrict__ rows, const int *__restrict__ rp,
                                                  const int *__restrict__ kc, const T *__restrict__ a,
                                                  const T *__restrict__ invd, const T *__restrict__ f, T *x,
                                                  T omega) {
  const int lane = threadIdx.x & (W - 1);
  for (int base = warp_first_row<W>(); base < nrows; base += rows_per_grid<W>()) {
    const int k = base + (threadIdx.x & 31) / W;
    const int row = k < nrows ? ldg(rows + k) : -1;
    T s = 0;
    if (row >= 0) {
      const int beg = ldg(rp + row), end = ldg(rp + row + 1);
      for (int j = beg + lane; j < end; j += W) s += ldg(a + j) * x[ldg(kc + j)];
    }
    s = group_sum<W>(s);
    if (lane == 0 && row >= 0) x[row] += omega * (ldg(f + row) - s) * ldg(invd + row);
  }
}

template <typename T>
__global__ void k_copy_dirichlet(int Na, int N, const T *__restrict__ f, T *__restrict__ x) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + Na;
  if (i < N) x[i] = f[i];
}

template <typename T>
int ssor_sweep(cudaStream_t s, const Level &L, const T *A, const T *invdiag, const T *f, T *x, double omega) {
  int nd = L.N - L.Na;
  if (nd > 0) { k_copy_dirichlet<T><<<(nd + 255) / 256, 256, 0, s>>>(L.Na, L.N, f, x); count_launches(1); }
  int W = pick_width(L);
  int nc = (int)L.rcolor_ptr.size() - 1;
  for (int pass = 0; pass < 2; pass++) {
    for (int cc = 0; cc < nc; cc++) {
      int c = pass == 0 ? cc : nc - 1 - cc;
      int beg = L.rcolor_ptr[c], n = L.rcolor_ptr[c + 1] - beg;
      if (n <= 0) continue;
      int g = grid_for(n, W, 148);
      const int *rows = L.row_list.p + beg;
      if (W == 32) { k_gs_color<32, T><<<g, 256, 0, s>>>(n, rows, L.rowptr.p, L.kcol.p, A, invdiag, f, x, (T)omega); count_launches(1); }
      else if (W == 16) { k_gs_color<16, T><<<g, 256, 0, s>>>(n, rows, L.rowptr.p, L.kcol.p, A, invdiag, f, x, (T)omega); count_launches(1); }
      else { k_gs_color<8, T><<<g, 256, 0, s>>>(n, rows, L.rowptr.p, L.kcol.p, A, invdiag, f, x, (T)omega); count_launches(1); }
    }
  }
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}
template int ssor_sweep<double>(cudaStream_t, const Level &, const double *, const double *, const double *, double *, double);
template int ssor_sweep<float>(cudaStream_t, const Level &, const float *, const float *, const float *, float *, double);

// ----------------------------------------------------------------- transfers
template <int W, typename T>
__global__ void __launch_bounds__(256) k_restrict(int Nc, int Nac, const int *__restrict__ rp, const int *__restrict__ col,
                                                  const T *__restrict__ val, const T *__restrict__ d, T *__restrict__ fc,
                                                  T *__restrict__ xc) {
  pdl_wait();
  pdl_trigger();
  const int lane = threadIdx.x & (W - 1);
  for (int base = warp_first_row<W>(); base < Nc; base += rows_per_grid<W>()) {
    const int row = base + (threadIdx.x & 31) / W;
    T s = 0;
    if (row < Nac) {
      const int beg = ldg(rp + row), end = ldg(rp + row + 1);
      for (int k = beg + lane; k < end; k += W) s += ldg(val + k) * ldg(d + ldg(col + k));
    }
    s = group_sum<W>(s);
    if (lane == 0 && row < Nc) {
      fc[row] = s;
      if (xc) xc[row] = (T)0;  // the coarse cycle starts from zero
    }
  }
}

template <int W, typename T>
__global__ void __launch_bounds__(256) k_prolong_add(int Naf, const int *__restrict__ rp, const int *__restrict__ col,
                                                     const T *__restrict__ val, const T *__restrict__ xc,
                                                     T *__restrict__ xf, T damp) {
  pdl_wait();
  pdl_trigger();
  const int lane = threadIdx.x & (W - 1);
  for (int base = warp_first_row<W>(); base < Naf; base += rows_per_grid<W>()) {
    const int row = base + (threadIdx.x & 31) / W;
    T s = 0;
    if (row < Naf) {
      const int beg = ldg(rp + row), end = ldg(rp + row + 1);
      for (int k = beg + lane; k < end; k += W) s += ldg(val + k) * ldg(xc + ldg(col + k));
    }
    s = group_sum<W>(s);
    if (lane == 0 && row < Naf) xf[row] += damp * s;
  }
}

template <typename T>
int restrict_defect(cudaStream_t s, const Level &Lf, const Level &Lc, const T *rval, const T *d, T *fc, T *xc) {
  // R = P^T has up to 27 (Q1) / 125 (Q2) entries per coarse row; 8 lanes a
  // row (64^3 Q2 FP32 V-cycle: 16 lanes 3.57 ms, 8 lanes 3.56, 32 lanes 3.58)
  int g = grid_for(Lc.N, 8, 148);
  PMG_CUDA(launch_pdl(k_restrict<8, T>, dim3(g), dim3(256), 0, s, Lc.N, Lc.Na, (const int *)Lf.rrp.p,
                      (const int *)Lf.rcol.p, rval, d, fc, xc));
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}
template <typename T>
int prolongate_add(cudaStream_t s, const Level &Lf, const T *pval, const T *xc, T *xf, double damp) {
  // 4 lanes a fine row (64^3 Q2 FP32 V-cycle: 8 lanes 3.53 ms, 4 lanes 3.47,
  // 2 lanes 3.46-3.47, 16 lanes 3.64)
  int g = grid_for(Lf.Na, 4, 148);
  PMG_CUDA(launch_pdl(k_prolong_add<4, T>, dim3(g), dim3(256), 0, s, Lf.Na, (const int *)Lf.prp.p,
                      (const int *)Lf.pcol.p, pval, xc, xf, (T)damp));
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}
template int restrict_defect<double>(cudaStream_t, const Level &, const Level &, const double *, const double *, double *, double *);
template int restrict_defect<float>(cudaStream_t, const Level &, const Level &, const float *, const float *, float *, float *);
template int prolongate_add<double>(cudaStream_t, const Level &, const double *, const double *, double *, double);
template int prolongate_add<float>(cudaStream_t, const Level &, const float *, const float *, float *, double);

// ----------------------------------------------------------------- diagonal
__global__ void k_invdiag(int N, const int *__restrict__ dpos, const double *__restrict__ a, double *invd,
                          float *invd32, int *flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int p = dpos[i];
  double v = p >= 0 ? a[p] : 0.0;
  if (v == 0.0 || !isfinite(v)) { atomicOr(flags, 4); v = 1.0; }
  invd[i] = 1.0 / v;
  if (invd32) invd32[i] = (float)(1.0 / v);
}



__global__ void k_f64_to_f32(size_t n, const double *__restrict__ a, float *__restrict__ b) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
static int vec_grid(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}
int convert_f64_f32(cudaStream_t s, const double *a, float *b, size_t n) {
  k_f64_to_f32<<<vec_grid(n), 256, 0, s>>>(n, a, b); count_launches(1);
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}
int copy_dirichlet(cudaStream_t s, int Na, int N, const double *f, double *x) {
  int nd = N - Na;
  if (nd > 0) { k_copy_dirichlet<double><<<(nd + 255) / 256, 256, 0, s>>>(Na, N, f, x); count_launches(1); }
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}

// ----------------------------------------------------------------- BLAS-1
constexpr int RED_BLOCKS = 296;  // 2 x 148 SMs
constexpr int RED_THREADS = 512;

// Fixed-order two-level reduction: every block writes its partial sum, the
// last block to finish adds the partials in index order (reproducible).
__global__ void __launch_bounds__(RED_THREADS) k_dot(size_t n, const double *__restrict__ a, const double *__restrict__ b,
                                                     double *partial, unsigned int *counter, double *result) {
  pdl_wait();
  pdl_trigger();
  __shared__ double sh[RED_THREADS / 32];
  __shared__ bool last;
  double s = 0;
  // four independent elements per thread and round (more loads in flight)
  const size_t st = (size_t)gridDim.x * blockDim.x;
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + 3 * st < n; i += 4 * st) {
    const double a0 = a[i], a1 = a[i + st], a2 = a[i + 2 * st], a3 = a[i + 3 * st];
    const double b0 = b[i], b1 = b[i + st], b2 = b[i + 2 * st], b3 = b[i + 3 * st];
    s += a0 * b0;
    s += a1 * b1;
    s += a2 * b2;
    s += a3 * b3;
  }
  for (; i < n; i += st) s += a[i] * b[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < RED_THREADS / 32; w++) t += sh[w];
    partial[blockIdx.x] = t;
    __threadfence();
    unsigned int prev = atomicAdd(counter, 1u);
    last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x < 32) {
    __threadfence();
    double t = 0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += 32) t += ((volatile double *)partial)[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) {
      *result = t;
      *counter = 0;
    }
  }
}

// One step of modified Gram-Schmidt fused with the next step's inner product:
//   w -= h_k v_k  (h_k read from device memory),  *h_next = w . u
// with u = v_{k+1}, or u = w for the squared norm after the last step.  The
// same fixed-order two-level reduction as k_dot.
__global__ void __launch_bounds__(RED_THREADS) k_mgs_step(size_t n, const double *__restrict__ hk,
                                                          const double *__restrict__ vk, const double *u, double *w,
                                                          double *partial, unsigned int *counter, double *h_next) {
  pdl_wait();
  pdl_trigger();
  __shared__ double sh[RED_THREADS / 32];
  __shared__ bool last;
  const double al = *hk;
  const bool self = u == w;
  double s = 0;
  // four independent elements per thread and round (more loads in flight)
  const size_t st = (size_t)gridDim.x * blockDim.x;
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + 3 * st < n; i += 4 * st) {
    double wv[4], uv[4];
#pragma unroll
    for (int q = 0; q < 4; q++) wv[q] = w[i + q * st] - al * __ldg(vk + i + q * st);
    if (!self) {
#pragma unroll
      for (int q = 0; q < 4; q++) uv[q] = u[i + q * st];
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      w[i + q * st] = wv[q];
      s += wv[q] * (self ? wv[q] : uv[q]);
    }
  }
  for (; i < n; i += st) {
    const double wi = w[i] - al * __ldg(vk + i);
    w[i] = wi;
    s += wi * (self ? wi : u[i]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int q = 0; q < RED_THREADS / 32; q++) t += sh[q];
    partial[blockIdx.x] = t;
    __threadfence();
    unsigned int prev = atomicAdd(counter, 1u);
    last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x < 32) {
    __threadfence();
    double t = 0;
    for (int q = threadIdx.x; q < (int)gridDim.x; q += 32) t += ((volatile double *)partial)[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) {
      *h_next = t;
      *counter = 0;
    }
  }
}

int mgs_step(Handle &h, size_t n, const double *hk_dev, const double *vk, const double *u, double *w, double *h_next) {
  PMG_CUDA(launch_pdl(k_mgs_step, dim3(RED_BLOCKS), dim3(RED_THREADS), 0, h.stream, n, hk_dev, vk, u, w,
                      h.red_partial.p, h.red_counter.p, h_next));
  count_launches(1);
  return PMG_OK;
}

int dot(Handle &h, const double *a, const double *b, size_t n, double *result_dev) {
  PMG_CUDA(launch_pdl(k_dot, dim3(RED_BLOCKS), dim3(RED_THREADS), 0, h.stream, n, a, b, h.red_partial.p,
                      h.red_counter.p, result_dev));
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}

// y = x / sqrt(*nrm2)   (nrm2 = squared norm in device memory; 0 -> y = 0)
__global__ void k_scale_inv_sqrt(size_t n, const double *__restrict__ nrm2, const double *__restrict__ x,
                                 double *__restrict__ y) {
  pdl_wait();
  pdl_trigger();
  double nv = sqrt(*nrm2);
  double s = nv > 0 ? 1.0 / nv : 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = x[i] * s;
}
int scale_by_inv_sqrt(cudaStream_t s, size_t n, const double *nrm2_dev, const double *x, double *y) {
  PMG_CUDA(launch_pdl(k_scale_inv_sqrt, dim3(vec_grid(n)), dim3(256), 0, s, n, nrm2_dev, x, y));
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}

__global__ void k_fill(size_t n, double *x, double v) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) x[i] = v;
}
int fill(cudaStream_t s, double *x, double v, size_t n) {
  k_fill<<<vec_grid(n), 256, 0, s>>>(n, x, v); count_launches(1);
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}
template <typename T>
int zero(cudaStream_t s, T *x, size_t n) {
  PMG_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), s));
  return PMG_OK;
}
template int zero<double>(cudaStream_t, double *, size_t);
template int zero<float>(cudaStream_t, float *, size_t);

__global__ void k_check_finite(size_t n, const double *x, int *flag) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (!isfinite(x[i])) { atomicOr(flag, 8); return; }
}
int check_finite(cudaStream_t s, const double *x, size_t n, int *flag) {
  k_check_finite<<<vec_grid(n), 256, 0, s>>>(n, x, flag); count_launches(1);
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}

// inverse diagonals of a level (FP64, and FP32 if the FP32 copy exists)
int level_invdiag(cudaStream_t s, Level &L, int *flags) {
  PMG_TRY(L.invdiag.alloc(L.N));
  float *i32 = nullptr;
  if (L.A32.p) {
    PMG_TRY(L.invdiag32.alloc(L.N));
    i32 = L.invdiag32.p;
  }
  k_invdiag<<<(L.N + 255) / 256, 256, 0, s>>>(L.N, L.diagpos.p, L.A.p, L.invdiag.p, i32, flags); count_launches(1);
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}

}  // namespace pmg
