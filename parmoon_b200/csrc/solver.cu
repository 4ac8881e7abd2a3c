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
#include <cmath>
#include <vector>

namespace pmg {

int level_invdiag(cudaStream_t s, Level &L, int *flags);

// ----------------------------------------------------------------- coarse LU
// One CTA factors the n x n row-major matrix in place (partial pivoting).
__global__ void __launch_bounds__(1024) k_dense_lu(int n, double *A, int *piv, int *flags) {
  __shared__ double sval[32];
  __shared__ int sidx[32];
  __shared__ int spiv;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int k = 0; k < n; k++) {
    // pivot search in column k
    double best = -1.0;
    int bi = k;
    for (int i = k + tid; i < n; i += nt) {
      double v = fabs(A[(size_t)i * n + k]);
      if (v > best) { best = v; bi = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_xor_sync(0xffffffffu, best, o);
      int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
    }
    if ((tid & 31) == 0) { sval[tid >> 5] = best; sidx[tid >> 5] = bi; }
    __syncthreads();
    if (tid == 0) {
      double b = -1.0;
      int p = k;
      for (int w = 0; w < (nt + 31) / 32; w++)
        if (sval[w] > b || (sval[w] == b && sidx[w] < p)) { b = sval[w]; p = sidx[w]; }
      spiv = p;
      piv[k] = p;
      if (!(b > 0.0)) atomicOr(flags, 16);
    }
    __syncthreads();
    const int p = spiv;
    if (p != k)
      for (int j = tid; j < n; j += nt) {
        double t = A[(size_t)k * n + j];
        A[(size_t)k * n + j] = A[(size_t)p * n + j];
        A[(size_t)p * n + j] = t;
      }
    __syncthreads();
    const double inv = 1.0 / A[(size_t)k * n + k];
    for (int i = k + 1 + tid; i < n; i += nt) A[(size_t)i * n + k] *= inv;
    __syncthreads();
    const int m = n - k - 1;
    for (int t = tid; t < m * m; t += nt) {
      int i = k + 1 + t / m, j = k + 1 + t % m;
      A[(size_t)i * n + j] -= A[(size_t)i * n + k] * A[(size_t)k * n + j];
    }
    __syncthreads();
  }
}

// Column c of the inverse: solve L U x = P e_c, one warp per column.
__global__ void k_dense_inverse(int n, const double *__restrict__ LU, const int *__restrict__ piv, double *work,
                                double *Inv) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  double *y = work + (size_t)warp * n;
  // b = P e_c: apply the row swaps to e_c
  for (int i = lane; i < n; i += 32) y[i] = (i == warp) ? 1.0 : 0.0;
  __syncwarp();
  if (lane == 0)
    for (int k = 0; k < n; k++) {
      int p = piv[k];
      if (p != k) { double t = y[k]; y[k] = y[p]; y[p] = t; }
    }
  __syncwarp();
  for (int i = 1; i < n; i++) {  // unit lower triangle
    double s = 0;
    for (int j = lane; j < i; j += 32) s += LU[(size_t)i * n + j] * y[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[i] -= s;
    __syncwarp();
  }
  for (int i = n - 1; i >= 0; i--) {  // upper triangle
    double s = 0;
    for (int j = i + 1 + lane; j < n; j += 32) s += LU[(size_t)i * n + j] * y[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[i] = (y[i] - s) / LU[(size_t)i * n + i];
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) Inv[(size_t)i * n + warp] = y[i];
}

__global__ void k_csr_to_dense(int n, const int *__restrict__ rp, const int *__restrict__ kc, const double *__restrict__ a,
                               double *D) {
  int i = blockIdx.x;
  if (i >= n) return;
  for (int j = threadIdx.x; j < n; j += blockDim.x) D[(size_t)i * n + j] = 0.0;
  __syncthreads();
  for (int k = rp[i] + threadIdx.x; k < rp[i + 1]; k += blockDim.x) D[(size_t)i * n + kc[k]] = a[k];
}

// x = Inv f  (dense GEMV in FP64; f, x in T)
template <typename T>
__global__ void __launch_bounds__(256) k_dense_apply(int n, const double *__restrict__ Inv, const T *__restrict__ f, T *x) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  double s = 0;
  for (int j = lane; j < n; j += 32) s += Inv[(size_t)warp * n + j] * (double)f[j];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) x[warp] = (T)s;
}

int coarse_factor(Handle &h) {
  Level &L = h.lv[0];
  int n = L.N;
  if (n > 4096) {
    set_error("coarsest level too large for the dense direct solve (n > 4096)");
    return PMG_ERR_UNSUPPORTED;
  }
  PMG_TRY(h.coarse_lu.alloc((size_t)n * n));
  PMG_TRY(h.coarse_inv.alloc((size_t)n * n));
  PMG_TRY(h.coarse_piv.alloc(n));
  DBuf<double> work;
  PMG_TRY(work.alloc((size_t)n * n));
  PMG_CUDA(cudaMemsetAsync(h.d_flags.p, 0, sizeof(int) * 4, h.stream));
  k_csr_to_dense<<<n, 256, 0, h.stream>>>(n, L.rowptr.p, L.kcol.p, L.A.p, h.coarse_lu.p); count_launches(1);
  k_dense_lu<<<1, 1024, 0, h.stream>>>(n, h.coarse_lu.p, h.coarse_piv.p, h.d_flags.p); count_launches(1);
  k_dense_inverse<<<(n * 32 + 255) / 256, 256, 0, h.stream>>>(n, h.coarse_lu.p, h.coarse_piv.p, work.p, h.coarse_inv.p); count_launches(1);
  PMG_CUDA(cudaGetLastError());
  int flags[4];
  PMG_CUDA(cudaMemcpyAsync(flags, h.d_flags.p, sizeof(flags), cudaMemcpyDeviceToHost, h.stream));
  PMG_CUDA(cudaStreamSynchronize(h.stream));
  if (flags[0] & 16) {
    set_error("zero pivot in the coarsest-level factorisation");
    return PMG_ERR_SINGULAR;
  }
  h.coarse_ready = true;
  return PMG_OK;
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
};
template <> struct Prec<float> {
  static const float *A(const Level &L) { return L.A32.p; }
  static const float *invd(const Level &L) { return L.invdiag32.p; }
  static float *x(Level &L) { return L.x32.p; }
  static float *f(Level &L) { return L.f32.p; }
  static float *d(Level &L) { return L.d32.p; }
  static const float *P(const Level &L) { return L.pval32.p; }
  static const float *R(const Level &L) { return L.rval32.p; }
};

template <typename T>
static int vcycle(Handle &h, int i) {
  cudaStream_t s = h.stream;
  Level &L = h.lv[i];
  using PT = Prec<T>;
  if (i == 0) {
    if (h.prm.coarse_smoother == PMG_COARSE_DIRECT) {
      k_dense_apply<T><<<(L.N * 32 + 255) / 256, 256, 0, s>>>(L.N, h.coarse_inv.p, PT::f(L), PT::x(L)); count_launches(1);
      PMG_CUDA(cudaGetLastError());
    } else {
      int it = h.prm.coarse_maxit > 0 ? h.prm.coarse_maxit : 1;
      for (int k = 0; k < it; k++) PMG_TRY(ssor_sweep<T>(s, L, PT::A(L), PT::invd(L), PT::f(L), PT::x(L), h.prm.smooth_omega));
    }
    return PMG_OK;
  }
  Level &C = h.lv[i - 1];
  for (int k = 0; k < h.prm.pre_smooth; k++)
    PMG_TRY(ssor_sweep<T>(s, L, PT::A(L), PT::invd(L), PT::f(L), PT::x(L), h.prm.smooth_omega));
  PMG_TRY(defect<T>(s, L, PT::A(L), PT::x(L), PT::f(L), PT::d(L)));
  PMG_TRY(restrict_defect<T>(s, L, C, PT::R(L), PT::d(L), PT::f(C)));
  PMG_TRY(zero<T>(s, PT::x(C), C.N));
  PMG_TRY(vcycle<T>(h, i - 1));
  PMG_TRY(prolongate_add<T>(s, L, PT::P(L), PT::x(C), PT::x(L), h.prm.gmg_damp));
  for (int k = 0; k < h.prm.post_smooth; k++)
    PMG_TRY(ssor_sweep<T>(s, L, PT::A(L), PT::invd(L), PT::f(L), PT::x(L), h.prm.smooth_omega));
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
    if (fp32) {
      PMG_TRY(L.A32.alloc(L.nnz));
      PMG_TRY(convert_f64_f32(h.stream, L.A.p, L.A32.p, L.nnz));
      PMG_TRY(L.x32.alloc(L.N)); PMG_TRY(L.f32.alloc(L.N)); PMG_TRY(L.d32.alloc(L.N));
      if (i > 0) {
        PMG_TRY(L.pval32.alloc(L.pval.n));
        PMG_TRY(convert_f64_f32(h.stream, L.pval.p, L.pval32.p, L.pval.n));
        PMG_TRY(L.rval32.alloc(L.rval.n));
        PMG_TRY(convert_f64_f32(h.stream, L.rval.p, L.rval32.p, L.rval.n));
      }
    }
    PMG_TRY(level_invdiag(h.stream, L, h.d_flags.p));
  }
  if (h.prm.coarse_smoother == PMG_COARSE_DIRECT && !h.coarse_ready) PMG_TRY(coarse_factor(h));
  return PMG_OK;
}

static int capture_vcycle(Handle &h) {
  if (h.vgraph && h.vgraph_prec == h.prm.precision) return PMG_OK;
  if (h.vgraph) { cudaGraphExecDestroy(h.vgraph); h.vgraph = nullptr; }
  cudaGraph_t g;
  const unsigned long long before = launches_so_far();
  PMG_CUDA(cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal));
  int top = (int)h.lv.size() - 1;
  int rc = h.prm.precision == PMG_PREC_FP32 ? vcycle<float>(h, top) : vcycle<double>(h, top);
  cudaError_t e = cudaStreamEndCapture(h.stream, &g);
  if (rc != PMG_OK) return rc;
  PMG_CUDA(e);
  PMG_CUDA(cudaGraphInstantiate(&h.vgraph, g, 0));
  cudaGraphDestroy(g);
  // kernels recorded during capture run at each replay, not now
  h.vgraph_kernels = launches_so_far() - before;
  count_launches(0ULL - h.vgraph_kernels);
  h.vgraph_prec = h.prm.precision;
  return PMG_OK;
}

// z = MG(v): one V-cycle with zero start (MultiGridScaIte.C:89-130)
static int precondition(Handle &h, const double *v, double *z) {
  Level &F = h.lv.back();
  int nb = (F.N + 255) / 256;
  if (h.prm.precision == PMG_PREC_FP32) {
    k_prec_in32<<<nb, 256, 0, h.stream>>>(F.Na, F.N, v, F.f32.p, F.x32.p); count_launches(1);
    PMG_CUDA(cudaGraphLaunch(h.vgraph, h.stream));
    count_launches(h.vgraph_kernels);
    k_prec_out32<<<nb, 256, 0, h.stream>>>(F.N, F.x32.p, z); count_launches(1);
  } else {
    k_prec_in64<<<nb, 256, 0, h.stream>>>(F.Na, F.N, v, F.f64.p, F.x64.p); count_launches(1);
    PMG_CUDA(cudaGraphLaunch(h.vgraph, h.stream));
    count_launches(h.vgraph_kernels);
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
  PMG_TRY(prepare_levels(h));
  PMG_TRY(capture_vcycle(h));
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
  else PMG_TRY(zero<double>(s, h.sol.p, N));
  // Dirichlet part of the start vector = rhs (TSystemCD3D::Assemble copies it, SystemCD3D.C:361)
  PMG_TRY(copy_dirichlet(s, F.Na, F.N, h.rhs.p, h.sol.p));
  PMG_CUDA(cudaEventRecord(h.ev[2], s));

  double *V = h.V.p, *Z = h.Z.p, *w = h.w.p;
  double *Hd = h.H.p;  // column i at Hd + i*(m+1); scratch scalars after (m+1)^2
  double *sc = Hd + (size_t)(m + 1) * (m + 1);
  std::vector<double> H((size_t)(m + 1) * m, 0.0), sv(m + 1), cs(m), sn(m), y(m);
  double *hcol = h.h_H;

  auto residual = [&](double *out_vec, double &nrm) -> int {
    PMG_TRY(defect<double>(s, F, F.A.p, h.sol.p, h.rhs.p, out_vec));
    PMG_TRY(dot(h, out_vec, out_vec, N, sc));
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
      PMG_TRY(precondition(h, vi, zi));
      PMG_TRY(spmv<double>(s, F, F.A.p, zi, w));
      double *Hc = Hd + (size_t)i * (m + 1);
      for (int k = 0; k <= i; k++) {
        PMG_TRY(dot(h, w, V + (size_t)k * N, N, Hc + k));
        PMG_TRY(axpy_dev(s, N, Hc + k, -1.0, V + (size_t)k * N, w));
      }
      PMG_TRY(dot(h, w, w, N, Hc + i + 1));
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
  PMG_CUDA(cudaEventRecord(h.ev[3], s));
  double res_final;
  PMG_TRY(residual(w, res_final));
  float ms = 0;
  PMG_CUDA(cudaEventElapsedTime(&ms, h.ev[2], h.ev[3]));
  h.t_solve = ms * 1e-3;
  if (sol_host) PMG_CUDA(cudaMemcpyAsync(sol_host, h.sol.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
  PMG_CUDA(cudaStreamSynchronize(s));
  if (st) {
    st->iterations = iters;
    st->res0 = res0;
    st->res_final = res_final;
    st->rel_res = res0 > 0 ? res_final / res0 : 0.0;
    st->mean_contraction = (iters > 0 && res0 > 0 && res_final > 0) ? pow(res_final / res0, 1.0 / iters) : 0.0;
    st->smoother_used = h.prm.smoother;
    st->seconds = h.t_solve;
  }
  return status;
}

}  // namespace pmg
