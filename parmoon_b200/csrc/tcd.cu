// Time-dependent convection-diffusion on the device: the theta-scheme system
// of TSystemTCD3D (src/System/SystemTCD3D.C:208-347).
//
//   pmg_assemble(MASS[_SUPG])         AssembleMRhs: M and f(t_0) on every level
//   pmg_assemble(GALERKIN / SUPG)     AssembleARhs: A and f(t_new)
//   pmg_tcd_system(tau, theta)        AssembleSystMat: right-hand side B, and
//                                     A := M + tau theta1 A on every level
//   pmg_solve                         Solve: FGMRES + V-cycle on M + tau theta1 A
//   pmg_tcd_restore                   RestoreMassMat: A back
//
// The reference forms M - tau theta2 A in place of M and then adds
// (tau theta2 + tau theta1) A; the device keeps M untouched and saves A
// instead, so "restore" is a copy back.  Active rows come first in the dof
// numbering, so the active part of a matrix is the contiguous entry range
// [0, row_ptr[Na]).
#include "pmg_internal.h"

namespace pmg {

// B = tau th3 f_old + tau th4 f_new + (M - tau th2 A) u_old on active rows;
// Dirichlet rows: B = f_new, start vector x0 = f_new (else u_old)
__global__ void k_tcd_rhs(int N, int Na, const int *__restrict__ rp, const int *__restrict__ kc,
                          const double *__restrict__ M, const double *__restrict__ A, const double *__restrict__ u_old,
                          const double *__restrict__ f_old, const double *__restrict__ f_new, double c3, double c4,
                          double c2, double *__restrict__ B, double *__restrict__ x0) {
  const int lane = threadIdx.x & 31;
  for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); base < N; base += (gridDim.x * blockDim.x) >> 5) {
    const int row = base;
    double sm = 0.0, sa = 0.0;
    if (row < Na)
      for (int k = rp[row] + lane; k < rp[row + 1]; k += 32) {
        const double u = u_old[kc[k]];
        sm += M[k] * u;
        sa += A[k] * u;
      }
    for (int o = 16; o > 0; o >>= 1) {
      sm += __shfl_xor_sync(0xffffffffu, sm, o);
      sa += __shfl_xor_sync(0xffffffffu, sa, o);
    }
    if (lane == 0) {
      if (row < Na) {
        B[row] = c3 * f_old[row] + c4 * f_new[row] + (sm - c2 * sa);
        x0[row] = u_old[row];
      } else {
        B[row] = f_new[row];
        x0[row] = f_new[row];
      }
    }
  }
}

// A := M + c A on the entries [0, n) (the active rows)
__global__ void k_tcd_matrix(size_t n, const double *__restrict__ M, double *__restrict__ A, double c) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    A[k] = M[k] + c * A[k];
}

}  // namespace pmg

using namespace pmg;

extern "C" int pmg_tcd_system(pmg_handle hh, double tau, const double theta[4], const double *f_old,
                              const double *u_old, double *rhs_out) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || !theta || !(tau > 0)) {
    set_error("pmg_tcd_system: bad arguments");
    return PMG_ERR_ARG;
  }
  for (auto &L : h->lv)
    if (!L.assembled || !L.M.p) {
      set_error("pmg_tcd_system: assemble the mass and the stiffness forms on every level first");
      return PMG_ERR_STATE;
    }
  if (h->tcd_active) {
    set_error("pmg_tcd_system: the system is assembled; call pmg_tcd_restore first (SystemTCD3D.C:266-270)");
    return PMG_ERR_STATE;
  }
  Level &F = h->lv.back();
  const size_t N = F.N;
  cudaStream_t s = h->stream;
  DBuf<double> uo_host, fo_host;
  const double *uo, *fo;
  if (u_old) {
    PMG_TRY(uo_host.upload(u_old, N, s));
    uo = uo_host.p;
  } else {
    if (!h->sol.p || h->krylov_n != (int)N) {
      set_error("pmg_tcd_system: no previous solution on the device; pass u_old");
      return PMG_ERR_STATE;
    }
    uo = h->sol.p;
  }
  if (f_old) {
    PMG_TRY(fo_host.upload(f_old, N, s));
    fo = fo_host.p;
  } else {
    if (!h->tcd_fold.p) {
      set_error("pmg_tcd_system: no previous rhs on the device; pass f_old");
      return PMG_ERR_STATE;
    }
    fo = h->tcd_fold.p;
  }
  // B into a scratch, the start vector into x0; f_new (the assembled rhs) is kept as the next f_old
  DBuf<double> B, x0;
  PMG_TRY(B.alloc(N));
  PMG_TRY(x0.alloc(N));
  const double c3 = tau * theta[2], c4 = tau * theta[3], c2 = tau * theta[1], c1 = tau * theta[0];
  int blocks = (int)std::min<size_t>((N + 7) / 8, (size_t)h->num_sms * 32);
  k_tcd_rhs<<<blocks, 256, 0, s>>>(F.N, F.Na, F.rowptr.p, F.kcol.p, F.M.p, F.A.p, uo, fo, F.rhs.p, c3, c4, c2, B.p, x0.p);
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  PMG_TRY(h->tcd_fold.alloc(N));
  PMG_CUDA(cudaMemcpyAsync(h->tcd_fold.p, F.rhs.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  PMG_CUDA(cudaMemcpyAsync(F.rhs.p, B.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  // the solve starts from u_old (with the new Dirichlet values)
  if (h->krylov_n != (int)N || !h->sol.p) {
    PMG_TRY(h->sol.alloc(N));
  }
  PMG_CUDA(cudaMemcpyAsync(h->sol.p, x0.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  h->sol_preset = true;
  // system matrix on every level, stiffness saved for pmg_tcd_restore
  for (auto &L : h->lv) {
    PMG_TRY(L.Astash.alloc(L.nnz));
    PMG_CUDA(cudaMemcpyAsync(L.Astash.p, L.A.p, sizeof(double) * L.nnz, cudaMemcpyDeviceToDevice, s));
    const size_t nact = L.h_rowptr[L.Na];
    int b2 = (int)std::min<size_t>((nact + 255) / 256, (size_t)h->num_sms * 32);
    if (nact > 0) {
      k_tcd_matrix<<<b2, 256, 0, s>>>(nact, L.M.p, L.A.p, c1);
      count_launches(1);
    }
    L.sell_val_fresh32 = L.sell_val_fresh64 = false;
    L.lw_fresh = false;
  }
  PMG_CUDA(cudaGetLastError());
  h->coarse_ready = false;
  h->tcd_active = true;
  if (rhs_out) PMG_CUDA(cudaMemcpyAsync(rhs_out, F.rhs.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
  PMG_CUDA(cudaStreamSynchronize(s));
  return PMG_OK;
}

extern "C" int pmg_tcd_restore(pmg_handle hh) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h) return PMG_ERR_ARG;
  if (!h->tcd_active) {
    set_error("pmg_tcd_restore: the system is not assembled (SystemTCD3D.C:340-345)");
    return PMG_ERR_STATE;
  }
  for (auto &L : h->lv) {
    PMG_CUDA(cudaMemcpyAsync(L.A.p, L.Astash.p, sizeof(double) * L.nnz, cudaMemcpyDeviceToDevice, h->stream));
    L.sell_val_fresh32 = L.sell_val_fresh64 = false;
    L.lw_fresh = false;
  }
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  h->coarse_ready = false;
  h->tcd_active = false;
  return PMG_OK;
}
