// The coarse end of the V-cycle in one launch: one thread-block cluster
// (up to 16 CTAs x 32 warps on one GPC) runs TMultiGrid3D::Cycle
// (src/FE/MultiGrid3D.C:449-695) for every level from `top` down to the
// coarsest and back up -- pre-smoothing, defect, restriction, the coarsest
// solve, prolongation, post-smoothing -- with a cluster barrier wherever the
// level-by-level path starts a new kernel.
//
// Why: below ~50k rows a colour sweep is a few microseconds of work, so the
// colour-by-colour launches (2 x 27 per Q2 SSOR step) are launch and L2
// latency: levels 1-2 of the 64^3 Q2 hierarchy cost about as much as the
// 2.1M-row finest level.
//
// Layout: every CTA keeps a full copy of the iterate x of each level of the
// cycle in its shared memory (35,937 + 4,913 + 729 floats for the 64^3 Q2
// hierarchy, 166 KB).  A colour pass gathers x from the local copy (no L2
// round trip) and a row update is stored to all copies through distributed
// shared memory; barrier.cluster.arrive.release / wait.acquire between passes
// makes the stores visible.  Matrices, f, d and the transfers stay in global
// memory (L2-resident at these sizes) and are loaded before the x gathers.
// The arithmetic is the level-by-level path's -- the same SELL-32 slices,
// colour order, omega, damping and coarsest solve -- up to the order of the
// partial sums inside a row.
#include "pmg_internal.h"
#include <cooperative_groups.h>
#include <algorithm>
#include <cstdlib>
#include <string>

namespace cg = cooperative_groups;

namespace pmg {

constexpr int CC_MAX_LEVELS = 8, CC_MAX_GROUPS = 64, CC_WARPS = 32;
constexpr size_t CC_SMEM_X = 200 * 1024;  // budget for the replicated iterates

template <typename T>
struct CcLevel {
  int N, Na, ncolors, xoff;  // xoff: offset of the level's x copy in shared memory
  int group[CC_MAX_GROUPS];  // slice range of colour c: [group[c], group[c+1]); group[ncolors+1] = all slices
  const int *perm, *sptr, *col;
  const T *val, *invd;
  // transfer between this level and the one below (this level is the fine side)
  const int *prp, *pcol, *rrp, *rcol;
  const T *pval, *rval;
  T *x, *f, *d;
};

template <typename T>
struct CcArgs {
  int nlev;  // levels 0 .. nlev-1; the cycle enters at nlev-1
  CcLevel<T> lv[CC_MAX_LEVELS];
  const double *inv;  // inverse of the coarsest level's active block (direct coarse solve) or NULL
  int direct, n0, na0, coarse_it, pre, post;
  const int *rp0, *kc0;  // coarsest CSR (FP64 values a0) for the Dirichlet columns of the rhs
  const double *a0;
  double *t0;            // reduced rhs f_a - A_ad f_d
  T omega, damp;
};

template <typename T>
struct CcCtx {
  cg::cluster_group cl;
  int warp, lane, gw, tw, rank, nblocks;
  T (*part)[32];
  T *xs;  // this CTA's shared memory holding the x copies
  __device__ void sync() { cl.sync(); }
  // x_i := v in every CTA's copy
  __device__ void bcast(int off, int i, T v) {
    for (int b = 0; b < nblocks; b++) *cl.map_shared_rank(xs + off + i, b) = v;
  }
};

// one pass over the slices [s0, s1): Gauss-Seidel update of x (GS) or d = f - A x
template <typename T, bool GS>
__device__ void cc_slices(CcCtx<T> &c, const CcLevel<T> &L, int s0, int s1, T omega) {
  const int nsl = s1 - s0;
  if (nsl <= 0) return;
  int K = c.tw / nsl;  // warps per slice: as many as the cluster offers, up to 16
  K = K >= 16 ? 16 : K >= 8 ? 8 : K >= 4 ? 4 : K >= 2 ? 2 : 1;
  const int spc = CC_WARPS / K;  // slices per CTA per round
  const int per_round = spc * c.nblocks;
  const int rounds = (nsl + per_round - 1) / per_round;
  const int k = c.warp % K;
  constexpr int PF = sizeof(T) == 4 ? 16 : 8;  // column steps loaded ahead (64 registers per thread)
  const T *x = c.xs + L.xoff;
  for (int r = 0; r < rounds; r++) {
    const int sl = s0 + r * per_round + c.rank * spc + c.warp / K;
    T sum = 0, fr = 0, id = 0;
    int row = -1;
    if (sl < s1) {
      const int off = __ldg(L.sptr + sl), lmax = (__ldg(L.sptr + sl + 1) - off) >> 5;
      const int *cp = L.col + off + c.lane;
      const T *vp = L.val + off + c.lane;
      int ci[PF];
      T cv[PF];
      // column steps in chunks of PF: loads of a chunk, then its gathers
      for (int c0 = 0; k + c0 * K < lmax; c0 += PF) {
#pragma unroll
        for (int u = 0; u < PF; u++) {
          const int j = k + (c0 + u) * K;
          ci[u] = j < lmax ? __ldg(cp + 32 * j) : -1;
          cv[u] = j < lmax ? __ldg(vp + 32 * j) : (T)0;
        }
        if (c0 == 0 && k == 0) {
          row = __ldg(L.perm + sl * 32 + c.lane);
          if (row >= 0) {
            fr = __ldcg(L.f + row);
            if (GS) id = __ldg(L.invd + sl * 32 + c.lane);
          }
        }
#pragma unroll
        for (int u = 0; u < PF; u++)
          if (ci[u] >= 0) sum += cv[u] * x[ci[u]];
      }
      if (k == 0 && lmax == 0) {
        row = __ldg(L.perm + sl * 32 + c.lane);
        if (row >= 0) {
          fr = __ldcg(L.f + row);
          if (GS) id = __ldg(L.invd + sl * 32 + c.lane);
        }
      }
    }
    c.part[c.warp][c.lane] = sum;
    __syncthreads();
    if (k == 0 && row >= 0) {
      for (int kk = 1; kk < K; kk++) sum += c.part[c.warp + kk][c.lane];
      if (GS) c.bcast(L.xoff, row, x[row] + omega * (fr - sum) * id);
      else __stcg(L.d + row, fr - sum);
    }
    __syncthreads();
  }
}

// SSOR step of TMGLevel3D::SSOR in colour order: Dirichlet rows from f, forward, backward
template <typename T>
__device__ void cc_ssor(CcCtx<T> &c, const CcLevel<T> &L, T omega) {
  // every CTA refreshes the Dirichlet rows of its own copy
  for (int i = L.Na + threadIdx.x; i < L.N; i += blockDim.x) c.xs[L.xoff + i] = __ldcg(L.f + i);
  __syncthreads();
  for (int cc = 0; cc < L.ncolors; cc++) {
    cc_slices<T, true>(c, L, L.group[cc], L.group[cc + 1], omega);
    c.sync();
  }
  for (int cc = L.ncolors - 1; cc >= 0; cc--) {
    cc_slices<T, true>(c, L, L.group[cc], L.group[cc + 1], omega);
    c.sync();
  }
}

template <typename T>
__global__ void __launch_bounds__(CC_WARPS * 32, 1) k_coarse_cycle(const __grid_constant__ CcArgs<T> a) {
  __shared__ T part[CC_WARPS][32];
  extern __shared__ __align__(16) unsigned char cc_dyn[];
  CcCtx<T> c{cg::this_cluster()};
  c.warp = threadIdx.x >> 5;
  c.lane = threadIdx.x & 31;
  c.rank = (int)c.cl.block_rank();
  c.nblocks = (int)c.cl.num_blocks();
  c.gw = c.rank * CC_WARPS + c.warp;
  c.tw = c.nblocks * CC_WARPS;
  c.part = part;
  c.xs = reinterpret_cast<T *>(cc_dyn);
  const int top = a.nlev - 1;
  // the entry level starts from x = 0 (the caller zeroed its global copy)
  for (int i = threadIdx.x; i < a.lv[top].N; i += blockDim.x) c.xs[a.lv[top].xoff + i] = (T)0;
  pdl_wait();
  pdl_trigger();
  c.sync();  // every copy initialised before any remote store
  // down: smooth, defect, restrict
  for (int l = top; l >= 1; l--) {
    const CcLevel<T> &L = a.lv[l];
    const CcLevel<T> &C = a.lv[l - 1];
    for (int s = 0; s < a.pre; s++) cc_ssor(c, L, a.omega);
    cc_slices<T, false>(c, L, 0, L.group[L.ncolors + 1], a.omega);
    // each CTA zeroes its own copy of the coarse iterate
    for (int i = threadIdx.x; i < C.N; i += blockDim.x) c.xs[C.xoff + i] = (T)0;
    c.sync();
    // restriction, 8 lanes per coarse row (R = P^T rows hold up to 125 entries)
    for (int base = c.gw * 4; base < C.N; base += c.tw * 4) {
      const int row = base + (c.lane >> 3), l8 = c.lane & 7;
      T v = 0;
      if (row < C.Na) {
        const int beg = __ldg(L.rrp + row), end = __ldg(L.rrp + row + 1);
#pragma unroll 4
        for (int q = beg + l8; q < end; q += 8) v += __ldg(L.rval + q) * __ldcg(L.d + __ldg(L.rcol + q));
      }
      v += __shfl_xor_sync(0xffffffffu, v, 4);
      v += __shfl_xor_sync(0xffffffffu, v, 2);
      v += __shfl_xor_sync(0xffffffffu, v, 1);
      if (l8 == 0 && row < C.N) __stcg(C.f + row, v);
    }
    c.sync();
  }
  // coarsest level: dense inverse (SolveExact) or SSOR steps
  const CcLevel<T> &Z = a.lv[0];
  if (a.direct) {
    // x_d = f_d; t = f_a - A_ad f_d
    for (int row = c.gw; row < a.n0; row += c.tw) {
      if (row >= a.na0) {
        if (c.lane == 0) c.bcast(Z.xoff, row, __ldcg(Z.f + row));
        continue;
      }
      double s = 0;
      for (int k = __ldg(a.rp0 + row) + c.lane; k < __ldg(a.rp0 + row + 1); k += 32) {
        const int j = __ldg(a.kc0 + k);
        if (j >= a.na0) s += __ldg(a.a0 + k) * (double)__ldcg(Z.f + j);
      }
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (c.lane == 0) __stcg(a.t0 + row, (double)__ldcg(Z.f + row) - s);
    }
    c.sync();
    // x_a = A_aa^{-1} t
    for (int row = c.gw; row < a.na0; row += c.tw) {
      double s = 0;
      const double *ir = a.inv + (size_t)row * a.na0;
      for (int j = c.lane; j < a.na0; j += 32) s += __ldg(ir + j) * __ldcg(a.t0 + j);
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (c.lane == 0) c.bcast(Z.xoff, row, (T)s);
    }
    c.sync();
  } else {
    for (int s = 0; s < a.coarse_it; s++) cc_ssor(c, Z, a.omega);
  }
  // up: prolongate, smooth
  for (int l = 1; l <= top; l++) {
    const CcLevel<T> &L = a.lv[l];
    const CcLevel<T> &C = a.lv[l - 1];
    // prolongation, one fine row per lane (P rows hold at most 27 entries)
    const T *xc = c.xs + C.xoff;
    for (int row = c.gw * 32 + c.lane; row < L.Na; row += c.tw * 32) {
      const int beg = __ldg(L.prp + row), end = __ldg(L.prp + row + 1);
      T v = 0;
#pragma unroll 4
      for (int q = beg; q < end; q++) v += __ldg(L.pval + q) * xc[__ldg(L.pcol + q)];
      c.bcast(L.xoff, row, c.xs[L.xoff + row] + a.damp * v);
    }
    c.sync();
    for (int s = 0; s < a.post; s++) cc_ssor(c, L, a.omega);
  }
  // the entry level's iterate back to global memory for the finer level
  const CcLevel<T> &E = a.lv[top];
  for (int i = c.rank * blockDim.x + threadIdx.x; i < E.N; i += c.nblocks * blockDim.x) __stcg(E.x + i, c.xs[E.xoff + i]);
}

template <typename T> static const T *lv_val(const Level &L);
template <> const float *lv_val<float>(const Level &L) { return L.sell_val32.p; }
template <> const double *lv_val<double>(const Level &L) { return L.sell_val64.p; }
template <typename T> static const T *lv_invd(const Level &L);
template <> const float *lv_invd<float>(const Level &L) { return L.sell_invd32.p; }
template <> const double *lv_invd<double>(const Level &L) { return L.sell_invd64.p; }
template <typename T> static T *lv_vec(Level &L, int which);
template <> float *lv_vec<float>(Level &L, int w) { return w == 0 ? L.x32.p : w == 1 ? L.f32.p : L.d32.p; }
template <> double *lv_vec<double>(Level &L, int w) { return w == 0 ? L.x64.p : w == 1 ? L.f64.p : L.d64.p; }
template <typename T> static const T *lv_p(const Level &L, bool r);
template <> const float *lv_p<float>(const Level &L, bool r) { return r ? L.rval32.p : L.pval32.p; }
template <> const double *lv_p<double>(const Level &L, bool r) { return r ? L.rval.p : L.pval.p; }

template <typename T>
static int cluster_ctas() {
  static int ctas = 0;
  if (ctas) return ctas;
  const void *kernel = (const void *)k_coarse_cycle<T>;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CC_SMEM_X);
  for (int want : {16, 8, 4}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(want);
    cfg.blockDim = dim3(CC_WARPS * 32);
    cfg.dynamicSmemBytes = CC_SMEM_X;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = want;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kernel, &cfg) == cudaSuccess && n > 0) {
      ctas = want;
      break;
    }
  }
  cudaGetLastError();
  return ctas;
}

// the highest level that, with every level below it, fits the cluster launch
// (0: none -- the level-by-level path runs)
// levels 0..top in one launch, opt-in: PMG_COARSE_CLUSTER=1 runs the levels
// of at most CC_ONE_CTA_ROWS rows on one CTA, PMG_COARSE_CLUSTER=16 every
// level whose iterates fit CC_SMEM_X on a 16-CTA cluster.  Both measured
// slower than the PDL-chained colour launches on the 64^3 Q2 hierarchy (a
// colour pass here ~5 us), so the default is the level-by-level path.
constexpr int CC_ONE_CTA_ROWS = 8192;

int coarse_cycle_top(Handle &h) {
  static int mode = -1;
  if (mode < 0) {
    const char *e = getenv("PMG_COARSE_CLUSTER");
    mode = !e ? 0 : (std::string(e) == "1") ? 1 : (std::string(e) == "16") ? 2 : 0;
  }
  if (mode == 0) return 0;
  const size_t vb = h.prm.precision == PMG_PREC_FP32 ? sizeof(float) : sizeof(double);
  size_t bytes = 0;
  int top = 0;
  for (int i = 0; i < (int)h.lv.size() - 1 && i < CC_MAX_LEVELS; i++) {
    const Level &L = h.lv[i];
    bytes += ((size_t)L.N * vb + 15) / 16 * 16;
    if (bytes > CC_SMEM_X || (int)L.sell_group.size() > CC_MAX_GROUPS) break;
    if (mode == 1 && L.N > CC_ONE_CTA_ROWS) break;
    top = i;
  }
  if (top < 1) return 0;
  if (mode == 1) {
    h.cc_ctas = 1;
  } else {
    // the launch shape is queried here, outside any stream capture
    const int c = std::min(cluster_ctas<float>(), cluster_ctas<double>());
    if (!c) return 0;
    h.cc_ctas = c;
  }
  return top;
}

template <typename T>
int coarse_cycle(Handle &h, int top) {
  if (top < 1 || top >= CC_MAX_LEVELS) {
    set_error("coarse_cycle: level out of range");
    return PMG_ERR_ARG;
  }
  CcArgs<T> a{};
  a.nlev = top + 1;
  size_t smem = 0;
  for (int i = 0; i <= top; i++) {
    Level &L = h.lv[i];
    CcLevel<T> &d = a.lv[i];
    d.N = L.N;
    d.Na = L.Na;
    d.xoff = (int)(smem / sizeof(T));
    smem += ((size_t)L.N * sizeof(T) + 15) / 16 * 16;
    d.ncolors = (int)L.sell_group.size() - 2;
    for (size_t g = 0; g < L.sell_group.size(); g++) d.group[g] = L.sell_group[g];
    d.perm = L.sell_perm.p;
    d.sptr = L.sell_ptr.p;
    d.col = L.sell_col.p;
    d.val = lv_val<T>(L);
    d.invd = lv_invd<T>(L);
    if (i > 0) {
      d.prp = L.prp.p; d.pcol = L.pcol.p; d.pval = lv_p<T>(L, false);
      d.rrp = L.rrp.p; d.rcol = L.rcol.p; d.rval = lv_p<T>(L, true);
    }
    d.x = lv_vec<T>(L, 0);
    d.f = lv_vec<T>(L, 1);
    d.d = lv_vec<T>(L, 2);
  }
  const bool direct = h.prm.coarse_smoother == PMG_COARSE_DIRECT;
  a.direct = direct ? 1 : 0;
  a.inv = direct ? h.coarse_inv.p : nullptr;
  a.n0 = h.lv[0].N;
  a.na0 = h.lv[0].Na;
  a.rp0 = h.lv[0].rowptr.p;
  a.kc0 = h.lv[0].kcol.p;
  a.a0 = h.lv[0].A.p;
  a.t0 = h.coarse_t.p;
  a.coarse_it = h.prm.coarse_maxit > 0 ? h.prm.coarse_maxit : 1;
  a.pre = h.prm.pre_smooth;
  a.post = h.prm.post_smooth;
  a.omega = (T)h.prm.smooth_omega;
  a.damp = (T)h.prm.gmg_damp;
  const int ctas = h.cc_ctas;
  if (ctas < 1) {
    set_error("coarse_cycle: launch shape not set");
    return PMG_ERR_STATE;
  }
  if (ctas == 1) {
    static bool attr = false;
    if (!attr) {
      PMG_CUDA(cudaFuncSetAttribute(k_coarse_cycle<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CC_SMEM_X));
      attr = true;
    }
  }
  if (smem > CC_SMEM_X) {
    set_error("coarse_cycle: iterates exceed the shared-memory budget");
    return PMG_ERR_ARG;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(CC_WARPS * 32);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = h.stream;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = ctas;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 2;
  PMG_CUDA(cudaLaunchKernelEx(&cfg, k_coarse_cycle<T>, a));
  count_launches(1);
  return PMG_OK;
}
template int coarse_cycle<float>(Handle &, int);
template int coarse_cycle<double>(Handle &, int);

}  // namespace pmg
