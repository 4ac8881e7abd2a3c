// A whole smoothing phase of a mid-size level in one launch (TMGLevel3D::SSOR,
// src/FE/MGLevel3D.C:363-467, in multicolour order).
//
// Why: on the levels between the finest and the cluster-resident coarse
// levels (35,937 and 274,625 rows on the 64^3 Q2 hierarchy) a colour pass is
// a few microseconds of work or less, so the colour-by-colour launches (2 x 27
// per SSOR step) cost mostly launch latency.
//
// How: the active rows are cut into R regions of consecutive row numbers; the
// SELL-32 copy orders the rows of each colour by region (slices never straddle
// a region), so region b owns the slice range seg[c][b] of every colour c.  One
// cooperative launch of R blocks runs the phase's pass list (the colours of
// the sweeps in order, with the same repeated-colour skips as the colour
// launches): block b updates the rows of its region and colour, then
// publishes "pass p done" in its progress counter with release semantics.
// Before pass p a block waits (acquire, bounded) until every region that
// shares a matrix coupling with its own has finished pass p-1: then the rows it
// reads carry the previous pass's values (read after write), and nobody still
// reads the rows it is about to overwrite (write after read).  No grid-wide
// barrier: a block waits only for its neighbours.  The iterate is read
// through L2 (ld.global.cg) because other SMs write it during the launch.
// The arithmetic is the colour launches' (same slices, order of the column
// steps within a warp, omega, 1/a_ii) with 4 warps per slice.
//
// Every wait is bounded (0.2 s by %globaltimer); a block that gives up sets
// the error word and returns, the blocks waiting on it then give up in turn,
// and the host reports PMG_ERR_STATE after the solve.  The launch is
// cooperative, so all R blocks are resident at once and no wait depends on an
// unscheduled block.
#include "pmg_internal.h"
#include <algorithm>
#include <cstdlib>
#include <set>

namespace pmg {

constexpr int RS_K = 4;        // warps per slice
constexpr int RS_SLOTS = 2;    // slices in flight per block
constexpr int RS_THREADS = 32 * RS_K * RS_SLOTS;
constexpr int RS_MAX_NEIGHBOURS = 32;

template <typename T>
struct RegionArgs {
  int nreg, npass, ncol;
  const int *passes;         // colour of every pass of the phase
  const int *seg;            // [c * (nreg + 1) + b]: first slice of region b in colour c
  const int *nb_ptr, *nb;    // regions coupled to region b: nb[nb_ptr[b] .. nb_ptr[b+1])
  int *prog;                 // passes finished per region (zero at launch)
  int *err;
  const int *perm, *sptr, *col;
  const short *c16;
  const unsigned char *wide;
  const T *val, *invd, *f;
  T *x;
  T omega;
};

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <typename T>
__global__ void __launch_bounds__(RS_THREADS) k_region_ssor(RegionArgs<T> a) {
  __shared__ T part[RS_SLOTS][RS_K][32];
  __shared__ int give_up;
  const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int slot = w / RS_K, wk = w % RS_K;
  const unsigned long long deadline = global_ns() + 200000000ull;  // 0.2 s for the whole phase
  for (int p = 0; p < a.npass; p++) {
    if (tid == 0) {
      int bad = 0;
      if (p > 0)
        for (int q = a.nb_ptr[b]; q < a.nb_ptr[b + 1] && !bad; q++) {
          const int *pr = a.prog + a.nb[q];
          while (ld_acquire(pr) < p) {
            if (ld_acquire(a.err) != 0 || global_ns() > deadline) { bad = 1; break; }
          }
        }
      give_up = bad;
    }
    __syncthreads();
    if (give_up) {
      if (tid == 0) atomicOr(a.err, 1);
      return;
    }
    const int c = a.passes[p];
    const int s0 = a.seg[c * (a.nreg + 1) + b], s1 = a.seg[c * (a.nreg + 1) + b + 1];
    for (int base = s0; base < s1; base += RS_SLOTS) {  // uniform trip count: the barriers below
      const int s = base + slot;
      const bool active = s < s1;
      T sum = 0;
      int r = -1;
      if (active) {
        const int off = a.sptr[s], lmax = (a.sptr[s + 1] - off) >> 5;
        r = a.perm[s * 32 + lane];
        const bool wd = a.wide[s] != 0;
        const T *xb = wd ? a.x : a.x + (r > 0 ? r : 0);
#pragma unroll 4
        for (int j = wk; j < lmax; j += RS_K) {
          const int idx = off + 32 * j + lane;
          const int ci = wd ? __ldcs(a.col + idx) : (int)__ldcs(a.c16 + idx);
          sum += __ldcs(a.val + idx) * __ldcg(xb + ci);
        }
      }
      part[slot][wk][lane] = sum;
      __syncthreads();
      if (active && wk == 0) {
#pragma unroll
        for (int k = 1; k < RS_K; k++) sum += part[slot][k][lane];
        if (r >= 0) a.x[r] = __ldcg(a.x + r) + a.omega * (__ldg(a.f + r) - sum) * __ldg(a.invd + s * 32 + lane);
      }
      __syncthreads();
    }
    if (tid == 0) {
      __threadfence();
      st_release(a.prog + b, p + 1);
    }
  }
}

// ------------------------------------------------------------------ host side

// regions of a level (0: colour launches): levels strictly between the
// cluster-resident coarse levels and the finest, at least 4 regions of ~1,500
// active rows, at most one per SM.  PMG_REGION_SWEEP=0 turns the path off.
int region_count(const Handle &h, const Level &L) {
  static int enabled = -1;
  if (enabled < 0) {
    const char *e = getenv("PMG_REGION_SWEEP");
    enabled = (e && e[0] == '0') ? 0 : 1;
  }
  if (!enabled) return 0;
  const int idx = (int)(&L - h.lv.data()), top = (int)h.lv.size() - 1;
  if (idx < 1 || idx >= top || L.Na <= 8192 || L.Na > 1000000) return 0;
  return std::max(4, std::min(h.num_sms, L.Na / 1500));
}

// region of an active row: consecutive row numbers
static inline int region_of(long r, long Na, int nreg) { return (int)(r * nreg / Na); }

int region_key(int r, int Na, int nreg) { return r < Na ? region_of(r, Na, nreg) : nreg; }

// after the SELL layout: slice ranges per (colour, region) and the coupled regions
int region_setup(Handle &h, Level &L, const std::vector<int> &perm, int nreg) {
  L.rs_nreg = 0;
  if (nreg <= 0) return PMG_OK;
  const int nc = (int)L.sell_group.size() - 2;
  std::vector<int> seg((size_t)nc * (nreg + 1));
  for (int c = 0; c < nc; c++) {
    const int s0 = L.sell_group[c], s1 = L.sell_group[c + 1];
    int s = s0;
    for (int b = 0; b <= nreg; b++) {
      // first slice of colour c whose first row lies in region >= b
      while (s < s1) {
        const int r = perm[(size_t)s * 32];
        if (r >= 0 && region_of(r, L.Na, nreg) >= b) break;
        s++;
      }
      seg[(size_t)c * (nreg + 1) + b] = b == 0 ? s0 : (b == nreg ? s1 : s);
    }
  }
  std::vector<std::set<int>> nbs(nreg);
  const std::vector<int> &rp = L.h_rowptr, &kc = L.h_kcol;
  for (int r = 0; r < L.Na; r++) {
    const int br = region_of(r, L.Na, nreg);
    for (int q = rp[r]; q < rp[r + 1]; q++) {
      const int col = kc[q];
      if (col >= L.Na) continue;
      const int bc = region_of(col, L.Na, nreg);
      if (bc == br) continue;
      nbs[br].insert(bc);
      nbs[bc].insert(br);
    }
  }
  std::vector<int> nb_ptr(nreg + 1, 0), nb;
  for (int b = 0; b < nreg; b++) {
    if ((int)nbs[b].size() > RS_MAX_NEIGHBOURS) return PMG_OK;  // numbering not local enough: colour launches
    nb.insert(nb.end(), nbs[b].begin(), nbs[b].end());
    nb_ptr[b + 1] = (int)nb.size();
  }
  if (nb.empty()) nb.push_back(0);
  PMG_TRY(L.rs_seg.upload(seg.data(), seg.size(), h.stream));
  PMG_TRY(L.rs_nb_ptr.upload(nb_ptr.data(), nb_ptr.size(), h.stream));
  PMG_TRY(L.rs_nb.upload(nb.data(), nb.size(), h.stream));
  PMG_TRY(L.rs_prog.alloc(nreg));
  if (!h.rs_err.p) {
    PMG_TRY(h.rs_err.alloc(1));
    PMG_CUDA(cudaMemsetAsync(h.rs_err.p, 0, sizeof(int), h.stream));
  }
  PMG_CUDA(cudaStreamSynchronize(h.stream));
  L.rs_nreg = nreg;
  return PMG_OK;
}

static bool cooperative_fits(int nreg, int num_sms, const void *kern) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, RS_THREADS, 0) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (long)per_sm * num_sms >= nreg;
}

// the colours of a phase of `steps` SSOR steps, in order: sell_ssor's
// sequence with its repeated-colour skips
static std::vector<int> phase_passes(int nc, int steps, double omega) {
  std::vector<int> passes;
  const bool skip = omega == 1.0;
  for (int k = 0; k < steps; k++)
    for (int pass = 0; pass < 2; pass++)
      for (int cc = 0; cc < nc; cc++) {
        if (skip && cc == 0 && (pass == 1 || k > 0)) continue;
        passes.push_back(pass == 0 ? cc : nc - 1 - cc);
      }
  return passes;
}

// before the V-cycle is captured: the pass lists of the pre- and post-smoothing
// phases on the device (a changed list drops the captured graphs, whose
// launches hold the list's address)
int region_prepare(Handle &h, Level &L) {
  if (L.rs_nreg <= 0) return PMG_OK;
  const int nc = (int)L.sell_group.size() - 2;
  const int steps[2] = {h.prm.pre_smooth, h.prm.post_smooth};
  for (int w = 0; w < 2; w++) {
    std::vector<int> passes = phase_passes(nc, steps[w], h.prm.smooth_omega);
    if (passes == L.rs_pass_host[w] && L.rs_pass[w].p) continue;
    L.rs_pass_host[w] = passes;
    if (passes.empty()) passes.push_back(0);
    PMG_TRY(L.rs_pass[w].upload(passes.data(), passes.size(), h.stream));
    invalidate_graphs(&h);
  }
  PMG_CUDA(cudaStreamSynchronize(h.stream));
  return PMG_OK;
}

// One smoothing phase (which = 0: pre, 1: post) as one launch; returns
// PMG_ERR_UNSUPPORTED when the level has no regions or the blocks cannot all
// be resident (the caller then launches colour by colour).  Only stream
// operations that graph capture accepts: a memset and a kernel launch.
template <typename T>
int region_ssor_phase(Handle &h, Level &L, const T *f, T *x, double omega, int which, bool dirichlet_first) {
  if (L.rs_nreg <= 0 || L.rs_pass_host[which].empty()) return PMG_ERR_UNSUPPORTED;
  if (!cooperative_fits(L.rs_nreg, h.num_sms, (const void *)k_region_ssor<T>)) return PMG_ERR_UNSUPPORTED;
  cudaStream_t s = h.stream;
  if (dirichlet_first) PMG_TRY(sell_copy_dirichlet<T>(s, L, f, x));
  PMG_CUDA(cudaMemsetAsync(L.rs_prog.p, 0, sizeof(int) * L.rs_nreg, s));
  RegionArgs<T> a{};
  a.nreg = L.rs_nreg;
  a.npass = (int)L.rs_pass_host[which].size();
  a.ncol = (int)L.sell_group.size() - 2;
  a.passes = L.rs_pass[which].p;
  a.seg = L.rs_seg.p;
  a.nb_ptr = L.rs_nb_ptr.p;
  a.nb = L.rs_nb.p;
  a.prog = L.rs_prog.p;
  a.err = h.rs_err.p;
  a.perm = L.sell_perm.p;
  a.sptr = L.sell_ptr.p;
  a.col = L.sell_col.p;
  a.c16 = L.sell_c16.p;
  a.wide = L.sell_wide.p;
  a.val = sell_val<T>(L);
  a.invd = sell_invd<T>(L);
  a.f = f;
  a.x = x;
  a.omega = (T)omega;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(L.rs_nreg);
  cfg.blockDim = dim3(RS_THREADS);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  PMG_CUDA(cudaLaunchKernelEx(&cfg, k_region_ssor<T>, a));
  count_launches(1);
  return PMG_OK;
}
template int region_ssor_phase<float>(Handle &, Level &, const float *, float *, double, int, bool);
template int region_ssor_phase<double>(Handle &, Level &, const double *, double *, double, int, bool);

int region_check(Handle &h) {
  if (!h.rs_err.p) return PMG_OK;
  int e = 0;
  PMG_CUDA(cudaMemcpy(&e, h.rs_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (!e) return PMG_OK;
  PMG_CUDA(cudaMemset(h.rs_err.p, 0, sizeof(int)));
  set_error("region sweep: a wait for a neighbouring region gave up");
  return PMG_ERR_STATE;
}

}  // namespace pmg
