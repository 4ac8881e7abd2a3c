// The coarse end of the V-cycle in one launch: one thread-block cluster
// (8 CTAs x 16 warps by default, on one GPC) runs TMultiGrid3D::Cycle
// (src/FE/MultiGrid3D.C:449-695) for every level from `top` down to the
// coarsest and back up -- pre-smoothing, defect, restriction, the coarsest
// solve, prolongation, post-smoothing.
//
// Why: on a level of a few thousand rows a colour sweep is well under a
// microsecond of work, so the colour-by-colour launches (2 x 27 per Q2 SSOR
// step, ~2.8 us each with programmatic dependent launch) are pure launch and
// L2 latency.
//
// Layout: every CTA keeps a full copy of the iterate x of each level of the
// cycle in its shared memory, plus the slice pointers and row permutation of
// the levels whose Gauss-Seidel passes are pipelined.  A colour pass gathers
// x from the local copy and sends each updated row to every copy with
// st.async, whose byte count completes a transaction on the receiving CTA's
// mbarrier: a CTA waits only for the rows of the pass, not for a
// cluster-wide barrier.  The matrix, f and 1/a_ii of a pass are loaded two
// passes ahead.  Defect, restriction, prolongation and the coarsest solve
// are separated by cluster barriers.  The arithmetic is the level-by-level
// path's -- the same SELL-32 slices, colour order, omega, damping and
// coarsest solve -- up to the order of the partial sums inside a row.
#include "pmg_internal.h"
#include <cooperative_groups.h>
#include <algorithm>
#include <cstdlib>
#include <string>

namespace cg = cooperative_groups;

namespace pmg {

// 16 warps per CTA: a GS pass keeps up to 32 column steps (64 registers in
// FP32) in flight per thread plus the next pass's slice, within the 128
// registers a 512-thread CTA allows
constexpr int CC_MAX_LEVELS = 8, CC_MAX_GROUPS = 64, CC_WARPS = 16;
constexpr size_t CC_SMEM_X = 200 * 1024;  // budget for the replicated iterates

template <typename T>
struct CcLevel {
  int N, Na, ncolors, xoff;  // xoff: offset of the level's x copy in shared memory
  int group[CC_MAX_GROUPS];  // slice range of colour c: [group[c], group[c+1]); group[ncolors+1] = all slices
  unsigned char lk[CC_MAX_GROUPS];  // log2 of the warps per slice of colour c in a GS pass
  int rows[CC_MAX_GROUPS];          // rows of colour c (the updates a GS pass sends to each CTA)
  int one_round;                    // pipelined GS passes: every colour's slices fit one round of the
                                    // cluster's warps, and sptr / perm are staged in shared memory
  int soff, nsl;                    // staged sptr at ints [soff, soff + nsl], perm (32 per slice) after it
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
  int *err;              // set to 1 when a bounded wait gives up
  unsigned extra_tx;     // bytes expected on top of a pass's updates: 0, except in the test of the give-up path
  T omega, damp;
};

template <typename T>
struct CcCtx {
  cg::cluster_group cl;
  int warp, lane, gw, tw, rank, nblocks;
  T (*part)[32];  // 2 x CC_WARPS rows: cross-warp sums, one buffer per pass parity
  T *xs;          // this CTA's shared memory holding the x copies
  const int *si;  // the same shared memory as ints (staged slice pointers and row permutations)
  unsigned mbar;  // shared address of the two pass mbarriers (8 bytes apart)
  unsigned pc;    // Gauss-Seidel passes completed so far (selects mbarrier and parity)
  int *err;       // set when a wait gives up
  unsigned extra_tx;  // see CcArgs
  bool failed;    // a wait of this CTA gave up: no further sends, expects or waits
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
    // warps beyond spc * K (K need not divide the warp count) take no slice
    const int sl = c.warp / K < spc ? s0 + r * per_round + c.rank * spc + c.warp / K : s1;
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

// ---- DSMEM row updates with transaction-count completion -------------------
// A Gauss-Seidel pass sends every updated row to every CTA's copy with
// st.async, which counts the bytes on the receiving CTA's mbarrier; a CTA
// starts the next pass once its mbarrier has seen all rows of the pass.  No
// cluster-wide barrier (and none of its release fence, which would wait for the
// warp's outstanding loads) sits between passes.  Ordering: CTA A sends pass
// p+1 only after it has received pass p from every CTA, and a CTA sends pass
// p only after its own pass-p gathers, so no update of pass p+1 reaches a copy
// that is still being read for pass p; and A cannot send pass p+2 before B
// has finished receiving pass p, so two mbarriers used by pass parity keep the
// byte counts of consecutive passes apart.
__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned cluster_addr(unsigned a, int rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_async(unsigned addr, float v, unsigned mbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];\n" ::"r"(addr),
               "r"(__float_as_uint(v)), "r"(mbar)
               : "memory");
}
__device__ __forceinline__ void st_async(unsigned addr, double v, unsigned mbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b64 [%0], %1, [%2];\n" ::"r"(addr),
               "l"(__double_as_longlong(v)), "r"(mbar)
               : "memory");
}
__device__ __forceinline__ void mbar_init(unsigned mbar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned mbar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// wait for the phase of the given parity, at most 0.2 s; false when it gave up
__device__ __forceinline__ bool mbar_wait(unsigned mbar, unsigned parity) {
  unsigned long long t0 = 0;
  for (int it = 0;; it++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (it == 0) t0 = global_ns();
    else if (global_ns() - t0 > 200000000ull) return false;
  }
}

// One warp's share of a Gauss-Seidel colour pass whose slices all fit one round
// (one slice per group of K warps): warp k of the group takes the column steps
// k, k+K, ...  K = 16 (lk = log2 K, kept per colour for other shapes), so
// that the column offsets are immediates.  head() (slice offset, length and the permuted row)
// is issued a whole pass ahead, body() (columns, values, f, 1/a_ii --
// everything but x) before the wait that ends the previous pass.
template <typename T>
struct CcGs {
  static constexpr int PF = 8;  // column steps held in registers: rows of up to 128 entries in one chunk
  int ci[PF];
  T cv[PF];
  int lk, k, sl, s1, off, lmax, row;  // sl >= s1: no slice for this warp; row < 0: no row for this lane
  T fr, id;

  template <int K>
  __device__ __forceinline__ void load_k(const CcLevel<T> &L, int lane) {
    const int rem = lmax - k;  // column steps u*K + k < lmax
    const int *cp = L.col + off + 32 * k + lane;
    const T *vp = L.val + off + 32 * k + lane;
#pragma unroll
    for (int u = 0; u < PF; u++) {
      ci[u] = u * K < rem ? __ldg(cp + 32 * K * u) : 0;
      cv[u] = u * K < rem ? __ldg(vp + 32 * K * u) : (T)0;
    }
    fr = id = 0;
    if (row >= 0) {
      fr = __ldcg(L.f + row);
      id = __ldg(L.invd + sl * 32 + lane);
    }
  }
  // this warp's slice of the colour's pass and everything of it but x: the
  // slice pointers and rows from shared memory, the rest from global memory
  __device__ __forceinline__ void load(const CcCtx<T> &c, const CcLevel<T> &L, int colour) {
    const int s0 = L.group[colour];
    s1 = L.group[colour + 1];
    lk = L.lk[colour];
    k = c.warp & ((1 << lk) - 1);
    const int spc = CC_WARPS >> lk, slot = c.warp >> lk;
    sl = slot < spc ? s0 + c.rank * spc + slot : s1;
    lmax = 0;
    row = -1;
    if (sl >= s1) return;  // no slice (warp-uniform)
    const int *sp = c.si + L.soff;
    off = sp[sl];
    lmax = (sp[sl + 1] - off) >> 5;
    row = sp[L.nsl + 1 + sl * 32 + c.lane];
    load_k<16>(L, c.lane);
  }
  // gathers from the local copy, the cross-warp sum (part: this pass's
  // buffer), and the update sent to every CTA's copy; the K warps of a slice
  // share the sends
  template <int K>
  __device__ __forceinline__ void run_k(CcCtx<T> &c, const CcLevel<T> &L, T omega, T (*part)[32], unsigned mbar) {
    const T *x = c.xs + L.xoff;
    const bool active = sl < s1;
    T sum = 0, xr = 0;
    if (active) {
      const int rem = lmax - k;
#pragma unroll
      for (int u = 0; u < PF; u++)
        if (u * K < rem) sum += cv[u] * x[ci[u]];
      // rows longer than K * PF column steps: the rest in further chunks
      for (int c0 = PF; c0 * K < rem; c0 += PF) {
        const int *cp = L.col + off + 32 * (k + c0 * K) + c.lane;
        const T *vp = L.val + off + 32 * (k + c0 * K) + c.lane;
        const int rem2 = rem - c0 * K;
#pragma unroll
        for (int u = 0; u < PF; u++) {
          ci[u] = u * K < rem2 ? __ldg(cp + 32 * K * u) : 0;
          cv[u] = u * K < rem2 ? __ldg(vp + 32 * K * u) : (T)0;
        }
#pragma unroll
        for (int u = 0; u < PF; u++)
          if (u * K < rem2) sum += cv[u] * x[ci[u]];
      }
      // x_row before the barrier: after it, an update of this row may already
      // have reached this CTA's copy
      if (row >= 0) xr = x[row];
    }
    part[c.warp][c.lane] = sum;
    // the CTA barrier of the cross-warp sum also makes a failed wait of the
    // previous pass (seen by any thread) known to the whole CTA
    c.failed = __syncthreads_or(c.failed) != 0;
    if (active && row >= 0 && !c.failed) {
      const int w0 = c.warp - k;
      T s = 0;
#pragma unroll
      for (int kk = 0; kk < K; kk++) s += part[w0 + kk][c.lane];
      const T v = xr + omega * (fr - s) * id;
      const unsigned a = smem_addr(c.xs + L.xoff + row);
      for (int b = k; b < c.nblocks; b += K) st_async(cluster_addr(a, b), v, cluster_addr(mbar, b));
    }
  }
  __device__ __forceinline__ void run(CcCtx<T> &c, const CcLevel<T> &L, T omega, T (*part)[32], unsigned mbar) {
    run_k<16>(c, L, omega, part, mbar);
  }
};

// SSOR step of TMGLevel3D::SSOR in colour order: Dirichlet rows from f (first
// step of a level visit; the sweeps never change them), forward, backward
template <typename T>
__device__ void cc_ssor(CcCtx<T> &c, const CcLevel<T> &L, T omega, bool dirichlet) {
  // every CTA refreshes the Dirichlet rows of its own copy
  if (dirichlet) {
    for (int i = L.Na + threadIdx.x; i < L.N; i += blockDim.x) c.xs[L.xoff + i] = __ldcg(L.f + i);
    __syncthreads();
  }
  const int nc = L.ncolors;
  if (!L.one_round) {  // colours that need several rounds: one pass at a time
    for (int cc = 0; cc < nc; cc++) {
      cc_slices<T, true>(c, L, L.group[cc], L.group[cc + 1], omega);
      c.sync();
    }
    for (int cc = nc - 1; cc >= 0; cc--) {
      cc_slices<T, true>(c, L, L.group[cc], L.group[cc + 1], omega);
      c.sync();
    }
    return;
  }
  // passes p = 0 .. 2nc-1 over colours 0..nc-1, nc-1..0 (an even count); A
  // runs the even passes and B the odd ones, each loading its next pass two
  // passes ahead
  auto colour = [&](int p) { return p < nc ? p : 2 * nc - 1 - p; };
  auto pass = [&](CcGs<T> &g, int p) {
    const unsigned mbar = c.mbar + 8 * (c.pc & 1);
    if (threadIdx.x == 0 && !c.failed) mbar_expect(mbar, (unsigned)(L.rows[colour(p)] * sizeof(T)) + c.extra_tx);
    g.run(c, L, omega, c.part + (c.pc & 1) * CC_WARPS, mbar);
    if (p + 2 < 2 * nc) g.load(c, L, colour(p + 2));
    // Give-up path: a CTA whose wait runs out flags the error and from its next
    // pass on (once its CTA barrier has spread the failure) sends, expects and
    // waits no more; a peer still waiting for its updates then runs out in turn,
    // so every CTA ends up failed, runs the rest of the control flow (the
    // cluster barriers) without waits and ends; the host discards the result
    // (PMG_ERR_STATE).  Updates sent before a CTA failed may still be in flight
    // towards a failed receiver: the grace period at the end of the kernel keeps
    // every receiver resident until they have landed.
    if (!c.failed && !mbar_wait(mbar, (c.pc >> 1) & 1)) {
      c.failed = true;
      atomicExch(c.err, 1);
    }
    c.pc++;
  };
  CcGs<T> A, B;
  A.load(c, L, colour(0));
  B.load(c, L, colour(1));
  for (int p = 0; p < 2 * nc; p += 2) {
    pass(A, p);
    pass(B, p + 1);
  }
  __syncthreads();  // the last pass's sums are read before part is reused
}

template <typename T>
__global__ void __launch_bounds__(CC_WARPS * 32, 1) k_coarse_cycle(const __grid_constant__ CcArgs<T> a) {
  __shared__ T part[2 * CC_WARPS][32];
  __shared__ __align__(8) unsigned long long mbars[2];
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
  c.si = reinterpret_cast<const int *>(cc_dyn);
  c.mbar = smem_addr(mbars);
  c.pc = 0;
  c.err = a.err;
  c.extra_tx = a.extra_tx;
  c.failed = false;
  if (threadIdx.x == 0) {
    mbar_init(c.mbar, 1);
    mbar_init(c.mbar + 8, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  const int top = a.nlev - 1;
  // the entry level starts from x = 0 (the caller zeroed its global copy)
  for (int i = threadIdx.x; i < a.lv[top].N; i += blockDim.x) c.xs[a.lv[top].xoff + i] = (T)0;
  // slice pointers and row permutations of the pipelined levels (constant data)
  for (int l = 0; l <= top; l++) {
    const CcLevel<T> &L = a.lv[l];
    if (!L.one_round) continue;
    int *sp = reinterpret_cast<int *>(cc_dyn) + L.soff;
    for (int i = threadIdx.x; i <= L.nsl; i += blockDim.x) sp[i] = __ldg(L.sptr + i);
    for (int i = threadIdx.x; i < L.nsl * 32; i += blockDim.x) sp[L.nsl + 1 + i] = __ldg(L.perm + i);
  }
  pdl_wait();
  pdl_trigger();
  c.sync();  // every copy initialised before any remote store
  // down: smooth, defect, restrict
  for (int l = top; l >= 1; l--) {
    const CcLevel<T> &L = a.lv[l];
    const CcLevel<T> &C = a.lv[l - 1];
    for (int s = 0; s < a.pre; s++) cc_ssor(c, L, a.omega, s == 0);
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
    for (int s = 0; s < a.coarse_it; s++) cc_ssor(c, Z, a.omega, s == 0);
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
    for (int s = 0; s < a.post; s++) cc_ssor(c, L, a.omega, s == 0);
  }
  // Without a failed wait every CTA has received all updates of every pass, so
  // no send is in flight once the cluster barrier below is passed.  After a
  // failure that does not hold: every CTA stopped sending before it arrived at
  // the barrier, and a send takes well under a microsecond to land, so a
  // failed CTA stays resident 200 us more (bounded) before it exits.
  const bool any_failed = __syncthreads_or(c.failed) != 0;
  c.sync();
  if (any_failed) {
    const unsigned long long t0 = global_ns();
    while (global_ns() - t0 < 200000ull) {
    }
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
// (0: none -- the level-by-level path runs).  PMG_COARSE_CLUSTER=<ctas>[:<max
// rows>] chooses the shape: the default "8:8192" runs the levels of at most
// 8192 rows on an 8-CTA cluster (measured: 64^3 Q2 FP32 V-cycle 4.17 ms
// against 4.31 ms level by level; larger levels stream more matrix per colour
// pass than one GPC's share of L2 bandwidth carries faster than the 148-SM
// colour launches); "1" runs the levels of at most CC_ONE_CTA_ROWS rows on one
// CTA, "16" (2, 4, 8) every level whose iterates fit CC_SMEM_X on a cluster of
// that size, "0" none.
constexpr int CC_ONE_CTA_ROWS = 8192;

int coarse_cycle_top(Handle &h) {
  static int mode = -1;  // 0 off, 1 one CTA, 2 cluster
  static long max_rows = 0;
  static int want = 0;   // CTAs asked for
  if (mode < 0) {
    const char *e = getenv("PMG_COARSE_CLUSTER");
    const std::string v(e ? e : "8:8192");
    const size_t colon = v.find(':');
    want = atoi(v.substr(0, colon).c_str());
    mode = want == 1 ? 1 : (want == 2 || want == 4 || want == 8 || want == 16) ? 2 : 0;
    max_rows = mode == 1 ? CC_ONE_CTA_ROWS : 0;
    if (mode && colon != std::string::npos) max_rows = atol(v.c_str() + colon + 1);
  }
  if (mode == 0) return 0;
  // the one-launch cycle runs SSOR pre/post steps without step-length control
  if (h.prm.smoother != PMG_SMOOTHER_SSOR && h.prm.smoother != PMG_SMOOTHER_LEARNED) return 0;
  if (h.prm.slc_all) return 0;
  // (and the dense coarsest solve; the iterative one checks its residual)
  if (h.prm.coarse_smoother != PMG_COARSE_DIRECT) return 0;
  const size_t vb = h.prm.precision == PMG_PREC_FP32 ? sizeof(float) : sizeof(double);
  size_t bytes = 0;
  int top = 0;
  for (int i = 0; i < (int)h.lv.size() - 1 && i < CC_MAX_LEVELS; i++) {
    const Level &L = h.lv[i];
    bytes += ((size_t)L.N * vb + 15) / 16 * 16;
    if (bytes > CC_SMEM_X || (int)L.sell_group.size() > CC_MAX_GROUPS) break;
    if (max_rows > 0 && L.N > max_rows) break;
    top = i;
  }
  if (top < 1) return 0;
  if (!h.cc_err.p) {
    if (h.cc_err.alloc(1) != PMG_OK) return 0;
    if (cudaMemset(h.cc_err.p, 0, sizeof(int)) != cudaSuccess) return 0;
  }
  if (mode == 1) {
    h.cc_ctas = 1;
  } else {
    // the launch shape is queried here, outside any stream capture
    const int c = std::min(cluster_ctas<float>(), cluster_ctas<double>());
    if (!c) return 0;
    h.cc_ctas = std::min(c, want);
  }
  return top;
}

int coarse_cycle_check(Handle &h) {
  if (!h.cc_err.p) return PMG_OK;
  int e = 0;
  PMG_CUDA(cudaMemcpy(&e, h.cc_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (!e) return PMG_OK;
  PMG_CUDA(cudaMemset(h.cc_err.p, 0, sizeof(int)));
  set_error("coarse cycle: a cluster wait gave up (updates of a pass never arrived)");
  return PMG_ERR_STATE;
}

template <typename T>
int coarse_cycle(Handle &h, int top) {
  if (top < 1 || top >= CC_MAX_LEVELS) {
    set_error("coarse_cycle: level out of range");
    return PMG_ERR_ARG;
  }
  if (h.cc_ctas < 1) {
    set_error("coarse_cycle: launch shape not set");
    return PMG_ERR_STATE;
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
    // warps per slice of each colour: the most (up to 16) that still cover the
    // colour's slices in one round of the cluster's warps
    d.one_round = 1;
    for (int cc = 0; cc < d.ncolors; cc++) {
      const int nsl = d.group[cc + 1] - d.group[cc];
      const int lk = 4;  // K = 16: the instantiated pass shape
      if (nsl > (CC_WARPS >> lk) * h.cc_ctas) d.one_round = 0;
      d.lk[cc] = (unsigned char)lk;
      d.rows[cc] = L.rcolor_ptr[cc + 1] - L.rcolor_ptr[cc];
    }
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
  // shared memory after the x copies: sptr and perm of the levels whose GS
  // passes are pipelined (a level that does not fit runs one pass at a time)
  for (int i = 0; i <= top; i++) {
    CcLevel<T> &d = a.lv[i];
    d.soff = 0;
    d.nsl = h.lv[i].sell_nslices;
    if (!d.one_round) continue;
    const size_t need = ((size_t)(d.nsl + 1) + (size_t)d.nsl * 32) * sizeof(int);
    if (smem + need > CC_SMEM_X) {
      d.one_round = 0;
      continue;
    }
    d.soff = (int)(smem / sizeof(int));
    smem += (need + 15) / 16 * 16;
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
  a.err = h.cc_err.p;
  // PMG_TEST_CC_EXTRA_TX=<bytes>: every pass expects that many bytes that no
  // CTA sends, so every wait runs out -- the test of the give-up path (read at
  // every launch; a captured V-cycle graph keeps the value it was captured with)
  {
    const char *e = getenv("PMG_TEST_CC_EXTRA_TX");
    a.extra_tx = e ? (unsigned)atoi(e) : 0u;
  }
  a.coarse_it = h.prm.coarse_maxit > 0 ? h.prm.coarse_maxit : 1;
  a.pre = h.prm.pre_smooth;
  a.post = h.prm.post_smooth;
  a.omega = (T)h.prm.smooth_omega;
  a.damp = (T)h.prm.gmg_damp;
  const int ctas = h.cc_ctas;
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
