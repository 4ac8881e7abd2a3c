// SELL-32 storage of the level matrices for the solve (sm_100a).
//
// The assembled matrix stays in the host's CSR pattern (that is what the
// slot map scatters into and what pmg_get_matrix returns).  For the solve
// every level also keeps a sliced-ELLPACK copy built once per pattern:
//
//   * rows are grouped by SSOR colour (Dirichlet rows form a last group),
//     sorted inside a group by decreasing length (ties: increasing row), and
//     cut into slices of 32 rows; a group is padded with empty rows to a
//     multiple of 32, so every colour owns a whole number of slices;
//   * slice s stores its 32 rows column-major with the slice's maximum row
//     length L_s: entry j of lane l sits at slice_ptr[s] + 32 j + l, so a warp
//     reads 128 contiguous bytes (FP32) per step; padding has value 0 and a
//     valid column, so no masking is needed.
//
// A block of SELL_K warps owns one slice (each warp takes every SELL_K-th
// column step of the 32 rows), so every row keeps several independent
// load chains in flight; the CSR kernels with a W-lane group per row stall
// on the row pointer of every row.  Vectors stay in the host's dof
// numbering: the kernels gather x through L2 and write each result row once.
//
// An SSOR step is one launch per colour and direction (2 x 27 launches for
// Q2), captured in the V-cycle's CUDA graph and chained with programmatic
// dependent launch.
#include "pmg_internal.h"
#include <algorithm>
#include <cstdlib>
#include <numeric>

namespace pmg {

int build_sell(Handle &h, Level &L) {
  if (L.sell_ready) return PMG_OK;
  const int N = L.N, Na = L.Na;
  const std::vector<int> &rp = L.h_rowptr, &kc = L.h_kcol;
  if ((int)rp.size() != N + 1) {
    set_error("build_sell: host copy of the CSR pattern missing");
    return PMG_ERR_STATE;
  }
  // entries of each row in the solve copy: an active row keeps its columns < Na
  // (columns are sorted, so that is a prefix), a Dirichlet row all of its own
  std::vector<int> alen(N);
  std::vector<int> dd_row, dd_beg;
  for (int r = 0; r < N; r++) {
    int n = rp[r + 1] - rp[r];
    if (r < Na) {
      n = (int)(std::lower_bound(kc.begin() + rp[r], kc.begin() + rp[r + 1], Na) - (kc.begin() + rp[r]));
      if (rp[r] + n < rp[r + 1]) {
        dd_row.push_back(r);
        dd_beg.push_back(rp[r] + n);
      }
    }
    alen[r] = n;
  }
  // groups: colours of the active rows, then the Dirichlet rows
  const int nc = (int)L.rcolor_ptr.size() - 1;
  std::vector<int> perm;
  std::vector<int> group_slice(nc + 2, 0);
  perm.reserve((size_t)N + 32 * (nc + 1));
  std::vector<int> rows;
  for (int g = 0; g <= nc; g++) {
    rows.clear();
    if (g < nc) rows.assign(L.h_row_list.begin() + L.rcolor_ptr[g], L.h_row_list.begin() + L.rcolor_ptr[g + 1]);
    else for (int r = Na; r < N; r++) rows.push_back(r);
    std::stable_sort(rows.begin(), rows.end(), [&](int a, int b) {
      return alen[a] > alen[b] || (alen[a] == alen[b] && a < b);
    });
    group_slice[g] = (int)(perm.size() / 32);
    perm.insert(perm.end(), rows.begin(), rows.end());
    while (perm.size() % 32) perm.push_back(-1);
  }
  group_slice[nc + 1] = (int)(perm.size() / 32);
  const int nslices = (int)(perm.size() / 32);
  std::vector<int> sptr(nslices + 1, 0);
  long total = 0;
  for (int s = 0; s < nslices; s++) {
    int lmax = 0;
    for (int l = 0; l < 32; l++) {
      int r = perm[(size_t)s * 32 + l];
      if (r >= 0) lmax = std::max(lmax, alen[r]);
    }
    sptr[s] = (int)total;
    total += 32L * lmax;
    if (total > 2147483647L) {
      set_error("build_sell: padded matrix exceeds 2^31 entries");
      return PMG_ERR_UNSUPPORTED;
    }
  }
  sptr[nslices] = (int)total;
  // columns: 32-bit for every slice (the one-launch coarse cycle reads these),
  // and column - row in 16 bits for the slices where every delta fits, which
  // the colour sweeps and products read instead (2 bytes per entry, not 4);
  // padding repeats the row (delta 0), padding lanes read x[0] with value 0
  std::vector<int> col((size_t)total);
  std::vector<short> c16((size_t)total);
  std::vector<unsigned char> wide(nslices, 0);
  long narrow_nnz = 0, wide_nnz = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : narrow_nnz, wide_nnz)
  for (int s = 0; s < nslices; s++) {
    const int off = sptr[s], lmax = (sptr[s + 1] - off) / 32;
    bool fits = true;
    long stored = 0;
    for (int l = 0; l < 32; l++) {
      const int r = perm[(size_t)s * 32 + l];
      const int len = r >= 0 ? alen[r] : 0;
      stored += len;
      for (int j = 0; j < lmax; j++) {
        const int c = j < len ? kc[rp[r] + j] : (r >= 0 ? r : 0);
        col[(size_t)off + 32 * j + l] = c;
        const long d = r >= 0 ? (long)c - r : 0;
        if (d < -32768 || d > 32767) fits = false;
        c16[(size_t)off + 32 * j + l] = (short)(fits ? d : 0);
      }
    }
    wide[s] = fits ? 0 : 1;
    if (fits) narrow_nnz += stored;
    else wide_nnz += stored;
  }
  PMG_TRY(L.sell_perm.upload(perm.data(), perm.size(), h.stream));
  PMG_TRY(L.sell_ptr.upload(sptr.data(), sptr.size(), h.stream));
  PMG_TRY(L.sell_col.upload(col.data(), col.size(), h.stream));
  PMG_TRY(L.sell_c16.upload(c16.data(), c16.size(), h.stream));
  PMG_TRY(L.sell_wide.upload(wide.data(), wide.size(), h.stream));
  PMG_TRY(L.sell_alen.upload(alen.data(), alen.size(), h.stream));
  L.n_dd = (int)dd_row.size();
  PMG_TRY(L.dd_row.upload(dd_row.data(), dd_row.size(), h.stream));
  PMG_TRY(L.dd_beg.upload(dd_beg.data(), dd_beg.size(), h.stream));
  PMG_CUDA(cudaStreamSynchronize(h.stream));
  L.sell_group = group_slice;
  L.sell_nslices = nslices;
  L.sell_nnz = total;
  L.sell_nnz_narrow = narrow_nnz;
  L.sell_nnz_wide = wide_nnz;
  L.sell_ready = true;
  L.sell_val_fresh32 = L.sell_val_fresh64 = false;
  return PMG_OK;
}

// values of the CSR matrix into the slice layout (and the permuted inverse diagonal)
template <typename T>
__global__ void k_csr_to_sell(int nslices, const int *__restrict__ perm, const int *__restrict__ sptr,
                              const int *__restrict__ rp, const int *__restrict__ alen, const double *__restrict__ a,
                              const int *__restrict__ dpos, T *__restrict__ val, T *__restrict__ invd) {
  const int lane = threadIdx.x & 31;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nslices; s += (gridDim.x * blockDim.x) >> 5) {
    const int off = sptr[s], lmax = (sptr[s + 1] - off) >> 5;
    const int r = perm[s * 32 + lane];
    const int beg = r >= 0 ? rp[r] : 0, len = r >= 0 ? alen[r] : 0;
    for (int j = 0; j < lmax; j++) val[off + 32 * j + lane] = j < len ? (T)a[beg + j] : (T)0;
    T dv = (T)1;
    if (r >= 0) {
      const double d = a[dpos[r]];
      dv = (T)(d != 0.0 ? 1.0 / d : 1.0);
    }
    invd[s * 32 + lane] = dv;
  }
}

template <typename T>
int sell_values(Handle &h, Level &L) {
  const bool f32 = sizeof(T) == 4;
  if (f32 ? L.sell_val_fresh32 : L.sell_val_fresh64) return PMG_OK;
  PMG_TRY(build_sell(h, L));
  T *val, *invd;
  if (f32) {
    PMG_TRY(L.sell_val32.alloc(L.sell_nnz));
    PMG_TRY(L.sell_invd32.alloc((size_t)L.sell_nslices * 32));
    val = reinterpret_cast<T *>(L.sell_val32.p);
    invd = reinterpret_cast<T *>(L.sell_invd32.p);
  } else {
    PMG_TRY(L.sell_val64.alloc(L.sell_nnz));
    PMG_TRY(L.sell_invd64.alloc((size_t)L.sell_nslices * 32));
    val = reinterpret_cast<T *>(L.sell_val64.p);
    invd = reinterpret_cast<T *>(L.sell_invd64.p);
  }
  int blocks = std::min((L.sell_nslices + 7) / 8, h.num_sms * 16);
  k_csr_to_sell<T><<<std::max(blocks, 1), 256, 0, h.stream>>>(L.sell_nslices, L.sell_perm.p, L.sell_ptr.p, L.rowptr.p,
                                                                L.sell_alen.p, L.A.p, L.diagpos.p, val, invd);
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  if (f32) L.sell_val_fresh32 = true; else L.sell_val_fresh64 = true;
  return PMG_OK;
}
template int sell_values<float>(Handle &, Level &);
template int sell_values<double>(Handle &, Level &);

// A block of K warps owns one slice: warp w accumulates the column steps
// j = w, w+K, ... of the slice's 32 rows (coalesced 32-wide loads), the K
// partial sums meet in shared memory and warp 0 finishes the rows.  K is
// chosen per launch (4, 8 or 16): small colours get more warps per slice so
// that each warp's chain of dependent loads (column index, then x) stays
// short; large colours already fill the GPU with K = 4.

// Column indices: a slice whose deltas fit (every slice of a lattice-ordered
// level) is read as 16-bit column - row deltas and gathered through x + row
// of the lane; the other slices read the 32-bit columns.  The choice is per
// slice and warp-uniform.  Matrix values and columns are read once per pass
// with streaming loads (ld.global.cs, evict-first), so they do not push the
// gathered iterate out of L1/L2: measured on the 64^3 finest level, FP32 SSOR
// step 0.490 -> 0.467 ms, FP64 SpMV 0.296 -> 0.272 ms.
template <int PF, int K>
__device__ __forceinline__ void sell_load_cols(bool wd, const int *__restrict__ col, const short *__restrict__ c16,
                                               int base, int j0, int lmax, int *ci) {
  if (wd) {
#pragma unroll
    for (int u = 0; u < PF; u++) ci[u] = j0 + u * K < lmax ? __ldcs(col + base + 32 * K * u) : 0;
  } else {
#pragma unroll
    for (int u = 0; u < PF; u++) ci[u] = j0 + u * K < lmax ? (int)__ldcs(c16 + base + 32 * K * u) : 0;
  }
}

// y = A x (MODE 0), d = f - A x (MODE 1), or the Jacobi update
// y = x + omega (f - A x) / a_rr (MODE 2, into a vector other than x) over
// slices [s0, s1)
template <typename T, int MODE, int K>
__global__ void __launch_bounds__(32 * K) k_sell_mv(int s0, int s1, const int *__restrict__ perm,
                                                    const int *__restrict__ sptr, const int *__restrict__ col,
                                                    const short *__restrict__ c16,
                                                    const unsigned char *__restrict__ wide,
                                                    const T *__restrict__ val, const T *__restrict__ x,
                                                    const T *__restrict__ f, T *__restrict__ y,
                                                    const T *__restrict__ invd, T omega) {
  // column steps per chunk: measured on the 64^3 Q2 finest level, FP64
  // product 0.275 ms with 8, 0.252 with 4, 0.253 with 2; FP32 defect 0.186
  // ms with 16, 0.164 with 8, 0.173 with 4
  constexpr int PF = sizeof(T) == 4 ? 8 : 4;
  __shared__ T part[K][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int s = s0 + blockIdx.x;
  int off = 0, lmax = 0, r = -1;
  bool wd = false;
  int ci[PF];
  T cv[PF];
  auto load_chunk = [&](int c0) {
    const int j0 = w + c0 * K;
    sell_load_cols<PF, K>(wd, col, c16, off + 32 * j0 + lane, j0, lmax, ci);
#pragma unroll
    for (int u = 0; u < PF; u++) cv[u] = j0 + u * K < lmax ? __ldcs(val + off + 32 * (j0 + u * K) + lane) : (T)0;
  };
  auto start = [&](int sl) {
    off = __ldg(sptr + sl);
    lmax = (__ldg(sptr + sl + 1) - off) >> 5;
    wd = __ldg(wide + sl) != 0;
    r = __ldg(perm + sl * 32 + lane);
    load_chunk(0);
  };
  // the matrix is not written by the predecessor: its first chunk streams in while that drains
  if (s < s1) start(s);
  pdl_wait();
  pdl_trigger();
  for (; s < s1; s += gridDim.x) {
    const T *xb = wd ? x : x + (r > 0 ? r : 0);
    T sum = 0;
    for (int c0 = 0;; c0 += PF) {
#pragma unroll
      for (int u = 0; u < PF; u++)
        if (w + (c0 + u) * K < lmax) sum += cv[u] * __ldg(xb + ci[u]);
      if (w + (c0 + PF) * K >= lmax) break;
      load_chunk(c0 + PF);
    }
    part[w][lane] = sum;
    const int rr = r;
    const int sn = s + gridDim.x;
    if (sn < s1) start(sn);  // next slice's first chunk before the reduction
    __syncthreads();
    if (w == 0) {
#pragma unroll
      for (int k = 1; k < K; k++) sum += part[k][lane];
      if (rr >= 0) {
        if (MODE == 2) y[rr] = __ldg(x + rr) + omega * (__ldg(f + rr) - sum) * __ldg(invd + s * 32 + lane);
        else y[rr] = MODE ? __ldg(f + rr) - sum : sum;
      }
    }
    __syncthreads();
  }
}

// Gauss-Seidel update of the rows of one colour (slices [s0, s1)).
// The first chunk of column steps of a warp's slice is loaded before
// pdl_wait(): the predecessor in the stream (the previous colour, a transfer
// or a defect) writes vectors only, never the matrix, so the colour's matrix
// streams in while the predecessor drains, and only the x gathers wait.

template <typename T, int K>
__global__ void __launch_bounds__(32 * K) k_sell_gs(int s0, int s1, const int *__restrict__ perm,
                                                    const int *__restrict__ sptr, const int *__restrict__ col,
                                                    const short *__restrict__ c16,
                                                    const unsigned char *__restrict__ wide,
                                                    const T *__restrict__ val, const T *__restrict__ invd,
                                                    const T *__restrict__ f, T *x, T omega) {
  constexpr int GS_PF = sizeof(T) == 4 ? 16 : 8;  // column steps per chunk (registers)
  __shared__ T part[K][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int s = s0 + blockIdx.x;
  int off = 0, lmax = 0, r = -1;
  bool wd = false;
  int ci[GS_PF];
  T cv[GS_PF];
  auto load_chunk = [&](int c0) {
    const int j0 = w + c0 * K;
    sell_load_cols<GS_PF, K>(wd, col, c16, off + 32 * j0 + lane, j0, lmax, ci);
#pragma unroll
    for (int u = 0; u < GS_PF; u++)
      cv[u] = j0 + u * K < lmax ? __ldcs(val + off + 32 * (j0 + u * K) + lane) : (T)0;
  };
  auto prefetch = [&](int sl) {
    off = __ldg(sptr + sl);
    lmax = (__ldg(sptr + sl + 1) - off) >> 5;
    wd = __ldg(wide + sl) != 0;
    r = __ldg(perm + sl * 32 + lane);
    load_chunk(0);
  };
  if (s < s1) prefetch(s);
  pdl_wait();
  pdl_trigger();
  for (; s < s1; s += gridDim.x) {
    const T *xb = wd ? x : x + (r > 0 ? r : 0);
    T sum = 0;
    // column steps in chunks of GS_PF: the gathers of a chunk go out, then the
    // next chunk's column / value loads, so a long row costs one latency per chunk
    for (int c0 = 0;; c0 += GS_PF) {
#pragma unroll
      for (int u = 0; u < GS_PF; u++)
        if (w + (c0 + u) * K < lmax) sum += cv[u] * xb[ci[u]];
      if (w + (c0 + GS_PF) * K >= lmax) break;
      load_chunk(c0 + GS_PF);
    }
    part[w][lane] = sum;
    __syncthreads();
    if (w == 0) {
#pragma unroll
      for (int k = 1; k < K; k++) sum += part[k][lane];
      if (r >= 0) x[r] += omega * (__ldg(f + r) - sum) * __ldg(invd + s * 32 + lane);
    }
    __syncthreads();
    if (s + gridDim.x < s1) prefetch(s + gridDim.x);
  }
}

// warps per slice for a launch over `slices` slices: the smallest K (>= 4;
// K = 2 and deeper unrolling measured slower on the 64^3 finest level) that
// still gives every SM 32 warps, at most kmax
static int pick_k(int slices, int num_sms, int kmax = 16) {
  static int kmin = -1;
  if (kmin < 0) {
    const char *e = getenv("PMG_SELL_KMIN");
    kmin = e ? atoi(e) : 4;
    if (kmin != 2 && kmin != 8 && kmin != 16) kmin = 4;
  }
  const long want = 32L * num_sms;  // warps to keep the load pipes busy
  int k = kmin;
  while (k < kmax && (long)slices * k < want) k *= 2;
  return k;
}

template <typename T>
__global__ void k_sell_copy_dirichlet(int Na, int N, const T *__restrict__ f, T *__restrict__ x) {
  pdl_wait();
  pdl_trigger();
  int i = blockIdx.x * blockDim.x + threadIdx.x + Na;
  if (i < N) x[i] = f[i];
}

// y_r -= sum over the Dirichlet columns j of active row r of A_rj v_j (the
// entries [dd_beg, row end) of the CSR row, FP64 values)
template <typename T>
__global__ void k_dirichlet_cols(int n, const int *__restrict__ rows, const int *__restrict__ beg,
                                 const int *__restrict__ rp, const int *__restrict__ kc, const double *__restrict__ a,
                                 const T *v, T *y, double sign) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = __ldg(rows + i);
  double s = 0;
  for (int k = __ldg(beg + i), e = __ldg(rp + r + 1); k < e; k++) s += __ldg(a + k) * (double)v[__ldg(kc + k)];
  y[r] = (T)((double)y[r] + sign * s);
}

template <typename T>
int dirichlet_cols(cudaStream_t s, const Level &L, const T *v, T *y, bool add) {
  if (L.n_dd == 0) return PMG_OK;
  PMG_CUDA(launch_pdl(k_dirichlet_cols<T>, dim3((L.n_dd + 255) / 256), dim3(256), 0, s, L.n_dd,
                      (const int *)L.dd_row.p, (const int *)L.dd_beg.p, (const int *)L.rowptr.p,
                      (const int *)L.kcol.p, (const double *)L.A.p, v, y, add ? 1.0 : -1.0));
  count_launches(1);
  return PMG_OK;
}
template int dirichlet_cols<float>(cudaStream_t, const Level &, const float *, float *, bool);
template int dirichlet_cols<double>(cudaStream_t, const Level &, const double *, double *, bool);

// grid of a SELL launch: one CTA per slice up to a cap, beyond which CTAs loop
// over slices (loading the next slice's first chunk before the reduction).
// Measured on the 64^3 Q2 finest level (K = 4, 4 / 8 column steps per chunk):
// 256 CTAs per SM, FP64 product 0.247 ms (64: 0.268, 1024: 0.252, the earlier
// 512: 0.252), FP32 defect 0.162 ms (64: 0.173, 128: 0.164, 1024: 0.165); a
// colour sweep stays below the cap.  PMG_SELL_CTAS_PER_SM overrides the cap.
template <typename T>
static int slice_grid(int nslices, int num_sms, int k) {
  static int cps = -1;
  if (cps < 0) {
    const char *e = getenv("PMG_SELL_CTAS_PER_SM");
    cps = e ? std::max(0, atoi(e)) : 0;
  }
  const long cap = (long)num_sms * (cps ? cps : 256);
  return (int)std::max(1L, std::min((long)nslices, cap));
}

template <typename T>
static const T *sell_val(const Level &L) {
  if (sizeof(T) == 4) return reinterpret_cast<const T *>(L.sell_val32.p);
  return reinterpret_cast<const T *>(L.sell_val64.p);
}
template <typename T>
static const T *sell_invd(const Level &L) {
  if (sizeof(T) == 4) return reinterpret_cast<const T *>(L.sell_invd32.p);
  return reinterpret_cast<const T *>(L.sell_invd64.p);
}

template <typename T, int MODE, int K>
static cudaError_t launch_mv(cudaStream_t s, const Level &L, const T *x, const T *f, T *y, int num_sms, int n = -1,
                             T omega = 0) {
  if (n < 0) n = L.sell_nslices;
  return launch_pdl(k_sell_mv<T, MODE, K>, dim3(slice_grid<T>(n, num_sms, K)), dim3(32 * K), 0, s, 0, n,
                    (const int *)L.sell_perm.p, (const int *)L.sell_ptr.p, (const int *)L.sell_col.p,
                    (const short *)L.sell_c16.p, (const unsigned char *)L.sell_wide.p, sell_val<T>(L), x, f, y,
                    sell_invd<T>(L), omega);
}

template <typename T>
int sell_spmv(cudaStream_t s, const Level &L, const T *x, const T *f, T *y, int mode, int num_sms) {
  int k = pick_k(L.sell_nslices, num_sms);
  cudaError_t e;
  if (k < 4) k = 4;  // a full-matrix product has enough slices for K = 4
  if (mode) e = k == 16 ? launch_mv<T, 1, 16>(s, L, x, f, y, num_sms) : k == 8 ? launch_mv<T, 1, 8>(s, L, x, f, y, num_sms)
                                                                             : launch_mv<T, 1, 4>(s, L, x, f, y, num_sms);
  else e = k == 16 ? launch_mv<T, 0, 16>(s, L, x, f, y, num_sms) : k == 8 ? launch_mv<T, 0, 8>(s, L, x, f, y, num_sms)
                                                                          : launch_mv<T, 0, 4>(s, L, x, f, y, num_sms);
  PMG_CUDA(e);
  count_launches(1);
  return PMG_OK;
}
template int sell_spmv<float>(cudaStream_t, const Level &, const float *, const float *, float *, int, int);
template int sell_spmv<double>(cudaStream_t, const Level &, const double *, const double *, double *, int, int);

template <typename T>
__global__ void k_copy_active(int Na, const T *__restrict__ src, T *__restrict__ dst) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < Na) dst[i] = src[i];
}

// One damped Jacobi step (TMGLevel3D::Jacobi, MGLevel3D.C:469-560):
// x_D := f_D, then x_a := x_a + omega (f_a - A_a x) / a_aa from the previous
// iterate, written into `tmp` (the active rows' slices are the colour groups)
// and copied back.  In the V-cycle x_D = f_D already holds when a level's
// smoothing starts, so the previous Dirichlet values the reference keeps in
// its aux copy equal the new ones.
template <typename T>
int sell_jacobi(cudaStream_t s, const Level &L, const T *f, T *x, T *tmp, double omega, int num_sms, bool dirichlet) {
  const int nc = (int)L.sell_group.size() - 2;
  const int nd = L.N - L.Na;
  if (nd > 0 && dirichlet) {
    PMG_CUDA(launch_pdl(k_sell_copy_dirichlet<T>, dim3((nd + 255) / 256), dim3(256), 0, s, L.Na, L.N, f, x));
    count_launches(1);
  }
  const int na_slices = L.sell_group[nc];
  if (na_slices <= 0) return PMG_OK;
  const int k = std::max(4, pick_k(na_slices, num_sms));
  cudaError_t e = k == 16 ? launch_mv<T, 2, 16>(s, L, x, f, tmp, num_sms, na_slices, (T)omega)
                : k == 8  ? launch_mv<T, 2, 8>(s, L, x, f, tmp, num_sms, na_slices, (T)omega)
                          : launch_mv<T, 2, 4>(s, L, x, f, tmp, num_sms, na_slices, (T)omega);
  PMG_CUDA(e);
  PMG_CUDA(launch_pdl(k_copy_active<T>, dim3((L.Na + 255) / 256), dim3(256), 0, s, L.Na, (const T *)tmp, x));
  count_launches(2);
  return PMG_OK;
}
template int sell_jacobi<float>(cudaStream_t, const Level &, const float *, float *, float *, double, int, bool);
template int sell_jacobi<double>(cudaStream_t, const Level &, const double *, double *, double *, double, int, bool);

// one SSOR step: Dirichlet rows from f (the sweeps never change them, so only the
// first step of a level visit needs it), forward over the colours, backward.
// skip_repeats (with omega = 1): a Gauss-Seidel update of a colour directly
// after an update of the same colour leaves x unchanged (the colour's rows have
// zero residual and are not coupled to each other), so the backward sweep
// starts with the second-to-last colour and, when the previous step was also
// an SSOR step of this level (after_ssor), the forward sweep with colour 1.
// forward_only: one SOR step (TMGLevel3D::SOR, MGLevel3D.C:280-361): the
// forward sweep over the colours alone.
template <typename T>
int sell_ssor(cudaStream_t s, const Level &L, const T *f, T *x, double omega, int num_sms, bool dirichlet,
              bool after_ssor, bool skip_repeats, bool forward_only) {
  const int nc = (int)L.sell_group.size() - 2;  // active colours
  const int nd = L.N - L.Na;
  if (nd > 0 && dirichlet) {
    PMG_CUDA(launch_pdl(k_sell_copy_dirichlet<T>, dim3((nd + 255) / 256), dim3(256), 0, s, L.Na, L.N, f, x));
    count_launches(1);
  }
  const bool skip = skip_repeats && omega == 1.0 && !forward_only;
  for (int pass = 0; pass < (forward_only ? 1 : 2); pass++)
    for (int cc = 0; cc < nc; cc++) {
      if (skip && cc == 0 && (pass == 1 || after_ssor)) continue;
      const int c = pass == 0 ? cc : nc - 1 - cc;
      const int s0 = L.sell_group[c], s1 = L.sell_group[c + 1];
      if (s1 <= s0) continue;
      // at most 8 warps per slice in FP32, 16 in FP64: the short colours of
      // levels 2-3 (42 and 318 slices), measured on the 64^3 bench: FP32
      // V-cycle 3.69 -> 3.61 ms with 8 (4: 3.96 ms); FP64 V-cycle 5.18 ->
      // 5.57 ms with 8
      const int k = pick_k(s1 - s0, num_sms, sizeof(T) == 4 ? 8 : 16);
      cudaError_t e;
#define PMG_GS(K_)                                                                                              \
  launch_pdl(k_sell_gs<T, K_>, dim3(slice_grid<T>(s1 - s0, num_sms, K_)), dim3(32 * K_), 0, s, s0, s1,           \
             (const int *)L.sell_perm.p, (const int *)L.sell_ptr.p, (const int *)L.sell_col.p,                   \
             (const short *)L.sell_c16.p, (const unsigned char *)L.sell_wide.p, sell_val<T>(L), sell_invd<T>(L), \
             f, x, (T)omega)
      e = k == 16 ? PMG_GS(16) : k == 8 ? PMG_GS(8) : k == 4 ? PMG_GS(4) : PMG_GS(2);
#undef PMG_GS
      PMG_CUDA(e);
      count_launches(1);
    }
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}
template int sell_ssor<float>(cudaStream_t, const Level &, const float *, float *, double, int, bool, bool, bool, bool);
template int sell_ssor<double>(cudaStream_t, const Level &, const double *, double *, double, int, bool, bool, bool,
                               bool);

}  // namespace pmg
