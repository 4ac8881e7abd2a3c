// Learned stencil smoother (no counterpart in the reference).
//
// For a level whose dofs sit on an n1 x n1 x n1 node lattice (Q1 hexahedra)
// a small convolutional network maps each node's local operator -- its
// matrix row as a 27-point stencil normalised by the diagonal -- to a
// 27-point correction stencil W(x).  A smoothing step is then
//     x_i += omega * sum_k W_k(i) r_{i + o_k},   r = f - A x,
// one launch for the stencil after the residual (no colouring).  W depends
// only on the matrix, so the network runs once per assembly; per V-cycle the
// smoother costs two streaming passes per step.
//
// Network: three 3x3x3 convolutions with zero padding on the lattice,
// 27 -> 32 (ReLU) -> 32 (ReLU) -> 27 channels, BF16 weights and BF16
// activations (every layer's input is rounded to BF16), FP32 accumulation.
// The forward runs on the tensor cores as an implicit GEMM per brick of the
// lattice (mma.sync m16n8k16 BF16: rows = nodes, columns = output channels,
// reduction = 27 offsets x 32 input channels); the backward (data and weight
// gradients) and Adam run on FP32 CUDA cores.  Training runs on the device
// through the pmg_learned_* entry points.
//
// Lattice order: node L = i + n1 (j + n1 k).  The forward's activations are
// node-major BF16 with the channels padded to 32 (L * 32 + c); the FP32
// arrays of the backward are channel-major (c * NL + L).  Offsets:
// k = (di+1) + 3 (dj+1) + 9 (dk+1).
#include "pmg_internal.h"
#include <cuda_bf16.h>
#include <cmath>
#include <vector>

namespace pmg {

constexpr int NET_C0 = 27, NET_C1 = 32, NET_C2 = 32, NET_C3 = 27;
constexpr int NET_W1 = NET_C1 * NET_C0 * 27, NET_W2 = NET_C2 * NET_C1 * 27, NET_W3 = NET_C3 * NET_C2 * 27;
constexpr int NET_OFF_W1 = 0, NET_OFF_B1 = NET_W1, NET_OFF_W2 = NET_OFF_B1 + NET_C1, NET_OFF_B2 = NET_OFF_W2 + NET_W2,
              NET_OFF_W3 = NET_OFF_B2 + NET_C2, NET_OFF_B3 = NET_OFF_W3 + NET_W3, NET_NPARAM = NET_OFF_B3 + NET_C3;

int learned_num_params() { return NET_NPARAM; }

__device__ __forceinline__ int lat_nb(int L, int k, int n1) {
  const int i = L % n1, j = (L / n1) % n1, kk = L / (n1 * n1);
  const int a = i + (k % 3) - 1, b = j + (k / 3) % 3 - 1, c = kk + k / 9 - 1;
  if (a < 0 || b < 0 || c < 0 || a >= n1 || b >= n1 || c >= n1) return -1;
  return a + n1 * (b + n1 * c);
}

// ------------------------------------------------------------- features
// feature k of node L = a(i, nb_k(i)) / a(i,i) for an active row i at node L
// (0 elsewhere), rounded to BF16: xf[L * 32 + k] (channels 27..31 stay 0) and,
// when feat != NULL (training), the same values FP32 channel-major;
// dscale[L] = 1 / a(i,i) for active rows, 0 for Dirichlet rows.  The caller
// zeroes xf (and feat).
__global__ void k_features(int N, int Na, int n1, const int *__restrict__ rp, const int *__restrict__ kc,
                           const double *__restrict__ a, const int *__restrict__ dof_lat, __nv_bfloat16 *__restrict__ xf,
                           float *__restrict__ feat, float *__restrict__ dscale) {
  const int NL = n1 * n1 * n1;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  const int L = dof_lat[r];
  if (r >= Na) { dscale[L] = 0.0f; return; }
  double diag = 1.0;
  for (int p = rp[r]; p < rp[r + 1]; p++) if (kc[p] == r) diag = a[p];
  const int i = L % n1, j = (L / n1) % n1, kk = L / (n1 * n1);
  for (int p = rp[r]; p < rp[r + 1]; p++) {
    const int Lc = dof_lat[kc[p]];
    const int di = Lc % n1 - i, dj = (Lc / n1) % n1 - j, dk = Lc / (n1 * n1) - kk;
    if (di < -1 || di > 1 || dj < -1 || dj > 1 || dk < -1 || dk > 1) continue;  // not on a 27-point stencil
    const int k = (di + 1) + 3 * (dj + 1) + 9 * (dk + 1);
    const __nv_bfloat16 v = __float2bfloat16((float)(a[p] / diag));
    xf[(size_t)L * 32 + k] = v;
    if (feat) feat[(size_t)k * NL + L] = __bfloat162float(v);
  }
  dscale[L] = (float)(1.0 / diag);
}

// Weights of one layer, [co][ci][27] BF16, repacked for the tensor-core
// forward as [k][co][ci] with both channel counts padded to 32 by zeros.
__global__ void k_pack_weights(int cin, int cout, const __nv_bfloat16 *__restrict__ w, __nv_bfloat16 *__restrict__ wpk) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 27 * 32 * 32) return;
  const int k = t >> 10, co = (t >> 5) & 31, ci = t & 31;
  wpk[t] = (co < cout && ci < cin) ? w[((size_t)co * cin + ci) * 27 + k] : __float2bfloat16(0.0f);
}

// ------------------------------------------------------------- tensor-core convolution
// One CTA (8 warps) owns a brick of CONV_BX x CONV_BY x CONV_BZ output nodes at
// a time (persistent over the bricks).  Shared memory holds the packed weights
// of the layer (27 x 32 x 32 BF16, loaded once) and the brick's input with a
// one-node halo (18 x 10 x 4 nodes x 64 bytes, zero outside the lattice).
// Warp w computes the nodes x = 0..15, y = w, z = 0..1 (two m16 tiles) for all
// 32 output channels (four n8 tiles): per offset and 16-channel chunk two
// ldmatrix.x4 for the activations, two for the weights and eight mma.
// Rows of 64 bytes are stored with their four 16-byte chunks permuted
// (chunk ^ ((row >> 1) & 3)), so the eight rows of one 8x8 ldmatrix read hit
// distinct banks.
constexpr int CONV_BX = 16, CONV_BY = 8, CONV_BZ = 2;
constexpr int CONV_HX = CONV_BX + 2, CONV_HY = CONV_BY + 2, CONV_HZ = CONV_BZ + 2;
constexpr int CONV_HALO = CONV_HX * CONV_HY * CONV_HZ;  // 720 nodes
constexpr int CONV_WROWS = 27 * 32;                     // weight rows [k][co]
constexpr int CONV_SMEM = (CONV_HALO + CONV_WROWS) * 64;  // 101,376 bytes: two CTAs per SM

__device__ __forceinline__ unsigned swz(int row, int chunk) {
  return (unsigned)(row * 64 + ((chunk ^ ((row >> 1) & 3)) << 4));
}

__device__ __forceinline__ void ldsm_x4(unsigned addr, unsigned (&r)[4]) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
}

// D += A (16x16, row) B (16x8, col), BF16 inputs, FP32 accumulators
__device__ __forceinline__ void mma_bf16(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// LAST = false: out = ReLU(conv + b) as BF16 node-major into xo; with a_cm /
//   z_cm (training) also the rounded activation and the pre-activation, FP32
//   channel-major.
// LAST = true: the stencil W[co][L] = (conv + b)[co] * dscale[L], co < cout.
template <bool LAST>
__global__ void __launch_bounds__(256, 2)
    k_conv_tc(int n1, int cout, const __nv_bfloat16 *__restrict__ xi, const __nv_bfloat16 *__restrict__ wpk,
              const __nv_bfloat16 *__restrict__ bias, __nv_bfloat16 *__restrict__ xo, float *__restrict__ a_cm,
              float *__restrict__ z_cm, const float *__restrict__ dscale, float *__restrict__ Wst) {
  extern __shared__ __align__(128) unsigned char conv_sm[];
  const unsigned s_halo = (unsigned)__cvta_generic_to_shared(conv_sm);
  const unsigned s_w = s_halo + CONV_HALO * 64;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const size_t NL = (size_t)n1 * n1 * n1;
  // weights: 864 rows x 4 chunks
  for (int t = tid; t < CONV_WROWS * 4; t += blockDim.x) {
    const int row = t >> 2, ch = t & 3;
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(wpk) + t);
    *reinterpret_cast<uint4 *>(conv_sm + CONV_HALO * 64 + swz(row, ch)) = v;
  }
  float bv[4][2];
#pragma unroll
  for (int nt = 0; nt < 4; nt++)
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int co = nt * 8 + 2 * (lane & 3) + e;
      bv[nt][e] = co < cout ? __bfloat162float(bias[co]) : 0.0f;
    }
  const int nbx = (n1 + CONV_BX - 1) / CONV_BX, nby = (n1 + CONV_BY - 1) / CONV_BY, nbz = (n1 + CONV_BZ - 1) / CONV_BZ;
  const int nbricks = nbx * nby * nbz;
  // per-lane ldmatrix rows: A (activations) row within the m16 tile and chunk half;
  // B (weights) output channel within a pair of n8 tiles and chunk half
  const int a_row = (lane & 7) + 8 * ((lane >> 3) & 1), a_half = lane >> 4;
  const int b_co = 8 * (lane >> 4) + (lane & 7), b_half = (lane >> 3) & 1;
  for (int br = blockIdx.x; br < nbricks; br += gridDim.x) {
    const int bx = br % nbx, by = (br / nbx) % nby, bz = br / (nbx * nby);
    const int x0 = bx * CONV_BX, y0 = by * CONV_BY, z0 = bz * CONV_BZ;
    __syncthreads();  // the previous brick's reads of the halo are done
    for (int t = tid; t < CONV_HALO * 4; t += blockDim.x) {
      const int node = t >> 2, ch = t & 3;
      const int hx = node % CONV_HX, hy = (node / CONV_HX) % CONV_HY, hz = node / (CONV_HX * CONV_HY);
      const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (gx >= 0 && gy >= 0 && gz >= 0 && gx < n1 && gy < n1 && gz < n1) {
        const size_t L = (size_t)gx + (size_t)n1 * ((size_t)gy + (size_t)n1 * gz);
        v = __ldg(reinterpret_cast<const uint4 *>(xi + L * 32) + ch);
      }
      *reinterpret_cast<uint4 *>(conv_sm + swz(node, ch)) = v;
    }
    __syncthreads();
    float acc[2][4][4];
#pragma unroll
    for (int m = 0; m < 2; m++)
#pragma unroll
      for (int nt = 0; nt < 4; nt++)
#pragma unroll
        for (int e = 0; e < 4; e++) acc[m][nt][e] = 0.0f;
#pragma unroll 3
    for (int k = 0; k < 27; k++) {
      const int dx = k % 3, dy = (k / 3) % 3, dz = k / 9;
#pragma unroll
      for (int kc = 0; kc < 2; kc++) {
        unsigned a[2][4], b[2][4];
#pragma unroll
        for (int m = 0; m < 2; m++) {
          const int row = (a_row + dx) + CONV_HX * ((warp + dy) + CONV_HY * (m + dz));
          ldsm_x4(s_halo + swz(row, 2 * kc + a_half), a[m]);
        }
#pragma unroll
        for (int p = 0; p < 2; p++) {
          const int row = k * 32 + 16 * p + b_co;
          ldsm_x4(s_w + swz(row, 2 * kc + b_half), b[p]);
        }
#pragma unroll
        for (int m = 0; m < 2; m++)
#pragma unroll
          for (int p = 0; p < 2; p++) {
            mma_bf16(acc[m][2 * p], a[m], b[p][0], b[p][1]);
            mma_bf16(acc[m][2 * p + 1], a[m], b[p][2], b[p][3]);
          }
      }
    }
    // epilogue: c0,c1 = (row g, channels 2q, 2q+1), c2,c3 = (row g+8, ...)
    const int g = lane >> 2, q = lane & 3;
    const int gy = y0 + warp;
#pragma unroll
    for (int m = 0; m < 2; m++) {
      const int gz = z0 + m;
#pragma unroll
      for (int hrow = 0; hrow < 2; hrow++) {
        const int gx = x0 + g + 8 * hrow;
        if (gx >= n1 || gy >= n1 || gz >= n1) continue;
        const size_t L = (size_t)gx + (size_t)n1 * ((size_t)gy + (size_t)n1 * gz);
        const float ds = LAST ? dscale[L] : 0.0f;
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
          const int co = nt * 8 + 2 * q;
          const float v0 = acc[m][nt][2 * hrow] + bv[nt][0], v1 = acc[m][nt][2 * hrow + 1] + bv[nt][1];
          if (LAST) {
            if (co < cout) Wst[(size_t)co * NL + L] = v0 * ds;
            if (co + 1 < cout) Wst[(size_t)(co + 1) * NL + L] = v1 * ds;
          } else {
            const __nv_bfloat162 r = __floats2bfloat162_rn(fmaxf(v0, 0.0f), fmaxf(v1, 0.0f));
            *reinterpret_cast<__nv_bfloat162 *>(xo + L * 32 + co) = r;
            if (a_cm) {
              a_cm[(size_t)co * NL + L] = __low2float(r);
              a_cm[(size_t)(co + 1) * NL + L] = __high2float(r);
              z_cm[(size_t)co * NL + L] = v0;
              z_cm[(size_t)(co + 1) * NL + L] = v1;
            }
          }
        }
      }
    }
  }
}

// dx[ci][L] = sum_{co,k} w[co][ci][k] dz[co][L - o_k]  (neighbour L' with nb_k(L') = L)
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_conv_bwd_data(int n1, const float *__restrict__ dz, const __nv_bfloat16 *__restrict__ w,
                                                       float *__restrict__ dx) {
  extern __shared__ float sw[];  // [co][k][ci]
  const int NL = n1 * n1 * n1;
  for (int t = threadIdx.x; t < COUT * CIN * 27; t += blockDim.x) {
    const int co = t / (CIN * 27), rem = t % (CIN * 27);
    const int ci = rem / 27, k = rem % 27;
    sw[(co * 27 + k) * CIN + ci] = __bfloat162float(w[t]);
  }
  __syncthreads();
  const int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= NL) return;
  float acc[CIN];
#pragma unroll
  for (int ci = 0; ci < CIN; ci++) acc[ci] = 0.0f;
  for (int k = 0; k < 27; k++) {
    const int src = lat_nb(L, 26 - k, n1);  // L - o_k
    if (src < 0) continue;
    for (int co = 0; co < COUT; co++) {
      const float g = dz[(size_t)co * NL + src];
      const float *wr = sw + (co * 27 + k) * CIN;
#pragma unroll
      for (int ci = 0; ci < CIN; ci++) acc[ci] += wr[ci] * g;
    }
  }
#pragma unroll
  for (int ci = 0; ci < CIN; ci++) dx[(size_t)ci * NL + L] = acc[ci];
}

// gw[co][ci][k] += sum_L dz[co][L] x[ci][nb_k(L)] ; gb[co] += sum_L dz[co][L]
// one block per (ci, k); threads stride over L with COUT accumulators
template <int CIN, int COUT>
__global__ void __launch_bounds__(256) k_conv_bwd_weight(int n1, const float *__restrict__ dz, const float *__restrict__ x,
                                                         float *__restrict__ gw, float *__restrict__ gb) {
  const int NL = n1 * n1 * n1;
  const int ci = blockIdx.x / 27, k = blockIdx.x % 27;
  const bool do_bias = (blockIdx.x == 0);
  float acc[COUT], accb[COUT];
#pragma unroll
  for (int co = 0; co < COUT; co++) { acc[co] = 0.0f; accb[co] = 0.0f; }
  for (int L = threadIdx.x; L < NL; L += blockDim.x) {
    const int nb = lat_nb(L, k, n1);
    const float xv = nb >= 0 ? x[(size_t)ci * NL + nb] : 0.0f;
#pragma unroll
    for (int co = 0; co < COUT; co++) {
      const float g = dz[(size_t)co * NL + L];
      acc[co] += g * xv;
      if (do_bias) accb[co] += g;
    }
  }
  __shared__ float red[256];
  for (int co = 0; co < COUT; co++) {
    red[threadIdx.x] = acc[co];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) gw[(size_t)(co * CIN + ci) * 27 + k] += red[0];
    __syncthreads();
    if (do_bias) {
      red[threadIdx.x] = accb[co];
      __syncthreads();
      for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
      }
      if (threadIdx.x == 0) gb[co] += red[0];
      __syncthreads();
    }
  }
}

// ReLU backward in place: g = g * (z > 0)
__global__ void k_relu_bwd(size_t n, const float *__restrict__ z, float *__restrict__ g) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (!(z[i] > 0.0f)) g[i] = 0.0f;
}

// ------------------------------------------------------------- smoothing step
// x_i += omega sum_k W_k(L_i) r_{dof(nb_k(L_i))} on active dofs (dof order vectors)
template <typename T>
__global__ void __launch_bounds__(256) k_stencil_smooth(int Na, int n1, const int *__restrict__ dof_lat,
                                                        const int *__restrict__ lat_dof, const float *__restrict__ W,
                                                        const T *__restrict__ r, T *__restrict__ x, T omega) {
  pdl_wait();
  pdl_trigger();
  const int NL = n1 * n1 * n1;
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= Na) return;
  const int L = dof_lat[d];
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 27; k++) {
    const int nb = lat_nb(L, k, n1);
    if (nb >= 0) s += W[(size_t)k * NL + L] * (float)r[lat_dof[nb]];
  }
  x[d] += omega * (T)s;
}

template <typename T>
int learned_smooth(cudaStream_t s, const Level &L, const T *r, T *x, double omega) {
  const int nb = (L.Na + 255) / 256;
  if (nb == 0) return PMG_OK;
  PMG_CUDA(launch_pdl(k_stencil_smooth<T>, dim3(nb), dim3(256), 0, s, L.Na, L.lat_n[0], (const int *)L.dof_ijk.p,
                      (const int *)L.lat_dof.p, (const float *)L.lw_stencil.p, r, x, (T)omega));
  count_launches(1);
  return PMG_OK;
}
template int learned_smooth<float>(cudaStream_t, const Level &, const float *, float *, double);
template int learned_smooth<double>(cudaStream_t, const Level &, const double *, double *, double);

// ------------------------------------------------------------- network driver
static int conv_smem(int cin, int cout) { return cin * cout * 27 * (int)sizeof(float); }

static int set_conv_attrs() {
  static bool done = false;
  if (done) return PMG_OK;
  PMG_CUDA(cudaFuncSetAttribute(k_conv_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, CONV_SMEM));
  PMG_CUDA(cudaFuncSetAttribute(k_conv_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, CONV_SMEM));
  PMG_CUDA(cudaFuncSetAttribute(k_conv_bwd_data<NET_C1, NET_C2>, cudaFuncAttributeMaxDynamicSharedMemorySize, conv_smem(NET_C1, NET_C2)));
  PMG_CUDA(cudaFuncSetAttribute(k_conv_bwd_data<NET_C2, NET_C3>, cudaFuncAttributeMaxDynamicSharedMemorySize, conv_smem(NET_C2, NET_C3)));
  done = true;
  return PMG_OK;
}

// persistent grid of the tensor-core convolution: two CTAs per SM, at most one per brick
static int conv_grid(int n1, int num_sms) {
  const long nb = (long)((n1 + CONV_BX - 1) / CONV_BX) * ((n1 + CONV_BY - 1) / CONV_BY) * ((n1 + CONV_BZ - 1) / CONV_BZ);
  return (int)std::min<long>(nb, 2L * num_sms);
}

// forward pass on one level: features -> W (stencil, L.lw_stencil); with
// train, the FP32 channel-major layer inputs and pre-activations stay in S
static int net_forward(cudaStream_t s, int num_sms, Level &L, const __nv_bfloat16 *wb, NetScratch &S, bool train) {
  const int n1 = L.lat_n[0], NL = n1 * n1 * n1;
  PMG_TRY(set_conv_attrs());
  PMG_TRY(S.alloc(NL, NET_C0, NET_C1, NET_C2, train));
  __nv_bfloat16 *xa = reinterpret_cast<__nv_bfloat16 *>(S.xa.p), *xb = reinterpret_cast<__nv_bfloat16 *>(S.xb.p);
  __nv_bfloat16 *wpk = reinterpret_cast<__nv_bfloat16 *>(S.wpk.p);
  const int WPK = 27 * 32 * 32;
  k_pack_weights<<<WPK / 256, 256, 0, s>>>(NET_C0, NET_C1, wb + NET_OFF_W1, wpk);
  k_pack_weights<<<WPK / 256, 256, 0, s>>>(NET_C1, NET_C2, wb + NET_OFF_W2, wpk + WPK);
  k_pack_weights<<<WPK / 256, 256, 0, s>>>(NET_C2, NET_C3, wb + NET_OFF_W3, wpk + 2 * WPK);
  PMG_CUDA(cudaMemsetAsync(xa, 0, sizeof(__nv_bfloat16) * 32 * (size_t)NL, s));
  PMG_CUDA(cudaMemsetAsync(S.dscale.p, 0, sizeof(float) * (size_t)NL, s));
  if (train) PMG_CUDA(cudaMemsetAsync(S.feat.p, 0, sizeof(float) * NET_C0 * (size_t)NL, s));
  k_features<<<(L.N + 255) / 256, 256, 0, s>>>(L.N, L.Na, n1, L.rowptr.p, L.kcol.p, L.A.p, L.dof_ijk.p, xa,
                                                train ? S.feat.p : nullptr, S.dscale.p);
  PMG_TRY(L.lw_stencil.alloc((size_t)27 * NL));
  const int g = conv_grid(n1, num_sms);
  k_conv_tc<false><<<g, 256, CONV_SMEM, s>>>(n1, NET_C1, xa, wpk, wb + NET_OFF_B1, xb, train ? S.a1.p : nullptr,
                                              train ? S.z1.p : nullptr, nullptr, nullptr);
  k_conv_tc<false><<<g, 256, CONV_SMEM, s>>>(n1, NET_C2, xb, wpk + WPK, wb + NET_OFF_B2, xa, train ? S.a2.p : nullptr,
                                              train ? S.z2.p : nullptr, nullptr, nullptr);
  k_conv_tc<true><<<g, 256, CONV_SMEM, s>>>(n1, NET_C3, xa, wpk + 2 * WPK, wb + NET_OFF_B3, nullptr, nullptr, nullptr,
                                             S.dscale.p, L.lw_stencil.p);
  count_launches(7);
  PMG_CUDA(cudaGetLastError());
  return PMG_OK;
}


int learned_forward(Handle &h, Level &L) {
  if (!h.has_learned || L.lat_n[0] <= 0) {
    set_error("learned smoother: the forward needs weights and a lattice");
    return PMG_ERR_STATE;
  }
  PMG_TRY(net_forward(h.stream, h.num_sms, L, reinterpret_cast<const __nv_bfloat16 *>(h.lw_bf16.p), h.net_scratch, false));
  L.lw_fresh = true;
  return PMG_OK;
}

// network -> stencil on every level that has a lattice (after assembly)
int learned_prepare(Handle &h) {
  if (!h.has_learned) {
    set_error("learned smoother: no weights (pmg_set_learned_weights)");
    return PMG_ERR_STATE;
  }
  for (auto &L : h.lv) {
    if (L.lat_n[0] <= 0) {
      set_error("learned smoother: every level needs a lattice (pmg_set_level_lattice)");
      return PMG_ERR_STATE;
    }
    if (L.lw_fresh) continue;
    PMG_TRY(learned_forward(h, L));
  }
  return PMG_OK;
}

// ------------------------------------------------------------- training
// loss for one sample (e, r = A e) on a level:  c = S r, u = e - c, v = A u,
// loss = |v|^2 / |r|^2 ; gradients w.r.t. the FP32 master weights accumulate in g.
__global__ void k_lat_gather(int N, const int *__restrict__ dof_lat, const double *__restrict__ v, float *__restrict__ vl) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < N) vl[dof_lat[d]] = (float)v[d];
}

// c[L] = sum_k W_k(L) r[nb_k(L)] (lattice order) ; u_dof = e_dof - c
__global__ void k_train_apply(int N, int Na, int n1, const int *__restrict__ dof_lat, const float *__restrict__ W,
                              const float *__restrict__ rl, const double *__restrict__ e, double *__restrict__ u) {
  const int NL = n1 * n1 * n1;
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= N) return;
  if (d >= Na) { u[d] = e[d]; return; }
  const int L = dof_lat[d];
  float s = 0.0f;
  for (int k = 0; k < 27; k++) {
    const int nb = lat_nb(L, k, n1);
    if (nb >= 0) s += W[(size_t)k * NL + L] * rl[nb];
  }
  u[d] = e[d] - (double)s;
}

// y_i = sum_j A_ji z_j through the transposed-entry map (pattern is structurally symmetric)
__global__ void k_spmv_t(int N, const int *__restrict__ rp, const int *__restrict__ kc, const int *__restrict__ tpos,
                         const double *__restrict__ a, const double *__restrict__ z, double *__restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double s = 0.0;
  for (int p = rp[i]; p < rp[i + 1]; p++) {
    const int t = tpos[p];
    if (t >= 0) s += a[t] * z[kc[p]];
  }
  y[i] = s;
}

// dout3[k][L] = -du[L] * r[nb_k(L)] * dscale[L]  (active nodes; du in lattice order)
__global__ void k_train_dout(int NL, int n1, const float *__restrict__ dul, const float *__restrict__ rl,
                             const float *__restrict__ dscale, float *__restrict__ dout) {
  const int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= NL) return;
  const float g = -dul[L] * dscale[L];
  for (int k = 0; k < 27; k++) {
    const int nb = lat_nb(L, k, n1);
    dout[(size_t)k * NL + L] = nb >= 0 ? g * rl[nb] : 0.0f;
  }
}

__global__ void k_scale_f(size_t n, float *x, const double *__restrict__ s2) {
  const float f = (float)(2.0 / (*s2 > 0 ? *s2 : 1.0));
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) x[i] *= f;
}

__global__ void k_adam(int n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       float lr, float b1, float b2, float eps, float c1, float c2, __nv_bfloat16 *__restrict__ pb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1 - b1) * gi, vi = b2 * v[i] + (1 - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pi;
  pb[i] = __float2bfloat16(pi);
}

}  // namespace pmg

using namespace pmg;

// Adam on the FP32 master weights (BF16 copy refreshed) from a host gradient
static int adam_step(pmg::Handle *h, const float *g, float lr) {
  using namespace pmg;
  cudaStream_t s = h->stream;
  PMG_CUDA(cudaMemcpyAsync(h->lw_grad.p, g, sizeof(float) * NET_NPARAM, cudaMemcpyHostToDevice, s));
  h->adam_t++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, (float)h->adam_t), c2 = 1.0f - powf(b2, (float)h->adam_t);
  k_adam<<<(NET_NPARAM + 255) / 256, 256, 0, s>>>(NET_NPARAM, h->lw_master.p, h->lw_grad.p, h->lw_m.p, h->lw_v.p, lr,
                                                   b1, b2, 1e-8f, c1, c2, reinterpret_cast<__nv_bfloat16 *>(h->lw_bf16.p));
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  PMG_CUDA(cudaStreamSynchronize(s));
  for (auto &Lv : h->lv) Lv.lw_fresh = false;
  return PMG_OK;
}

extern "C" {

int pmg_learned_num_params(int *n) {
  if (!n) return PMG_ERR_ARG;
  *n = NET_NPARAM;
  return PMG_OK;
}

int pmg_set_level_lattice(pmg_handle hh, int level, int nx, int ny, int nz, const int *dof_lat) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || level < 0 || level >= (int)h->lv.size() || !dof_lat) return PMG_ERR_ARG;
  Level &L = h->lv[level];
  if (!L.has_csr) { set_error("pmg_set_level_lattice: set the CSR first"); return PMG_ERR_STATE; }
  if (nx != ny || ny != nz || nx < 2 || (long)nx * nx * nx != L.N) {
    set_error("pmg_set_level_lattice: the learned smoother needs a cubic lattice with one dof per node");
    return PMG_ERR_UNSUPPORTED;
  }
  std::vector<int> inv((size_t)L.N, -1);
  for (int d = 0; d < L.N; d++) {
    if (dof_lat[d] < 0 || dof_lat[d] >= L.N || inv[dof_lat[d]] >= 0) {
      set_error("pmg_set_level_lattice: dof_lat is not a permutation of the lattice");
      return PMG_ERR_ARG;
    }
    inv[dof_lat[d]] = d;
  }
  PMG_TRY(L.dof_ijk.upload(dof_lat, L.N, h->stream));
  PMG_TRY(L.lat_dof.upload(inv.data(), inv.size(), h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  L.lat_n[0] = nx; L.lat_n[1] = ny; L.lat_n[2] = nz;
  L.lw_fresh = false;
  return PMG_OK;
}

int pmg_set_learned_weights(pmg_handle hh, const float *weights) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || !weights) return PMG_ERR_ARG;
  std::vector<__nv_bfloat16> wb(NET_NPARAM);
  for (int i = 0; i < NET_NPARAM; i++) {
    if (!std::isfinite(weights[i])) { set_error("pmg_set_learned_weights: non-finite weight"); return PMG_ERR_NONFINITE; }
    wb[i] = __float2bfloat16(weights[i]);
  }
  PMG_TRY(h->lw_bf16.upload(reinterpret_cast<const uint16_t *>(wb.data()), wb.size(), h->stream));
  PMG_TRY(h->lw_master.upload(weights, NET_NPARAM, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  h->has_learned = true;
  for (auto &L : h->lv) L.lw_fresh = false;
  return PMG_OK;
}

int pmg_get_learned_weights(pmg_handle hh, float *weights) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || !weights || !h->lw_master.p) return PMG_ERR_STATE;
  PMG_CUDA(cudaMemcpy(weights, h->lw_master.p, sizeof(float) * NET_NPARAM, cudaMemcpyDeviceToHost));
  return PMG_OK;
}

// Stencil W of a level (27 x NL FP32, lattice order) for inspection / tests.
int pmg_learned_stencil(pmg_handle hh, int level, float *W_out) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || level < 0 || level >= (int)h->lv.size() || !W_out) return PMG_ERR_ARG;
  Level &L = h->lv[level];
  if (!L.assembled) { set_error("pmg_learned_stencil: assemble first"); return PMG_ERR_STATE; }
  PMG_TRY(learned_prepare(*h));
  PMG_CUDA(cudaMemcpyAsync(W_out, L.lw_stencil.p, sizeof(float) * 27 * (size_t)L.N, cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  return PMG_OK;
}

// One training step on `level` over n_samples pairs (e_s, r_s = A e_s) given as
// device arrays of n_samples x N doubles: loss = mean_s |A (e_s - S r_s)|^2 / |r_s|^2.
// lr > 0 applies one Adam step (beta 0.9 / 0.999) to the master weights;
// grad_out (host, n_params floats, may be NULL) receives the mean gradient.
int pmg_learned_train_step(pmg_handle hh, int level, int n_samples, const double *e_dev, const double *r_dev, float lr,
                           double *loss_out, float *grad_out) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || level < 0 || level >= (int)h->lv.size() || n_samples < 1 || !e_dev || !r_dev) return PMG_ERR_ARG;
  if (!h->has_learned) { set_error("pmg_learned_train_step: set initial weights first"); return PMG_ERR_STATE; }
  Level &L = h->lv[level];
  if (!L.assembled || L.lat_n[0] <= 0) { set_error("pmg_learned_train_step: level needs a matrix and a lattice"); return PMG_ERR_STATE; }
  cudaStream_t s = h->stream;
  const int n1 = L.lat_n[0], NL = n1 * n1 * n1, N = L.N;
  // transposed-entry map (once per pattern)
  if (L.tpos.n != (size_t)L.nnz) {
    std::vector<int> tp(L.nnz, -1);
    const std::vector<int> &rp = L.h_rowptr, &kc = L.h_kcol;
    for (int i = 0; i < N; i++)
      for (int p = rp[i]; p < rp[i + 1]; p++) {
        const int j = kc[p];
        int lo = rp[j], hi = rp[j + 1] - 1;
        while (lo <= hi) {
          int mid = (lo + hi) >> 1;
          if (kc[mid] == i) { tp[p] = mid; break; }
          if (kc[mid] < i) lo = mid + 1; else hi = mid - 1;
        }
      }
    PMG_TRY(L.tpos.upload(tp.data(), tp.size(), s));
  }
  NetScratch &S = h->net_scratch;
  PMG_TRY(net_forward(s, h->num_sms, L, reinterpret_cast<const __nv_bfloat16 *>(h->lw_bf16.p), S, true));
  PMG_TRY(h->lw_grad.alloc(NET_NPARAM));
  PMG_TRY(h->lw_m.alloc(NET_NPARAM));
  PMG_TRY(h->lw_v.alloc(NET_NPARAM));
  if (h->adam_t == 0) {
    PMG_CUDA(cudaMemsetAsync(h->lw_m.p, 0, sizeof(float) * NET_NPARAM, s));
    PMG_CUDA(cudaMemsetAsync(h->lw_v.p, 0, sizeof(float) * NET_NPARAM, s));
  }
  PMG_CUDA(cudaMemsetAsync(h->lw_grad.p, 0, sizeof(float) * NET_NPARAM, s));
  DBuf<float> rl, dul, dout, d2, d1;
  DBuf<double> u, v, du, nrm;
  PMG_TRY(rl.alloc(NL)); PMG_TRY(dul.alloc(NL));
  PMG_TRY(dout.alloc((size_t)NET_C3 * NL)); PMG_TRY(d2.alloc((size_t)NET_C2 * NL)); PMG_TRY(d1.alloc((size_t)NET_C1 * NL));
  PMG_TRY(u.alloc(N)); PMG_TRY(v.alloc(N)); PMG_TRY(du.alloc(N)); PMG_TRY(nrm.alloc(2 * n_samples));
  const int gN = (N + 255) / 256, gL = (NL + 255) / 256, gC = (NL + 127) / 128;
  float *gw = h->lw_grad.p;
  const __nv_bfloat16 *wb = reinterpret_cast<const __nv_bfloat16 *>(h->lw_bf16.p);
  for (int smp = 0; smp < n_samples; smp++) {
    const double *e = e_dev + (size_t)smp * N, *r = r_dev + (size_t)smp * N;
    PMG_CUDA(cudaMemsetAsync(rl.p, 0, sizeof(float) * NL, s));
    k_lat_gather<<<gN, 256, 0, s>>>(N, L.dof_ijk.p, r, rl.p);
    k_train_apply<<<gN, 256, 0, s>>>(N, L.Na, n1, L.dof_ijk.p, L.lw_stencil.p, rl.p, e, u.p);
    PMG_TRY(spmv<double>(s, L, L.A.p, u.p, v.p));
    PMG_TRY(dot(*h, v.p, v.p, N, nrm.p + 2 * smp));
    PMG_TRY(dot(*h, r, r, N, nrm.p + 2 * smp + 1));
    // dL/dv = 2 v / |r|^2 ; du = A^T dL/dv ; dL/dc = -du
    k_spmv_t<<<gN, 256, 0, s>>>(N, L.rowptr.p, L.kcol.p, L.tpos.p, L.A.p, v.p, du.p);
    PMG_CUDA(cudaMemsetAsync(dul.p, 0, sizeof(float) * NL, s));
    k_lat_gather<<<gN, 256, 0, s>>>(N, L.dof_ijk.p, du.p, dul.p);
    k_train_dout<<<gL, 256, 0, s>>>(NL, n1, dul.p, rl.p, S.dscale.p, dout.p);
    k_scale_f<<<std::min(gL * 27, 148 * 16), 256, 0, s>>>((size_t)NET_C3 * NL, dout.p, nrm.p + 2 * smp + 1);
    // layer 3 (no ReLU), layer 2, layer 1
    k_conv_bwd_weight<NET_C2, NET_C3><<<NET_C2 * 27, 256, 0, s>>>(n1, dout.p, S.a2.p, gw + NET_OFF_W3, gw + NET_OFF_B3);
    k_conv_bwd_data<NET_C2, NET_C3><<<gC, 128, conv_smem(NET_C2, NET_C3), s>>>(n1, dout.p, wb + NET_OFF_W3, d2.p);
    k_relu_bwd<<<std::min(gL * 32, 148 * 16), 256, 0, s>>>((size_t)NET_C2 * NL, S.z2.p, d2.p);
    k_conv_bwd_weight<NET_C1, NET_C2><<<NET_C1 * 27, 256, 0, s>>>(n1, d2.p, S.a1.p, gw + NET_OFF_W2, gw + NET_OFF_B2);
    k_conv_bwd_data<NET_C1, NET_C2><<<gC, 128, conv_smem(NET_C1, NET_C2), s>>>(n1, d2.p, wb + NET_OFF_W2, d1.p);
    k_relu_bwd<<<std::min(gL * 32, 148 * 16), 256, 0, s>>>((size_t)NET_C1 * NL, S.z1.p, d1.p);
    k_conv_bwd_weight<NET_C0, NET_C1><<<NET_C0 * 27, 256, 0, s>>>(n1, d1.p, S.feat.p, gw + NET_OFF_W1, gw + NET_OFF_B1);
    count_launches(14);
    PMG_CUDA(cudaGetLastError());
  }
  std::vector<double> nr(2 * n_samples);
  PMG_CUDA(cudaMemcpyAsync(nr.data(), nrm.p, sizeof(double) * nr.size(), cudaMemcpyDeviceToHost, s));
  PMG_CUDA(cudaStreamSynchronize(s));
  double loss = 0;
  for (int smp = 0; smp < n_samples; smp++) loss += nr[2 * smp] / (nr[2 * smp + 1] > 0 ? nr[2 * smp + 1] : 1.0);
  loss /= n_samples;
  if (loss_out) *loss_out = loss;
  // mean over samples
  std::vector<float> g(NET_NPARAM);
  PMG_CUDA(cudaMemcpy(g.data(), gw, sizeof(float) * NET_NPARAM, cudaMemcpyDeviceToHost));
  for (auto &x : g) x /= (float)n_samples;
  if (grad_out) std::copy(g.begin(), g.end(), grad_out);
  if (lr > 0) PMG_TRY(adam_step(h, g.data(), lr));
  return PMG_OK;
}

int pmg_learned_apply_gradient(pmg_handle hh, const float *grad, float lr) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || !grad || !(lr > 0)) {
    set_error("pmg_learned_apply_gradient: bad arguments");
    return PMG_ERR_ARG;
  }
  if (!h->lw_master.p) {
    set_error("pmg_learned_apply_gradient: set the weights first");
    return PMG_ERR_STATE;
  }
  for (int k = 0; k < NET_NPARAM; k++)
    if (!std::isfinite(grad[k])) {
      set_error("pmg_learned_apply_gradient: non-finite gradient");
      return PMG_ERR_NONFINITE;
    }
  PMG_TRY(h->lw_grad.alloc(NET_NPARAM));
  PMG_TRY(h->lw_m.alloc(NET_NPARAM));
  PMG_TRY(h->lw_v.alloc(NET_NPARAM));
  if (h->adam_t == 0) {
    PMG_CUDA(cudaMemsetAsync(h->lw_m.p, 0, sizeof(float) * NET_NPARAM, h->stream));
    PMG_CUDA(cudaMemsetAsync(h->lw_v.p, 0, sizeof(float) * NET_NPARAM, h->stream));
  }
  return adam_step(h, grad, lr);
}

}  // extern "C"
