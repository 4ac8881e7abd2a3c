// pmg_defect_noalloc: the defect r = b - A x and its norm without any device
// allocation at call time.
//
// pmg_defect copies host vectors into freshly allocated device buffers and
// reduces the norm through the handle's reduction buffers.  Some callers
// cannot take that route: a host that hands the library memory from its own
// device pool (an inference server or a framework allocator that has already
// reserved the GPU's memory) cannot let a library call cudaMalloc behind its
// back, and a latency-critical loop cannot afford cudaFree, which waits for
// the whole device.  This entry point takes device pointers for x, b, r and
// the norm, and keeps its only scratch -- one partial sum of squares per
// block of rows -- in a fixed array compiled into the library.
//
// The scratch array is a file-scope __device__ array: every GPU that loads the
// library holds it (512 KiB) until the process exits, and every call shares
// it.  Each call overwrites the partials it uses before reading them, so no
// clearing is needed between calls; two calls whose kernels overlap on the
// GPU (different streams, or different handles on one device running at the
// same time) race on it.
#include "pmg_internal.h"
#include <mutex>

namespace pmg {

constexpr int kNoallocRowsPerBlock = 256;
constexpr size_t kNoallocPartials = (size_t)PMG_NOALLOC_MAX_ROWS / kNoallocRowsPerBlock;  // 65,536 doubles

static __device__ __align__(256) double g_noalloc_partials[kNoallocPartials];

// Host code must not pass g_noalloc_partials itself to a kernel: on the host
// that name is only a stand-in for the device array.  The device address is
// looked up once per device, with that device current.
static std::mutex g_noalloc_mu;
static double *g_noalloc_addr[128] = {};

static int noalloc_scratch(int device, double **out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (device < 0 || device >= 128) {
    set_error("pmg_defect_noalloc: device index out of range");
    return PMG_ERR_ARG;
  }
  if (!g_noalloc_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p) {
      set_error(std::string("pmg_defect_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      return PMG_ERR_CUDA;
    }
    g_noalloc_addr[device] = static_cast<double *>(p);
  }
  *out = g_noalloc_addr[device];
  return PMG_OK;
}

// Block b owns rows [256 b, 256 b + 256): W lanes per row, the block's sum of
// squared defects goes to partials[b].  Loops are warp-uniform (shuffles).
template <int W>
__global__ void __launch_bounds__(256) k_defect_partials(int N, const int *__restrict__ rp, const int *__restrict__ kc,
                                                         const double *__restrict__ a, const double *__restrict__ x,
                                                         const double *__restrict__ f, double *__restrict__ d,
                                                         double *__restrict__ partials) {
  constexpr int GROUPS = 256 / W;
  __shared__ double sh[GROUPS];
  const int g = threadIdx.x / W, lane = threadIdx.x & (W - 1);
  const int row0 = blockIdx.x * kNoallocRowsPerBlock;
  double acc = 0.0;
  for (int rr = g; rr < kNoallocRowsPerBlock; rr += GROUPS) {
    const int row = row0 + rr;
    double s = 0.0;
    if (row < N)
      for (int k = __ldg(rp + row) + lane; k < __ldg(rp + row + 1); k += W) s += __ldg(a + k) * __ldg(x + __ldg(kc + k));
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, W);
    if (lane == 0 && row < N) {
      const double v = __ldg(f + row) - s;
      d[row] = v;
      acc += v * v;
    }
  }
  if (lane == 0) sh[g] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < GROUPS; k++) t += sh[k];
    partials[blockIdx.x] = t;
  }
}

// One block adds the nb partials in a fixed order and writes the norm.
__global__ void __launch_bounds__(256) k_noalloc_norm(int nb, const double *__restrict__ partials, double *norm) {
  __shared__ double sh[256];
  double t = 0.0;
  for (int k = threadIdx.x; k < nb; k += 256) t += partials[k];
  sh[threadIdx.x] = t;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *norm = sqrt(sh[0]);
}

}  // namespace pmg

using namespace pmg;

extern "C" int pmg_defect_noalloc(pmg_handle hh, int level, const double *x, const double *b, double *r,
                                  double *norm) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  // the same checks as pmg_defect: an existing level whose matrix holds values
  PMG_TRY(check_matrix(h, level, "pmg_defect_noalloc"));
  if (!x || !b || !r || !norm) {
    set_error("pmg_defect_noalloc: x, b, r and norm must be device pointers");
    return PMG_ERR_ARG;
  }
  Level &L = h->lv[level];
  if ((long)L.N > (long)PMG_NOALLOC_MAX_ROWS) {
    set_error("pmg_defect_noalloc: the level has more rows than PMG_NOALLOC_MAX_ROWS (16,777,216); "
              "use pmg_defect");
    return PMG_ERR_ARG;
  }
  int prev = -1;
  PMG_CUDA(cudaGetDevice(&prev));
  if (prev != h->device) PMG_CUDA(cudaSetDevice(h->device));
  double *scratch = nullptr;
  int rc = noalloc_scratch(h->device, &scratch);
  if (rc == PMG_OK) {
    const int nb = (L.N + kNoallocRowsPerBlock - 1) / kNoallocRowsPerBlock;
    const int W = L.avg_row >= 48 ? 32 : (L.avg_row >= 16 ? 16 : 8);
    if (W == 32) k_defect_partials<32><<<nb, 256, 0, h->stream>>>(L.N, L.rowptr.p, L.kcol.p, L.A.p, x, b, r, scratch);
    else if (W == 16) k_defect_partials<16><<<nb, 256, 0, h->stream>>>(L.N, L.rowptr.p, L.kcol.p, L.A.p, x, b, r, scratch);
    else k_defect_partials<8><<<nb, 256, 0, h->stream>>>(L.N, L.rowptr.p, L.kcol.p, L.A.p, x, b, r, scratch);
    k_noalloc_norm<<<1, 256, 0, h->stream>>>(nb, scratch, norm);
    count_launches(2);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
      set_error(std::string("pmg_defect_noalloc: ") + cudaGetErrorString(e));
      rc = PMG_ERR_CUDA;
    }
  }
  if (prev != h->device) cudaSetDevice(prev);
  return rc;
}
