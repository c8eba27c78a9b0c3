// hg_noalloc.cu -- hg_residuals_noalloc: Mesh_ComputeResiduals of a caller-owned device array
// without allocating device memory (declared in include/horses_gpu.h).
//
// The per-block partial maxima and the four results live in one file-scope device array of fixed
// size (na_scratch, 512 KB + 32 B).  Every call looks up its address on the current device with
// cudaGetSymbolAddress (a host-side lookup; nothing is cached, so a reset device or another host
// thread never sees a stale address).  Nothing in the scratch has to start at zero: every slot a call
// reads was written earlier in the same call, on the same stream.  Two calls that overlap in time on
// one device (different streams or host threads) share the scratch and race; callers serialise them.
#include "../../include/horses_gpu.h"

#include <cuda_runtime.h>

namespace {

constexpr int NA_THREADS = 256;
constexpr int64_t NA_NODES_PER_BLOCK = 8192;   // 32 nodes per thread
constexpr int NA_MAX_BLOCKS = 16384;           // partials: 16384 x 4 doubles = 512 KB
static_assert(int64_t(NA_MAX_BLOCKS) * NA_NODES_PER_BLOCK * 4 == HG_NOALLOC_MAX_NDOF, "scratch size and limit");

static __device__ __align__(256) double na_scratch[NA_MAX_BLOCKS * 4 + 4];

__device__ __forceinline__ double na_max(double m, double v) { return (v > m || v != v) ? v : m; }

// block b: max |x[node][k]| over nodes [b*NPB, min((b+1)*NPB, n_nodes)) -> part[b][k]
__global__ void __launch_bounds__(NA_THREADS) na_partial_kernel(const double* x, int64_t n_nodes, double* part) {
  __shared__ double s[4][NA_THREADS / 32];
  const int64_t n0 = int64_t(blockIdx.x) * NA_NODES_PER_BLOCK;
  const int64_t n1 = n0 + NA_NODES_PER_BLOCK < n_nodes ? n0 + NA_NODES_PER_BLOCK : n_nodes;
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t n = n0 + threadIdx.x; n < n1; n += NA_THREADS) {
    const double4 v = reinterpret_cast<const double4*>(x)[n];
    m[0] = na_max(m[0], fabs(v.x));
    m[1] = na_max(m[1], fabs(v.y));
    m[2] = na_max(m[2], fabs(v.z));
    m[3] = na_max(m[3], fabs(v.w));
  }
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int k = 0; k < 4; ++k) m[k] = na_max(m[k], __shfl_xor_sync(0xffffffffu, m[k], off));
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) s[k][threadIdx.x >> 5] = m[k];
  __syncthreads();
  if (threadIdx.x < 4) {
    double r = 0.0;
    for (int w = 0; w < NA_THREADS / 32; ++w) r = na_max(r, s[threadIdx.x][w]);
    part[size_t(blockIdx.x) * 4 + threadIdx.x] = r;
  }
}

__global__ void __launch_bounds__(NA_THREADS) na_reduce_kernel(int nblocks, const double* part, double* out) {
  __shared__ double s[4][NA_THREADS];
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += NA_THREADS)
#pragma unroll
    for (int k = 0; k < 4; ++k) m[k] = na_max(m[k], part[size_t(b) * 4 + k]);
#pragma unroll
  for (int k = 0; k < 4; ++k) s[k][threadIdx.x] = m[k];
  __syncthreads();
  for (int w = NA_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < 4; ++k) s[k][threadIdx.x] = na_max(s[k][threadIdx.x], s[k][threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = s[threadIdx.x][0];
}

}  // namespace

extern "C" int hg_residuals_noalloc(const double* qdot, int64_t ndof, void* cuda_stream, double out[4]) {
  if (!qdot || !out || ndof <= 0 || ndof % 4 != 0 || ndof > HG_NOALLOC_MAX_NDOF) return 1;
  if ((reinterpret_cast<uintptr_t>(qdot) & 31) != 0) return 1;
  // an error left pending by earlier work on this thread is not this call's: report it as such and
  // leave it pending for the code that caused it
  if (cudaPeekAtLastError() != cudaSuccess) return 4;
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, na_scratch) != cudaSuccess || !p) return 2;
  double* part = static_cast<double*>(p);
  double* res = part + size_t(NA_MAX_BLOCKS) * 4;
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  const int64_t n_nodes = ndof / 4;
  const int nblocks = int((n_nodes + NA_NODES_PER_BLOCK - 1) / NA_NODES_PER_BLOCK);
  na_partial_kernel<<<nblocks, NA_THREADS, 0, st>>>(qdot, n_nodes, part);
  if (cudaGetLastError() != cudaSuccess) return 3;
  na_reduce_kernel<<<1, NA_THREADS, 0, st>>>(nblocks, part, res);
  if (cudaGetLastError() != cudaSuccess) return 3;
  if (cudaMemcpyAsync(out, res, 4 * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess) return 3;
  if (cudaStreamSynchronize(st) != cudaSuccess) return 3;
  return 0;
}
