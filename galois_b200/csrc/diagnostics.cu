// Bounded-wait diagnostics: run the device waits the persistent kernels use
// with a wait that nothing will ever satisfy and a short limit, so that a
// host (or a test) can see the wait give up, the error word reach the host
// as GB_ERR_TIMEOUT and the context stay usable -- without faulting, trapping
// or hanging the GPU.  Two waits:
//   0: the software grid barrier (device_common.cuh) with one CTA that never
//      arrives;
//   1: a worklist ticket (gb_worklist.cuh) whose chunk is never published
//      while the work count says a busy warp still exists.
#include "device_common.cuh"
#include "device_graph.cuh"
#include "gb_worklist.cuh"

namespace gb {
namespace {

__global__ void missing_arrival_kernel(GridBar* bar, int* err, uint64_t limit_ns) {
  if (blockIdx.x == 0) return;  // this CTA never arrives at the barrier
  grid_barrier(bar, gridDim.x, err, ~0ull, limit_ns);
}

__global__ void unpublished_ticket_kernel(worklists::Ring r, int* err, uint64_t limit_ns) {
  __shared__ uint4 s_lq[8][64];
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    for (uint64_t i = 0; i <= r.mask; ++i) r.seq[i] = i;  // an empty ring
  }
  __syncthreads();
  __threadfence();
  const uint64_t deadline = worklists::timer_ns() + limit_ns;
  worklists::WarpQueue<64> q(s_lq[threadIdx.x >> 5], r, err, deadline);
  uint4 ent;
  bool has;
  q.next(ent, has);  // takes a ticket; work stays 1 and nothing is published
}

}  // namespace
}  // namespace gb

extern "C" int gb_probe_bounded_waits(int which, uint32_t limit_us, void* stream) {
  using namespace gb;
  clear_error();
  if (which != 0 && which != 1) GB_FAIL(GB_ERR_ARG, "gb_probe_bounded_waits: which must be 0 or 1");
  if (limit_us == 0 || limit_us > 2000000) GB_FAIL(GB_ERR_ARG, "gb_probe_bounded_waits: limit must be 1 us .. 2 s");
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0, sms = 0;
  GB_CUDA(cudaGetDevice(&dev));
  GB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const unsigned long long cap = 1024;
  const size_t bytes = 256 + worklists::ring_bytes(cap);
  char* mem = nullptr;
  GB_CUDA(cudaMalloc(&mem, bytes));
  GB_CUDA(cudaMemsetAsync(mem, 0, bytes, s));
  GridBar* bar = reinterpret_cast<GridBar*>(mem);
  int* err = reinterpret_cast<int*>(mem + 64);
  worklists::Ring ring = worklists::ring_layout(mem + 256, cap);
  const uint64_t limit_ns = (uint64_t)limit_us * 1000ull;
  cudaError_t e = cudaSuccess;
  if (which == 0) {
    // every CTA resident at once (cooperative launch), one per SM
    void* args[] = {&bar, &err, const_cast<uint64_t*>(&limit_ns)};
    e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&missing_arrival_kernel), sms, 64, args, 0, s);
  } else {
    const int one = 1;  // a busy warp that never finishes: the count never reaches zero
    e = cudaMemcpyAsync(&ring.rc->work, &one, sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) unpublished_ticket_kernel<<<1, 256, 0, s>>>(ring, err, limit_ns);
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(mem);
  if (e != cudaSuccess) return cuda_fail(e, "gb_probe_bounded_waits");
  if (herr == kDevTimeout) GB_FAIL(GB_ERR_TIMEOUT, "gb_probe_bounded_waits: the wait gave up after %u us as designed",
                                   limit_us);
  GB_FAIL(GB_ERR_CUDA, "gb_probe_bounded_waits: the wait ended without its timeout (device error word %d)", herr);
}
