// Failure detection without a GPU fault: a grid barrier that one CTA never reaches.  Every other
// CTA's wait (the bounded spin of grid_barrier, the barrier of the persistent CG / PCG kernels)
// runs out after `limit` polls, records ERR_TIMEOUT in the error word and returns; the host
// reads the word and the context stays usable.  No trap, assert, bad address or endless loop.
#include "spx_internal.cuh"

namespace spx {

namespace {

__global__ void k_barrier_probe(unsigned int* __restrict__ bar, int* __restrict__ err, int absent, long long limit,
                                unsigned int* __restrict__ timed_out) {
  if (static_cast<int>(blockIdx.x) == absent) return;  // this CTA never arrives
  if (!grid_barrier(bar, bar + 1, gridDim.x, err, limit) && threadIdx.x == 0) atomicAdd(timed_out, 1u);
}

// nbar grid barriers in a row (the cost of one phase boundary of the persistent solvers)
__global__ void k_barrier_chain(unsigned int* __restrict__ bar, int* __restrict__ err, int nbar) {
  for (int i = 0; i < nbar; ++i)
    if (!grid_barrier(bar, bar + 1, gridDim.x, err)) return;
}

}  // namespace

// average time of one grid barrier over nbar in a row on nblocks CTAs of `threads` threads
// (a cooperative launch, so all CTAs are resident); microseconds
double barrier_time_us(int nblocks, int threads, int nbar) {
  SPX_CHECK(nblocks >= 1 && nblocks <= num_sms(), "nblocks must be in [1, number of SMs]");
  SPX_CHECK(threads >= 32 && threads <= 1024 && threads % 32 == 0, "threads must be a multiple of 32 in [32, 1024]");
  SPX_CHECK(nbar >= 1 && nbar <= (1 << 20), "nbar must be in [1, 2^20]");
  DevBuf<unsigned int> bar(2);
  DevBuf<int> err(1);
  cudaEvent_t e0, e1;
  SPX_CUDA(cudaEventCreate(&e0));
  SPX_CUDA(cudaEventCreate(&e1));
  float ms = 0.0f;
  for (int rep = 0; rep < 2; ++rep) {  // the first launch warms up
    bar.zero();
    err.zero();
    void* args[] = {&bar.p, &err.p, &nbar};
    SPX_CUDA(cudaEventRecord(e0));
    SPX_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_barrier_chain), dim3(nblocks), dim3(threads), args,
                                         0, nullptr));
    SPX_CUDA(cudaEventRecord(e1));
    SPX_CUDA(cudaEventSynchronize(e1));
    SPX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int h_err = 0;
  SPX_CUDA(cudaMemcpy(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost));
  SPX_CHECK(h_err == 0, "a barrier wait ran out");
  return 1000.0 * ms / nbar;
}

// runs the probe on nblocks CTAs (at most one per SM, so that all are resident); returns the
// recorded error code and the number of CTAs whose wait ran out
int barrier_timeout_probe(int nblocks, long long limit, int* timed_out_ctas) {
  SPX_CHECK(nblocks >= 2 && nblocks <= num_sms(), "nblocks must be in [2, number of SMs]");
  SPX_CHECK(limit >= 1 && limit <= (1ll << 24), "limit must be in [1, 2^24] polls");
  DevBuf<unsigned int> bar(2), cnt(1);
  DevBuf<int> err(1);
  bar.zero();
  cnt.zero();
  err.zero();
  k_barrier_probe<<<nblocks, 128>>>(bar.p, err.p, nblocks - 1, limit, cnt.p);
  SPX_LAUNCH_CHECK();
  SPX_CUDA(cudaDeviceSynchronize());
  int h_err = 0;
  unsigned int h_cnt = 0;
  SPX_CUDA(cudaMemcpy(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost));
  SPX_CUDA(cudaMemcpy(&h_cnt, cnt.p, sizeof(unsigned int), cudaMemcpyDeviceToHost));
  *timed_out_ctas = static_cast<int>(h_cnt);
  return h_err;
}

}  // namespace spx
