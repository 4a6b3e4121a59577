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

}  // namespace

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
