// The bounded-wait failure path of the TMA-fed kernels, run on purpose (qpd_probe_wait_timeout).
//
// Every kernel that waits on an mbarrier for its tile loads gives up after a bounded number of polls,
// records QPD_DEVERR_TIMEOUT in the context's device status word and returns, so a load that never
// lands ends in an error the host reads instead of a hung GPU.  This kernel takes that path with a
// small bound: it arms a barrier for 16 bytes that no copy ever delivers (nothing is loaded, nothing is
// in flight when it exits) and waits on it.
#include "qpd_tma.cuh"

namespace qpd {
namespace {

__global__ void wait_probe(int* status, long long polls) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_expect_tx(&bar, 16);  // the one arrival, expecting bytes that never come
    __syncthreads();
    mbar_wait(&bar, 0, status, polls);
}

}  // namespace

cudaError_t launch_wait_probe(int* status, long long polls, cudaStream_t st) {
    wait_probe<<<1, 32, 0, st>>>(status, polls);
    return cudaGetLastError();
}

}  // namespace qpd
