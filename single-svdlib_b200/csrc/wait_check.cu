// svdb_wait_selftest: makes the library's two bounded device waits run out on
// purpose and reports what they returned, so that the timeout path is tested
// without hanging or faulting a GPU.
//
//   which = 0: the grid barrier of the cooperative Lanczos block (grid_sync),
//              in a one-block grid that expects two arrivals: the second
//              never comes, so the generation counter is never advanced.
//   which = 1: the mbarrier wait of the tensor-core Gram (mbar_wait_bounded),
//              on a barrier initialised for one arrival that nothing makes.
//
// Each kernel gives up after limit_ns of %globaltimer, records
// SVDB_ERR_TIMEOUT in device memory and returns; the host reads the status
// and returns it.  Nothing else is in flight, no tensor memory is held, and
// the context stays usable.
#include "device_common.cuh"
#include "svdb_internal.h"

namespace svdb {

__global__ void k_wait_grid_selftest(GridBarrier* bar) {
    // the first block to arrive waits for one more block than the grid has
    grid_sync(bar, gridDim.x + 1);
}

__global__ void k_wait_mbar_selftest(unsigned long long limit_ns, int* status) {
    __shared__ __align__(8) uint64_t bar;
    const uint32_t addr = (uint32_t)__cvta_generic_to_shared(&bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(addr) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) *status = mbar_wait_bounded(addr, 0, limit_ns) ? SVDB_OK : SVDB_ERR_TIMEOUT;
}

}  // namespace svdb

extern "C" int svdb_wait_selftest(int which, uint64_t limit_ns) {
    using namespace svdb;
    try {
        if (which != 0 && which != 1) throw Error(SVDB_ERR_ARG, "svdb_wait_selftest: which must be 0 or 1");
        if (limit_ns == 0 || limit_ns > 2000000000ull)
            throw Error(SVDB_ERR_ARG, "svdb_wait_selftest: limit_ns must be in 1 .. 2e9");
        cudaStream_t s = nullptr;
        SVDB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        int status = -1;
        try {
            if (which == 0) {
                DevBuf<GridBarrier> bar(1, s);
                GridBarrier b0;
                std::memset(&b0, 0, sizeof b0);
                b0.limit_ns = limit_ns;
                SVDB_CUDA(cudaMemcpyAsync(bar.p, &b0, sizeof b0, cudaMemcpyHostToDevice, s));
                k_wait_grid_selftest<<<1, 32, 0, s>>>(bar.p);
                SVDB_CHECK_LAUNCH();
                SVDB_CUDA(cudaMemcpyAsync(&b0, bar.p, sizeof b0, cudaMemcpyDeviceToHost, s));
                SVDB_CUDA(cudaStreamSynchronize(s));
                status = b0.err;
            } else {
                DevBuf<int> st(1, s);
                SVDB_CUDA(cudaMemsetAsync(st.p, 0xff, sizeof(int), s));
                k_wait_mbar_selftest<<<1, 32, 0, s>>>(limit_ns, st.p);
                SVDB_CHECK_LAUNCH();
                SVDB_CUDA(cudaMemcpyAsync(&status, st.p, sizeof(int), cudaMemcpyDeviceToHost, s));
                SVDB_CUDA(cudaStreamSynchronize(s));
            }
        } catch (...) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
            throw;
        }
        SVDB_CUDA(cudaStreamDestroy(s));
        if (status != SVDB_OK && status != SVDB_ERR_TIMEOUT)
            throw Error(SVDB_ERR_CUDA, "svdb_wait_selftest: the kernel left no status");
        if (status == SVDB_ERR_TIMEOUT) set_last_error("svdb_wait_selftest: the wait gave up after its limit");
        return status;
    } catch (Error& e) {
        set_last_error(e.what());
        return e.code;
    }
}
