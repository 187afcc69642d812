// svdb_opb_device_noalloc: y = A^T (A x) (or A (A^T x)) on device buffers
// without allocating any memory.
//
// Who needs it: callers that cannot call cudaMalloc / cudaFree at the point
// where they apply the operator -- a host application whose own allocator has
// already reserved all of the GPU's memory, or a latency-critical loop in which
// an allocation (and the device-wide synchronisation cudaFree implies) is not
// acceptable.  They pass x and y in their own device memory; the intermediate
// vector A x lives in a fixed array compiled into this library.
//
// The array is a file-scope __device__ variable (kScratchDoubles doubles =
// 8 MiB).  This file is its own CUDA module, and CUDA loads modules lazily by
// default, so the array is placed in device memory when its address is first
// taken.  Host code may not use the variable's name as a device address; the
// address is taken with cudaGetSymbolAddress once per device, with that
// device current, by noalloc_reserve(), which every matrix handle's creation
// calls.  So the 8 MiB are reserved on a GPU when the first matrix handle is
// created there (an allocating call anyway), and held until the process
// exits; a call of svdb_opb_device_noalloc itself never loads or allocates
// anything.  The handle's device must be current when it is called: the
// scratch address is looked up for the current device.
//
// All calls share the one array: calls whose work overlaps on the GPU (on
// different streams, or from different host threads) race on it and must be
// serialised by the caller.  The array keeps the previous call's contents; the
// first sparse product overwrites every entry that the second one reads, so
// nothing has to be cleared.
#include <mutex>

#include "svdb_internal.h"

namespace svdb {

// Largest intermediate length accepted: rows of A (or columns when transposed).
constexpr uint64_t kScratchDoubles = uint64_t(1) << 20;

static __device__ __align__(256) double g_opb_scratch[kScratchDoubles];

static std::mutex g_scratch_mu;
static void* g_scratch_addr[64];  // per device ordinal

static double* scratch_for_current_device() {
    int dev = 0;
    SVDB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Error(SVDB_ERR_UNSUPPORTED, "device ordinal above 63");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_opb_scratch);
        if (e != cudaSuccess || !p)
            throw Error(SVDB_ERR_CUDA, std::string("cudaGetSymbolAddress(g_opb_scratch): ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = p;
    }
    return static_cast<double*>(g_scratch_addr[dev]);
}

void noalloc_reserve() { (void)scratch_for_current_device(); }

}  // namespace svdb

extern "C" int svdb_opb_device_noalloc(const svdb_matrix* a, const double* d_x, double* d_y, int transposed,
                                       void* stream) {
    using namespace svdb;
    try {
        if (!a || !d_x || !d_y) throw Error(SVDB_ERR_ARG, "null argument");
        const DevCompressed& o1 = transposed ? csc_of(a) : csr_of(a);
        const DevCompressed& o2 = transposed ? csr_of(a) : csc_of(a);
        if ((uint64_t)o1.nmajor > kScratchDoubles)
            throw Error(SVDB_ERR_UNSUPPORTED,
                        "svdb_opb_device_noalloc: intermediate vector of " + std::to_string(o1.nmajor) +
                            " doubles exceeds the fixed scratch of " + std::to_string(kScratchDoubles) +
                            " doubles; use svdb_opb or the allocating entry points");
        int cur = -1;
        SVDB_CUDA(cudaGetDevice(&cur));
        if (cur != a->device) throw Error(SVDB_ERR_ARG, "the matrix lives on another device than the current one");
        double* temp = scratch_for_current_device();
        cudaStream_t s = stream ? (cudaStream_t)stream : a->stream;
        spmv(o1, false, d_x, temp, s, false);  // temp = A x  (every entry written); gather kernel, no plan
        spmv(o2, false, temp, d_y, s, false);  // y = A^T temp
        return SVDB_OK;
    } catch (Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (std::exception& e) {
        set_last_error(e.what());
        return SVDB_ERR_ARG;
    }
}
