// Allocation-free variant of the batched triangular solve.
//
// Who needs it: callers that must not allocate device memory at solve time --
// a host simulator that runs its Newton loop against a fixed memory budget,
// code running inside another framework's memory pool or allocator (which
// forbids raw cudaMalloc/cudaFree), or latency-critical loops where an
// allocation's implicit device synchronisation is unacceptable.  The regular
// nsg_batch_solve needs an n-double sweep workspace per instance, which the
// batch allocates with cudaMalloc when it is created; this variant takes that
// workspace from a fixed array compiled into the library instead, so the call
// itself allocates nothing.
//
// The array, g_static_sweep_scratch, holds kStaticScratchDoubles doubles
// (8 MiB) and lives on every GPU that loads the library until the process
// exits.  Host code cannot use the array's name as a device address: it asks
// the runtime for the address once per device (cudaGetSymbolAddress, with
// that device current) and passes it to the kernel.
#include "capi_internal.hpp"
#include "kernels/lu_cta.cuh"

#include <mutex>

namespace {

constexpr long long kStaticScratchDoubles = NSG_STATIC_SCRATCH_DOUBLES;

static __device__ __align__(256) double g_static_sweep_scratch[kStaticScratchDoubles];

// Same sweep as solve_kernel (SparseMatrix::solve, src/solver/solve.cpp:6-47),
// with the workspace taken from the static array's device address.
__global__ void __launch_bounds__(256)
solve_static_scratch_kernel(const nsg::PlanDesc* __restrict__ plans,
                            const int32_t* __restrict__ pool,
                            const nsg::InstDesc* __restrict__ insts,
                            const double* __restrict__ LU, double* __restrict__ X,
                            double* __restrict__ scratch) {
    const nsg::InstDesc inst = insts[blockIdx.x];
    nsg::cta_solve(plans[inst.plan], pool, LU + inst.lu_off, X + inst.x_off,
                   scratch + inst.w_off);
}

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of the static array on device `dev` (which is current),
// looked up on the first call for that device and kept for the life of the
// process.  A cudaDeviceReset after that first call reloads the module, so
// the kept address would be stale: resetting a device that this entry point
// has used is not supported.
cudaError_t scratch_address(int dev, double** out) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_sweep_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

}  // namespace

using namespace nsg_internal;

extern "C" {

int nsg_batch_solve_static_scratch(nsg_batch* b, double* d_x, void* stream) {
    if (!b || !d_x) return fail(NSG_ERR_INVALID, "nsg_batch_solve_static_scratch: null argument");
    const long long need = b->x_off[b->count];
    if (need > kStaticScratchDoubles)
        return fail(NSG_ERR_INVALID,
                    "nsg_batch_solve_static_scratch: the batch has " + std::to_string(need) +
                        " unknowns in total; the static workspace holds at most " +
                        std::to_string(kStaticScratchDoubles));
    // The plans, factors and workspace live on the batch's device; the static
    // array used must be that device's copy.
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail("nsg_batch_solve_static_scratch: current device", e);
    if (dev != b->device)
        return fail(NSG_ERR_INVALID,
                    "nsg_batch_solve_static_scratch: the current device (" + std::to_string(dev) +
                        ") is not the batch's device (" + std::to_string(b->device) + ")");
    double* scratch = nullptr;
    e = scratch_address(dev, &scratch);
    if (e != cudaSuccess) return cuda_fail("nsg_batch_solve_static_scratch: symbol address", e);
    // The sweep writes every workspace entry before reading it, so nothing in
    // the array has to be cleared between calls.
    solve_static_scratch_kernel<<<b->count, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        b->d_plans, b->d_pool, b->d_insts, b->d_lu, d_x, scratch);
    e = cudaGetLastError();
    return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_batch_solve_static_scratch", e);
}

}  // extern "C"
