// Evaluate entry point that allocates no device memory.
//
// Who needs it: applications that call the solver from code which must not
// allocate device memory once it is running -- for example a simulation
// engine whose own caching allocator already owns the GPU's memory pool (a
// further cudaMalloc can fail or fragment that pool), or a time-stepping loop
// that cannot afford the implicit device-wide synchronisation cudaMalloc and
// cudaFree perform.  Such callers build the tree during their set-up phase
// (pdmk_create_double allocates the tree's own buffers there) and then call
// pdmk_evaluate_device_noalloc_double in the loop with charges and potentials
// in device buffers they own.
//
// The only temporary memory the evaluate needs beyond the tree's own buffers
// is the scratch of the separable plane-wave / Chebyshev transforms.  Here it
// lives in one file-scope __device__ array of kNoAllocScratchBytes (32 MiB),
// which every GPU that loads this library holds until the process exits.  The
// transforms run level by level in chunks of boxes that fit in it (the same
// pass as the regular evaluate, with a smaller scratch); a tree whose single
// box needs more scratch than the array holds is rejected with an error.
//
// Rules for callers:
//   * The array belongs to this file's device code, which CUDA loads onto a
//     device lazily (CUDA_MODULE_LOADING=LAZY is the default): the 32 MiB are
//     reserved on a device when its address is first looked up.  Creating a
//     double tree (pdmk_create_double) does that look-up, with the tree's
//     device current, so the reservation happens during the caller's set-up,
//     together with the tree's own buffers, before the caller's allocator
//     takes the memory pool.  If that look-up fails at creation (the device
//     has no 32 MiB left), the first no-allocation call repeats it and fails
//     with -2 if it still cannot reserve the array.  Either way the first
//     call on a device should come before any CUDA stream capture.
//   * All calls share the one array and it keeps the last call's contents
//     (every value is written before it is read, so nothing needs clearing).
//     Calls that overlap on the GPU -- two trees evaluated concurrently on
//     different streams of the same device -- race on it and must be
//     serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <stdexcept>
#include <string>

#include "device_tree.hpp"

namespace pdmkb {

namespace {

constexpr size_t kNoAllocScratchBytes = 32u << 20;
constexpr int64_t kNoAllocScratchElems = (int64_t)(kNoAllocScratchBytes / sizeof(dev::cd));

static __device__ __align__(256) dev::cd g_noalloc_scratch[kNoAllocScratchElems];

std::mutex g_addr_mutex;
void* g_addr[256] = {};  // device address of g_noalloc_scratch per device ordinal

dev::cd* scratch_address(int device) {
    if (device < 0 || device >= 256) throw std::runtime_error("CUDA error: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[device]) {
        int cur = -1;
        PDMK_CUDA_CHECK(cudaGetDevice(&cur));
        if (cur != device) PDMK_CUDA_CHECK(cudaSetDevice(device));
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (cur != device) cudaSetDevice(cur);
        if (e != cudaSuccess || !p)
            throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(e) +
                                     " while looking up the no-allocation scratch array");
        g_addr[device] = p;
    }
    return static_cast<dev::cd*>(g_addr[device]);
}

}  // namespace

void noalloc_reserve(int device) {
    try {
        scratch_address(device);
    } catch (const std::exception&) {
        cudaGetLastError();  // not sticky; the no-allocation call retries and reports it
    }
}

void DeviceTree::evaluate_device_noalloc(const double* q, double* pot) {
    require_periodic("evaluate");
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    last_was_multi_ = false;
    if (!proxy_up_)
        throw std::invalid_argument("the no-allocation evaluate needs a tree built with its FP64 buffers (double tree)");
    dev::cd* scratch = scratch_address(device_);
    const int64_t need = fp64_need_max();
    if (need > kNoAllocScratchElems)
        throw std::invalid_argument("tree needs " + std::to_string(need * sizeof(dev::cd)) +
                                    " bytes of transform scratch per box; the no-allocation evaluate provides " +
                                    std::to_string(kNoAllocScratchBytes));
    cudaStream_t s = stream_;
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[0], s));
    PDMK_CUDA_CHECK(cudaMemsetAsync(pot_sorted_, 0, sizeof(double) * n_, s));
    run_fp64_tree(q, scratch, kNoAllocScratchElems, s);
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[1], s));
    dev::launch_near(near_, s);
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[2], s));
    dev::launch_nufft_gather_q(trg_perm_, q, q_sorted_, n_, s);
    PDMK_CUDA_CHECK(cudaMemsetAsync(grid_, 0, sizeof(double) * n_grid_, s));
    dev::launch_spread(nufft_, nufft_max_jk_, nufft_max_ex_, s);
    if (cufftExecD2Z(plan_fwd_, grid_, reinterpret_cast<cufftDoubleComplex*>(spec_)) != CUFFT_SUCCESS)
        throw std::runtime_error("cuFFT error in the forward far-field transform");
    dev::launch_multiply(spec_, mult_, n_spec_, s);
    if (cufftExecZ2D(plan_inv_, reinterpret_cast<cufftDoubleComplex*>(spec_), grid_) != CUFFT_SUCCESS)
        throw std::runtime_error("cuFFT error in the inverse far-field transform");
    dev::launch_interp(nufft_, s);
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[3], s));
    dev::launch_finalize(pot_sorted_, far_sorted_, trg_, trg_perm_, q, pot, n_, s);
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[4], s));
    PDMK_CUDA_CHECK(cudaGetLastError());
    PDMK_CUDA_CHECK(cudaStreamSynchronize(s));
}

}  // namespace pdmkb
