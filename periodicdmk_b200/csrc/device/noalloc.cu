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
// transforms are run in chunks of boxes that fit in it; a tree whose single
// box needs more scratch than the array holds is rejected with an error.
//
// Rules for callers:
//   * The first call on a device looks up the array's device address (set-up
//     done once per device, with that device current).  Make that first call
//     before any CUDA stream capture.
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

#include "../api/impl.hpp"
#include "device_tree.hpp"
#include "pdmk/pdmk_capi.h"

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

void DeviceTree::evaluate_device_noalloc(const double* q, double* pot) {
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    if (!proxy_up_)
        throw std::invalid_argument("the no-allocation evaluate needs a tree built with its FP64 buffers (double tree)");
    dev::cd* scratch = scratch_address(device_);
    const int64_t cap = kNoAllocScratchElems;
    const int p = p_, n = npw_, n2 = npw2_, M = M_;
    const int64_t ncoef = (int64_t)p * p * p;
    const int64_t ncoef_c = (ncoef + 1) / 2;  // a real (p,p,p) tensor in complex-sized slots
    // per-box scratch of each phase (complex elements)
    const int64_t need_c2p = 2 * ncoef_c;
    const int64_t need_pw = (int64_t)p * p * n + (int64_t)p * n * n;
    const int64_t need_eval = (int64_t)M + (int64_t)n * n2 * p + (int64_t)n2 * p * p;
    const int64_t need = std::max(need_c2p, std::max(need_pw, need_eval));
    if (need > cap)
        throw std::invalid_argument("tree needs " + std::to_string(need * sizeof(dev::cd)) +
                                    " bytes of transform scratch per box; the no-allocation evaluate provides " +
                                    std::to_string(kNoAllocScratchBytes));
    auto chunk = [&](int64_t per) { return (int)std::max<int64_t>(1, cap / per); };
    cudaStream_t s = stream_;
    PDMK_CUDA_CHECK(cudaEventRecord(ev_[0], s));
    PDMK_CUDA_CHECK(cudaMemsetAsync(pot_sorted_, 0, sizeof(double) * n_, s));
    PDMK_CUDA_CHECK(cudaMemsetAsync(proxy_up_, 0, sizeof(double) * std::max<int64_t>(n_up_ * ncoef, 1), s));
    PDMK_CUDA_CHECK(cudaMemsetAsync(proxy_down_, 0, sizeof(double) * std::max<int64_t>(n_down_ * ncoef, 1), s));
    dev::launch_gather(src_, src_charge_idx_, q, n_all_, s);
    dev::launch_c2proxy(c2x_, p, s);
    // upward child -> parent, in chunks of parents
    for (const auto& g : c2p_groups_) {
        const double* mx = c2p_ + (int64_t)g.child * 3 * p * p;
        const int C = chunk(need_c2p);
        double* s1 = reinterpret_cast<double*>(scratch);
        double* s2 = reinterpret_cast<double*>(scratch + (int64_t)C * ncoef_c);
        for (int c0 = 0; c0 < g.n; c0 += C) {
            dev::ContractArgs a{};
            a.n_entries = std::min(C, g.n - c0);
            a.in = proxy_up_; a.in_off = g.in_off + c0; a.out = s1; a.out_stride = ncoef;
            a.mat = mx; a.ni = p; a.na = p; a.R = p * p; a.mode = dev::kStore;
            dev::launch_contract(a, dev::kRRR, s);
            a.in = s1; a.in_off = nullptr; a.in_stride = ncoef; a.out = s2; a.mat = mx + p * p;
            dev::launch_contract(a, dev::kRRR, s);
            a.in = s2; a.out = proxy_up_; a.out_off = g.out_off + c0; a.mat = mx + 2 * p * p; a.mode = dev::kAdd;
            dev::launch_contract(a, dev::kRRR, s);
        }
    }
    // outgoing plane waves
    for (const auto& g : pw_groups_) {
        const auto& L = lev_[g.level];
        const int C = chunk(need_pw);
        dev::cd* s1 = scratch;
        dev::cd* s2 = scratch + (int64_t)C * p * p * n;
        for (int c0 = 0; c0 < g.n; c0 += C) {
            dev::ContractArgs a{};
            a.n_entries = std::min(C, g.n - c0);
            a.in = proxy_up_; a.in_off = g.in_off + c0; a.out = s1; a.out_stride = (int64_t)p * p * n;
            a.mat = L.poly2pw; a.ni = p; a.na = n; a.R = p * p; a.mode = dev::kStore;
            dev::launch_contract(a, dev::kRCC, s);
            a.in = s1; a.in_off = nullptr; a.in_stride = (int64_t)p * p * n; a.out = s2;
            a.out_stride = (int64_t)p * n * n; a.R = p * n;
            dev::launch_contract(a, dev::kCCC, s);
            a.in = s2; a.in_stride = (int64_t)p * n * n; a.out = pw_out_; a.out_off = g.out_off + c0;
            a.mat = L.poly2pw_half; a.na = n2; a.R = n * n;
            dev::launch_contract(a, dev::kCCC, s);
        }
    }
    // downward per level: shift -> pw2proxy in chunks, then parent -> child
    for (const auto& E : eval_levels_) {
        const auto& L = lev_[E.level];
        const int C = chunk(need_eval);
        dev::cd* pin = scratch;
        dev::cd* s1 = scratch + (int64_t)C * M;
        dev::cd* s2 = s1 + (int64_t)C * n * n2 * p;
        for (int c0 = 0; c0 < E.n; c0 += C) {
            const int ne = std::min(C, E.n - c0);
            dev::ShiftArgs sa{pw_out_, L.shift, pin, M, ne, E.term_start + c0, E.term_slot, E.term_stencil};
            dev::launch_shift(sa, s);
            dev::ContractArgs a{};
            a.n_entries = ne;
            a.in = pin; a.in_stride = M; a.out = s1; a.out_stride = (int64_t)n * n2 * p;
            a.mat = L.pw2polyT; a.ni = n; a.na = p; a.R = n * n2; a.mode = dev::kStore;
            dev::launch_contract(a, dev::kCCC, s);
            a.in = s1; a.in_stride = (int64_t)n * n2 * p; a.out = s2; a.out_stride = (int64_t)n2 * p * p;
            a.R = n2 * p;
            dev::launch_contract(a, dev::kCCC, s);
            a.in = s2; a.in_stride = (int64_t)n2 * p * p; a.out = proxy_down_; a.out_off = E.down_off + c0;
            a.mat = L.pw2polyTw; a.ni = n2; a.R = p * p; a.mode = dev::kAddRealScaled; a.scale = 2.0;
            dev::launch_contract(a, dev::kCCR, s);
        }
        if (E.n_p2c) {
            const int Cp = chunk(need_c2p);
            double* t1 = reinterpret_cast<double*>(scratch);
            double* t2 = reinterpret_cast<double*>(scratch + (int64_t)Cp * ncoef_c);
            for (int c0 = 0; c0 < E.n_p2c; c0 += Cp) {
                dev::ContractArgs b{};
                b.n_entries = std::min(Cp, E.n_p2c - c0);
                b.in = proxy_down_; b.in_off = E.p2c_in + c0; b.out = t1; b.out_stride = ncoef;
                b.mat = p2c_; b.mat_off = E.p2c_mat + c0; b.ni = p; b.na = p; b.R = p * p; b.mode = dev::kStore;
                dev::launch_contract(b, dev::kRRR, s);
                b.in = t1; b.in_off = nullptr; b.in_stride = ncoef; b.out = t2; b.mat = p2c_ + p * p;
                dev::launch_contract(b, dev::kRRR, s);
                b.in = t2; b.out = proxy_down_; b.out_off = E.p2c_out + c0; b.mat = p2c_ + 2 * p * p; b.mode = dev::kAdd;
                dev::launch_contract(b, dev::kRRR, s);
            }
        }
    }
    dev::launch_eval(eval_, p, s);
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

extern "C" int pdmk_evaluate_device_noalloc_double(void* h, const double* charges_dev, double* pot_dev) {
    if (!h) {
        std::fprintf(stderr, "pdmk_evaluate_device_noalloc_double: null handle\n");
        return -1;
    }
    try {
        if (!charges_dev || !pot_dev) throw std::invalid_argument("null device pointer");
        auto* t = static_cast<pdmk::PeriodicDMKTreeT<double, 3>*>(h);
        t->impl()->dev->evaluate_device_noalloc(charges_dev, pot_dev);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "pdmk_evaluate_device_noalloc_double: %s\n", e.what());
        const std::string m = e.what();
        return (m.rfind("CUDA error", 0) == 0 || m.rfind("cuFFT error", 0) == 0) ? -2 : -1;
    }
}
