// Batch of independent periodic systems (the many-systems form of the
// reference's build-once / evaluate-many API, cpp/src/periodic_dmk.cpp:41-186,
// one PeriodicDMKTreeT per system).
//
// Construction: the host plans (tree, lists, tables) of all systems are built
// on all host threads, then uploaded one by one.  Evaluate: one host->device
// copy of all charges, every system's evaluate enqueued on its own stream
// after that copy (replayed from a CUDA graph from the second evaluate on), one
// device->host copy of all potentials after every system has finished.
// Pageable host buffers pass through pinned staging buffers, filled and
// drained by up to 8 persistent host threads (a pageable cudaMemcpy moves
// 3-10 GB/s); page-locked ones are copied directly.  Both transfers run in
// about 8 chunks of whole systems: a chunk's systems start as soon as its
// charges are on the device, and a chunk of potentials is copied out of the
// staging while the later chunks are still in flight.
// Float trees (one charge vector per system) leave their near field and final
// gather out of the per-system sequences: after all systems' other stages one
// persistent kernel pulls (system, leaf) items from a device queue, largest
// first, and writes every system's potentials (batch_near.cu).  Its targets per
// thread are chosen at the first evaluate by timing the candidates (an
// autotuner whose choice is cached per batch shape for the process).
#include "batch.hpp"

#include "../device/tree_build.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <exception>
#include <map>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <thread>
#include <tuple>

#include "../host/plan.hpp"

namespace pdmkb {

TreeBatch::TreeBatch(int nsys, const double* cells, const int* Ns, const double* positions, int n_digits,
                     int n_per_leaf, int nz, bool single)
    : single_(single) {
    if (nsys <= 0) throw std::invalid_argument("nsys must be positive");
    if (!cells || !Ns || !positions) throw std::invalid_argument("null cells, Ns or positions");
    off_.assign(nsys + 1, 0);
    for (int i = 0; i < nsys; ++i) {
        if (Ns[i] <= 0) throw std::invalid_argument("every system needs at least one point");
        off_[i + 1] = off_[i] + Ns[i];
    }
    PDMK_CUDA_CHECK(cudaGetDevice(&device_));
    // plans in parallel on host threads (the point steps of the larger
    // systems on the GPU)
    std::vector<std::unique_ptr<Plan>> plans(nsys);
    std::atomic<int> next{0};
    std::exception_ptr first_error;
    std::mutex err_mu;
    auto work = [&]() {
        cudaSetDevice(device_);
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= nsys) return;
            try {
                const double* c = cells + 9 * (size_t)i;
                const double* x = positions + 3 * off_[i];
                plans[i] = std::make_unique<Plan>(tree_build_on_device(Ns[i], 20000)
                                                      ? build_plan_device(c, Ns[i], x, n_digits, n_per_leaf, nz)
                                                      : build_plan(c, Ns[i], x, n_digits, n_per_leaf, nz));
            } catch (...) {
                std::lock_guard<std::mutex> g(err_mu);
                if (!first_error) first_error = std::current_exception();
            }
        }
    };
    const int nthr = std::max(1, std::min<int>(nsys, (int)std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (int t = 0; t < nthr; ++t) pool.emplace_back(work);
    for (auto& t : pool) t.join();
    if (first_error) std::rethrow_exception(first_error);
    try {
        // device trees (uploads, cuFFT plans) on host threads too: each system's
        // upload is a sequence of small allocations and copies
        trees_.resize(nsys);
        next = 0;
        auto upload = [&]() {
            cudaSetDevice(device_);
            for (;;) {
                const int i = next.fetch_add(1);
                if (i >= nsys) return;
                try {
                    trees_[i] = std::make_unique<DeviceTree>(*plans[i], device_, /*fp64_working_set=*/!single_);
                    plans[i].reset();  // the device tree keeps what it needs
                } catch (...) {
                    std::lock_guard<std::mutex> g(err_mu);
                    if (!first_error) first_error = std::current_exception();
                }
            }
        };
        std::vector<std::thread> up;
        for (int t = 0; t < nthr; ++t) up.emplace_back(upload);
        for (auto& t : up) t.join();
        if (first_error) std::rethrow_exception(first_error);
        PDMK_CUDA_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        profile_ = std::getenv("PDMK_BATCH_PROFILE") != nullptr;
        if (profile_)
            for (auto& e : prof_) PDMK_CUDA_CHECK(cudaEventCreate(&e));
        done_.assign(nsys, nullptr);
        for (auto& e : done_) PDMK_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        // transfer chunks: about 8 of equal points, at system boundaries
        {
            const int64_t tot = off_.back(), want = std::max<int64_t>(1, (tot + 7) / 8);
            chunk_sys_.assign(1, 0);
            for (int i = 1; i <= nsys; ++i)
                if (i == nsys || off_[i] - off_[chunk_sys_.back()] >= want) chunk_sys_.push_back(i);
            const size_t nch = chunk_sys_.size() - 1;
            ev_up_.assign(nch, nullptr);
            ev_dn_.assign(nch, nullptr);
            for (auto& e : ev_up_) PDMK_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            for (auto& e : ev_dn_) PDMK_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        const size_t n = (size_t)total_points();
        PDMK_CUDA_CHECK(cudaMalloc(&q_dev_, sizeof(double) * n));
        PDMK_CUDA_CHECK(cudaMalloc(&pot_dev_, sizeof(double) * n));
        PDMK_CUDA_CHECK(cudaMalloc(&potf_dev_, sizeof(float) * n));
        PDMK_CUDA_CHECK(cudaMallocHost(&err_host_, sizeof(int) * nsys));
        PDMK_CUDA_CHECK(cudaMallocHost(&q_pin_, sizeof(double) * n));
        PDMK_CUDA_CHECK(cudaMallocHost(&p_pin_, sizeof(double) * n));
        graphs_.assign(nsys, nullptr);
        if (single_) {
            for (auto& t : trees_) t->defer_near_ = true;
            // queue items: every system's near-field leaves, largest work first
            std::vector<std::tuple<int64_t, int, int>> items;
            for (int i = 0; i < nsys; ++i) {
                const auto& cost = trees_[i]->near_leaf_cost();
                for (int e = 0; e < trees_[i]->near_leaves(); ++e) items.emplace_back(-cost[e], i, e);
            }
            std::stable_sort(items.begin(), items.end());
            std::vector<int2> it(items.size());
            for (size_t k = 0; k < items.size(); ++k) it[k] = make_int2(std::get<1>(items[k]), std::get<2>(items[k]));
            n_items_ = (int)it.size();
            PDMK_CUDA_CHECK(cudaMalloc(&items_dev_, sizeof(int2) * std::max<size_t>(it.size(), 1)));
            PDMK_CUDA_CHECK(cudaMemcpy(items_dev_, it.data(), sizeof(int2) * it.size(), cudaMemcpyHostToDevice));
            PDMK_CUDA_CHECK(cudaMalloc(&sys_dev_, sizeof(dev::NearLeafSys) * nsys));
            // leaf-evaluation items: every system's evaluated leaves, most targets first
            std::vector<std::tuple<int, int, int>> ev;
            for (int i = 0; i < nsys; ++i) {
                const auto& nt = trees_[i]->eval_leaf_targets();
                for (int e = 0; e < trees_[i]->eval_leaves(); ++e) ev.emplace_back(-nt[e], i, e);
            }
            std::stable_sort(ev.begin(), ev.end());
            std::vector<int2> ei(ev.size());
            for (size_t k = 0; k < ev.size(); ++k) ei[k] = make_int2(std::get<1>(ev[k]), std::get<2>(ev[k]));
            n_eitems_ = (int)ei.size();
            PDMK_CUDA_CHECK(cudaMalloc(&eitems_dev_, sizeof(int2) * std::max<size_t>(ei.size(), 1)));
            PDMK_CUDA_CHECK(cudaMemcpy(eitems_dev_, ei.data(), sizeof(int2) * ei.size(), cudaMemcpyHostToDevice));
            PDMK_CUDA_CHECK(cudaMalloc(&esys_dev_, sizeof(dev::EvalLeafSys) * nsys));
            p_ = trees_[0]->expansion_order();
            // interpolation items: 128-target blocks of every system
            std::vector<int2> ii;
            for (int i = 0; i < nsys; ++i)
                for (int64_t b = 0; b * 128 < off_[i + 1] - off_[i]; ++b) ii.push_back(make_int2(i, (int)b));
            n_iitems_ = (int)ii.size();
            PDMK_CUDA_CHECK(cudaMalloc(&iitems_dev_, sizeof(int2) * std::max<size_t>(ii.size(), 1)));
            PDMK_CUDA_CHECK(cudaMemcpy(iitems_dev_, ii.data(), sizeof(int2) * ii.size(), cudaMemcpyHostToDevice));
            PDMK_CUDA_CHECK(cudaMalloc(&isys_dev_, sizeof(dev::InterpSys) * nsys));
            w_ = trees_[0]->nufft_width();
            PDMK_CUDA_CHECK(cudaMalloc(&head_dev_, sizeof(int)));
            nc_ = trees_[0]->near_coeffs();
            for (int i = 0; i < nc_; ++i) coef32_[i] = (float)trees_[0]->near_coef()[i];
        }
    } catch (...) {
        release();
        throw;
    }
}

void TreeBatch::release() {
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    for (auto& g : graphs_)
        if (g) cudaGraphExecDestroy(g);
    graphs_.clear();
    if (err_host_) cudaFreeHost(err_host_);
    err_host_ = nullptr;
    if (q_pin_) cudaFreeHost(q_pin_);
    if (p_pin_) cudaFreeHost(p_pin_);
    q_pin_ = p_pin_ = nullptr;
    trees_.clear();
    for (auto& e : done_)
        if (e) cudaEventDestroy(e);
    done_.clear();
    for (auto& e : ev_up_)
        if (e) cudaEventDestroy(e);
    for (auto& e : ev_dn_)
        if (e) cudaEventDestroy(e);
    ev_up_.clear();
    ev_dn_.clear();
    pool_.reset();
    for (auto& e : prof_)
        if (e) cudaEventDestroy(e);
    if (stream_) cudaStreamDestroy(stream_);
    if (q_dev_) cudaFree(q_dev_);
    if (pot_dev_) cudaFree(pot_dev_);
    if (potf_dev_) cudaFree(potf_dev_);
    if (sys_dev_) cudaFree(sys_dev_);
    if (esys_dev_) cudaFree(esys_dev_);
    if (eitems_dev_) cudaFree(eitems_dev_);
    if (isys_dev_) cudaFree(isys_dev_);
    if (iitems_dev_) cudaFree(iitems_dev_);
    esys_dev_ = nullptr;
    eitems_dev_ = nullptr;
    isys_dev_ = nullptr;
    iitems_dev_ = nullptr;
    if (items_dev_) cudaFree(items_dev_);
    if (head_dev_) cudaFree(head_dev_);
    sys_dev_ = nullptr;
    items_dev_ = nullptr;
    head_dev_ = nullptr;
    stream_ = nullptr;
    q_dev_ = pot_dev_ = nullptr;
    potf_dev_ = nullptr;
}

TreeBatch::~TreeBatch() { release(); }

size_t TreeBatch::device_bytes() const {
    size_t b = (sizeof(double) * 2 + sizeof(float)) * (size_t)total_points();
    for (const auto& t : trees_) b += t->device_bytes();
    return b;
}

namespace {
// page-locked (or device-registered) host memory: copied by DMA directly
bool pinned(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

// memcpy split over persistent host threads (pageable <-> pinned staging)
class CopyPool {
  public:
    explicit CopyPool(int n) {
        for (int i = 0; i < n; ++i) workers_.emplace_back([this, i] { run(i); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (auto& w : workers_) w.join();
    }
    void copy(void* dst, const void* src, size_t bytes) {
        if (bytes < ((size_t)1 << 20) || workers_.empty()) {
            std::memcpy(dst, src, bytes);
            return;
        }
        std::unique_lock<std::mutex> lk(mu_);
        dst_ = static_cast<char*>(dst);
        src_ = static_cast<const char*>(src);
        bytes_ = bytes;
        pending_ = (int)workers_.size();
        ++gen_;
        cv_.notify_all();
        done_.wait(lk, [&] { return pending_ == 0; });
    }

  private:
    void run(int id) {
        uint64_t seen = 0;
        for (;;) {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return gen_ != seen; });
            seen = gen_;
            if (stop_) return;
            const size_t nw = workers_.size();
            const size_t part = ((bytes_ + nw - 1) / nw + 63) & ~(size_t)63;
            const size_t o = std::min(bytes_, part * (size_t)id), b = std::min(part, bytes_ - o);
            char* d = dst_;
            const char* sp = src_;
            lk.unlock();
            if (b) std::memcpy(d + o, sp + o, b);
            lk.lock();
            if (--pending_ == 0) done_.notify_one();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    uint64_t gen_ = 0;
    bool stop_ = false;
    char* dst_ = nullptr;
    const char* src_ = nullptr;
    size_t bytes_ = 0;
    int pending_ = 0;
};

void CopyPoolDeleter::operator()(CopyPool* p) const { delete p; }

void TreeBatch::evaluate(const double* charges, void* pot, bool pot_float) {
    if (!charges || !pot) throw std::invalid_argument("null charges or output");
    PDMK_CUDA_CHECK(cudaSetDevice(device_));
    const int64_t n = total_points();
    const auto h0 = std::chrono::steady_clock::now();
    if (profile_) PDMK_CUDA_CHECK(cudaEventRecord(prof_[0], stream_));
    // Pageable buffers go through the pinned staging (a pageable cudaMemcpy
    // moves 3-10 GB/s): host threads fill it chunk by chunk, each chunk's DMA
    // starts as soon as it is staged and the systems of that chunk start once
    // their charges are on the device.
    const bool q_pinned = pinned(charges), p_pinned = pinned(pot);
    if ((!q_pinned || !p_pinned) && !pool_)
        pool_.reset(new CopyPool((int)std::min(8u, std::max(1u, std::thread::hardware_concurrency()))));
    // The first evaluate runs the systems directly (it creates their multi-RHS
    // state); the second captures each system's launch sequence into a CUDA
    // graph (device buffers and tables are fixed per system), later ones
    // replay the graphs.
    const bool capture = evaluates_ == 1;
    const int nch = (int)chunk_sys_.size() - 1;
    for (int c = 0; c < nch; ++c) {
        const int s0 = chunk_sys_[c], s1 = chunk_sys_[c + 1];
        const int64_t o0 = off_[s0], cnt = off_[s1] - o0;
        const double* src = charges + o0;
        if (!q_pinned) {
            pool_->copy(q_pin_ + o0, charges + o0, sizeof(double) * (size_t)cnt);
            src = q_pin_ + o0;
        }
        PDMK_CUDA_CHECK(cudaMemcpyAsync(q_dev_ + o0, src, sizeof(double) * (size_t)cnt, cudaMemcpyHostToDevice,
                                        stream_));
        PDMK_CUDA_CHECK(cudaEventRecord(ev_up_[c], stream_));
        for (int i = s0; i < s1; ++i) {
            DeviceTree& t = *trees_[i];
            cudaStream_t ts = t.stream();
            PDMK_CUDA_CHECK(cudaStreamWaitEvent(ts, ev_up_[c], 0));
            auto enqueue = [&]() {
                if (single_)
                    t.enqueue_multi_device(q_dev_ + off_[i], 1, pot_dev_ + off_[i], /*fp32=*/true);
                else
                    t.evaluate_device(q_dev_ + off_[i], pot_dev_ + off_[i], nullptr);
            };
            if (graphs_[i]) {
                PDMK_CUDA_CHECK(cudaGraphLaunch(graphs_[i], ts));
            } else if (capture) {
                cudaGraph_t g = nullptr;
                PDMK_CUDA_CHECK(cudaStreamBeginCapture(ts, cudaStreamCaptureModeThreadLocal));
                try {
                    enqueue();
                } catch (...) {
                    cudaStreamEndCapture(ts, &g);
                    if (g) cudaGraphDestroy(g);
                    throw;
                }
                PDMK_CUDA_CHECK(cudaStreamEndCapture(ts, &g));
                cudaGraphExec_t ge = nullptr;
                const cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
                cudaGraphDestroy(g);
                PDMK_CUDA_CHECK(ie);
                graphs_[i] = ge;
                PDMK_CUDA_CHECK(cudaGraphLaunch(ge, ts));
            } else {
                enqueue();
            }
            PDMK_CUDA_CHECK(cudaEventRecord(done_[i], ts));
        }
    }
    if (profile_) PDMK_CUDA_CHECK(cudaEventRecord(prof_[1], stream_));
    // the main stream joins every system (after all uploads are enqueued, so
    // that no upload waits for a system)
    for (size_t i = 0; i < trees_.size(); ++i) PDMK_CUDA_CHECK(cudaStreamWaitEvent(stream_, done_[i], 0));
    const auto h1 = std::chrono::steady_clock::now();
    const bool prof = profile_;
    if (prof) PDMK_CUDA_CHECK(cudaEventRecord(prof_[2], stream_));
    if (single_) {
        if (!queue_built_) build_queue();
        dev::launch_batch_eval(esys_dev_, eitems_dev_, n_eitems_, p_, stream_);
        dev::launch_batch_interp(isys_dev_, iitems_dev_, n_iitems_, w_, stream_);
        if (prof) PDMK_CUDA_CHECK(cudaEventRecord(prof_[3], stream_));
        run_queue();
    } else if (prof) {
        PDMK_CUDA_CHECK(cudaEventRecord(prof_[3], stream_));
    }
    if (prof) PDMK_CUDA_CHECK(cudaEventRecord(prof_[4], stream_));
    const size_t es = pot_float ? sizeof(float) : sizeof(double);
    char* p_dst = static_cast<char*>(p_pinned ? pot : static_cast<void*>(p_pin_));
    if (pot_float) dev::launch_to_float(pot_dev_, potf_dev_, n, stream_);
    const char* p_src = pot_float ? reinterpret_cast<const char*>(potf_dev_) : reinterpret_cast<const char*>(pot_dev_);
    for (int c = 0; c < nch; ++c) {
        const int64_t o0 = off_[chunk_sys_[c]], cnt = off_[chunk_sys_[c + 1]] - o0;
        PDMK_CUDA_CHECK(cudaMemcpyAsync(p_dst + es * o0, p_src + es * o0, es * (size_t)cnt, cudaMemcpyDeviceToHost,
                                        stream_));
        PDMK_CUDA_CHECK(cudaEventRecord(ev_dn_[c], stream_));
    }
    // error words of the tensor-core kernels: one asynchronous copy each, one wait
    int n_err = 0;
    if (single_) {
        for (size_t i = 0; i < trees_.size(); ++i) {
            const int* w = trees_[i]->multi_error_word(true);
            err_host_[i] = 0;
            if (w) {
                PDMK_CUDA_CHECK(cudaMemcpyAsync(err_host_ + i, w, sizeof(int), cudaMemcpyDeviceToHost, stream_));
                ++n_err;
            }
        }
    }
    if (prof) PDMK_CUDA_CHECK(cudaEventRecord(prof_[5], stream_));
    // drain each chunk of the staging as soon as its DMA is done
    double out_ms = 0.0;  // host copy time (profile)
    if (!p_pinned)
        for (int c = 0; c < nch; ++c) {
            const int64_t o0 = off_[chunk_sys_[c]], cnt = off_[chunk_sys_[c + 1]] - o0;
            PDMK_CUDA_CHECK(cudaEventSynchronize(ev_dn_[c]));
            const auto c0 = std::chrono::steady_clock::now();
            pool_->copy(static_cast<char*>(pot) + es * o0, p_dst + es * o0, es * (size_t)cnt);
            out_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - c0).count();
        }
    PDMK_CUDA_CHECK(cudaStreamSynchronize(stream_));
    PDMK_CUDA_CHECK(cudaGetLastError());
    if (prof) {
        float ms[5];
        for (int i = 0; i < 5; ++i) PDMK_CUDA_CHECK(cudaEventElapsedTime(&ms[i], prof_[i], prof_[i + 1]));
        const double enq = std::chrono::duration<double, std::milli>(h1 - h0).count();
        std::fprintf(stderr, "pdmk batch: upload %.2f ms, systems %.2f ms (host staging + enqueue %.2f ms), leaf "
                             "evaluation + interpolation %.2f ms, queue %.2f ms, download %.2f ms + host copy %.2f ms\n",
                     ms[0], ms[1], enq, ms[2], ms[3], ms[4], out_ms);
    }
    ++evaluates_;
    if (n_err)
        for (size_t i = 0; i < trees_.size(); ++i)
            if (err_host_[i]) trees_[i]->check_device_error();  // clears the word and throws
}

void TreeBatch::build_queue() {
    // descriptors of every system's buffers (its single-RHS float state exists
    // after the first deferred evaluate)
    std::vector<dev::NearLeafSys> d(trees_.size());
    std::vector<dev::EvalLeafSys> ed(trees_.size());
    std::vector<dev::InterpSys> id(trees_.size());
    for (size_t i = 0; i < trees_.size(); ++i) {
        trees_[i]->near_leaf_sys(d[i], pot_dev_ + off_[i]);
        trees_[i]->eval_leaf_sys(ed[i]);
        trees_[i]->interp_sys(id[i]);
        if (trees_[i]->nufft_width() != w_) throw std::logic_error("batch systems with different NUFFT widths");
    }
    PDMK_CUDA_CHECK(cudaMemcpyAsync(isys_dev_, id.data(), sizeof(dev::InterpSys) * id.size(), cudaMemcpyHostToDevice,
                                    stream_));
    PDMK_CUDA_CHECK(cudaMemcpyAsync(sys_dev_, d.data(), sizeof(dev::NearLeafSys) * d.size(), cudaMemcpyHostToDevice,
                                    stream_));
    PDMK_CUDA_CHECK(cudaMemcpyAsync(esys_dev_, ed.data(), sizeof(dev::EvalLeafSys) * ed.size(),
                                    cudaMemcpyHostToDevice, stream_));
    PDMK_CUDA_CHECK(cudaStreamSynchronize(stream_));
    queue_built_ = true;
}

namespace {
// autotuner cache: (items, total points, polynomial length, device) -> targets per thread
std::mutex g_tune_mu;
std::map<std::tuple<int, int64_t, int, int>, int> g_tune;
}  // namespace

void TreeBatch::run_queue() {
    if (!queue_built_) build_queue();
    dev::BatchNearArgs a{};
    a.sys = sys_dev_;
    a.items = items_dev_;
    a.n_items = n_items_;
    a.head = head_dev_;
    for (int i = 0; i < 32; ++i) a.coef32[i] = coef32_[i];
    if (tpt_ == 0) {
        const auto key = std::make_tuple(n_items_, total_points(), nc_, device_);
        {
            std::lock_guard<std::mutex> g(g_tune_mu);
            auto it = g_tune.find(key);
            if (it != g_tune.end()) tpt_ = it->second;
        }
        if (tpt_ == 0) {
            // time each candidate once on this batch (the kernel writes the
            // potentials from inputs it does not modify, so repeats are harmless)
            cudaEvent_t e0, e1;
            PDMK_CUDA_CHECK(cudaEventCreate(&e0));
            PDMK_CUDA_CHECK(cudaEventCreate(&e1));
            float best = 1e30f;
            for (int tpt : {1, 2, 4}) {
                const int ctas = dev::batch_near_ctas(nc_, tpt);
                PDMK_CUDA_CHECK(cudaEventRecord(e0, stream_));
                dev::launch_batch_near(a, nc_, tpt, ctas, stream_);
                PDMK_CUDA_CHECK(cudaEventRecord(e1, stream_));
                PDMK_CUDA_CHECK(cudaEventSynchronize(e1));
                float ms = 0;
                PDMK_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
                if (ms < best) {
                    best = ms;
                    tpt_ = tpt;
                }
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            std::lock_guard<std::mutex> g(g_tune_mu);
            g_tune[key] = tpt_;
        }
        ctas_ = dev::batch_near_ctas(nc_, tpt_);
    }
    dev::launch_batch_near(a, nc_, tpt_, ctas_, stream_);
    PDMK_CUDA_CHECK(cudaGetLastError());
}

}  // namespace pdmkb
