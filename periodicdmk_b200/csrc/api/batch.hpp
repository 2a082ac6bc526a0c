// Batch of independent periodic systems: host trees built in parallel, device
// evaluates enqueued concurrently (one stream per system).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "../device/device_tree.hpp"

namespace pdmkb {

class CopyPool;  // host threads copying between pageable and pinned buffers (batch.cpp)
struct CopyPoolDeleter {
    void operator()(CopyPool* p) const;
};

class TreeBatch {
  public:
    // cells: nsys x 9 (column-major 3x3 each); positions: 3 x Ns[i] blocks in order.
    // single: float (mixed-precision) trees, else double.
    TreeBatch(int nsys, const double* cells, const int* Ns, const double* positions, int n_digits, int n_per_leaf,
              int nz, bool single);
    ~TreeBatch();
    TreeBatch(const TreeBatch&) = delete;
    TreeBatch& operator=(const TreeBatch&) = delete;

    // charges / pot: concatenated host arrays of total_points() entries.
    void evaluate(const double* charges, void* pot, bool pot_float);
    int n_systems() const { return (int)trees_.size(); }
    int64_t total_points() const { return off_.empty() ? 0 : off_.back(); }
    size_t device_bytes() const;
    bool single() const { return single_; }

  private:
    void release();
    std::vector<std::unique_ptr<DeviceTree>> trees_;
    std::vector<int64_t> off_;  // prefix sums of N (size nsys + 1)
    bool single_ = false;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    // PDMK_BATCH_PROFILE: per-evaluate phase times on stderr (upload, systems, leaf evaluation and
    // interpolation, queue, download)
    bool profile_ = false;
    cudaEvent_t prof_[6]{};
    std::vector<cudaEvent_t> done_;
    double* q_dev_ = nullptr;
    double* pot_dev_ = nullptr;
    float* potf_dev_ = nullptr;
    // pinned staging of pageable host buffers (filled and drained by host threads)
    double* q_pin_ = nullptr;
    double* p_pin_ = nullptr;
    std::unique_ptr<CopyPool, CopyPoolDeleter> pool_;
    // transfers in chunks of whole systems: chunk c = systems chunk_sys_[c] ..
    // chunk_sys_[c + 1] - 1; its upload / download is complete at ev_up_[c] / ev_dn_[c]
    std::vector<int> chunk_sys_;
    std::vector<cudaEvent_t> ev_up_, ev_dn_;
    // after the first evaluate, each system's evaluate is replayed from a CUDA graph
    std::vector<cudaGraphExec_t> graphs_;
    int* err_host_ = nullptr;  // pinned, one word per system
    int evaluates_ = 0;
    // Float trees: the near field and final gather of all systems run as one
    // persistent launch over a device queue of (system, leaf) items.
    void build_queue();
    void run_queue();
    dev::NearLeafSys* sys_dev_ = nullptr;
    // the leaf evaluations of all systems in one launch: descriptors and
    // (system, leaf) items, most targets first
    dev::EvalLeafSys* esys_dev_ = nullptr;
    int2* eitems_dev_ = nullptr;
    int n_eitems_ = 0;
    int p_ = 0;
    // the far-field interpolations of all systems in one launch: descriptors
    // and (system, block of 128 targets) items
    dev::InterpSys* isys_dev_ = nullptr;
    int2* iitems_dev_ = nullptr;
    int n_iitems_ = 0;
    int w_ = 0;
    int2* items_dev_ = nullptr;
    int* head_dev_ = nullptr;
    int n_items_ = 0;
    int nc_ = 0;
    float coef32_[32] = {};
    bool queue_built_ = false;
    int tpt_ = 0, ctas_ = 0;  // targets per thread and grid of the queue kernel (autotuned)

  public:
    // targets per thread chosen by the autotuner (0 before the first evaluate)
    int queue_targets_per_thread() const { return tpt_; }
};

}  // namespace pdmkb
