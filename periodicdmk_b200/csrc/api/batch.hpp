// Batch of independent periodic systems: host trees built in parallel, device
// evaluates enqueued concurrently (one stream per system).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "../device/device_tree.hpp"

namespace pdmkb {

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
    cudaEvent_t ready_ = nullptr;
    std::vector<cudaEvent_t> done_;
    double* q_dev_ = nullptr;
    double* pot_dev_ = nullptr;
    float* potf_dev_ = nullptr;
    // after the first evaluate, each system's evaluate is replayed from a CUDA graph
    std::vector<cudaGraphExec_t> graphs_;
    int* err_host_ = nullptr;  // pinned, one word per system
    int evaluates_ = 0;
    // Float trees: the near field and final gather run as persistent launches
    // over device queues of (system, leaf) items, one per group of systems in
    // launch order, each as soon as its group's systems are done (so a
    // group's near field overlaps the later groups' tree passes).
    void build_queue();
    void run_queue(int g, cudaStream_t s);
    void launch_group(int g);  // group g's queue on its stream; the batch stream waits for it
    dev::NearLeafSys* sys_dev_ = nullptr;
    int2* items_dev_ = nullptr;  // grouped: group g's items at [group_item_[g], group_item_[g + 1])
    int* head_dev_ = nullptr;    // one queue head per group
    int n_items_ = 0;
    int n_groups_ = 1;
    std::vector<int> group_of_;    // system -> group
    std::vector<int> group_last_;  // group -> last system (launch order)
    std::vector<int> group_item_;  // group -> first item (size n_groups_ + 1)
    std::vector<cudaStream_t> group_stream_;
    std::vector<cudaEvent_t> group_done_;
    int nc_ = 0;
    float coef32_[32] = {};
    bool queue_built_ = false;
    int tpt_ = 0, ctas_ = 0;  // targets per thread and grid of the queue kernel (autotuned)

  public:
    // targets per thread chosen by the autotuner (0 before the first evaluate)
    int queue_targets_per_thread() const { return tpt_; }
};

}  // namespace pdmkb
