// Device-resident periodic DMK tree: uploads a host Plan once and runs the
// evaluate path on one GPU.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <functional>
#include <memory>
#include <vector>

#include "../host/plan.hpp"
#include "batch_near.cuh"
#include "grad.cuh"
#include "kernels.cuh"

namespace pdmkb {

struct StageTimes {
    double dmk_ms = 0;     // charge gather, upward pass, plane-wave downward pass, leaf evaluation
    double direct_ms = 0;  // residual near field + self correction + desort
    double nufft_ms = 0;   // periodic far field
    double near_ms = 0;    // residual near-field kernel alone
    double finalize_ms = 0;
};

// Looks up (and so, under lazy module loading, reserves) the static scratch
// array of the no-allocation evaluate on `device`; failures are left to that
// evaluate to report.  Defined in noalloc.cu.
void noalloc_reserve(int device);

class DeviceTree {
  public:
    // fp64_working_set: allocate the single-RHS FP64 expansion and transform
    // buffers now (double trees); float trees leave them to the first FP64
    // evaluate, if any, since their evaluates use the multi-RHS state.
    DeviceTree(const Plan& P, int device = -1, bool fp64_working_set = true);
    ~DeviceTree();
    DeviceTree(const DeviceTree&) = delete;
    DeviceTree& operator=(const DeviceTree&) = delete;

    int n_points() const { return n_; }
    int device() const { return device_; }
    cudaStream_t stream() const { return stream_; }

    // Host buffers in, host buffers out (copies inside).  times may be null.
    void evaluate_host(const double* q_user, double* pot_user, StageTimes* times = nullptr);
    // Device buffers (N doubles each) on this tree's device; enqueued on stream_.
    // With times != null the call synchronises to read the stage events.
    void evaluate_device(const double* q_user_d, double* pot_user_d, StageTimes* times = nullptr);
    // k charge vectors (N x k column-major, device buffers): potentials N x k.
    // fp32: mixed-precision path, else FP64.  RHS processed in blocks sized to
    // the free device memory (at most 64).  times (optional) sums the blocks.
    void evaluate_multi_device(const double* Q_dev, int k, double* pot_dev, bool fp32, StageTimes* times = nullptr);
    // Same computation, enqueued on stream() without any host synchronisation
    // (no stage times); check_device_error() after the stream has finished
    // reports a tensor-core pipeline timeout of the enqueued work.
    void enqueue_multi_device(const double* Q_dev, int k, double* pot_dev, bool fp32);
    void check_device_error();
    // Device word a tensor-core kernel of the multi-RHS state sets on a pipeline
    // timeout (null before the first multi-RHS call of that precision).
    int* multi_error_word(bool fp32) const;
    // Host buffers (pinned or pageable).  pot is double* or, with pot_float,
    // float* (converted on the device before the copy back).
    void evaluate_multi_host(const double* Q, int k, void* pot, bool pot_float, bool fp32,
                             StageTimes* times = nullptr);
    // Same with float charges (N x k column-major): the host variant copies
    // float charges in and float potentials out; the device variant takes a
    // float charge buffer on this tree's device and writes double potentials.
    // The charges are widened to double on the device before the evaluate.
    void evaluate_multi_host_f32(const float* Q, int k, float* pot, bool fp32);
    void evaluate_multi_device_f32(const float* Q, int k, double* pot, bool fp32, StageTimes* times = nullptr);
    // Whether the mixed-precision path is used for this tree's digit count
    // (it is for n_digits <= 6; above that the FP64 path runs).
    bool mixed_allowed() const { return n_digits_ <= 6; }
    // Stage times of the last multi-RHS evaluate (summed over RHS blocks).
    StageTimes last_multi_times() const { return last_multi_; }
    // Same as evaluate_device, but the transform scratch is the library's fixed
    // static device array instead of the tree's buffers, and nothing is
    // allocated; synchronous.  Defined in noalloc.cu.
    void evaluate_device_noalloc(const double* q_user_d, double* pot_user_d);
    // Potentials and their gradients d u / d x (user frame, grad[3 i + d], user
    // order) of the plain FP64 path: device buffers (N, 3N doubles) or host
    // buffers.  Synchronous.  Defined with the gradient kernels' drivers in
    // device_tree.cu (kernels in grad.cu).
    void evaluate_grad_device(const double* q_user_d, double* pot_user_d, double* grad_user_d);
    void evaluate_grad_host(const double* q_user, double* pot_user, double* grad_user);
    // Quasi-periodic trees (built from a plan with a Bloch vector): complex
    // potentials u(x_i) = sum_j q_j sum_R e^{i bloch.R} G(x_i - x_j - R),
    // interleaved (Re, Im) per point in user order (2N doubles), computed in
    // FP64 as two real right-hand sides (the phased charges' real and
    // imaginary parts) through the tree, and a two-transform quasi-periodic
    // far field.  Device buffers, or host buffers.  Synchronous.  Defined in
    // multi.cu (kernels in qp.cu).
    bool quasi_periodic() const { return qp_; }
    void evaluate_complex_device(const double* q_user_d, double* pot2_user_d, StageTimes* times = nullptr);
    void evaluate_complex_host(const double* q_user, double* pot2_user, StageTimes* times = nullptr);
    // Tree part (near + plane-wave levels - self) and far field, user order, host buffers.
    void evaluate_parts_host(const double* q_user, double* tree_part, double* far_part);
    // Number of kernels one evaluate launches (for reporting).
    int launches_per_evaluate() const { return launches_; }
    // Stage times of the most recent evaluate (synchronises on its last event).
    StageTimes last_times();
    // Near-field pairs the reference evaluates after its contact-geometry cull
    // (the algorithmic work of the residual sum) and before it (all list pairs).
    int64_t near_pairs_culled() const { return near_pairs_culled_; }
    int64_t near_pairs_nominal() const { return near_pairs_nominal_; }
    int near_coeffs() const { return near_.nc; }
    size_t device_bytes() const { return bytes_; }
    // image boxes sharing an original box's proxy moments and outgoing expansions
    int64_t translate_boxes() const { return n_alias_; }

  private:
    struct MultiState;
    struct MultiStateDeleter {
        void operator()(MultiState* m) const;
    };
    int multi_block(int k, bool fp32);
    int multi_block_size(int k, bool fp32) const;
    int kb_cache_k_[2] = {0, 0}, kb_cache_[2] = {0, 0};  // last (k -> kb) per precision
    MultiState& multi_state(int kb, bool fp32);
    template <typename T>
    void run_multi_block(MultiState& m, const double* Q, int kvalid, double* pot_user);
    // far field of the columns [c0, c0 + cols) of a multi-RHS block (q_t -> far)
    int far_columns(MultiState& m, int c0, int cols, bool qp, cufftHandle fwd, cufftHandle inv, cudaStream_t s,
                    bool interp = true);
    // Host-buffer multi-RHS evaluate with the charge upload in column chunks:
    // upload(c0, cols) enqueues a chunk's copy on stream_; the far field of each
    // chunk runs on a second stream as soon as it has arrived, the tree passes
    // after the last chunk.  False when the shape does not allow it (nothing
    // enqueued then).
    bool multi_host_overlapped(int k, bool fp32, double* qd, double* pd,
                               const std::function<void(int, int)>& upload);
    // run_multi_block leaves the far field (and the target-charge gather) to
    // the caller, whose work is complete at far_ext_event_
    bool far_ext_ = false;
    cudaEvent_t far_ext_event_ = nullptr;
    int overlap_h2d_ = 1;  // PDMK_E2E_OVERLAP=0 keeps the upload in one copy before the evaluate
    std::unique_ptr<MultiState, MultiStateDeleter> multi_[2];
    StageTimes last_multi_{};
    // device staging of the host-buffer multi-RHS calls (grow-only, freed with the tree)
    double* stage_q_ = nullptr;
    double* stage_p_ = nullptr;
    size_t stage_elems_ = 0;
    void ensure_stage(int64_t n);  // grow both staging buffers to n doubles

  public:
    bool last_was_multi_ = false;
    // Set by a batch of systems: single-RHS float evaluates leave out the leaf
    // evaluation, the far-field interpolation, the near field and the final
    // gather, which the batch does for all systems in one launch each
    // (multi.cu, nufft_multi.cu, batch_near.cu).
    bool defer_near_ = false;
    // Descriptor of this tree's leaf-evaluation inputs for the batch's launch
    // (the single-RHS float state must exist).
    void eval_leaf_sys(dev::EvalLeafSys& d) const;
    int eval_leaves() const { return eval_.n_leaves; }
    // Descriptor of this tree's far-field interpolation for the batch's launch
    // (the single-RHS float state must exist).
    void interp_sys(dev::InterpSys& d) const;
    int nufft_width() const { return nufft_.w; }
    int expansion_order() const { return p_; }
    const std::vector<int>& eval_leaf_targets() const { return eval_leaf_trg_; }
    // Descriptor of this tree's buffers for the batch near-field kernel (the
    // single-RHS float state must exist: one deferred evaluate has run);
    // out = this system's potentials in user order.
    void near_leaf_sys(dev::NearLeafSys& d, double* out) const;
    // Near-field leaves (target leaves) and their estimated work (targets x
    // sources over the leaf's near pairs), host copies.
    int near_leaves() const { return near_.n_leaves; }
    const std::vector<int64_t>& near_leaf_cost() const { return near_leaf_cost_; }
    const double* near_coef() const { return near_.coef; }
    int multi_launches_ = 0;  // kernels launched by the last multi-RHS evaluate
    // Tensor-core kernels the mixed-precision path may use (bit 0 proxy
    // moments, bit 1 near field, bit 2 leaf evaluation, bit 3 the separable
    // translation and plane-wave transform steps); the CUDA-core kernels cover
    // the rest.  Initialised from PDMK_TC_MASK (default 7).
    int tc_mask_ = 7;
    // FP64 child <-> parent translations on the FP64 tensor cores (DMMA)
    // instead of the CUDA cores.  Initialised from PDMK_FP64_DMMA (default 0).
    int fp64_dmma_ = -1;  // translations on DMMA: 1 on, 0 off, -1 at p = 28 only (measured faster there)
    // Proxy moments of the FP64 path at p = 28, 38 on DMMA (dmma.cu) instead of
    // the register-tiled CUDA-core kernel.  Initialised from PDMK_MOMENTS_DMMA
    // (default 1: 86 -> 42 ms per 12-digit evaluate of 2e6 clustered points).
    int moments_dmma_ = 1;

  private:
    void init(const Plan& P, int device, bool fp64_working_set);
    void ensure_fp64_working_set();
    void release();
    template <typename T>
    T* alloc(size_t n);
    template <typename T>
    T* upload(const std::vector<T>& v);
    void run(const double* q_user_d, double* pot_user_d);
    // Chunk sizes (boxes per launch) of the FP64 transforms for a scratch of cap complex elements.
    struct Fp64Chunks {
        int c2p = 1, pw_out = 1, pw_in = 1;
    };
    Fp64Chunks fp64_chunks(int64_t cap) const;
    // Transform scratch per box (complex elements) of the child/parent
    // translations, the outgoing and the incoming plane-wave transforms.
    int64_t fp64_need_c2p() const;
    int64_t fp64_need_pw_out() const;
    int64_t fp64_need_pw_in() const;
    int64_t fp64_need_max() const;
    // Gather, proxy moments, upward pass and the level-by-level downward pass
    // with leaf evaluation of the single-RHS FP64 path; transform scratch of
    // cap complex elements.  Returns the number of kernels launched.
    int run_fp64_tree(const double* q_user_d, dev::cd* scratch, int64_t cap, cudaStream_t s);

    int device_ = 0;
    int n_digits_ = 6;
    int n_ = 0, n_all_ = 0, p_ = 0, npw_ = 0, npw2_ = 0, M_ = 0;
    size_t bytes_ = 0;
    int launches_ = 0;
    int64_t near_pairs_culled_ = 0, near_pairs_nominal_ = 0;
    int near_max_trg_ = 0, near_max_pairs_ = 0;  // largest target count / source-box count of a near-field leaf
    int near_max_chunks_ = 0;                     // largest number of 32-source chunks of a near-field leaf
    std::vector<int64_t> near_leaf_cost_;         // per near-field leaf: targets x near sources
    std::vector<int> eval_leaf_trg_;              // per evaluated leaf: targets
    int* near_pair_chunk_base_ = nullptr;         // per near pair: first chunk bounding box of its source box
    float4* near_chunk_lo_ = nullptr;
    float4* near_chunk_hi_ = nullptr;
    int eval_max_trg_ = 0;  // largest target count of an evaluated leaf
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev_[5]{};
    std::vector<void*> allocs_;

    // points
    double4* src_ = nullptr;
    int* src_charge_idx_ = nullptr;
    double4* trg_ = nullptr;  // .w = self-interaction weight of the target's leaf
    int* trg_perm_ = nullptr;
    double* pot_sorted_ = nullptr;
    double* far_sorted_ = nullptr;
    double* q_sorted_ = nullptr;
    double* q_dev_ = nullptr;    // staging for host-buffer evaluate
    double* pot_dev_ = nullptr;
    // expansions
    double* proxy_up_ = nullptr;
    int64_t n_up_ = 0, n_down_ = 0, n_pw_ = 0;
    int64_t n_alias_ = 0;  // image boxes sharing an original box's expansions (exact lattice translates)
    // tables
    double* c2p_ = nullptr;
    double* p2c_ = nullptr;
    struct LevelDev {
        dev::cd* poly2pw = nullptr;      // n x p
        dev::cd* poly2pw_half = nullptr; // n2 x p
        dev::cd* pw2polyT = nullptr;     // p x n
        dev::cd* pw2polyTw = nullptr;    // p x n2, half-space weights folded in
        double* shift = nullptr;         // 27 x 2M
    };
    std::vector<LevelDev> lev_;
    // upward
    dev::C2ProxyArgs c2x_{};
    struct C2PGroup {  // one (level, child index) group of children -> parents
        int n = 0;
        int64_t* in_off = nullptr;
        int64_t* out_off = nullptr;
        int child = 0;
    };
    std::vector<C2PGroup> c2p_groups_;
    struct PwGroup {  // boxes of one level whose outgoing expansion is formed
        int level = 0, n = 0;
        int64_t* in_off = nullptr;   // proxy_up element offset
        int64_t* out_off = nullptr;  // pw_out element offset
    };
    std::vector<PwGroup> pw_groups_;
    struct EvalLevel {  // boxes of one level that receive incoming expansions
        int level = 0, n = 0;
        int* term_start = nullptr;
        int* term_slot = nullptr;
        int* term_stencil = nullptr;
        int64_t* down_off = nullptr;
        int n_p2c = 0;
        int64_t* p2c_in = nullptr;
        int64_t* p2c_out = nullptr;
        int64_t* p2c_mat = nullptr;  // element offset of the child's x matrix in p2c_
    };
    std::vector<EvalLevel> eval_levels_;
    dev::EvalArgs eval_{};
    dev::NearArgs near_{};
    // Single-RHS FP64 path, one level at a time.  Besides proxy_up it holds the
    // outgoing plane waves of one level, the downward proxy coefficients of two
    // consecutive levels (ping-pong by level parity) and one transform scratch
    // of bounded size; every offset below is local to its level's buffer.
    struct Fp64Level {
        int level = 0;
        int64_t n_down = 0;             // boxes of this level with downward storage
        int n_pw = 0;                   // outgoing expansions formed at this level
        int64_t* pw_in_off = nullptr;   // proxy_up element offset
        int64_t* pw_out_off = nullptr;  // element offset in the level's plane-wave buffer
        int n_in = 0;                   // boxes that receive incoming expansions
        int* term_start = nullptr;      // CSR over those boxes
        int* term_slot = nullptr;       // plane-wave slot (units of M) in the level buffer
        int* term_stencil = nullptr;
        int64_t* down_off = nullptr;    // element offset in the level's proxy_down buffer
        dev::EvalArgs eval{};           // leaves of this level (slot: level-local proxy_down slot)
        int n_p2c = 0;                  // parent (this level) -> child (next level) translations
        int64_t* p2c_in = nullptr;
        int64_t* p2c_out = nullptr;
        int64_t* p2c_mat = nullptr;
    };
    std::vector<Fp64Level> f64_levels_;
    double* down_level_[2] = {nullptr, nullptr};  // proxy_down of even / odd levels
    int64_t down_level_boxes_[2] = {0, 0};
    dev::cd* pw_level_ = nullptr;                  // outgoing plane waves of the current level
    int64_t pw_level_boxes_ = 0;
    dev::cd* f64_scratch_ = nullptr;
    int64_t f64_scratch_elems_ = 0;
    // far field
    dev::NufftArgs nufft_{};
    int nufft_max_jk_ = 0, nufft_max_ex_ = 0, nufft_max_cells_ = 0;
    double* grid_ = nullptr;
    dev::cd* spec_ = nullptr;
    double* mult_ = nullptr;
    int64_t n_spec_ = 0, n_grid_ = 0;
    cufftHandle plan_fwd_ = 0, plan_inv_ = 0;
    // gradients (allocated on the first gradient evaluate)
    void ensure_grad();
    bool grad_on_ = false;          // leaf-evaluation gradients launched by run_fp64_tree
    double* grad_sorted_ = nullptr; // near + local-expansion gradient, [3][n] sorted targets
    double* far_grad_ = nullptr;    // far-field gradient, [3][n]
    double* grad_dev_ = nullptr;    // staging for host-buffer gradient evaluates, [n][3]
    dev::cd* spec_save_ = nullptr;  // far-field spectrum after the multiplier
    dev::cd* spec_tmp_ = nullptr;   // i K_d times it
    dev::GradFrame frame_{};
    // quasi-periodic state (qp.cu)
    bool qp_ = false;
    bool qp_run_ = false;               // run_multi_block<double> computes the two QP columns
    double2* qp_src_phase_ = nullptr;   // (cos, sin) of bloch.R per sorted source
    double2* qp_trg_phase_ = nullptr;   // (cos, sin) of bloch.x per sorted target
    double* qp_s_ = nullptr;            // even part of the far-field multiplier, half spectrum
    double* qp_d_ = nullptr;            // odd part
    void require_periodic(const char* what) const;  // throws std::logic_error on QP trees
};

}  // namespace pdmkb
