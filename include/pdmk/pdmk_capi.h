/* C ABI of the B200 periodic DMK library (libpdmk_b200.so).
 *
 * The first block replaces, symbol for symbol, the reference's
 * cpp/include/pdmk/pdmk_capi.h:20-51 (exported from libpdmk_jl.so and bound by
 * julia/PeriodicDMK/src/PeriodicDMK.jl:120-126,135-137,172-181,198-209):
 * same names, argument order, layouts and return conventions.
 *   - cell_3x3: column-major 3x3, cell[i + 3*j] = component i of lattice vector j
 *   - positions_3xN: column-major 3xN, positions[d + 3*i] = coordinate d of point i
 *   - int-returning calls: 0 on success, -1 on a null handle or an exception
 *     (message on stderr), -2 on a CUDA error reported by the device.
 *   - create calls return NULL on error (message on stderr).
 *   - the caller owns all buffers; the library owns a handle until destroy.
 * The second block is additive (no reference counterpart, same conventions).
 */
#ifndef PDMK_CAPI_H
#define PDMK_CAPI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- reference entry points ------------------------------------------- */

/* Ewald summation reference (replaces cpp/include/pdmk/pdmk_capi.h:23-28;
 * reference implementation cpp/src/ewald_nufft.cpp:445-654, same parameter
 * choice).  Runs on the current CUDA device: cell-list real-space sum and a
 * NUFFT reciprocal sum, O(N log N).  s sets the accuracy: erfc(s) ~ exp(-s^2);
 * the NUFFT tolerance is 1e-12. */
int pdmk_ewald_nufft(const double* cell_3x3, int N, const double* positions_3xN, const double* charges, double s,
                     double* potentials_out, double* energy_out);

/* Cubic cover of a cell (replaces cpp/include/pdmk/pdmk_capi.h:32-35;
 * reference cpp/src/cubic_cover_optimizer.cpp:33-89).  Returns 1 for nz <= 0. */
int pdmk_optimize_cubic_cover(const double* cell_3x3, int nz, int* m_out, int* n_out, int* p_out, double* e1_out,
                              double* e2_out, double* e3_out, double* s_out, double* cost_out);

/* Build a tree (replaces cpp/include/pdmk/pdmk_capi.h:39-41 / :45-47,
 * cpp/src/pdmk_capi.cpp:48-59).  The tree is built on the host and uploaded to
 * the current CUDA device. */
void* pdmk_create_double(const double* cell_3x3, int N, const double* positions_3xN, int n_digits, int n_per_leaf,
                         int nz);
void* pdmk_create_float(const double* cell_3x3, int N, const double* positions_3xN, int n_digits, int n_per_leaf,
                        int nz);

/* Evaluate potentials for N charges in user order (replaces
 * cpp/include/pdmk/pdmk_capi.h:40-43 / :46-49, cpp/src/pdmk_capi.cpp:61-77).
 * N and positions_3xN are ignored, as in the reference. */
int pdmk_evaluate_double(void* h, int N, const double* positions_3xN, const double* charges, double* pot_out);
int pdmk_evaluate_float(void* h, int N, const double* positions_3xN, const double* charges, float* pot_out);

void pdmk_destroy_double(void* h);
void pdmk_destroy_float(void* h);

/* ---- additive entry points (no reference counterpart) ----------------- */

/* evaluate with a device-time breakdown: timing[0..3] = nufft_ms, dmk_ms,
 * direct_ms, build_ms (the fields of the reference's EvalTiming). */
int pdmk_evaluate_timed_double(void* h, int N, const double* positions_3xN, const double* charges, double* pot_out,
                               double* timing4);
int pdmk_evaluate_timed_float(void* h, int N, const double* positions_3xN, const double* charges, float* pot_out,
                              double* timing4);

/* k charge vectors on one tree: charges_Nxk[i + N*c], pot_Nxk[i + N*c]. */
int pdmk_evaluate_multi_double(void* h, int N, int k, const double* charges_Nxk, double* pot_Nxk);
int pdmk_evaluate_multi_float(void* h, int N, int k, const double* charges_Nxk, float* pot_Nxk);

/* Device-resident evaluate: charges_dev / pot_dev are device pointers (N
 * doubles for the double tree; charges double and pot float for the float
 * tree) on the tree's device.  The call returns after the work completes. */
int pdmk_evaluate_device_double(void* h, const double* charges_dev, double* pot_dev);
int pdmk_evaluate_device_float(void* h, const double* charges_dev, float* pot_dev);

/* k charge vectors on device buffers (Q_dev and pot_dev: N x k doubles,
 * column-major).  mixed != 0 selects the mixed-precision path (FP32 near field
 * and transforms, FP64 far field and accumulation); 0 the plain FP64 path.
 * The float-tree variant always uses the mixed path.  Synchronous. */
int pdmk_evaluate_multi_device_double(void* h, int k, const double* Q_dev, double* pot_dev, int mixed);
int pdmk_evaluate_multi_device_float(void* h, int k, const double* Q_dev, double* pot_dev);

/* Charges stored in float32 (N x k column-major, charges_Nxk[i + N*c]) on a
 * float tree (mixed-precision path): the host variant copies half the bytes of
 * the double form in and float potentials out; the device variant takes a
 * float charge buffer and writes double potentials.  The charges are widened
 * to double on the device, so the results equal the double-charge calls on
 * the same (float-representable) charges. */
int pdmk_evaluate_multi_float_qf32(void* h, int N, int k, const float* charges_Nxk, float* pot_Nxk);
int pdmk_evaluate_multi_device_float_qf32(void* h, int k, const float* Q_dev, double* pot_dev);

/* Potentials and their gradients (the field is -grad; the force on charge i
 * is -q_i grad_i) of a double tree, user order: grad_3xN[d + 3*i] = d u_i /
 * d x_d in the caller's frame.  No counterpart in the reference's C ABI: its
 * lower layers compute target gradients (pgh_trg = DMK_POTENTIAL_GRAD;
 * cpp/src/dmk/proxy.cpp:307-448, cpp/include/dmk/vector_kernels.hpp:391-417)
 * but PeriodicDMKTreeT exposes potentials only.  N and positions_3xN are
 * ignored, as in pdmk_evaluate_double.  The device form takes device buffers
 * (N, N and 3N doubles). */
int pdmk_evaluate_grad_double(void* h, int N, const double* positions_3xN, const double* charges, double* pot_out,
                              double* grad_3xN);
int pdmk_evaluate_grad_device_double(void* h, const double* charges_dev, double* pot_dev, double* grad_dev);

/* Quasi-periodic trees (the reference's PeriodicDMKTreeT constructed with a
 * Bloch vector and its evaluate_complex, cpp/src/periodic_dmk.cpp:41-47,
 * 251-276; not in the reference's C ABI, whose create takes no Bloch vector).
 * bloch3 is in the lattice-QR frame, as the reference takes it.  The complex
 * potentials u_i = sum_j q_j sum_R e^{i bloch.R} G(x_i - x_j - R) come out
 * interleaved, pot_2N[2 i] = Re u_i, pot_2N[2 i + 1] = Im u_i (the layout of
 * the reference's pbcdmk_adaptive output), computed in FP64 for both tree
 * types.  The real evaluates of a quasi-periodic tree, and the complex
 * evaluate of a periodic one, fail with -1.  The device form takes device
 * buffers (N charges, 2N doubles out). */
void* pdmk_create_qp_double(const double* cell_3x3, int N, const double* positions_3xN, int n_digits, int n_per_leaf,
                            int nz, const double* bloch3);
void* pdmk_create_qp_float(const double* cell_3x3, int N, const double* positions_3xN, int n_digits, int n_per_leaf,
                           int nz, const double* bloch3);
int pdmk_evaluate_complex_double(void* h, int N, const double* positions_3xN, const double* charges, double* pot_2N);
int pdmk_evaluate_complex_float(void* h, int N, const double* positions_3xN, const double* charges, float* pot_2N);
int pdmk_evaluate_complex_device_double(void* h, const double* charges_dev, double* pot_2N_dev);

/* The two parts of the potential in user order: the tree part (near field +
 * plane-wave levels - self term) and the periodic far field. */
int pdmk_evaluate_parts_double(void* h, const double* charges, double* tree_part, double* far_part);

/* Tree facts: out[0..15] = N, n_all (originals + images), boxes, levels,
 * target leaves, expansion order p, plane waves per axis, kernel launches per
 * single-RHS evaluate, device bytes, far-field modes (ms, mt, mu product),
 * near-field box pairs, plane-wave boxes, kernel launches of the last
 * multi-RHS evaluate, tree digit count, mixed path available (1/0), image
 * boxes that share an original box's expansions (exact lattice translates). */
int pdmk_info_double(void* h, int64_t* out16);
int pdmk_info_float(void* h, int64_t* out16);

/* Stage times of the most recent evaluate (multi-RHS: summed over its RHS
 * blocks): out8[0..7] =
 * dmk_ms, near_ms (residual near-field kernel), nufft_ms, finalize_ms,
 * total_ms, near-field pairs after the reference's contact-geometry cull,
 * near-field pairs before it, residual polynomial length. */
int pdmk_stage_times_double(void* h, double* out8);
int pdmk_stage_times_float(void* h, double* out8);

/* Measured FMA throughput of the current device in TFLOP/s (fp64 != 0: FP64,
 * else FP32), 2 flops per FMA; the denominator of CUDA-core rooflines. */
int pdmk_fma_peak(int fp64, double* tflops);

/* Measured tensor-core throughput of the current device in TFLOP/s (2 flops
 * per multiply-add): kind 0 = tcgen05 TF32 MMA with the operands in shared
 * memory (one of the three products of a 3xTF32 split), kind 1 = FP64 DMMA
 * (mma.sync m8n8k4, the FP64 tensor-core form of sm_100a).  The denominators
 * of tensor-core rooflines.  Returns -1 for an unknown kind. */
int pdmk_tc_peak(int kind, double* tflops);

/* Evaluate that allocates no device memory (no counterpart in the reference).
 * For callers that cannot allocate device memory while they run -- e.g. an
 * engine whose caching allocator owns the GPU memory pool, or a time-step
 * loop that cannot take the device-wide synchronisation of cudaMalloc/cudaFree.
 * The tree is created beforehand (pdmk_create_double allocates its buffers);
 * charges_dev / pot_dev are N doubles on the tree's device, owned by the caller.
 * Transform scratch lives in one static 32 MiB device array, held until exit by
 * every GPU it has been reserved on; trees needing more per box are rejected
 * (-1).  CUDA loads the array lazily: pdmk_create_double reserves it on the
 * tree's device (so the reservation belongs to the caller's set-up, before its
 * allocator takes the pool); if that fails, the first call here retries and
 * returns -2 when the device has no room.  Make the first call before any
 * stream capture.  Calls share the array, so calls that overlap on the GPU
 * race and must be serialised by the caller.  Synchronous. */
int pdmk_evaluate_device_noalloc_double(void* h, const double* charges_dev, double* pot_dev);

/* ---- batches of independent systems ------------------------------------ */

/* Many independent periodic systems built and evaluated together (no
 * reference counterpart; each system is what pdmk_create_* / pdmk_evaluate_*
 * of cpp/include/pdmk/pdmk_capi.h:39-49 build and evaluate one at a time).
 *   cells:     nsys column-major 3x3 cells, concatenated (9 doubles each)
 *   Ns:        points per system
 *   positions: column-major 3 x Ns[i] blocks, concatenated in system order
 * pdmk_batch_create picks the precision as the reference's
 * AutoPeriodicDMKTree (cpp/src/periodic_dmk.cpp:326-336): the float
 * (mixed-precision) trees for n_digits <= 6, double above;
 * pdmk_batch_create_double always uses double trees.  Host tree construction
 * runs on all host threads.  Returns NULL on error. */
void* pdmk_batch_create(int nsys, const double* cells, const int* Ns, const double* positions, int n_digits,
                        int n_per_leaf, int nz);
void* pdmk_batch_create_double(int nsys, const double* cells, const int* Ns, const double* positions, int n_digits,
                               int n_per_leaf, int nz);
/* Potentials of all systems; charges and pot_out are concatenated in system
 * order (sum of Ns entries).  The systems run concurrently on the device. */
int pdmk_batch_evaluate(void* h, const double* charges, double* pot_out);
int pdmk_batch_evaluate_float(void* h, const double* charges, float* pot_out);
/* out4 = {number of systems, total points, device bytes, 1 if float trees} */
int pdmk_batch_info(void* h, int64_t* out4);
void pdmk_batch_destroy(void* h);

/* Campaign reference files: oracle potentials at M sampled points of an
 * N-point system, stored with the system in the reference's 'PDMC' format
 * (cpp/include/pdmk/campaign_ref_io.hpp:13-186, header-only C++ there; the C++
 * form here is include/pdmk/campaign_ref_io.hpp).  No counterpart in the
 * reference's C ABI.  cell9 is column-major as cell_3x3 above; pos_3N as
 * positions_3xN.  pdmk_campaign_read_header: out5 = {config_id, N, M, digits,
 * prec}; pdmk_campaign_read fills buffers of those sizes.  -1 on an I/O error,
 * a malformed file or a digest mismatch.  pdmk_sha256: SHA-256 (FIPS 180-4)
 * of len bytes into out32. */
int pdmk_sha256(const void* data, uint64_t len, unsigned char* out32);
int pdmk_campaign_write(const char* path, uint32_t config_id, uint32_t digits, uint32_t prec, uint64_t seed,
                        const double* cell9, uint32_t N, const double* pos_3N, const double* chg_N, uint32_t M,
                        const uint32_t* ref_idx, const double* ref_u);
int pdmk_campaign_read_header(const char* path, uint32_t* out5, uint64_t* seed);
int pdmk_campaign_read(const char* path, double* cell9, double* pos_3N, double* chg_N, uint32_t* ref_idx,
                       double* ref_u);

/* Tree construction check: builds the plan of a system with its point steps
 * on the host (on_device = 0) or on the current CUDA device (1) and writes the
 * SHA-256 of the plan's point order, image list, box topology and interaction
 * lists to out32, and the build time to build_ms (may be null).  The two forms
 * give the same digest. */
int pdmk_plan_digest(const double* cell_3x3, int N, const double* positions_3xN, int n_digits, int n_per_leaf,
                     int nz, int on_device, unsigned char* out32, double* build_ms);

/* Last error message of the calling thread ("" if none). */
const char* pdmk_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* PDMK_CAPI_H */
