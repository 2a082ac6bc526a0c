// Tree construction with the points on the GPU (DevicePoints): the
// point-heavy steps of the reference's PBCTree constructor
// (cpp/src/dmk/pbc_tree.cpp:138-740; images, cpp/include/pdmk/image_layout.hpp:14-88)
// run here, while build_plan (host/tree.cpp) decides the box topology from the
// counts these steps return.  Each step performs the floating-point operations
// of the host form (host/tree.cpp, HostPoints) on the same values, so the
// plans agree exactly:
//   * lattice images: per shift, a flag per original, an exclusive scan and a
//     compaction (shift-major, input order, as the host loop appends them);
//   * level-0 binning: a stable LSD radix sort (8-bit digits) of the box keys;
//   * refinement and 2:1-balance splits: one CTA per splitting box partitions
//     its range stably into the 8 octants (warp ballots give each point's rank
//     among the earlier points of its octant);
//   * Morton order inside each leaf: one CTA per leaf ranks its keys (stable:
//     ties by position) and scatters;
//   * the inside-the-leaf check: one CTA per leaf counts the points outside.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "../host/plan.hpp"
#include "../host/points.hpp"
#include "common.cuh"
#include "tree_build.hpp"

namespace pdmkb {
namespace dev {
namespace {

constexpr int kScanThreads = 1024, kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kRsThreads = 256, kRsItems = 16, kRsTile = kRsThreads * kRsItems;

// ---------------------------------------------------------------- scan
// exclusive scan of each 4096-element tile in place; tile totals to sums
__global__ void __launch_bounds__(kScanThreads) k_scan_tile(int* __restrict__ d, int64_t n, int* __restrict__ sums) {
    __shared__ int sh[kScanThreads];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int v[kScanItems], t = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? d[base + k] : 0;
        t += v[k];
    }
    sh[threadIdx.x] = t;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {  // Hillis-Steele inclusive scan of thread totals
        const int add = threadIdx.x >= (unsigned)off ? sh[threadIdx.x - off] : 0;
        __syncthreads();
        sh[threadIdx.x] += add;
        __syncthreads();
    }
    int run = sh[threadIdx.x] - t;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) d[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = sh[threadIdx.x];
}

__global__ void k_scan_add(int* __restrict__ d, int64_t n, const int* __restrict__ offs) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] += offs[i / kScanTile];
}

// In-place exclusive scan of n ints; returns the total (synchronises).
int64_t exclusive_scan(int* d, int64_t n, cudaStream_t s) {
    if (n <= 0) return 0;
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    int* sums = nullptr;
    PDMK_CUDA_CHECK(cudaMallocAsync(&sums, sizeof(int) * (tiles + 1), s));
    k_scan_tile<<<(unsigned)tiles, kScanThreads, 0, s>>>(d, n, sums);
    PDMK_CUDA_CHECK(cudaGetLastError());
    int64_t total = 0;
    if (tiles > 1) {
        total = exclusive_scan(sums, tiles, s);
        k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d, n, sums);
        PDMK_CUDA_CHECK(cudaGetLastError());
    } else {
        int t = 0;
        PDMK_CUDA_CHECK(cudaMemcpyAsync(&t, sums, sizeof(int), cudaMemcpyDeviceToHost, s));
        PDMK_CUDA_CHECK(cudaStreamSynchronize(s));
        total = t;
    }
    PDMK_CUDA_CHECK(cudaFreeAsync(sums, s));
    PDMK_CUDA_CHECK(cudaStreamSynchronize(s));
    return total;
}

// ---------------------------------------------------------------- radix sort (stable, 8-bit digits)
__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const uint32_t* __restrict__ key, int64_t n, int shift,
                                                        int* __restrict__ hist, int64_t tiles) {
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kRsTile;
    for (int k = 0; k < kRsItems; ++k) {
        const int64_t i = base + (int64_t)k * kRsThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(key[i] >> shift) & 255u], 1);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const uint32_t* __restrict__ key, const int* __restrict__ val,
                                                           int64_t n, int shift, const int* __restrict__ offs,
                                                           int64_t tiles, uint32_t* __restrict__ key_out,
                                                           int* __restrict__ val_out) {
    __shared__ int base[256];
    __shared__ int wcnt[kRsThreads / 32][256];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    base[tid] = offs[(int64_t)tid * tiles + blockIdx.x];
    for (int w = 0; w < kRsThreads / 32; ++w) wcnt[w][tid] = 0;
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    for (int c = 0; c < kRsItems; ++c) {
        // items of a chunk are consecutive: warp order, then lane order, is input order
        const int64_t i = (int64_t)blockIdx.x * kRsTile + (int64_t)c * kRsThreads + tid;
        const bool ok = i < n;
        const uint32_t k = ok ? key[i] : 0u;
        const int dg = ok ? (int)((k >> shift) & 255u) : 256 + lane;  // no match for missing items
        const unsigned peers = __match_any_sync(0xffffffffu, dg);
        const int rank = __popc(peers & lt);
        if (ok && rank == 0) wcnt[warp][dg] = __popc(peers);
        __syncthreads();
        if (ok) {
            int pre = 0;
            for (int w = 0; w < warp; ++w) pre += wcnt[w][dg];
            const int dst = base[dg] + pre + rank;
            key_out[dst] = k;
            val_out[dst] = val[i];
        }
        __syncthreads();
        int tot = 0;
        for (int w = 0; w < kRsThreads / 32; ++w) {
            tot += wcnt[w][tid];
            wcnt[w][tid] = 0;
        }
        base[tid] += tot;
        __syncthreads();
    }
}

// Stable sort of (key, val) by the low `bits` bits of key; results in key/val.
void radix_sort(uint32_t*& key, int*& val, uint32_t*& key_tmp, int*& val_tmp, int64_t n, int bits, cudaStream_t s) {
    if (n <= 1) return;
    const int64_t tiles = (n + kRsTile - 1) / kRsTile;
    int* hist = nullptr;
    PDMK_CUDA_CHECK(cudaMallocAsync(&hist, sizeof(int) * 256 * tiles, s));
    for (int shift = 0; shift < bits; shift += 8) {
        k_rs_hist<<<(unsigned)tiles, kRsThreads, 0, s>>>(key, n, shift, hist, tiles);
        PDMK_CUDA_CHECK(cudaGetLastError());
        exclusive_scan(hist, 256 * tiles, s);
        k_rs_scatter<<<(unsigned)tiles, kRsThreads, 0, s>>>(key, val, n, shift, hist, tiles, key_tmp, val_tmp);
        PDMK_CUDA_CHECK(cudaGetLastError());
        std::swap(key, key_tmp);
        std::swap(val, val_tmp);
    }
    PDMK_CUDA_CHECK(cudaFreeAsync(hist, s));
    PDMK_CUDA_CHECK(cudaStreamSynchronize(s));
}

// ---------------------------------------------------------------- images
struct Shift {
    double x, y, z;
};

__device__ __forceinline__ bool in_ext(const double4& p, const Shift& sh, const double* lo, const double* hi) {
    const double x0 = p.x + sh.x, x1 = p.y + sh.y, x2 = p.z + sh.z;
    return !(x0 < lo[0] || x0 > hi[0] || x1 < lo[1] || x1 > hi[1] || x2 < lo[2] || x2 > hi[2]);
}

struct ExtBox {
    double lo[3], hi[3];
};

__global__ void k_img_count(const double4* __restrict__ x, int n, const Shift* __restrict__ sh, int nsh, ExtBox b,
                            int* __restrict__ cnt) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (j >= n || k >= nsh) return;
    if (in_ext(x[j], sh[k], b.lo, b.hi)) atomicAdd(&cnt[k], 1);
}

__global__ void k_img_flag(const double4* __restrict__ x, int n, Shift sh, ExtBox b, int* __restrict__ flag) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) flag[j] = in_ext(x[j], sh, b.lo, b.hi) ? 1 : 0;
}

__global__ void k_img_write(const double4* __restrict__ x, int n, Shift sh, ExtBox b, const int* __restrict__ off,
                            double4* __restrict__ out, int* __restrict__ idx, int64_t at) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n || !in_ext(x[j], sh, b.lo, b.hi)) return;
    const double4 p = x[j];
    const int64_t o = at + off[j];
    out[o] = make_double4(p.x + sh.x, p.y + sh.y, p.z + sh.z, 0.0);
    idx[o] = j;
}

// ---------------------------------------------------------------- level-0 keys, gathers
struct Grid0 {
    double xelo[3], rcinv;
    int m[3];
};

__global__ void k_bin_keys(const double4* __restrict__ x, int64_t n, Grid0 g, uint32_t* __restrict__ key,
                           int* __restrict__ val, int* __restrict__ cnt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = x[i];
    const double c[3] = {p.x, p.y, p.z};
    int ii[3];
    for (int k = 0; k < 3; ++k) {
        ii[k] = (int)((c[k] - g.xelo[k]) * g.rcinv);
        ii[k] = min(max(ii[k], 0), g.m[k] - 1);
    }
    const uint32_t b = (uint32_t)(ii[2] * g.m[0] * g.m[1] + ii[1] * g.m[0] + ii[0]);
    key[i] = b;
    val[i] = (int)i;
    atomicAdd(&cnt[b], 1);
}

__global__ void k_gather(const double4* __restrict__ x, const int* __restrict__ perm, const int* __restrict__ order,
                         int64_t n, double4* __restrict__ x_out, int* __restrict__ perm_out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = order[i];
    x_out[i] = x[j];
    perm_out[i] = perm[j];
}

// ---------------------------------------------------------------- octant partition
struct RangeD {
    int start, count;
    double c[3];
};

constexpr int kPartThreads = 256;

__device__ __forceinline__ int octant(const double4& p, const double* c) {
    return (p.x >= c[0] ? 1 : 0) | (p.y >= c[1] ? 2 : 0) | (p.z >= c[2] ? 4 : 0);
}

// One CTA per range: counts, then a stable scatter into tmp, then the range is
// copied back.  counts[8 r + o] = points of range r in octant o.
__global__ void __launch_bounds__(kPartThreads) k_partition(const RangeD* __restrict__ rg, double4* __restrict__ x,
                                                            int* __restrict__ perm, double4* __restrict__ xt,
                                                            int* __restrict__ pt, int* __restrict__ counts) {
    __shared__ int cnt[8], base[8];
    __shared__ int wcnt[kPartThreads / 32][8];
    const RangeD r = rg[blockIdx.x];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid < 8) cnt[tid] = 0;
    __syncthreads();
    for (int i = tid; i < r.count; i += kPartThreads) atomicAdd(&cnt[octant(x[r.start + i], r.c)], 1);
    __syncthreads();
    if (tid == 0) {
        int o = r.start;
        for (int k = 0; k < 8; ++k) {
            base[k] = o;
            o += cnt[k];
            counts[8 * (int64_t)blockIdx.x + k] = cnt[k];
        }
    }
    const unsigned lt = (1u << lane) - 1u;
    for (int c0 = 0; c0 < r.count; c0 += kPartThreads) {
        const int i = c0 + tid;
        const bool ok = i < r.count;
        const double4 p = ok ? x[r.start + i] : make_double4(0, 0, 0, 0);
        const int o = ok ? octant(p, r.c) : -1;
        int rank = 0;
        for (int k = 0; k < 8; ++k) {
            const unsigned m = __ballot_sync(0xffffffffu, o == k);
            if (o == k) rank = __popc(m & lt);
            if (lane == 0) wcnt[warp][k] = __popc(m);
        }
        __syncthreads();
        if (ok) {
            int pre = 0;
            for (int w = 0; w < warp; ++w) pre += wcnt[w][o];
            const int dst = base[o] + pre + rank;
            xt[dst] = p;
            pt[dst] = perm[r.start + i];
        }
        __syncthreads();
        if (tid < 8) {
            int tot = 0;
            for (int w = 0; w < kPartThreads / 32; ++w) tot += wcnt[w][tid];
            base[tid] += tot;
        }
        __syncthreads();
    }
    // the range's own writes are visible to the CTA after the barrier above
    for (int i = tid; i < r.count; i += kPartThreads) {
        x[r.start + i] = xt[r.start + i];
        perm[r.start + i] = pt[r.start + i];
    }
}

// ---------------------------------------------------------------- Morton order, inside check
struct LeafD {
    int start, count;
    double c[3], h;
};

constexpr int kMortonThreads = 256, kMortonSmem = 4096;

__device__ __forceinline__ uint64_t spread3(uint32_t v) {
    uint64_t x = v & 0x3FF;
    x = (x | (x << 16)) & 0x030000FF;
    x = (x | (x << 8)) & 0x0300F00F;
    x = (x | (x << 4)) & 0x030C30C3;
    x = (x | (x << 2)) & 0x09249249;
    return x;
}

__device__ __forceinline__ uint64_t morton_key(const double4& p, const LeafD& L) {
    const double c[3] = {p.x, p.y, p.z};
    uint64_t k = 0;
    for (int d = 0; d < 3; ++d) {
        const double f = (c[d] - (L.c[d] - L.h)) / (2.0 * L.h);
        const int q = min(1023, max(0, (int)(f * 1024.0)));
        k |= spread3((uint32_t)q) << d;
    }
    return k;
}

// One CTA per leaf: the keys go to shared memory (or, for large leaves, to
// kscratch at the leaf's own range), each point's rank = #(smaller keys) +
// #(equal keys earlier), then scatter into tmp and copy back.
__global__ void __launch_bounds__(kMortonThreads) k_morton(const LeafD* __restrict__ lv, double4* __restrict__ x,
                                                           int* __restrict__ perm, double4* __restrict__ xt,
                                                           int* __restrict__ pt, uint64_t* __restrict__ kscratch) {
    __shared__ uint64_t sk[kMortonSmem];
    const LeafD L = lv[blockIdx.x];
    const int m = L.count;
    uint64_t* keys = m <= kMortonSmem ? sk : kscratch + L.start;
    for (int i = threadIdx.x; i < m; i += kMortonThreads) keys[i] = morton_key(x[L.start + i], L);
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += kMortonThreads) {
        const uint64_t ki = keys[i];
        int rank = 0;
        for (int j = 0; j < m; ++j) {
            const uint64_t kj = keys[j];
            rank += (kj < ki || (kj == ki && j < i)) ? 1 : 0;
        }
        xt[L.start + rank] = x[L.start + i];
        pt[L.start + rank] = perm[L.start + i];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += kMortonThreads) {
        x[L.start + i] = xt[L.start + i];
        perm[L.start + i] = pt[L.start + i];
    }
}

__global__ void k_outside(const LeafD* __restrict__ lv, const double4* __restrict__ x,
                          unsigned long long* __restrict__ bad) {
    const LeafD L = lv[blockIdx.x];
    int nb = 0;
    for (int i = threadIdx.x; i < L.count; i += blockDim.x) {
        const double4 p = x[L.start + i];
        if (fabs(p.x - L.c[0]) > L.h || fabs(p.y - L.c[1]) > L.h || fabs(p.z - L.c[2]) > L.h) ++nb;
    }
    if (nb) atomicAdd(bad, (unsigned long long)nb);
}

__global__ void k_iota(int* __restrict__ v, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int)i;
}

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

template <typename T>
T* dalloc(int64_t n, cudaStream_t s) {
    T* p = nullptr;
    PDMK_CUDA_CHECK(cudaMallocAsync(&p, sizeof(T) * (size_t)std::max<int64_t>(n, 1), s));
    return p;
}

}  // namespace

// ---------------------------------------------------------------- DevicePoints
class DevicePoints final : public PointOps {
  public:
    DevicePoints() { PDMK_CUDA_CHECK(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking)); }
    ~DevicePoints() override {
        for (int k = 0; k < 2; ++k) {
            if (x_[k]) cudaFreeAsync(x_[k], s_);
            if (p_[k]) cudaFreeAsync(p_[k], s_);
        }
        if (xt_) cudaFreeAsync(xt_, s_);
        if (pt_) cudaFreeAsync(pt_, s_);
        cudaStreamSynchronize(s_);
        cudaStreamDestroy(s_);
    }
    DevicePoints(const DevicePoints&) = delete;
    DevicePoints& operator=(const DevicePoints&) = delete;

    void load(int n, const double* r) override {
        n_[0] = n_[1] = n;
        std::vector<double4> h(n);
        for (int i = 0; i < n; ++i) h[i] = make_double4(r[3 * (size_t)i], r[3 * (size_t)i + 1], r[3 * (size_t)i + 2], 0.0);
        for (int k = 0; k < 2; ++k) {
            x_[k] = dalloc<double4>(n, s_);
            p_[k] = dalloc<int>(n, s_);
            PDMK_CUDA_CHECK(cudaMemcpyAsync(x_[k], h.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, s_));
            k_iota<<<nblk(n), 256, 0, s_>>>(p_[k], n);
        }
        PDMK_CUDA_CHECK(cudaStreamSynchronize(s_));
        PDMK_CUDA_CHECK(cudaGetLastError());
    }

    std::vector<int> add_images(const std::vector<std::array<double, 3>>& shifts, const double* lo,
                                const double* hi) override {
        const int n = n_[0], nsh = (int)shifts.size();
        ExtBox b{};
        for (int d = 0; d < 3; ++d) {
            b.lo[d] = lo[d];
            b.hi[d] = hi[d];
        }
        std::vector<Shift> hs(nsh);
        for (int k = 0; k < nsh; ++k) hs[k] = {shifts[k][0], shifts[k][1], shifts[k][2]};
        std::vector<int> per(nsh, 0);
        if (nsh > 65535) throw std::invalid_argument("too many image shifts");
        if (nsh > 0) {
            Shift* dsh = dalloc<Shift>(nsh, s_);
            int* dcnt = dalloc<int>(nsh, s_);
            PDMK_CUDA_CHECK(cudaMemcpyAsync(dsh, hs.data(), sizeof(Shift) * nsh, cudaMemcpyHostToDevice, s_));
            PDMK_CUDA_CHECK(cudaMemsetAsync(dcnt, 0, sizeof(int) * nsh, s_));
            k_img_count<<<dim3(nblk(n), nsh), 256, 0, s_>>>(x_[0], n, dsh, nsh, b, dcnt);
            PDMK_CUDA_CHECK(cudaGetLastError());
            PDMK_CUDA_CHECK(cudaMemcpyAsync(per.data(), dcnt, sizeof(int) * nsh, cudaMemcpyDeviceToHost, s_));
            PDMK_CUDA_CHECK(cudaFreeAsync(dsh, s_));
            PDMK_CUDA_CHECK(cudaFreeAsync(dcnt, s_));
            PDMK_CUDA_CHECK(cudaStreamSynchronize(s_));
        }
        int64_t nimg = 0;
        for (int c : per) nimg += c;
        if ((int64_t)n + nimg > (int64_t)0x7fffffff) throw std::invalid_argument("too many source images");
        const int64_t na = n + nimg;
        double4* xs = dalloc<double4>(na, s_);
        int* idx = dalloc<int>(nimg, s_);
        int* flag = dalloc<int>(n, s_);
        PDMK_CUDA_CHECK(cudaMemcpyAsync(xs, x_[0], sizeof(double4) * n, cudaMemcpyDeviceToDevice, s_));
        int64_t at = 0;
        for (int k = 0; k < nsh; ++k) {
            if (!per[k]) continue;
            k_img_flag<<<nblk(n), 256, 0, s_>>>(x_[0], n, hs[k], b, flag);
            PDMK_CUDA_CHECK(cudaGetLastError());
            const int64_t tot = exclusive_scan(flag, n, s_);
            if (tot != per[k]) throw std::runtime_error("CUDA error: image count mismatch");
            k_img_write<<<nblk(n), 256, 0, s_>>>(x_[0], n, hs[k], b, flag, xs + n, idx, at);
            PDMK_CUDA_CHECK(cudaGetLastError());
            at += per[k];
        }
        std::vector<int> out(nimg);
        if (nimg) PDMK_CUDA_CHECK(cudaMemcpyAsync(out.data(), idx, sizeof(int) * nimg, cudaMemcpyDeviceToHost, s_));
        PDMK_CUDA_CHECK(cudaFreeAsync(flag, s_));
        PDMK_CUDA_CHECK(cudaFreeAsync(idx, s_));
        PDMK_CUDA_CHECK(cudaFreeAsync(x_[0], s_));
        PDMK_CUDA_CHECK(cudaFreeAsync(p_[0], s_));
        x_[0] = xs;
        p_[0] = dalloc<int>(na, s_);
        k_iota<<<nblk(na), 256, 0, s_>>>(p_[0], na);
        n_[0] = (int)na;
        // scratch for the partitions and orderings, sized for the larger set
        xt_ = dalloc<double4>(na, s_);
        pt_ = dalloc<int>(na, s_);
        PDMK_CUDA_CHECK(cudaStreamSynchronize(s_));
        PDMK_CUDA_CHECK(cudaGetLastError());
        return out;
    }

    std::vector<int> bin0(int s, const double* xelo, double rcinv, const int* m) override {
        const int64_t n = n_[s];
        const int64_t nb0 = (int64_t)m[0] * m[1] * m[2];
        if (nb0 <= 0 || nb0 > ((int64_t)1 << 30)) throw std::invalid_argument("level-0 grid size");
        Grid0 g{};
        for (int d = 0; d < 3; ++d) {
            g.xelo[d] = xelo[d];
            g.m[d] = m[d];
        }
        g.rcinv = rcinv;
        uint32_t* key = dalloc<uint32_t>(n, s_);
        uint32_t* key2 = dalloc<uint32_t>(n, s_);
        int* val = dalloc<int>(n, s_);
        int* val2 = dalloc<int>(n, s_);
        int* cnt = dalloc<int>(nb0, s_);
        PDMK_CUDA_CHECK(cudaMemsetAsync(cnt, 0, sizeof(int) * nb0, s_));
        k_bin_keys<<<nblk(n), 256, 0, s_>>>(x_[s], n, g, key, val, cnt);
        PDMK_CUDA_CHECK(cudaGetLastError());
        int bits = 1;
        while (bits < 32 && ((int64_t)1 << bits) < nb0) ++bits;
        radix_sort(key, val, key2, val2, n, bits, s_);
        k_gather<<<nblk(n), 256, 0, s_>>>(x_[s], p_[s], val, n, xt_, pt_);
        PDMK_CUDA_CHECK(cudaGetLastError());
        PDMK_CUDA_CHECK(cudaMemcpyAsync(x_[s], xt_, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s_));
        PDMK_CUDA_CHECK(cudaMemcpyAsync(p_[s], pt_, sizeof(int) * n, cudaMemcpyDeviceToDevice, s_));
        std::vector<int> ip(nb0 + 1, 0);
        PDMK_CUDA_CHECK(cudaMemcpyAsync(ip.data() + 1, cnt, sizeof(int) * nb0, cudaMemcpyDeviceToHost, s_));
        for (void* p : {(void*)key, (void*)key2, (void*)val, (void*)val2, (void*)cnt}) PDMK_CUDA_CHECK(cudaFreeAsync(p, s_));
        PDMK_CUDA_CHECK(cudaStreamSynchronize(s_));
        for (int64_t b = 0; b < nb0; ++b) ip[b + 1] += ip[b];
        return ip;
    }

    std::vector<std::array<int, 8>> partition(int s, const std::vector<Range>& r) override {
        const int nr = (int)r.size();
        std::vector<std::array<int, 8>> out(nr);
        if (!nr) return out;
        std::vector<RangeD> h(nr);
        for (int k = 0; k < nr; ++k) {
            if (r[k].start < 0 || r[k].count < 0 || (int64_t)r[k].start + r[k].count > n_[s])
                throw std::invalid_argument("partition range outside the point set");
            h[k] = {r[k].start, r[k].count, {r[k].c[0], r[k].c[1], r[k].c[2]}};
        }
        RangeD* d = dalloc<RangeD>(nr, s_);
        int* cnt = dalloc<int>(8 * (int64_t)nr, s_);
        PDMK_CUDA_CHECK(cudaMemcpyAsync(d, h.data(), sizeof(RangeD) * nr, cudaMemcpyHostToDevice, s_));
        k_partition<<<nr, kPartThreads, 0, s_>>>(d, x_[s], p_[s], xt_, pt_, cnt);
        PDMK_CUDA_CHECK(cudaGetLastError());
        PDMK_CUDA_CHECK(cudaMemcpyAsync(out.data(), cnt, sizeof(int) * 8 * nr, cudaMemcpyDeviceToHost, s_));
        PDMK_CUDA_CHECK(cudaFreeAsync(d, s_));
        PDMK_CUDA_CHECK(cudaFreeAsync(cnt, s_));
        PDMK_CUDA_CHECK(cudaStreamSynchronize(s_));
        return out;
    }

    void morton(int s, const std::vector<Leaf>& leaves) override {
        const int nl = (int)leaves.size();
        if (!nl) return;
        std::vector<LeafD> h(nl);
        bool big = false;
        for (int k = 0; k < nl; ++k) {
            const Leaf& L = leaves[k];
            if (L.start < 0 || L.count < 0 || (int64_t)L.start + L.count > n_[s])
                throw std::invalid_argument("leaf range outside the point set");
            h[k] = {L.start, L.count, {L.c[0], L.c[1], L.c[2]}, L.h};
            big = big || L.count > kMortonSmem;
        }
        LeafD* d = dalloc<LeafD>(nl, s_);
        uint64_t* ks = big ? dalloc<uint64_t>(n_[s], s_) : nullptr;
        PDMK_CUDA_CHECK(cudaMemcpyAsync(d, h.data(), sizeof(LeafD) * nl, cudaMemcpyHostToDevice, s_));
        k_morton<<<nl, kMortonThreads, 0, s_>>>(d, x_[s], p_[s], xt_, pt_, ks);
        PDMK_CUDA_CHECK(cudaGetLastError());
        PDMK_CUDA_CHECK(cudaFreeAsync(d, s_));
        if (ks) PDMK_CUDA_CHECK(cudaFreeAsync(ks, s_));
        PDMK_CUDA_CHECK(cudaStreamSynchronize(s_));
    }

    int64_t outside(int s, const std::vector<Leaf>& leaves) override {
        std::vector<LeafD> h;
        for (const Leaf& L : leaves) {
            if (L.count <= 0) continue;
            if (L.start < 0 || (int64_t)L.start + L.count > n_[s])
                throw std::invalid_argument("leaf range outside the point set");
            h.push_back({L.start, L.count, {L.c[0], L.c[1], L.c[2]}, L.h});
        }
        if (h.empty()) return 0;
        const int nl = (int)h.size();
        LeafD* d = dalloc<LeafD>(nl, s_);
        unsigned long long* bad = dalloc<unsigned long long>(1, s_);
        PDMK_CUDA_CHECK(cudaMemcpyAsync(d, h.data(), sizeof(LeafD) * nl, cudaMemcpyHostToDevice, s_));
        PDMK_CUDA_CHECK(cudaMemsetAsync(bad, 0, sizeof(unsigned long long), s_));
        k_outside<<<nl, 128, 0, s_>>>(d, x_[s], bad);
        PDMK_CUDA_CHECK(cudaGetLastError());
        unsigned long long hb = 0;
        PDMK_CUDA_CHECK(cudaMemcpyAsync(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost, s_));
        PDMK_CUDA_CHECK(cudaFreeAsync(d, s_));
        PDMK_CUDA_CHECK(cudaFreeAsync(bad, s_));
        PDMK_CUDA_CHECK(cudaStreamSynchronize(s_));
        return (int64_t)hb;
    }

    void fetch(int s, std::vector<double>& pos, std::vector<int>& perm) override {
        const int64_t n = n_[s];
        std::vector<double4> h(n);
        perm.resize(n);
        PDMK_CUDA_CHECK(cudaMemcpyAsync(h.data(), x_[s], sizeof(double4) * n, cudaMemcpyDeviceToHost, s_));
        PDMK_CUDA_CHECK(cudaMemcpyAsync(perm.data(), p_[s], sizeof(int) * n, cudaMemcpyDeviceToHost, s_));
        PDMK_CUDA_CHECK(cudaStreamSynchronize(s_));
        pos.resize(3 * (size_t)n);
        for (int64_t i = 0; i < n; ++i) {
            pos[3 * i] = h[i].x;
            pos[3 * i + 1] = h[i].y;
            pos[3 * i + 2] = h[i].z;
        }
    }

    int size(int s) const override { return n_[s]; }

  private:
    cudaStream_t s_ = nullptr;
    int n_[2] = {0, 0};
    double4* x_[2] = {nullptr, nullptr};
    int* p_[2] = {nullptr, nullptr};
    double4* xt_ = nullptr;  // partition / ordering scratch (sources' size)
    int* pt_ = nullptr;
};

}  // namespace dev

bool tree_build_on_device(int n, int min_device_points) {
    if (const char* e = std::getenv("PDMK_TREE_BUILD")) {
        if (std::strcmp(e, "host") == 0) return false;
        if (std::strcmp(e, "device") == 0) return true;
    }
    return n >= min_device_points;
}

Plan build_plan_device(const double* cell, int n, const double* pos, int n_digits, int n_per_leaf, int nz,
                       const double* bloch) {
    dev::DevicePoints points;
    return build_plan(cell, n, pos, n_digits, n_per_leaf, nz, bloch, &points);
}

}  // namespace pdmkb
