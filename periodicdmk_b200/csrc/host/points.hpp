// The point-heavy steps of the tree build behind one interface, so that the
// points can live on the host (HostPoints, tree.cpp) or on the GPU
// (DevicePoints, device/tree_build.cu) while the box topology is decided on the
// host by the same code (build_plan).  Both back ends perform the same
// floating-point operations on the same inputs, so they produce the same plan.
//
// Two point sets: 0 = sources (originals, then their lattice images), 1 =
// targets (the originals).  Each set is held in its current sorted order with
// the input index of every sorted point.
#pragma once
#include <array>
#include <cstdint>
#include <vector>

namespace pdmkb {

class PointOps {
  public:
    struct Range {  // a box's points [start, start + count) and its centre
        int start, count;
        double c[3];
    };
    struct Leaf {  // a leaf's points, its centre and half side
        int start, count;
        double c[3];
        double h;
    };
    virtual ~PointOps() = default;
    // Originals: r[3 i + d], i < n (rotated positions, user order).
    virtual void load(int n, const double* r) = 0;
    // Appends to the sources, for each shift in order and each original j in
    // order, the copy r_j + shift when it lies in [lo, hi] on every axis
    // (inclusive); returns the original index of every appended image.
    virtual std::vector<int> add_images(const std::vector<std::array<double, 3>>& shifts, const double lo[3],
                                        const double hi[3]) = 0;
    // Stable counting sort of set s into the level-0 grid of m[0] x m[1] x
    // m[2] boxes: box index ix + m0 (iy + m1 iz) with i_d =
    // clamp((int)((x_d - xelo_d) * rcinv), 0, m_d - 1).  Returns the first
    // sorted point of every box (nbox + 1 entries).
    virtual std::vector<int> bin0(int s, const double xelo[3], double rcinv, const int m[3]) = 0;
    // Stable partition of every range into the octants of its centre (octant
    // bit d set when x_d >= c_d); returns the 8 counts of every range.
    virtual std::vector<std::array<int, 8>> partition(int s, const std::vector<Range>& r) = 0;
    // Reorders every leaf's points by the Morton key of the leaf box (10 bits
    // per axis, q_d = min(1023, max(0, (int)((x_d - (c_d - h)) / (2 h) * 1024)))),
    // stable among equal keys.
    virtual void morton(int s, const std::vector<Leaf>& leaves) = 0;
    // Number of points of the leaves with |x_d - c_d| > h on some axis.
    virtual int64_t outside(int s, const std::vector<Leaf>& leaves) = 0;
    // Sorted positions pos[3 i + d] and sorted -> input index of set s.
    virtual void fetch(int s, std::vector<double>& pos, std::vector<int>& perm) = 0;
    virtual int size(int s) const = 0;
};

}  // namespace pdmkb
