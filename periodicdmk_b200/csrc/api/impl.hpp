// Private state behind pdmk::PeriodicDMKTreeT (host plan + device tree).
#pragma once
#include <memory>

#include "../device/device_tree.hpp"
#include "../host/plan.hpp"
#include "pdmk/periodic_dmk.hpp"

namespace pdmk {

template <typename Real, int DIM>
struct PeriodicDMKTreeT<Real, DIM>::Impl {
    std::unique_ptr<pdmkb::Plan> plan;
    std::unique_ptr<pdmkb::DeviceTree> dev;
    bool single = false;
};

}  // namespace pdmk
