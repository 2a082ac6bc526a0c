// Per-evaluation stage timing (replaces the reference's
// cpp/include/pdmk/eval_timing.hpp:10-20; same fields and meaning).  The three
// stage times are measured on the GPU with CUDA events and partition the
// device time of one evaluate.
#pragma once

namespace pdmk {

struct EvalTiming {
    double nufft_ms = 0.0;   ///< periodic far field
    double dmk_ms = 0.0;     ///< charge gather + upward pass + plane-wave downward pass (incl. leaf evaluation)
    double direct_ms = 0.0;  ///< residual near field + self correction + desort
    double build_ms = 0.0;   ///< 0 for 3D: the tree is built once at construction
};

}  // namespace pdmk
