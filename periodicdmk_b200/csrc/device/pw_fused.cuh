// Fused three-step plane-wave transforms for blocks of RHS (one CTA per (box, RHS)).
#pragma once
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace pdmkb {
namespace dev {

// Entry ge = e0 + blockIdx.x is (box eb = ge / rhs, RHS ec = ge % rhs).
// Outgoing: in = proxy_up + in_off[eb]*rhs + ec*p^3 (real), out = pw + out_off[eb]*rhs + ec*M (complex, stored).
// Incoming: in = pw_in + blockIdx.x*in_stride (complex), out = proxy_down + out_off[eb]*rhs + ec*p^3 (real, +=).
struct PwFused {
    const void* in;
    const int64_t* in_off;
    int64_t in_stride;
    void* out;
    const int64_t* out_off;
    const void* mat_a;  // outgoing: poly2pw (n x p); incoming: pw2polyT (p x n)
    const void* mat_b;  // outgoing: poly2pw_half (n2 x p); incoming: pw2polyTw (p x n2)
    int rhs;
    int64_t e0;
};

// true for the (p, n, n2) of 3 and 6 digits when the intermediates fit in shared memory
template <typename T>
bool pw_fused_supported(int p, int n, int n2);
template <typename T>
void launch_pw_out_fused(const PwFused& a, int p, int n, int n2, int n_entries, cudaStream_t s);
template <typename T>
void launch_pw_in_fused(const PwFused& a, int p, int n, int n2, int n_entries, cudaStream_t s);

}  // namespace dev
}  // namespace pdmkb
