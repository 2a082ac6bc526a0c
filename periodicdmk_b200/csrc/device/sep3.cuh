// Fused separable p x p x p transform (child <-> parent Chebyshev maps):
// out(a,b,c) (+)= sum Ux(a,i) Uy(b,j) Uz(c,k) in(i,j,k), one CTA per (box, RHS)
// entry with the tensor in shared memory.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace pdmkb {
namespace dev {

// Entry ge = e0 + blockIdx.x is (box eb = ge / rhs, RHS ec = ge % rhs):
// in = in + in_off[eb]*rhs + ec*p^3, out likewise; matrices U_x, U_y, U_z are
// column-major p x p at mat + (mat_off ? mat_off[eb] : 0) + d*p*p.
struct Sep3 {
    const void* in;
    const int64_t* in_off;
    void* out;
    const int64_t* out_off;
    const void* mat;
    const int64_t* mat_off;  // null: mat
    int rhs;
    int64_t e0;
    int accumulate;
    int tri;  // 0 dense; 1 U(a,i) = 0 for i > a (child -> parent); 2 U(a,i) = 0 for i < a (parent -> child)
};

// true if the fused kernel handles (T, p) (the tensor pair fits in shared memory)
template <typename T>
bool sep3_supported(int p);
template <typename T>
void launch_sep3(const Sep3& a, int p, int n_entries, cudaStream_t s);

}  // namespace dev
}  // namespace pdmkb
