// FP64 tensor-core (DMMA) forms of the FP64 path's contraction steps (dmma.cu).
#pragma once
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace pdmkb {
namespace dev {

// Real x real step (the child <-> parent translations) of ContractArgs with
// mode kStore or kAdd and structure kDense / kTriUpper / kTriLower, on
// mma.sync.m8n8k4.f64.  Covers ni <= 64, na <= 40 (p <= 38).
bool translate_dmma_supported(int ni, int na);
void launch_translate_dmma(const ContractArgs& a, cudaStream_t s);

// Proxy moments of the FP64 path (launch_c2proxy's sum) on mma.sync.m8n8k4.f64,
// for the orders of 9 and 12 digits (p = 28, 38).
bool c2proxy_dmma_supported(int p);
void launch_c2proxy_dmma(const C2ProxyArgs& a, int p, cudaStream_t s);

}  // namespace dev
}  // namespace pdmkb
