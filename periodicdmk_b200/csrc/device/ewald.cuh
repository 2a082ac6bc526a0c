// Ewald summation on the GPU (ewald.cu).
#pragma once

namespace pdmkb {

struct EwaldInfo {
    double alpha = 0, rcut = 0, kmax = 0;
    int bins[3]{};   // real-space bins per fractional axis
    int modes[3]{};  // reciprocal modes per axis (2 mmax + 1)
    int grid[3]{};   // NUFFT grid
};

// Potentials pot[N] (and the energy, if energy is not null) of N charges q at
// pos[3 i + d] in the cell cell[3 j + i] (component i of lattice vector j);
// s sets the accuracy, erfc(s) ~ e^{-s^2}.  Runs on the current CUDA device,
// synchronously; throws std::invalid_argument on bad input and
// std::runtime_error ("CUDA error" / "cuFFT error") on device failures.
void ewald_gpu(const double* cell, int n, const double* pos, const double* q, double s, double* pot, double* energy,
               EwaldInfo* info = nullptr);

}  // namespace pdmkb
