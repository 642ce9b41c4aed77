// Cooperative kernel for runs of speculative Lanczos steps on short vectors
// (coop.cu).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

struct trlx_operator;

namespace trlb {

template <class C>
struct CoopArgs {
    int nrow;
    long n_pad;
    long chunk;    // rows per block (multiple of 64)
    int maxcols;   // capacity of h (basis columns)
    const long long *rp;
    const int *ci;
    const C *va;
    C *const *cols;  // basis column table
    int j0, S;       // steps j0 + 1 .. j0 + S
    double beta0;    // beta of the first step's recurrence
    double *log;     // [s][4]: alpha, |r|^2 before, |h|^2, |r|^2 after (s = 1..S)
    C *part;         // (maxcols + 2) * G partials
    C *h;            // maxcols coefficients
};

// Runs S steps (CSR operators only).  Returns 0, -1 if the cooperative
// kernel does not apply (operator format, device, sizes), -1001 on a CUDA
// error.
template <class C>
int launch_spec_coop(const trlx_operator *A, C *const *cols, long n_pad, int maxcols, int j0, int S, double beta0,
                     double *log, C *part, long part_elems, C *h, cudaStream_t st);

}  // namespace trlb
