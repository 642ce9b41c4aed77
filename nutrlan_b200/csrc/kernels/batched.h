// Device-side types of the persistent batched solver (batched.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace trlb {
namespace batched {

enum Format { kFormatStencil5 = 0, kFormatCSR = 1 };

// One problem of the batch (offsets index the shared device arrays).
struct Problem {
    int n;               // rows
    int L;               // grid side of the 5-point stencil (n = L * L)
    int ld;              // basis leading dimension (n rounded up to 32)
    int pad;
    long long diag_off;  // stencil: diagonal potential d[0..n) (operator 4 + d, -1 couplings)
    long long rp_off;    // CSR: row pointers (n + 1, local entry indices)
    long long ent_off;   // CSR: first entry in col/val
    long long basis_off; // basis ((maxlan + 1) * ld doubles)
    long long evec_off;  // output eigenvectors (ned * n doubles)
    long long start_off; // caller start vector (n doubles) or -1: seeded random
};

struct Params {
    int nprob, ned, maxlan, lohi, restart, maxmv, format;
    double tol;
    unsigned long long seed;
    const Problem *probs;
    const int *order;  // solve order (largest first)
    const double *diag;
    const long long *row_ptr;
    const int *col;
    const double *val;
    const double *start;
    double *basis;
    double *evec;
    double *eval;  // nprob * ned
    double *res;   // nprob * ned
    int *info_out; // nprob * 4: stat, nec, matvec, nloop
    unsigned *queue; // one counter per phase (zero before the launch)
    // Threads per CTA of the launch: 1024 (groups of 1024, 512 or 256) or
    // 512 (groups of 512, 256 or 128; twice the registers per thread).
    int cta;
    // Phases over order[]: problems order[phase_begin[f] .. phase_end[f])
    // are solved by groups of phase_threads[f] threads.
    int nphases;
    int phase_threads[4];
    int phase_begin[4];
    int phase_end[4];
    size_t smem_total;  // dynamic shared memory of the launch (set by launch())
};

size_t group_bytes(int maxlan);
size_t smem_bytes(int maxlan, int min_threads, int cta);
int launch(const Params &P, int blocks, cudaStream_t st);
int max_blocks_per_sm(int min_threads, int maxlan, int cta);

}  // namespace batched
}  // namespace trlb
