// Launch helper of the general-layout Gram-Schmidt projection kernel
// (gdot.cu): wrk = [v1 v2]^H rr for any device pointers / leading dimensions.
#pragma once

#include <cuda_runtime.h>

namespace trlb {

// Grid for n rows: number of blocks (<= max_blocks) and rows per block.
int gdot_grid(int n, int max_blocks, long *chunk);

// part must hold nblocks * (m1 + m2) elements; *ticket must be zero (the
// kernel leaves it zero).
template <class C>
int launch_gdot(int nrow, const C *v1, int ld1, int m1, const C *v2, int ld2, int m2, const C *rr, C *wrk,
                C *part, unsigned *ticket, int nblocks, long chunk, cudaStream_t st);

}  // namespace trlb
