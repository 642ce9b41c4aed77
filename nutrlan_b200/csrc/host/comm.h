// Communicators for block-row solves over several GPUs (one rank per GPU).
//
// The reference's parallel build splits every vector into contiguous row
// blocks, one per MPI rank, and sums the partial dot products over the ranks
// (trl_g_sum, trl_g_dot_, SRC/trl_comm_mpi.c); the user's operator exchanges
// whatever it needs itself.  Here the same operations exist for two
// transports:
//   * NCCL (libnccl.so.2 loaded at run time): device buffers, queued on the
//     solver's stream, no host round trip;
//   * a host callback (any allreduce on host doubles, e.g. MPI_Allreduce or
//     a gloo process group): device values are staged through pinned host
//     memory around each call.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <vector>

namespace trlb {

enum { kOpSum = 0, kOpMax = 1, kOpMin = 2 };

class Comm {
   public:
    virtual ~Comm() {}
    int rank = 0, size = 1;
    // In-place sum over the ranks of n doubles of device memory, ordered on st.
    virtual int sum_device(double *d, size_t n, cudaStream_t st) = 0;
    // In-place sum / max / min over the ranks of n host doubles (blocking).
    virtual int reduce_host(double *h, size_t n, int op) = 0;
    // Point-to-point exchange of device doubles, ordered on st: to every peer
    // p, send[soff[p] .. soff[p+1]) goes out and recv[roff[p] .. roff[p+1])
    // comes in.  `counts` is the size x size matrix (row = sender) of all
    // ranks' message lengths, which the host transport needs.
    virtual int exchange(const double *send, const std::vector<long> &soff, double *recv,
                         const std::vector<long> &roff, const std::vector<long> &counts, cudaStream_t st) = 0;
};

}  // namespace trlb

// Opaque handle of the C API.
struct trlx_comm {
    trlb::Comm *impl = nullptr;
};
