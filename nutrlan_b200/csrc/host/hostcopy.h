// Copies between pageable host memory and device memory at PCIe speed.
//
// A plain cudaMemcpy from pageable memory runs at 11 GB/s host-to-device and
// 17 GB/s device-to-host on a B200 host, a third of what the link moves from
// pinned memory (55 GB/s): the driver stages through a small pinned buffer
// with one CPU thread.  These functions stage through a ring of larger pinned
// buffers instead, fill or drain each buffer with several host threads, and
// keep the DMA engine busy while the threads work on the next buffer.
//
// Both functions are synchronous with respect to the host, like cudaMemcpy on
// pageable memory: on return the host source may be reused (host-to-device)
// or the host destination holds the data (device-to-host).  The copies are
// ordered on `st` after the work already queued there.  Pinned or registered
// host memory and copies below a few MB go straight to cudaMemcpy2DAsync.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace trlb {

// `rows` rows of `width` bytes; `dpitch`/`spitch` are the byte strides of the
// destination and source rows.  kind is cudaMemcpyHostToDevice or
// cudaMemcpyDeviceToHost.  Returns the first CUDA error, or cudaSuccess.
cudaError_t host_copy_2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width, size_t rows,
                         cudaMemcpyKind kind, cudaStream_t st);

inline cudaError_t host_copy(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind, cudaStream_t st) {
    return host_copy_2d(dst, bytes, src, bytes, bytes, 1, kind, st);
}

// Frees the pinned staging buffers and stops the copy threads (they are
// created again by the next large copy).
void release_staging();

}  // namespace trlb
