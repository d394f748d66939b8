// Host-to-device copies of caller buffers (host interface; see upload.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace fpls {

// Copies `bytes` from the host buffer src to the device buffer dst, ordered
// on stream s. Pageable sources of at least kUploadStagedMin bytes go through
// pinned staging slots: host threads copy each chunk into a slot while the
// previous chunk's DMA runs (a pageable cudaMemcpyAsync moves one chunk at a
// time through the driver's own staging, ~11 GB/s on the B200 hosts). Pinned
// and small sources are one cudaMemcpyAsync. As with a pageable
// cudaMemcpyAsync, src has been read completely when the call returns; the
// DMA of the last chunks may still be running on s.
constexpr size_t kUploadStagedMin = size_t(8) << 20;
void upload_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s);

}  // namespace fpls
