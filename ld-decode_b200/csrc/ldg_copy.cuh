// Copies done by SMs through host-mapped pinned memory.  A small transfer
// that the host waits on (a run count, run lists, field plans, TBC
// descriptors) issued as cudaMemcpyAsync queues on the copy engines behind
// the bulk capture and output copies of an end-to-end pipeline; a kernel
// that reads or writes the pinned buffer directly over PCIe does not.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ldg {

// Device-accessible address of `p`: device memory as is, pinned host memory
// through its mapping; nullptr for pageable host memory (or on error).
void* device_view(const void* p);

// dst[0, nbytes) = src[0, nbytes) by a kernel on `stream`; both are
// device-accessible addresses (device_view).
cudaError_t sm_copy(void* dst, const void* src, size_t nbytes, cudaStream_t stream);

}  // namespace ldg
