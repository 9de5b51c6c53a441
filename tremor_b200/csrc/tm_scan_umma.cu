// Split-BF16 tensor-core contraction (tcgen05). Placeholder until the kernel lands:
// reports "not supported" so the FP32 kernel runs.
#include "tm_epilogue.cuh"

namespace tmb {

bool umma_supported(int, int, uint64_t) { return false; }

cudaError_t launch_scan_umma(const ScanArgs &, cudaStream_t) { return cudaErrorNotSupported; }

} // namespace tmb
