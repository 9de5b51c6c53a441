// Split-BF16 tensor-core contraction (tcgen05). Placeholder until the kernel lands:
// reports "not supported" so the FP32 kernel runs.
#include "tm_epilogue.cuh"

namespace tmb {

cudaError_t launch_scan_umma(const ScanArgs &, cudaStream_t, bool *supported)
{
    *supported = false;
    return cudaSuccess;
}

} // namespace tmb
