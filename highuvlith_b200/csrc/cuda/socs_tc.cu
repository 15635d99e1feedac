// Tensor-core (split-BF16x3 tcgen05) form of the SOCS sum.  Placeholder
// until the tcgen05 kernels land: reports the form as unsupported.
#include <cuda_runtime.h>

#include "../engine.hpp"

namespace huv_launch {
cudaError_t tc_prepare(huv::TcState&, const huv::DeviceSet&, int, int, cudaStream_t) { return cudaErrorNotSupported; }
cudaError_t tc_socs(const huv::TcState&, const huv::DeviceSet&, const float2*, int, int, float, float,
                    const float*, float*, void*, cudaStream_t) {
  return cudaErrorNotSupported;
}
size_t tc_workspace_bytes(const huv::DeviceSet&, int, int) { return 0; }
void tc_release(huv::TcState& tc) { tc = huv::TcState(); }
}  // namespace huv_launch

namespace huv {
bool Engine::tc_supported(const DeviceSet&, int) const { return false; }
void Engine::run_tc_form(const huv_batch&, DeviceSet&, int, float*, cudaStream_t) {
  throw Error(HUV_ERR_UNSUPPORTED, "TC form not available in this build");
}
}  // namespace huv
