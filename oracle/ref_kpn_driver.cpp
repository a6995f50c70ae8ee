// ref_kpn_driver.cpp - exposes the reference's KPN CUDA functions as PyTorch operators (TEST
// INFRASTRUCTURE ONLY).  modules/kpn_module/src/Kernel.cu and perPixelKernel.cpp are compiled unmodified
// from the reference tree (oracle/ref_build.py); the reference registers only per_pixel_kernel::forward,
// so getInvIterBaseCuda is registered here as ref_kpn::inv_iter_base.
#include <torch/script.h>

#include "perPixelKernel.hpp"

namespace {
torch::Tensor inv_iter_base(torch::Tensor x, torch::Tensor low_res_pred, torch::Tensor low_res_x, torch::Tensor prev,
                            torch::Tensor fused_weights, bool use_previous, int64_t kernel_size) {
    return getInvIterBaseCuda(x, low_res_pred, low_res_x, prev, fused_weights, use_previous, (int)kernel_size);
}
}  // namespace

TORCH_LIBRARY(ref_kpn, m) { m.def("inv_iter_base", inv_iter_base); }
