/*
 * kernels_aux.cu - the adjoint passes and the preview renderers, which share
 * the sampling, tracing and shading device code of kernels_device.cuh.
 */
#include "kernels_device.cuh"

namespace ssolb {

#include "adjoint.cuh"
#include "draw.cuh"

} /* namespace ssolb */
