// Host shim counterpart of the reference's src/device/dg_kernels.hpp: the
// extracted kernel bodies include it; the launchers are not part of the host
// build, so it only pulls in the runtime shim.  TEST INFRASTRUCTURE ONLY.
#ifndef NW_DEVICE_DG_KERNELS_HPP
#define NW_DEVICE_DG_KERNELS_HPP
#include <cstddef>
#include "gpu_runtime.hpp"
#endif
