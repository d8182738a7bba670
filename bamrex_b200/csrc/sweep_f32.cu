// FP32-storage instantiations of the sweep kernels.
#include "sweep_pick.cuh"

namespace bamrex {
template const void* pick_sweep_kernel<float>(int, int, int, int, bool);
}  // namespace bamrex
