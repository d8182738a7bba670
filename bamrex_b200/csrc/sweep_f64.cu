// FP64 (drop-in) instantiations of the sweep kernels.
#include "sweep_pick.cuh"

namespace bamrex {
template const void* pick_sweep_kernel<double>(int, int, int, int, bool);
}  // namespace bamrex
