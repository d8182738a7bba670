// FP32-storage instantiations of the TMA-staged sweeps.
#include "sweep_tma_pick.cuh"

namespace bamrex {
template const void* pick_tma_kernel<float>(int, int, int, bool, bool);
}  // namespace bamrex
