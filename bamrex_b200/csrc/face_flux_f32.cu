// FP32-storage flux-register face kernels (see face_flux.cuh).
#include "face_flux.cuh"

namespace bamrex {
template const void* pick_register_kernel<float>(int, int, int, int);
}
