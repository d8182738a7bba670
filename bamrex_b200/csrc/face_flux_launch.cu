// Launch of the flux-register face kernels: one thread per register slot.
#include <cuda_runtime.h>

#include "level_impl.h"

namespace bamrex {

template <typename T>
const void* pick_register_kernel(int D, int dir, int method, int fast_lim);
extern template const void* pick_register_kernel<double>(int, int, int, int);
extern template const void* pick_register_kernel<float>(int, int, int, int);

cudaError_t launch_register_faces(int D, int dir, int method, bool fp32, const Consts& k, const FabDev* in,
                                  const RegisterTask& t, int NC, double dt, double dx_dir, double scale,
                                  const StepScalars* scal, double area1, double area2, cudaStream_t s,
                                  const SweepBox* xsw)
{
    (void)NC;
    const int lim = fast_limiter(D, method, k);
    const void* fn = fp32 ? pick_register_kernel<float>(D, dir, method, lim)
                          : pick_register_kernel<double>(D, dir, method, lim);
    if (!fn) return cudaErrorInvalidValue;
    if (t.nslots <= 0) return cudaSuccess;
    constexpr int threads = 128;  // kRegThreads
    const int grid = (t.nslots + threads - 1) / threads;
    RegisterTask tt = t;
    Consts kc = k;
    void* args[] = { (void*)&in, (void*)&tt, (void*)&kc, (void*)&dt, (void*)&dx_dir, (void*)&scale,
                     (void*)&scal, (void*)&area1, (void*)&area2, (void*)&xsw };
    return cudaLaunchKernel(fn, dim3(grid), dim3(threads), args, 0, s);
}

}  // namespace bamrex
