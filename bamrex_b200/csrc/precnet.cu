// Learned preconditioner for the pressure Helmholtz solve: a small 2D
// convolutional network M(r) ~ A^{-1} r with BF16 weights and FP32
// accumulation, its training (forward, backward and Adam kernels written
// here), and a flexible GMRES solve that applies it, falling back to the
// plain BiCGStab/multigrid solve when it does not reach the tolerance.
// This component has no counterpart in the reference; the solve it
// accelerates is setup_pressure_op / solve_pressure
// (Source/IMEX/IMEX_O1.cpp:570-640).
//
// Network (all convolutions 3x3, periodic padding, ReLU after every
// convolution except the last; C = 16 channels):
//   level 0 (n):     conv(2->C), conv(C->C)                       -> h0
//   level 1 (n/2):   avgpool(h0), conv, conv                      -> h1
//   level 2 (n/4):   avgpool(h1), conv, conv                      -> h2
//   level 3 (n/8):   avgpool(h2), conv, conv                      -> h3
//   up:              conv(up(h3) + h2) -> g2; conv(up(g2) + h1) -> g1;
//                    conv(up(g1) + h0) -> g0; conv(C->1)(g0)     -> out
// Input channels: r / s (s = RMS of r) and log(beta) on cells; the
// correction is e = out * s * dx^2 / B.  Activations are FP32 in NCHW
// layout; the forward uses weights rounded to BF16.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "bamrex_cuda.h"
#include "level_impl.h"

using namespace bamrex;

namespace {

constexpr int C = 16;
constexpr int kT = 256;
constexpr int kNLevels = 4;

enum Kind { K_CONV = 0, K_POOL = 1, K_UPADD = 2 };

struct Layer {
    int kind;
    int in, in2, out;   // activation ids (in2: skip input of K_UPADD)
    int cin, cout;
    int relu;
    int w_off, b_off;   // parameter offsets (conv)
};

struct Act {
    int c, lev;         // channels, level (size n >> lev)
    size_t off;         // float offset in the activation arena (batch-major)
};

// ------------------------------------------------------------------ kernels
__device__ __forceinline__ int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// y[b][co][p] = bias[co] + sum_{ci,tap} w[co][ci][tap] x[b][ci][p + tap].
// Weights are staged in shared memory as [tap][ci][co] so the COUT weights
// of one (tap, ci) are contiguous (vector loads); taps and input channels
// are loops, the COUT accumulators stay in registers.
template <int CIN, int COUT>
__global__ void __launch_bounds__(kT) conv_fwd_kernel(const float* __restrict__ x, float* __restrict__ y,
                                                      const float* __restrict__ w, const float* __restrict__ bias,
                                                      int H, int W, int batch, int relu)
{
    __shared__ __align__(16) float sw[9 * CIN * COUT];
    __shared__ float sb[COUT];
    for (int q = threadIdx.x; q < COUT * CIN * 9; q += blockDim.x) {
        const int co = q / (CIN * 9), ci = (q / 9) % CIN, tap = q % 9;
        sw[(tap * CIN + ci) * COUT + co] = w[q];
    }
    for (int q = threadIdx.x; q < COUT; q += blockDim.x) sb[q] = bias[q];
    __syncthreads();
    const long long HW = (long long)H * W;
    const long long total = HW * batch;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / HW);
        const int p = (int)(t % HW);
        const int i = p % W, j = p / W;
        const float* xb = x + (long long)b * CIN * HW;
        float acc[COUT];
#pragma unroll
        for (int co = 0; co < COUT; ++co) acc[co] = sb[co];
#pragma unroll 1
        for (int tap = 0; tap < 9; ++tap) {
            const int ii = wrap(i + tap % 3 - 1, W), jj = wrap(j + tap / 3 - 1, H);
            const float* xq = xb + (long long)jj * W + ii;
            const float* wt = sw + tap * CIN * COUT;
#pragma unroll 2
            for (int ci = 0; ci < CIN; ++ci) {
                const float v = __ldg(xq + (long long)ci * HW);
                const float* wc = wt + ci * COUT;
#pragma unroll
                for (int co = 0; co < COUT; ++co) acc[co] = fmaf(wc[co], v, acc[co]);
            }
        }
        float* yb = y + (long long)b * COUT * HW;
#pragma unroll
        for (int co = 0; co < COUT; ++co) yb[(long long)co * HW + p] = relu ? fmaxf(acc[co], 0.0f) : acc[co];
    }
}

// dx[b][ci][p] += sum_{co,tap} w[co][ci][tap] g[b][co][p - tap], g = dy * relu'(y).
// Weights staged as [tap][co][ci].
template <int CIN, int COUT>
__global__ void __launch_bounds__(kT) conv_bwd_data_kernel(const float* __restrict__ dy, const float* __restrict__ y,
                                                           const float* __restrict__ w, float* __restrict__ dx, int H,
                                                           int W, int batch, int relu)
{
    __shared__ __align__(16) float sw[9 * COUT * CIN];
    for (int q = threadIdx.x; q < COUT * CIN * 9; q += blockDim.x) {
        const int co = q / (CIN * 9), ci = (q / 9) % CIN, tap = q % 9;
        sw[(tap * COUT + co) * CIN + ci] = w[q];
    }
    __syncthreads();
    const long long HW = (long long)H * W;
    const long long total = HW * batch;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / HW);
        const int p = (int)(t % HW);
        const int i = p % W, j = p / W;
        const float* dyb = dy + (long long)b * COUT * HW;
        const float* yb = y + (long long)b * COUT * HW;
        float acc[CIN];
#pragma unroll
        for (int ci = 0; ci < CIN; ++ci) acc[ci] = 0.0f;
#pragma unroll 1
        for (int tap = 0; tap < 9; ++tap) {
            // output pixel o with o + tap_offset = p
            const int ii = wrap(i - (tap % 3 - 1), W), jj = wrap(j - (tap / 3 - 1), H);
            const long long q = (long long)jj * W + ii;
            const float* wt = sw + tap * COUT * CIN;
#pragma unroll 2
            for (int co = 0; co < COUT; ++co) {
                float g = __ldg(dyb + (long long)co * HW + q);
                if (relu && !(__ldg(yb + (long long)co * HW + q) > 0.0f)) g = 0.0f;
                const float* wc = wt + co * CIN;
#pragma unroll
                for (int ci = 0; ci < CIN; ++ci) acc[ci] = fmaf(wc[ci], g, acc[ci]);
            }
        }
        float* dxb = dx + (long long)b * CIN * HW;
#pragma unroll
        for (int ci = 0; ci < CIN; ++ci) dxb[(long long)ci * HW + p] += acc[ci];
    }
}

// The 16 -> 16 channel convolution on the tensor cores (inference):
// implicit GEMM with M = pixels, N = 16 output channels, K = 9 taps x 16
// input channels, mma.sync m16n8k16 with BF16 operands and FP32
// accumulators.  A block of 4 warps takes a tile of 4 rows x 32 pixels; the
// input rows the taps read (6 rows x 34 pixels x 16 channels) are staged in
// shared memory as BF16, pixel-major with a 24-element pixel stride so the
// fragment loads of a warp hit 32 distinct banks.  Each warp keeps the
// weight fragments of all 9 taps in registers and computes its row as two
// m16 tiles x two n8 tiles.  Requires W % 32 == 0 and H % 4 == 0.
constexpr int kMmaTW = 32, kMmaTH = 4, kMmaPS = 24;

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi)
{
    const unsigned l = __bfloat16_as_ushort(__float2bfloat16_rn(lo));
    const unsigned h = __bfloat16_as_ushort(__float2bfloat16_rn(hi));
    return l | (h << 16);
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__global__ void __launch_bounds__(128) conv16_mma_kernel(const float* __restrict__ x, float* __restrict__ y,
                                                         const float* __restrict__ w, const float* __restrict__ bias,
                                                         int H, int W, int batch, int relu)
{
    __shared__ __align__(16) __nv_bfloat16 xs[(kMmaTH + 2) * (kMmaTW + 2) * kMmaPS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    // weight fragments: B[k = ci][n = co] for every tap and both n8 tiles
    unsigned bw[9][2][2];
#pragma unroll
    for (int tap = 0; tap < 9; ++tap)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
            const int co = nt * 8 + g;
            bw[tap][nt][0] = pack_bf16(w[(co * C + 2 * t) * 9 + tap], w[(co * C + 2 * t + 1) * 9 + tap]);
            bw[tap][nt][1] = pack_bf16(w[(co * C + 2 * t + 8) * 9 + tap], w[(co * C + 2 * t + 9) * 9 + tap]);
        }
    float bv[2][2];
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
        bv[nt][0] = bias[nt * 8 + 2 * t];
        bv[nt][1] = bias[nt * 8 + 2 * t + 1];
    }
    const long long HW = (long long)H * W;
    const int tx = W / kMmaTW, ty = H / kMmaTH;
    const long long ntiles = (long long)batch * tx * ty;
    constexpr int SR = kMmaTH + 2, SC = kMmaTW + 2;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int b = (int)(tile / ((long long)tx * ty));
        const int rem = (int)(tile % ((long long)tx * ty));
        const int j0 = (rem / tx) * kMmaTH, i0 = (rem % tx) * kMmaTW;
        const float* xb = x + (long long)b * C * HW;
        __syncthreads();  // the previous tile's fragments are consumed
        for (int q = threadIdx.x; q < C * SR * SC; q += blockDim.x) {
            const int ci = q / (SR * SC), r = (q / SC) % SR, c = q % SC;
            const int jj = wrap(j0 + r - 1, H), ii = wrap(i0 + c - 1, W);
            xs[(r * SC + c) * kMmaPS + ci] = __float2bfloat16_rn(xb[(long long)ci * HW + (long long)jj * W + ii]);
        }
        __syncthreads();
        float acc[2][2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                acc[mt][nt][0] = acc[mt][nt][2] = bv[nt][0];
                acc[mt][nt][1] = acc[mt][nt][3] = bv[nt][1];
            }
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
            const int dy = tap / 3, dx = tap % 3;  // smem row warp + dy, column pixel + dx
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const __nv_bfloat16* base = xs + ((warp + dy) * SC + mt * 16 + dx) * kMmaPS;
                unsigned a[4];
                a[0] = *reinterpret_cast<const unsigned*>(base + g * kMmaPS + 2 * t);
                a[1] = *reinterpret_cast<const unsigned*>(base + (g + 8) * kMmaPS + 2 * t);
                a[2] = *reinterpret_cast<const unsigned*>(base + g * kMmaPS + 2 * t + 8);
                a[3] = *reinterpret_cast<const unsigned*>(base + (g + 8) * kMmaPS + 2 * t + 8);
#pragma unroll
                for (int nt = 0; nt < 2; ++nt) mma_bf16_16816(acc[mt][nt], a, bw[tap][nt][0], bw[tap][nt][1]);
            }
        }
        float* yb = y + (long long)b * C * HW + (long long)(j0 + warp) * W + i0;
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                const int p0 = mt * 16 + g, co = nt * 8 + 2 * t;
                float v[4] = { acc[mt][nt][0], acc[mt][nt][1], acc[mt][nt][2], acc[mt][nt][3] };
                if (relu)
#pragma unroll
                    for (int e = 0; e < 4; ++e) v[e] = fmaxf(v[e], 0.0f);
                yb[(long long)co * HW + p0] = v[0];
                yb[(long long)(co + 1) * HW + p0] = v[1];
                yb[(long long)co * HW + p0 + 8] = v[2];
                yb[(long long)(co + 1) * HW + p0 + 8] = v[3];
            }
    }
}

// Partial weight gradients.  Work is split into tiles of one row segment
// (TW pixels) of one sample; each block loops over tiles, stages the masked
// output gradient g = dy * relu'(y) and the three input rows the 3x3 taps
// read in shared memory, and each thread accumulates a fixed set of entries
// (weights [co][ci][tap], then biases).  part[block][entry]; the blocks'
// partials are added in a fixed order afterwards.
constexpr int kTW = 128;
template <int CIN, int COUT>
__global__ void __launch_bounds__(kT) conv_bwd_weight_kernel(const float* __restrict__ dy, const float* __restrict__ y,
                                                             const float* __restrict__ x, float* __restrict__ part,
                                                             int H, int W, int batch, int relu, int TW)
{
    constexpr int NW = COUT * CIN * 9 + COUT;
    constexpr int PER = (NW + kT - 1) / kT;
    __shared__ float sg[COUT][kTW];
    __shared__ float sx[CIN][3][kTW + 2];
    const long long HW = (long long)H * W;
    const int segs = W / TW;  // TW divides W, TW <= kTW
    const long long ntiles = (long long)batch * H * segs;
    float acc[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) acc[q] = 0.0f;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int seg = (int)(tile % segs);
        const int j = (int)((tile / segs) % H);
        const int b = (int)(tile / ((long long)segs * H));
        const int i0 = seg * TW;
        for (int q = threadIdx.x; q < COUT * TW; q += blockDim.x) {
            const int co = q / TW, t = q % TW;
            const long long o = (long long)b * COUT * HW + (long long)co * HW + (long long)j * W + i0 + t;
            float g = dy[o];
            if (relu && !(y[o] > 0.0f)) g = 0.0f;
            sg[co][t] = g;
        }
        for (int q = threadIdx.x; q < CIN * 3 * (TW + 2); q += blockDim.x) {
            const int ci = q / (3 * (TW + 2)), r = (q / (TW + 2)) % 3, t = q % (TW + 2);
            const int jj = wrap(j + r - 1, H), ii = wrap(i0 + t - 1, W);
            sx[ci][r][t] = x[(long long)b * CIN * HW + (long long)ci * HW + (long long)jj * W + ii];
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int e = threadIdx.x + q * kT;
            if (e >= NW) break;
            float a = acc[q];
            if (e < COUT * CIN * 9) {
                const int co = e / (CIN * 9), ci = (e / 9) % CIN, tap = e % 9;
                const int di = tap % 3, dj = tap / 3;  // x column t + di - 1, row j + dj - 1
                for (int t = 0; t < TW; ++t) a = fmaf(sg[co][t], sx[ci][dj][t + di], a);
            } else {
                const int co = e - COUT * CIN * 9;
                for (int t = 0; t < TW; ++t) a += sg[co][t];
            }
            acc[q] = a;
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int e = threadIdx.x + q * kT;
        if (e < NW) part[(long long)blockIdx.x * NW + e] = acc[q];
    }
}

// grad[e] = sum over blocks of part (fixed order)
__global__ void sum_parts_kernel(const float* __restrict__ part, int nblocks, int nw, float* __restrict__ grad)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nw; e += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int k = 0; k < nblocks; ++k) s += part[(long long)k * nw + e];
        grad[e] = s;
    }
}

// Forward pool and upsample-add walk rows over blocks and the pixels of a
// row over threads (one division per row).
__global__ void pool_fwd_kernel(const float* __restrict__ x, float* __restrict__ y, int c, int H, int W, int batch)
{
    const int h = H / 2, w = W / 2;
    const long long rows = (long long)batch * c * h;
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
        const long long plane = row / h;
        const int j = (int)(row - plane * h);
        const float* x0 = x + (plane * H + 2 * j) * (long long)W;
        const float* x1 = x0 + W;
        float* yr = y + row * w;
        for (int i = threadIdx.x; i < w; i += blockDim.x)
            yr[i] = 0.25f * (x0[2 * i] + x0[2 * i + 1] + x1[2 * i] + x1[2 * i + 1]);
    }
}

__global__ void pool_bwd_kernel(const float* __restrict__ dy, float* __restrict__ dx, int c, int H, int W, int batch)
{
    const long long total = (long long)batch * c * H * W;
    const int h = H / 2, w = W / 2;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % W), j = (int)((t / W) % H);
        const long long plane = t / ((long long)H * W);
        dx[t] += 0.25f * dy[plane * h * w + (j / 2) * w + i / 2];
    }
}

// y = up(a) + s, a at half resolution
__global__ void upadd_fwd_kernel(const float* __restrict__ a, const float* __restrict__ s, float* __restrict__ y, int c,
                                 int H, int W, int batch)
{
    const int h = H / 2, w = W / 2;
    const long long rows = (long long)batch * c * H;
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
        const long long plane = row / H;
        const int j = (int)(row - plane * H);
        const float* ar = a + (plane * h + j / 2) * (long long)w;
        const float* sr = s + row * W;
        float* yr = y + row * W;
        for (int i = threadIdx.x; i < W; i += blockDim.x) yr[i] = ar[i / 2] + sr[i];
    }
}

__global__ void upadd_bwd_kernel(const float* __restrict__ dy, float* __restrict__ da, float* __restrict__ ds, int c,
                                 int H, int W, int batch)
{
    const int h = H / 2, w = W / 2;
    const long long total = (long long)batch * c * h * w;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % w), j = (int)((t / w) % h);
        const long long plane = t / ((long long)h * w);
        const float* d = dy + plane * H * W;
        da[t] += d[(2 * j) * W + 2 * i] + d[(2 * j) * W + 2 * i + 1] + d[(2 * j + 1) * W + 2 * i] +
                 d[(2 * j + 1) * W + 2 * i + 1];
    }
    const long long full = (long long)batch * c * H * W;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < full; t += (long long)gridDim.x * blockDim.x)
        ds[t] += dy[t];
}

__global__ void round_bf16_kernel(const float* __restrict__ src, float* __restrict__ dst, int n)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
        dst[q] = __bfloat162float(__float2bfloat16_rn(src[q]));
}

// The training loss is the residual the network leaves, in the operator's
// own norm: with d = out - target and A_beta the periodic beta-weighted
// Laplacian of the normalised operator (face beta = mean of the two cells,
// beta = exp(input channel 1)), loss_b = ||A_beta d||^2 / HW (||A_beta
// target||^2 = ||r / rms(r)||^2 = HW up to the tiny a-term).  Every frequency
// of the residual weighs the same, which is what a preconditioner needs.
// mode 0: q = A_beta (o - t); mode 1: g = 2 A_beta q / (HW batch)
__global__ void abeta_kernel(const float* __restrict__ in, const float* __restrict__ o, const float* __restrict__ t,
                             float* __restrict__ dst, int H, int W, int batch, int mode)
{
    const long long HW = (long long)H * W;
    const long long total = HW * batch;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(q / HW);
        const int p = (int)(q % HW);
        const int i = p % W, j = p / W;
        const float* lb = in + (long long)b * 2 * HW + HW;
        const float* ob = o + (long long)b * HW;
        const float* tb = mode == 0 ? t + (long long)b * HW : nullptr;
        auto val = [&](int ii, int jj) {
            const long long k = (long long)jj * W + ii;
            return mode == 0 ? ob[k] - tb[k] : ob[k];
        };
        const float bc = __expf(lb[p]);
        const float dc = val(i, j);
        float acc = 0.0f;
        const int nb[4][2] = { { wrap(i - 1, W), j }, { wrap(i + 1, W), j }, { i, wrap(j - 1, H) }, { i, wrap(j + 1, H) } };
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const float bf = 0.5f * (bc + __expf(lb[(long long)nb[f][1] * W + nb[f][0]]));
            acc += bf * (dc - val(nb[f][0], nb[f][1]));
        }
        dst[q] = mode == 0 ? acc : 2.0f * acc / (float)(HW * batch);
    }
}

__global__ void sumsq_kernel(const float* __restrict__ q, long long n, double* __restrict__ part)
{
    __shared__ double red[kT];
    double acc = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        acc += (double)q[t] * (double)q[t];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                            int n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const float gq = g[q];
        m[q] = b1 * m[q] + (1.0f - b1) * gq;
        v[q] = b2 * v[q] + (1.0f - b2) * gq * gq;
        const float mh = m[q] / c1, vh = v[q] / c2;
        w[q] -= lr * mh / (sqrtf(vh) + eps);
    }
}

int gridn(long long n) { return (int)std::max(1LL, std::min((n + kT - 1) / kT, (long long)device_sm_count() * 16)); }

}  // namespace

struct bamrex_precnet {
    int ny = 0, nx = 0, batch = 0;
    std::vector<Layer> layers;
    std::vector<Act> acts;
    int nparams = 0;
    float* d_w = nullptr;      // FP32 master weights
    float* d_wb = nullptr;     // BF16-rounded copy used by the forward
    float* d_g = nullptr;      // gradients
    float* d_m = nullptr;      // Adam moments
    float* d_v = nullptr;
    float* d_act = nullptr;    // activations
    float* d_grad = nullptr;   // activation gradients
    float* d_part = nullptr;   // weight-gradient partials
    size_t part_cap = 0;
    float* d_tgt = nullptr;
    float* d_q = nullptr;
    double* d_tn = nullptr;
    double* d_lpart = nullptr;
    size_t act_floats = 0;
    int adam_t = 0;
    bool wb_dirty = true;
    // the 16 -> 16 convolutions of inference: 0 FP32 CUDA cores, 1 tensor
    // cores (tcgen05 where the width is a multiple of 128, mma.sync
    // elsewhere), 2 mma.sync only
    int tc_mode = 1;
    int* d_status = nullptr;   // set by a tcgen05 convolution that gave up waiting
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
};

namespace {

int pfail(bamrex_precnet* N, int code, const std::string& m)
{
    const int rc = fail(code, m);
    if (N) N->err = last_error_text();
    return rc;
}

int pck(bamrex_precnet* N, cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        const int rc = cuda_fail(e, what);
        N->err = last_error_text();
        return rc;
    }
    return BAMREX_OK;
}

#define P_TRY(call)                       \
    do {                                  \
        int rc_ = (call);                 \
        if (rc_ != BAMREX_OK) return rc_; \
    } while (0)

// A tcgen05 convolution that gave up waiting for its MMAs leaves a
// status: reported (and cleared) by the calls that wait for the stream.
int check_status(bamrex_precnet* N)
{
    int st = 0;
    P_TRY(pck(N, cudaMemcpy(&st, N->d_status, sizeof(int), cudaMemcpyDeviceToHost), "status"));
    if (!st) return BAMREX_OK;
    cudaMemset(N->d_status, 0, sizeof(int));
    return pfail(N, BAMREX_ERR_TIMEOUT, "a tensor-core convolution gave up waiting for its MMAs");
}


void build_graph(bamrex_precnet* N)
{
    N->layers.clear();
    N->acts.clear();
    auto act = [&](int c, int lev) {
        N->acts.push_back({ c, lev, 0 });
        return (int)N->acts.size() - 1;
    };
    int p = 0;
    auto conv = [&](int in, int cin, int cout, int relu, int lev) {
        const int out = act(cout, lev);
        Layer L{ K_CONV, in, -1, out, cin, cout, relu, p, p + cout * cin * 9 };
        p += cout * cin * 9 + cout;
        N->layers.push_back(L);
        return out;
    };
    auto pool = [&](int in, int lev) {
        const int out = act(C, lev + 1);
        N->layers.push_back({ K_POOL, in, -1, out, C, C, 0, 0, 0 });
        return out;
    };
    auto upadd = [&](int a, int s, int lev) {
        const int out = act(C, lev);
        N->layers.push_back({ K_UPADD, a, s, out, C, C, 0, 0, 0 });
        return out;
    };
    const int x = act(2, 0);  // id 0: the input
    int h0 = conv(conv(x, 2, C, 1, 0), C, C, 1, 0);
    int h1 = conv(conv(pool(h0, 0), C, C, 1, 1), C, C, 1, 1);
    int h2 = conv(conv(pool(h1, 1), C, C, 1, 2), C, C, 1, 2);
    int h3 = conv(conv(pool(h2, 2), C, C, 1, 3), C, C, 1, 3);
    int g2 = conv(upadd(h3, h2, 2), C, C, 1, 2);
    int g1 = conv(upadd(g2, h1, 1), C, C, 1, 1);
    int g0 = conv(upadd(g1, h0, 0), C, C, 1, 0);
    conv(g0, C, 1, 0, 0);  // the output (last activation)
    N->nparams = p;
}

size_t level_hw(const bamrex_precnet* N, int lev) { return (size_t)(N->ny >> lev) * (size_t)(N->nx >> lev); }

int alloc_acts(bamrex_precnet* N)
{
    size_t off = 0;
    for (auto& a : N->acts) {
        a.off = off;
        off += (size_t)N->batch * a.c * level_hw(N, a.lev);
    }
    N->act_floats = off;
    if (N->d_act) cudaFree(N->d_act);
    if (N->d_grad) cudaFree(N->d_grad);
    if (N->d_tgt) cudaFree(N->d_tgt);
    if (N->d_tn) cudaFree(N->d_tn);
    N->d_act = N->d_grad = N->d_tgt = nullptr;
    N->d_tn = nullptr;
    P_TRY(pck(N, cudaMalloc((void**)&N->d_act, sizeof(float) * off), "activations"));
    P_TRY(pck(N, cudaMalloc((void**)&N->d_grad, sizeof(float) * off), "activation gradients"));
    if (N->d_q) cudaFree(N->d_q);
    N->d_q = nullptr;
    P_TRY(pck(N, cudaMalloc((void**)&N->d_tgt, sizeof(float) * N->batch * level_hw(N, 0)), "targets"));
    P_TRY(pck(N, cudaMalloc((void**)&N->d_q, sizeof(float) * N->batch * level_hw(N, 0)), "loss residual"));
    P_TRY(pck(N, cudaMalloc((void**)&N->d_tn, sizeof(double) * (N->batch + 1024)), "target norms"));
    N->d_lpart = N->d_tn + N->batch;
    return BAMREX_OK;
}

float* A(bamrex_precnet* N, int id) { return N->d_act + N->acts[id].off; }
float* G(bamrex_precnet* N, int id) { return N->d_grad + N->acts[id].off; }

int launch_conv_fwd(bamrex_precnet* N, const Layer& L)
{
    const int lev = N->acts[L.out].lev;
    const int H = N->ny >> lev, W = N->nx >> lev;
    const long long n = (long long)H * W * N->batch;
    const float* w = N->d_wb + L.w_off;
    const float* b = N->d_wb + L.b_off;
    if (N->tc_mode == 1 && conv_tc_supported(L.cin, L.cout, H, W))
        return pck(N, launch_conv_tc(L.cin, L.cout, A(N, L.in), A(N, L.out), w, b, H, W, N->batch, L.relu, N->d_status,
                                     N->stream),
                   "conv forward (tcgen05)");
    if (L.cin == 2 && L.cout == C)
        conv_fwd_kernel<2, C><<<gridn(n), kT, 0, N->stream>>>(A(N, L.in), A(N, L.out), w, b, H, W, N->batch, L.relu);
    else if (L.cin == C && L.cout == C && N->tc_mode != 0 && W % kMmaTW == 0 && H % kMmaTH == 0) {
        const long long tiles = (long long)N->batch * (W / kMmaTW) * (H / kMmaTH);
        const int grid = (int)std::max(1LL, std::min(tiles, (long long)device_sm_count() * 8));
        conv16_mma_kernel<<<grid, 128, 0, N->stream>>>(A(N, L.in), A(N, L.out), w, b, H, W, N->batch, L.relu);
    } else if (L.cin == C && L.cout == C)
        conv_fwd_kernel<C, C><<<gridn(n), kT, 0, N->stream>>>(A(N, L.in), A(N, L.out), w, b, H, W, N->batch, L.relu);
    else
        conv_fwd_kernel<C, 1><<<gridn(n), kT, 0, N->stream>>>(A(N, L.in), A(N, L.out), w, b, H, W, N->batch, L.relu);
    return pck(N, cudaGetLastError(), "conv forward");
}

int forward(bamrex_precnet* N)
{
    if (N->wb_dirty) {
        round_bf16_kernel<<<gridn(N->nparams), kT, 0, N->stream>>>(N->d_w, N->d_wb, N->nparams);
        P_TRY(pck(N, cudaGetLastError(), "bf16 weights"));
        N->wb_dirty = false;
    }
    for (const Layer& L : N->layers) {
        const int lev = N->acts[L.out].lev;
        const int H = N->ny >> lev, W = N->nx >> lev;
        if (L.kind == K_CONV) {
            P_TRY(launch_conv_fwd(N, L));
        } else if (L.kind == K_POOL) {
            const long long n = (long long)N->batch * C * H * W;
            pool_fwd_kernel<<<gridn(n), kT, 0, N->stream>>>(A(N, L.in), A(N, L.out), C, H * 2, W * 2, N->batch);
            P_TRY(pck(N, cudaGetLastError(), "pool forward"));
        } else {
            const long long n = (long long)N->batch * C * H * W;
            upadd_fwd_kernel<<<gridn(n), kT, 0, N->stream>>>(A(N, L.in), A(N, L.in2), A(N, L.out), C, H, W, N->batch);
            P_TRY(pck(N, cudaGetLastError(), "upsample forward"));
        }
    }
    return BAMREX_OK;
}

int backward(bamrex_precnet* N)
{
    // d(out) is in G(last); every other activation gradient starts at zero
    const int last = (int)N->acts.size() - 1;
    P_TRY(pck(N, cudaMemsetAsync(N->d_grad, 0, sizeof(float) * N->acts[last].off, N->stream), "memset"));
    P_TRY(pck(N, cudaMemsetAsync(N->d_g, 0, sizeof(float) * N->nparams, N->stream), "memset"));
    for (int li = (int)N->layers.size() - 1; li >= 0; --li) {
        const Layer& L = N->layers[li];
        const int lev = N->acts[L.out].lev;
        const int H = N->ny >> lev, W = N->nx >> lev;
        if (L.kind == K_CONV) {
            const long long n = (long long)H * W * N->batch;
            const float* w = N->d_wb + L.w_off;
            const int nw = L.cout * L.cin * 9 + L.cout;
            int TW = kTW;
            while (TW > 1 && (W % TW != 0)) TW /= 2;
            const long long tiles = (long long)N->batch * H * (W / TW);
            const int nblocks = (int)std::min<long long>(tiles, (long long)device_sm_count() * 4);
            if ((size_t)nblocks * nw > N->part_cap) {
                if (N->d_part) cudaFree(N->d_part);
                N->part_cap = (size_t)nblocks * nw;
                P_TRY(pck(N, cudaMalloc((void**)&N->d_part, sizeof(float) * N->part_cap), "partials"));
            }
#define BX_BWD(CI, CO)                                                                                               \
    conv_bwd_weight_kernel<CI, CO><<<nblocks, kT, 0, N->stream>>>(G(N, L.out), A(N, L.out), A(N, L.in), N->d_part, H, \
                                                                  W, N->batch, L.relu, TW);                          \
    if (L.in != 0)                                                                                                   \
        conv_bwd_data_kernel<CI, CO><<<gridn(n), kT, 0, N->stream>>>(G(N, L.out), A(N, L.out), w, G(N, L.in), H, W,  \
                                                                     N->batch, L.relu);
            if (L.cin == 2 && L.cout == C) {
                BX_BWD(2, C)
            } else if (L.cin == C && L.cout == C) {
                BX_BWD(C, C)
            } else {
                BX_BWD(C, 1)
            }
#undef BX_BWD
            P_TRY(pck(N, cudaGetLastError(), "conv backward"));
            sum_parts_kernel<<<(nw + kT - 1) / kT, kT, 0, N->stream>>>(N->d_part, nblocks, nw, N->d_g + L.w_off);
            P_TRY(pck(N, cudaGetLastError(), "weight gradient sum"));
        } else if (L.kind == K_POOL) {
            const long long n = (long long)N->batch * C * (H * 2) * (W * 2);
            pool_bwd_kernel<<<gridn(n), kT, 0, N->stream>>>(G(N, L.out), G(N, L.in), C, H * 2, W * 2, N->batch);
            P_TRY(pck(N, cudaGetLastError(), "pool backward"));
        } else {
            const long long n = (long long)N->batch * C * H * W;
            upadd_bwd_kernel<<<gridn(n), kT, 0, N->stream>>>(G(N, L.out), G(N, L.in), G(N, L.in2), C, H, W, N->batch);
            P_TRY(pck(N, cudaGetLastError(), "upsample backward"));
        }
    }
    return BAMREX_OK;
}

}  // namespace

extern "C" int bamrex_precnet_create(bamrex_precnet** out, int nx, int ny, int batch, unsigned long long seed, void* stream)
{
    if (!out) return fail(BAMREX_ERR_ARG, "NULL argument");
    *out = nullptr;
    if (nx < 8 || ny < 8 || nx % 8 || ny % 8 || batch < 1)
        return fail(BAMREX_ERR_ARG, "grid sides must be multiples of 8 (four levels) and batch >= 1");
    std::unique_ptr<bamrex_precnet> N(new (std::nothrow) bamrex_precnet());
    if (!N) return fail(BAMREX_ERR_OOM, "host allocation failed");
    N->nx = nx;
    N->ny = ny;
    N->batch = batch;
    build_graph(N.get());
    if (stream) {
        N->stream = (cudaStream_t)stream;
    } else {
        BX_CK(cudaStreamCreateWithFlags(&N->stream, cudaStreamNonBlocking));
        N->own_stream = true;
    }
    const size_t P = (size_t)N->nparams;
    P_TRY(pck(N.get(), cudaMalloc((void**)&N->d_w, sizeof(float) * (P * 5 + 4)), "parameters"));
    N->d_status = reinterpret_cast<int*>(N->d_w + 5 * P);
    P_TRY(pck(N.get(), cudaMemsetAsync(N->d_status, 0, sizeof(int), N->stream), "status"));
    N->d_wb = N->d_w + P;
    N->d_g = N->d_w + 2 * P;
    N->d_m = N->d_w + 3 * P;
    N->d_v = N->d_w + 4 * P;
    // He initialisation from the seed; zero biases; the output layer small
    std::vector<float> w(P, 0.0f);
    std::mt19937_64 rng(seed);
    for (const Layer& L : N->layers) {
        if (L.kind != K_CONV) continue;
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (9.0f * L.cin)) * (L.cout == 1 ? 0.1f : 1.0f));
        for (int q = 0; q < L.cout * L.cin * 9; ++q) w[L.w_off + q] = nd(rng);
    }
    P_TRY(pck(N.get(), cudaMemcpy(N->d_w, w.data(), sizeof(float) * P, cudaMemcpyHostToDevice), "weights"));
    P_TRY(pck(N.get(), cudaMemset(N->d_m, 0, sizeof(float) * P * 2), "moments"));
    P_TRY(alloc_acts(N.get()));
    // complete before the network's kernels run on another stream
    P_TRY(pck(N.get(), cudaDeviceSynchronize(), "set-up"));
    *out = N.release();
    return BAMREX_OK;
}

extern "C" int bamrex_precnet_destroy(bamrex_precnet* N)
{
    if (!N) return BAMREX_OK;
    if (N->stream) cudaStreamSynchronize(N->stream);
    cudaFree(N->d_w);
    cudaFree(N->d_act);
    cudaFree(N->d_grad);
    cudaFree(N->d_part);
    cudaFree(N->d_tgt);
    cudaFree(N->d_q);
    cudaFree(N->d_tn);
    if (N->own_stream) cudaStreamDestroy(N->stream);
    delete N;
    return BAMREX_OK;
}

extern "C" const char* bamrex_precnet_last_error(const bamrex_precnet* N) { return N ? N->err.c_str() : ""; }

extern "C" int bamrex_precnet_num_params(const bamrex_precnet* N) { return N ? N->nparams : 0; }

extern "C" int bamrex_precnet_resize(bamrex_precnet* N, int nx, int ny, int batch)
{
    if (!N) return fail(BAMREX_ERR_ARG, "NULL network");
    if (nx < 8 || ny < 8 || nx % 8 || ny % 8 || batch < 1) return pfail(N, BAMREX_ERR_ARG, "bad size");
    P_TRY(pck(N, cudaStreamSynchronize(N->stream), "sync"));
    N->nx = nx;
    N->ny = ny;
    N->batch = batch;
    return alloc_acts(N);
}

extern "C" int bamrex_precnet_get_weights(bamrex_precnet* N, float* w)
{
    if (!N || !w) return fail(BAMREX_ERR_ARG, "NULL argument");
    P_TRY(pck(N, cudaMemcpyAsync(w, N->d_w, sizeof(float) * N->nparams, cudaMemcpyDeviceToHost, N->stream), "copy"));
    return pck(N, cudaStreamSynchronize(N->stream), "sync");
}

extern "C" int bamrex_precnet_set_weights(bamrex_precnet* N, const float* w)
{
    if (!N || !w) return fail(BAMREX_ERR_ARG, "NULL argument");
    P_TRY(pck(N, cudaMemcpyAsync(N->d_w, w, sizeof(float) * N->nparams, cudaMemcpyHostToDevice, N->stream), "copy"));
    N->wb_dirty = true;
    N->adam_t = 0;
    P_TRY(pck(N, cudaMemsetAsync(N->d_m, 0, sizeof(float) * N->nparams * 2, N->stream), "memset"));
    return pck(N, cudaStreamSynchronize(N->stream), "sync");
}

// inputs: batch x 2 x ny x nx floats; out: batch x ny x nx floats (host or device)
extern "C" int bamrex_precnet_forward(bamrex_precnet* N, const float* in, float* out)
{
    if (!N || !in || !out) return fail(BAMREX_ERR_ARG, "NULL argument");
    const size_t nin = (size_t)N->batch * 2 * level_hw(N, 0), nout = (size_t)N->batch * level_hw(N, 0);
    P_TRY(pck(N, cudaMemcpyAsync(A(N, 0), in, sizeof(float) * nin, cudaMemcpyDefault, N->stream), "input"));
    P_TRY(forward(N));
    P_TRY(pck(N, cudaMemcpyAsync(out, A(N, (int)N->acts.size() - 1), sizeof(float) * nout, cudaMemcpyDefault, N->stream),
              "output"));
    P_TRY(pck(N, cudaStreamSynchronize(N->stream), "sync"));
    return check_status(N);
}

// Gradient of sum(out * dout) w.r.t. the parameters (after a forward on
// the same input): grad receives nparams floats.
extern "C" int bamrex_precnet_backward(bamrex_precnet* N, const float* dout, float* grad)
{
    if (!N || !dout || !grad) return fail(BAMREX_ERR_ARG, "NULL argument");
    const int last = (int)N->acts.size() - 1;
    const size_t nout = (size_t)N->batch * level_hw(N, 0);
    P_TRY(pck(N, cudaMemcpyAsync(G(N, last), dout, sizeof(float) * nout, cudaMemcpyDefault, N->stream), "dout"));
    P_TRY(backward(N));
    P_TRY(pck(N, cudaMemcpyAsync(grad, N->d_g, sizeof(float) * N->nparams, cudaMemcpyDefault, N->stream), "grad"));
    return pck(N, cudaStreamSynchronize(N->stream), "sync");
}

// One Adam step on the relative squared error of the batch: inputs batch x
// 2 x ny x nx, targets batch x ny x nx (host or device).  *loss: the mean
// relative squared error before the step.
extern "C" int bamrex_precnet_train_step(bamrex_precnet* N, const float* in, const float* target, float lr, double* loss)
{
    if (!N || !in || !target) return fail(BAMREX_ERR_ARG, "NULL argument");
    const long long HW = (long long)level_hw(N, 0);
    const size_t nin = (size_t)N->batch * 2 * HW, nout = (size_t)N->batch * HW;
    P_TRY(pck(N, cudaMemcpyAsync(A(N, 0), in, sizeof(float) * nin, cudaMemcpyDefault, N->stream), "input"));
    P_TRY(pck(N, cudaMemcpyAsync(N->d_tgt, target, sizeof(float) * nout, cudaMemcpyDefault, N->stream), "target"));
    const int tc = N->tc_mode;
    N->tc_mode = 0;  // the backward differentiates the FP32 forward
    const int frc = forward(N);
    N->tc_mode = tc;
    P_TRY(frc);
    const int last = (int)N->acts.size() - 1;
    const int nb = 512;
    float* qbuf = N->d_q;  // q = A_beta (out - target)
    const int H0 = N->ny, W0 = N->nx;
    abeta_kernel<<<gridn((long long)nout), kT, 0, N->stream>>>(A(N, 0), A(N, last), N->d_tgt, qbuf, H0, W0, N->batch, 0);
    P_TRY(pck(N, cudaGetLastError(), "loss residual"));
    sumsq_kernel<<<nb, kT, 0, N->stream>>>(qbuf, (long long)nout, N->d_lpart);
    P_TRY(pck(N, cudaGetLastError(), "loss"));
    abeta_kernel<<<gridn((long long)nout), kT, 0, N->stream>>>(A(N, 0), qbuf, nullptr, G(N, last), H0, W0, N->batch, 1);
    P_TRY(pck(N, cudaGetLastError(), "loss gradient"));
    P_TRY(backward(N));
    N->adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)N->adam_t), c2 = 1.0f - std::pow(b2, (float)N->adam_t);
    adam_kernel<<<gridn(N->nparams), kT, 0, N->stream>>>(N->d_w, N->d_g, N->d_m, N->d_v, N->nparams, lr, b1, b2, 1e-8f, c1, c2);
    P_TRY(pck(N, cudaGetLastError(), "adam"));
    N->wb_dirty = true;
    std::vector<double> lp(nb);
    P_TRY(pck(N, cudaMemcpyAsync(lp.data(), N->d_lpart, sizeof(double) * nb, cudaMemcpyDeviceToHost, N->stream), "loss"));
    P_TRY(pck(N, cudaStreamSynchronize(N->stream), "sync"));
    double s = 0.0;
    for (double v : lp) s += v;
    if (loss) *loss = s / ((double)HW * N->batch);
    return BAMREX_OK;
}

namespace bamrex {

float* precnet_input(bamrex_precnet* N) { return A(N, 0); }
const float* precnet_output(bamrex_precnet* N) { return A(N, (int)N->acts.size() - 1); }
void precnet_size(const bamrex_precnet* N, int* nx, int* ny, int* batch)
{
    *nx = N->nx;
    *ny = N->ny;
    *batch = N->batch;
}
int precnet_run(bamrex_precnet* N, cudaStream_t s)
{
    cudaStream_t keep = N->stream;
    N->stream = s;
    const int rc = forward(N);
    N->stream = keep;
    return rc;
}

}  // namespace bamrex

extern "C" int bamrex_precnet_set_tensor_cores(bamrex_precnet* N, int on)
{
    if (!N) return fail(BAMREX_ERR_ARG, "NULL network");
    if (on < 0 || on > 2) return pfail(N, BAMREX_ERR_ARG, "tensor-core mode must be 0, 1 or 2");
    N->tc_mode = on;
    return BAMREX_OK;
}
