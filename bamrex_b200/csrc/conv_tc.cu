// The preconditioner network's 3x3 convolutions on the fifth-generation
// tensor cores (inference): implicit GEMM with M = 128 output pixels of one
// row, N = 16 output channels, K = 16 input channels per tap, the 9 taps
// accumulated in tensor memory by tcgen05.mma (BF16 operands, FP32
// accumulators).  The 16 -> 16 layers fill N and K; the input layer (2 -> 16)
// pads K and the output layer (16 -> 1) pads N with zero weights, which
// costs the tensor core nothing next to the memory traffic.
//
// Shared-memory operands (no swizzle, K-major canonical layout: rows of 16
// bytes, 8-row core matrices 128 bytes apart, the two 8-channel halves of
// K a "plane" apart):
//   * an input row holds 130 pixels (x0 - 1 .. x0 + 128, periodic in x) as
//     two planes of [pixel][8 channels] BF16; row m of the A operand of tap
//     (dy, dx) is pixel x0 + m + dx - 1 of input row y + dy - 1, so the tap's
//     descriptor is the row's start shifted by 16 dx bytes;
//   * the weights of tap t are B(k = ci, n = co) as two planes of
//     [co][8 input channels].
// A CTA of 4 warps takes a strip of 128 pixels and up to 16 output rows
// (fewer on small levels, so every SM has work),
// keeps the input rows in a ring of 4 slots (the next row is converted from
// the FP32 NCHW activations while the tensor core works on the current
// one), one thread issues the 9 MMAs of a row and commits them to an
// mbarrier, and the 4 warps read their 32 lanes x 16 columns of the
// accumulator (tcgen05.ld), add the bias, apply the ReLU and store the
// FP32 NCHW output.  Two accumulator buffers (32 TMEM columns) let a row's
// MMAs start while the previous row's epilogue is still reading.  Every
// wait is bounded; a CTA that gives up sets *status and still releases its
// tensor memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "tma.cuh"

namespace bamrex {

int device_sm_count();

namespace {

constexpr int kTcThreads = 128;
constexpr int kTcM = 128;                 // output pixels per MMA (one row strip)
constexpr int kTcRows = 16;               // most output rows per work item
constexpr int kTcPix = kTcM + 2;          // staged input pixels of a row
constexpr int kTcPlane = kTcPix * 16;     // bytes of one 8-channel plane (2080)
constexpr int kTcRowBytes = 2 * kTcPlane; // 4160
constexpr int kTcSlots = 4;
constexpr int kTcWBytes = 9 * 512;        // weights: 9 taps x 2 planes x 16 rows x 16 bytes
constexpr int kTcSmem = 1024 + kTcSlots * kTcRowBytes + kTcWBytes + 64;
constexpr int kTcCols = 32;               // TMEM columns: two 16-column accumulators
constexpr long long kTcWaitCycles = 2000000000LL;

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1),
// BF16 A and B (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0),
// N >> 3 in bits 17-22, M >> 4 in bits 24-28.
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(16 >> 3) << 17) |
                              ((uint32_t)(kTcM >> 4) << 24);

// Shared-memory matrix descriptor, no swizzle: start address, leading byte
// offset (between the K halves), stride byte offset (between 8-row core
// matrices), each in 16-byte units, and the descriptor version 1 (bit 46).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ int wrapi(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// Convert input row r (periodic) of the strip into its ring slot: one
// thread per (plane, pixel), 8 channels -> one 16-byte store; channels at
// and above CIN are zero (K padded to 16).
template <int CIN>
__device__ __forceinline__ void stage_row(unsigned char* rows, const float* __restrict__ xb, long long HW, int H, int W,
                                          int x0, int r)
{
    const int rr = wrapi(r, H);
    unsigned char* slot = rows + ((r + kTcSlots) & (kTcSlots - 1)) * kTcRowBytes;
    const float* xr = xb + (long long)rr * W;
    // every item's loads first (up to 3 x 8 in flight per thread), then the
    // conversions and stores
    constexpr int kItems = (2 * kTcPix + kTcThreads - 1) / kTcThreads;
    float v[kItems][8];
#pragma unroll
    for (int u = 0; u < kItems; ++u) {
        const int q = threadIdx.x + u * kTcThreads;
        if (q < 2 * kTcPix) {
            const int plane = q / kTcPix, p = q - plane * kTcPix;
            const float* src = xr + (long long)(plane * 8) * HW + wrapi(x0 - 1 + p, W);
#pragma unroll
            for (int c = 0; c < 8; ++c) v[u][c] = (plane * 8 + c < CIN) ? src[(long long)c * HW] : 0.0f;
        }
    }
#pragma unroll
    for (int u = 0; u < kItems; ++u) {
        const int q = threadIdx.x + u * kTcThreads;
        if (q < 2 * kTcPix) {
            const int plane = q / kTcPix, p = q - plane * kTcPix;
            __nv_bfloat162 h[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) h[c] = __floats2bfloat162_rn(v[u][2 * c], v[u][2 * c + 1]);
            *reinterpret_cast<uint4*>(slot + plane * kTcPlane + p * 16) = *reinterpret_cast<const uint4*>(h);
        }
    }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kTcThreads, 5) conv_tc_kernel(const float* __restrict__ x, float* __restrict__ y,
                                                               const float* __restrict__ w,
                                                               const float* __restrict__ bias, int H, int W,
                                                               int batch, int relu, int rows_per_item, int* status)
{
    extern __shared__ unsigned char tc_smem_raw[];
    const uint32_t raw = smem_u32(tc_smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* sm = tc_smem_raw + (base - raw);
    unsigned char* rows = sm;
    unsigned char* wsm = sm + kTcSlots * kTcRowBytes;
    const uint32_t rows_s = base, w_s = base + kTcSlots * kTcRowBytes;
    const uint32_t bar0 = w_s + kTcWBytes;     // two mbarriers, 8 bytes each
    uint32_t* tslot = reinterpret_cast<uint32_t*>(wsm + kTcWBytes + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // weights [co][ci][9] of the real channels, zero elsewhere (N and K
    // padded to 16)
    for (int q = tid; q < 9 * 16 * 16; q += kTcThreads) {
        const int t = q >> 8, co = (q >> 4) & 15, ci = q & 15;
        const float wv = (co < COUT && ci < CIN) ? w[(co * CIN + ci) * 9 + t] : 0.0f;
        *reinterpret_cast<__nv_bfloat16*>(wsm + t * 512 + (ci >> 3) * 256 + co * 16 + (ci & 7) * 2) =
            __float2bfloat16_rn(wv);
    }
    float bv[COUT];
#pragma unroll
    for (int co = 0; co < COUT; ++co) bv[co] = bias[co];
    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"((uint32_t)kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    const long long HW = (long long)H * W;
    const int strips = W / kTcM, rblocks = (H + rows_per_item - 1) / rows_per_item;
    const long long items = (long long)batch * rblocks * strips;
    uint32_t phase = 0;  // bit b: the next completion parity of mbarrier b
    int nrow = 0;        // rows computed by this CTA (alternates the accumulators)
    bool ok = true;
    for (long long it = blockIdx.x; it < items && ok; it += gridDim.x) {
        const int b = (int)(it / ((long long)rblocks * strips));
        const int rem = (int)(it - (long long)b * rblocks * strips);
        const int y0 = (rem / strips) * rows_per_item, x0 = (rem % strips) * kTcM;
        const int y1 = min(y0 + rows_per_item, H);
        const float* xb = x + (long long)b * CIN * HW;
        float* yb = y + (long long)b * COUT * HW;
        // the ring's slots are free: the previous item's MMAs have completed
#pragma unroll 1
        for (int r = y0 - 1; r <= y0 + 1; ++r) stage_row<CIN>(rows, xb, HW, H, W, x0, r);
        for (int yy = y0; yy < y1; ++yy) {
            fence_async_smem();
            __syncthreads();
            const int buf = nrow & 1;
            if (tid == 0) {
                tc_fence_after();
#pragma unroll
                for (int tap = 0; tap < 9; ++tap) {
                    const int dy = tap / 3, dx = tap - 3 * dy;
                    const uint32_t slot = (uint32_t)((yy - 1 + dy + kTcSlots) & (kTcSlots - 1));
                    const uint64_t ad = umma_desc(rows_s + slot * kTcRowBytes + dx * 16, kTcPlane, 128);
                    const uint64_t bd = umma_desc(w_s + tap * 512, 256, 128);
                    umma_bf16(tmem + (uint32_t)(buf * 16), ad, bd, kTcIdesc, tap > 0 ? 1u : 0u);
                }
                umma_commit(bar0 + 8 * buf);
            }
            // the next row of the ring while the tensor core works (its slot
            // is none of the three this row's MMAs read)
            if (yy + 1 < y1) stage_row<CIN>(rows, xb, HW, H, W, x0, yy + 2);
            const bool done = mbar_wait_bounded(bar0 + 8 * buf, (phase >> buf) & 1u, kTcWaitCycles);
            phase ^= 1u << buf;
            ok = __syncthreads_and(done) != 0;
            if (!ok) break;
            tc_fence_after();
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(buf * 16), v);
            tc_fence_before();
            float* yo = yb + (long long)yy * W + x0 + warp * 32 + lane;
#pragma unroll
            for (int co = 0; co < COUT; ++co) {
                float o = v[co] + bv[co];
                if (relu) o = fmaxf(o, 0.0f);
                yo[(long long)co * HW] = o;
            }
            ++nrow;
        }
    }
    if (!ok && tid == 0 && status) atomicExch(status, 4 /* BAMREX_ERR_TIMEOUT */);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTcCols)
                     : "memory");
    }
}

}  // namespace

bool conv_tc_supported(int cin, int cout, int H, int W)
{
    return W % kTcM == 0 && H >= 1 && ((cin == 16 && cout == 16) || (cin == 2 && cout == 16) || (cin == 16 && cout == 1));
}

cudaError_t launch_conv_tc(int cin, int cout, const float* x, float* y, const float* w, const float* bias, int H, int W,
                           int batch, int relu, int* status, cudaStream_t s)
{
    if (!conv_tc_supported(cin, cout, H, W)) return cudaErrorInvalidValue;
    // rows per work item: up to 16 (each item re-reads two halo rows), fewer
    // on small levels so that every SM gets about two items
    const int sms = device_sm_count();
    const long long strip_rows = (long long)batch * H * (W / kTcM);
    const int rpi = (int)std::max(1LL, std::min((long long)kTcRows, strip_rows / (2LL * sms)));
    const long long items = (long long)batch * ((H + rpi - 1) / rpi) * (W / kTcM);
    const int grid = (int)std::max(1LL, std::min(items, (long long)sms * 5));  // 5 resident per SM
    if (cin == 16 && cout == 16)
        conv_tc_kernel<16, 16><<<grid, kTcThreads, kTcSmem, s>>>(x, y, w, bias, H, W, batch, relu, rpi, status);
    else if (cin == 2)
        conv_tc_kernel<2, 16><<<grid, kTcThreads, kTcSmem, s>>>(x, y, w, bias, H, W, batch, relu, rpi, status);
    else
        conv_tc_kernel<16, 1><<<grid, kTcThreads, kTcSmem, s>>>(x, y, w, bias, H, W, batch, relu, rpi, status);
    return cudaGetLastError();
}

}  // namespace bamrex
