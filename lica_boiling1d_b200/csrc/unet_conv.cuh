// 3x3 convolution (stride 1, zero padding 1) of NHWC BF16 activations on the tcgen05
// tensor cores, as an implicit GEMM:
//   D[m, co] = sum_{tap, ci} A[m, (tap, ci)] * W[co, (tap, ci)],  m = a tile of 128 pixels,
// with A[m, (tap, ci)] = x[n, y + dy - 1, x + dx - 1, ci] fetched by one TMA box copy per
// (tap, channel block): the box is the pixel tile shifted by the tap, and the copy's
// out-of-bounds zero fill is the padding.  The weight slice of the same (tap, channel
// block) is a second box copy.  Up to two input tensors are concatenated along the
// channels (the decoder's [upsampled, skip] input) without being materialised.
//
// One CTA = 4 warps and one 128-pixel tile (th rows x tw columns of one image):
//   warp 0 lane 0 : TMA producer over a ring of kStages stages (full/empty mbarriers)
//   warp 1 lane 0 : MMA issuer, 128 x cout x 16 per instruction, FP32 accumulator in
//                   tensor memory (cout columns, lane = pixel)
//   all warps     : epilogue, tensor memory -> registers (warp w reads lanes 32w..32w+31),
//                   + bias, optional ReLU, BF16 NHWC store (optionally an FP32 copy)
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>

#include "tc_sm100.cuh"

namespace lica {
namespace unet {

constexpr int kStages = 4;
constexpr int kTileM = 128;
constexpr int kStageA = kTileM * 128;  // bytes: 128 pixels x up to 64 BF16 channels

struct ConvParams {
    int n, h, w;          // image count and size (output = input size)
    int tw, th;           // pixel tile: th rows x tw columns, tw * th = 128
    int nsrc;             // input tensors (1 or 2), concatenated along channels
    int cin[2], cblk[2];  // channels of each input, channels per TMA box (16, 32 or 64)
    int ctot;             // cin[0] + cin[1]; the weight matrix is cout x (9 * ctot), k = tap*ctot + c
    int cout;             // output channels = MMA N (multiple of 16, <= 256)
    int tmem_cols;        // power of two >= max(32, cout)
    int out_c, out_c0;    // channel count of the output tensor and the first channel written
    int relu;             // 1: max(0, .) before the store
    const float* bias;    // [cout] or null
    __nv_bfloat16* out;   // NHWC output (or null)
    float* out32;         // NHWC FP32 output (or null)
    int* err;             // set to 1 when a bounded wait runs out
};

__host__ __device__ inline size_t conv_smem_bytes(int cout) {
    return 1024 /* alignment slack */ + (size_t)kStages * (kStageA + (size_t)cout * 128) + 256;
}

__global__ void __launch_bounds__(128, 1)
    k_conv3x3_tc(const __grid_constant__ CUtensorMap tm_x0, const __grid_constant__ CUtensorMap tm_x1,
                 const __grid_constant__ CUtensorMap tm_w0, const __grid_constant__ CUtensorMap tm_w1,
                 const ConvParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int stage_b = P.cout * 128;
    unsigned char* sa = base;                      // kStages x kStageA
    unsigned char* sb = base + kStages * kStageA;  // kStages x stage_b
    uint64_t* bars = reinterpret_cast<uint64_t*>(sb + kStages * stage_b);
    uint64_t* full = bars;
    uint64_t* empty = bars + kStages;
    uint64_t* done = bars + 2 * kStages;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 1);
    int* s_ok = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_x = P.w / P.tw, tiles_y = P.h / P.th;
    int t = blockIdx.x;
    const int tx = t % tiles_x;
    t /= tiles_x;
    const int ty = t % tiles_y;
    const int img = t / tiles_y;
    const int x0 = tx * P.tw, y0 = ty * P.th;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(done, 1);
        tc::fence_barrier_init();
        tc::prefetch_tmap(&tm_x0);
        tc::prefetch_tmap(&tm_w0);
        if (P.nsrc > 1) {
            tc::prefetch_tmap(&tm_x1);
            tc::prefetch_tmap(&tm_w1);
        }
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, (uint32_t)P.tmem_cols);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // K blocks: tap-major, then source, then channel block
    const int nb0 = P.cin[0] / P.cblk[0], nb1 = P.nsrc > 1 ? P.cin[1] / P.cblk[1] : 0;
    const int nkb = 9 * (nb0 + nb1);

    if (warp == 0 && lane == 0) {
        int tap = 0, src = 0, cb = 0;
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % kStages, u = kb / kStages;
            if (kb >= kStages && !tc::mbar_wait(&empty[s], (u - 1) & 1)) { atomicExch(P.err, 1); break; }
            const int cblk = P.cblk[src];
            const uint32_t bytes = (uint32_t)(kTileM + P.cout) * cblk * 2;
            tc::mbar_expect_tx(&full[s], bytes);
            const int dy = tap / 3, dx = tap - 3 * dy;
            const void* tmx = src ? (const void*)&tm_x1 : (const void*)&tm_x0;
            const void* tmw = src ? (const void*)&tm_w1 : (const void*)&tm_w0;
            tc::tma_load_4d(sa + s * kStageA, tmx, &full[s], cb * cblk, x0 + dx - 1, y0 + dy - 1, img);
            tc::tma_load_2d(sb + s * stage_b, tmw, &full[s], tap * P.ctot + (src ? P.cin[0] : 0) + cb * cblk, 0);
            if (++cb == (src ? nb1 : nb0)) {
                cb = 0;
                if (++src == P.nsrc) { src = 0; ++tap; }
            }
        }
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = tc::idesc_bf16_f32(kTileM, (uint32_t)P.cout);
        int src = 0, cb = 0;
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % kStages, u = kb / kStages;
            if (!tc::mbar_wait(&full[s], u & 1)) { atomicExch(P.err, 1); break; }
            tc::tc_fence_after();
            const int cblk = P.cblk[src];
            const uint32_t rb = (uint32_t)cblk * 2;
            const uint64_t da = tc::smem_desc(sa + s * kStageA, rb);
            const uint64_t db = tc::smem_desc(sb + s * stage_b, rb);
            for (int k = 0; k < cblk / 16; ++k)
                tc::mma_bf16(tmem, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc, (kb | k) != 0);
            tc::mma_commit(&empty[s]);
            if (++cb == (src ? nb1 : nb0)) {
                cb = 0;
                if (++src == P.nsrc) src = 0;
            }
        }
        tc::mma_commit(done);  // also after a failed wait: done then tracks the MMAs in flight
    }
    __syncwarp();

    // epilogue: pixel m = threadIdx.x (tensor-memory lane), columns = output channels
    if (threadIdx.x == 0) {
        const bool ok = tc::mbar_wait(done, 0);
        if (!ok) atomicExch(P.err, 1);
        *s_ok = ok ? 1 : 0;
    }
    __syncthreads();
    tc::tc_fence_after();
    if (*s_ok) {
        const int m = threadIdx.x;
        const int y = y0 + m / P.tw, x = x0 + m % P.tw;
        const size_t pix = ((size_t)img * P.h + y) * P.w + x;
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < P.cout; c0 += 16) {
            float v[16];
            tc::tmem_ld16(taddr + (uint32_t)c0, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float a = v[i] + (P.bias ? P.bias[c0 + i] : 0.f);
                if (P.relu) a = fmaxf(a, 0.f);
                v[i] = a;
            }
            if (P.out) {
                uint32_t pk[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
                    pk[i] = *reinterpret_cast<const uint32_t*>(&b2);
                }
                uint4* dst = reinterpret_cast<uint4*>(P.out + pix * P.out_c + P.out_c0 + c0);
                dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
            if (P.out32) {
                float4* dst = reinterpret_cast<float4*>(P.out32 + pix * P.out_c + P.out_c0 + c0);
#pragma unroll
                for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, (uint32_t)P.tmem_cols);
    }
}

}  // namespace unet
}  // namespace lica
