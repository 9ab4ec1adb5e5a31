// 3x3 convolution (stride 1, zero padding 1) of NHWC BF16 activations on the tcgen05
// tensor cores, as an implicit GEMM:
//   D[m, co] = sum_{tap, ci} A[m, (tap, ci)] * W[co, (tap, ci)],  m = a tile of 128 pixels,
// with A[m, (tap, ci)] = x[n, y + dy - 1, x + dx - 1, ci] fetched by one TMA box copy per
// (tap, channel block): the box is the pixel tile shifted by the tap, and the copy's
// out-of-bounds zero fill is the padding.  The weight slice of the same (tap, channel
// block) is a second box copy.  Up to two input tensors are concatenated along the
// channels (the decoder's [upsampled, skip] input) without being materialised.
//
// A tile is 16 x 8 pixels of one image.  Per (dx, channel block) one TMA box of 18 x 8
// pixels (the tile shifted by dx, with one row of halo above and below) serves the three
// taps dy = 0, 1, 2: 8 pixel rows are one swizzle atom, so the A operand of tap dy starts
// dy atoms into the box.  Persistent CTAs of 6 warps
// walk the tiles t = blockIdx.x, + gridDim.x, ...:
//   warp 4        : TMA producer, streaming the K blocks of consecutive tiles through a
//                   ring of stages (full/empty mbarriers) without draining it
//   warp 5        : MMA issuer, 128 x cout x 16 per instruction, FP32 accumulators in
//                   tensor memory, two of them (tile parity)
//   warps 0-3, 6-9: epilogue, one group of four warps per accumulator so that two tiles
//                   drain while the next is multiplied: tensor memory -> registers (warp w
//                   reads lanes 32 (w % 4) + 0..31 = pixels), + bias, optional ReLU, BF16
//                   NHWC store (optionally FP32), optional fused 2x2 pool or 1x1 head
// Warps 4 and 5 run their loops converged; one elected lane issues each TMA copy, MMA and
// commit.
// Stage sizes follow the layer's channel block (A: kdx x 144 x cblk, B: 3 x cout x cblk
// BF16).  When the whole weight matrix fits in shared memory beside the ring it is loaded
// once per CTA (resident weights), the stages carry only activations, and a stage holds
// all three dx boxes of its channel block (kdx = 3): every K block is then 9 taps of MMAs,
// which amortises the fixed cost of a pipeline step (barrier wait, issue, commit) over
// three times as many tensor-core instructions.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>

#include "tc_sm100.cuh"

namespace lica {
namespace unet {

constexpr int kStages = 32;  // cap of the stage ring: deep enough for ~5 tiles of loads in flight per SM
constexpr int kBarBytes = 1024;  // mbarriers and the tensor-memory slot, after the tiles
static_assert((2 * kStages + 5) * 8 + 4 <= kBarBytes, "barrier region too small");
constexpr int kTileM = 128;
constexpr int kTileW = 8, kTileH = 16;          // pixel tile: 16 rows x 8 columns
constexpr int kHaloRows = kTileW * (kTileH + 2);  // A box: 18 rows x 8 columns = 144 pixel rows
// wide mode: A box of 10 rows x 16 columns (160 pixel rows), output tile 8 rows x 14 columns
constexpr int kWideBoxW = 16, kWideBoxH = 10, kWideRows = kWideBoxW * kWideBoxH;
constexpr int kWideTileW = 14, kWideTileH = 8;

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
    int stage_a, stage_b; // bytes of one pipeline stage's A and B tiles (multiples of 1 KB)
    int nstages;          // stages in the ring (<= kStages; fewer for wide layers)
    int wres;             // bytes of the resident weights (0: weight slices stream with A)
    int kdx;              // dx taps per K block: 3 (all three halo boxes in one stage; resident
                          // weights only) or 1
    int tiles;            // pixel tiles of the whole launch
    int wide;             // 1: one MMA covers the three dx taps (N = 3 cout, resident weights in
                          // the order [dy][channel block][dx]); the A box is the 16-column
                          // window x0 - 1 .. x0 + 14 and the epilogue adds the partial sums
                          // E_dx shifted by dx pixels (lanes) to the 14 output columns
    // fused consumers of the BF16 output (cout <= 64, out_c0 = 0), or null:
    __nv_bfloat16* pool;       // 2x2 average, NHWC (h/2, w/2, cout): 0.25 ((a + b) + (c + d)) in FP32
    const float* head_w;       // 1x1 head over cout = 32 channels: [wh (32), bh]
    float* head_out;           // head output per pixel, FP32 (bh + sum_c wh[c] y[c], c ascending)
    double* head_x0;           // (or null) x0 = head_out * sigma[img] * hsq * rho
    const double* head_rho;
    const double* head_sigma;
    double hsq;
};

constexpr int kConvThreads = 320;  // epilogue warps 0-3 and 6-9, producer warp 4, MMA warp 5

constexpr int kBiasBytes = 2048;  // the bias (cout <= 256 floats) and the head [wh, bh], after the barriers

__host__ __device__ inline size_t conv_p_smem_bytes(int stage_a, int stage_b, int nstages, int wres) {
    return 1024 + (size_t)nstages * (stage_a + stage_b) + (size_t)wres + kBarBytes + kBiasBytes;
}

// Bias, ReLU, BF16 (and FP32) stores of the columns c0 .. c0 + min(ncols, NC) - 1 of one
// pixel held in registers, and the fused consumers of the BF16 values: the 2x2 pool (the
// four pixels of a block are lanes l, l^1, l^8, l^9 of one warp; the lane with both bits
// clear stores) and the head's running dot product.  Called by whole warps.
template <int NC>
__device__ __forceinline__ void conv_epilogue_store(const ConvParams& P, const float* sbias, const float* shead,
                                                    size_t pix, size_t ppix, int lane, bool valid, int c0,
                                                    const uint32_t* r, int ncols, float& head) {
    const int yx = P.wide ? 16 : 8;  // lane distance of the pixel below
#pragma unroll
    for (int g = 0; g < NC / 16; ++g) {
        if (16 * g < ncols) {
            float v[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float a = __uint_as_float(r[16 * g + i]) + sbias[c0 + 16 * g + i];
                if (P.relu) a = fmaxf(a, 0.f);
                v[i] = a;
            }
            const size_t o = pix * P.out_c + P.out_c0 + c0 + 16 * g;
            uint32_t pk[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
                pk[i] = *reinterpret_cast<const uint32_t*>(&b2);
            }
            if (P.out && valid) {
                uint4* dst = reinterpret_cast<uint4*>(P.out + o);
                dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
            if (P.out32 && valid) {
                float4* dst = reinterpret_cast<float4*>(P.out32 + o);
#pragma unroll
                for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
            }
            if (P.pool || P.head_w) {
                float vb[16];  // the stored BF16 values
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&pk[i]));
                    vb[2 * i] = f.x;
                    vb[2 * i + 1] = f.y;
                }
                if (P.pool) {
                    float q[16];
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const float pair = vb[i] + __shfl_xor_sync(0xffffffffu, vb[i], 1);  // a + b | c + d
                        q[i] = 0.25f * (pair + __shfl_xor_sync(0xffffffffu, pair, yx));
                    }
                    if (valid && (lane & (1 | yx)) == 0) {
                        uint32_t qk[8];
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            const __nv_bfloat162 b2 = __floats2bfloat162_rn(q[2 * i], q[2 * i + 1]);
                            qk[i] = *reinterpret_cast<const uint32_t*>(&b2);
                        }
                        uint4* dst = reinterpret_cast<uint4*>(P.pool + ppix * P.cout + c0 + 16 * g);
                        dst[0] = make_uint4(qk[0], qk[1], qk[2], qk[3]);
                        dst[1] = make_uint4(qk[4], qk[5], qk[6], qk[7]);
                    }
                }
                if (P.head_w) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) head += shead[c0 + 16 * g + i] * vb[i];
                }
            }
        }
    }
}

__device__ __forceinline__ void tile_origin(const ConvParams& P, int t, int& img, int& x0, int& y0) {
    const int tiles_x = (P.w + P.tw - 1) / P.tw, tiles_y = P.h / P.th;
    const int tx = t % tiles_x;
    t /= tiles_x;
    const int ty = t % tiles_y;
    img = t / tiles_y;
    x0 = tx * P.tw;
    y0 = ty * P.th;
}

__global__ void __launch_bounds__(kConvThreads, 1)
    k_conv3x3_tcp(const __grid_constant__ CUtensorMap tm_x0, const __grid_constant__ CUtensorMap tm_x1,
                  const __grid_constant__ CUtensorMap tm_w0, const __grid_constant__ CUtensorMap tm_w1,
                  const ConvParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* sa = base;
    const int NS = P.nstages;
    unsigned char* sb = base + NS * P.stage_a;
    // resident weights (P.wres > 0): [tap][channel block][cout rows][cblk], loaded once
    unsigned char* sw = sb + NS * P.stage_b;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sw + P.wres);
    uint64_t* full = bars;
    uint64_t* empty = bars + kStages;
    uint64_t* tfull = bars + 2 * kStages;       // [2]: accumulator ready for the epilogue
    uint64_t* tempty = bars + 2 * kStages + 2;  // [2]: accumulator drained by the epilogue
    uint64_t* wready = bars + 2 * kStages + 4;  // resident weights landed
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 5);
    float* sbias = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(bars) + kBarBytes);
    float* shead = sbias + 256;  // [wh (32), bh]

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            tc::mbar_init(&tfull[a], 1);
            tc::mbar_init(&tempty[a], 128);
        }
        tc::mbar_init(wready, 1);
        tc::fence_barrier_init();
        tc::prefetch_tmap(&tm_x0);
        tc::prefetch_tmap(&tm_w0);
        if (P.nsrc > 1) {
            tc::prefetch_tmap(&tm_x1);
            tc::prefetch_tmap(&tm_w1);
        }
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, (uint32_t)(2 * P.tmem_cols));
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const int nb0 = P.cin[0] / P.cblk[0], nb1 = P.nsrc > 1 ? P.cin[1] / P.cblk[1] : 0;
    const int kdx = P.kdx;  // 3 in wide mode (every K block covers the three dx taps)
    const int nkb = (3 / kdx) * (nb0 + nb1);  // K blocks: (dx group, source, channel block)

    // Warps 4 and 5 run their loops with all 32 lanes (warp-uniform control and descriptor
    // arithmetic); one elected lane issues the copies, MMAs and commits.
    if (warp == 4) {
        // TMA producer
        if (P.wres) {
            if (tc::elect_one()) {
                tc::mbar_expect_tx(wready, (uint32_t)P.wres);
                for (int tap = 0; tap < 9; ++tap)
                    for (int src = 0; src < P.nsrc; ++src) {
                        const int cblk = (src ? P.cblk[1] : P.cblk[0]), off = src ? P.cin[0] : 0;
                        const void* tmw = src ? (const void*)&tm_w1 : (const void*)&tm_w0;
                        const int dy = tap / 3, dx = tap % 3;
                        for (int cb = 0; cb < (src ? nb1 : nb0); ++cb) {
                            const int col = off + cb * cblk, c = tap * P.ctot + col;
                            // narrow: [tap][column]; wide: [dy][column block][dx]
                            const int at = P.wide ? 3 * dy * P.ctot + 3 * col + dx * cblk : c;
                            tc::tma_load_2d(sw + 2 * P.cout * at, tmw, wready, c, 0);
                        }
                    }
            }
            __syncwarp();
        }
        int s = 0, g = 0;  // ring stage, K blocks issued over all tiles
        uint32_t ph = 0;   // parity of the stage's current use
        bool ok = true;
        for (int t = blockIdx.x; t < P.tiles && ok; t += gridDim.x) {
            int img, x0, y0;
            tile_origin(P, t, img, x0, y0);
            int dx = 0, src = 0, cb = 0;
            for (int kb = 0; kb < nkb; ++kb, ++g) {
                if (g >= NS && !tc::mbar_wait_warp(&empty[s], ph ^ 1u, lane)) {
                    if (lane == 0) atomicExch(P.err, 1);
                    ok = false;
                    break;
                }
                const int cblk = (src ? P.cblk[1] : P.cblk[0]);
                if (P.wide) {
                    // the 16 x 10 window (output columns x0 .. x0 + 13 need inputs x0 - 1 ..
                    // x0 + 14; rows y0 - 1 .. y0 + 8)
                    if (tc::elect_one()) {
                        tc::mbar_expect_tx(&full[s], (uint32_t)kWideRows * cblk * 2);
                        const void* tmx = src ? (const void*)&tm_x1 : (const void*)&tm_x0;
                        tc::tma_load_4d(sa + s * P.stage_a, tmx, &full[s], cb * cblk, x0 - 1, y0 - 1, img);
                    }
                } else if (tc::elect_one()) {
                    const int bsub = P.cout * cblk * 2;  // bytes of one tap's weight slice
                    tc::mbar_expect_tx(&full[s],
                                       (uint32_t)(kdx * kHaloRows + (P.wres ? 0 : 3 * P.cout)) * cblk * 2);
                    const void* tmx = src ? (const void*)&tm_x1 : (const void*)&tm_x0;
                    // 8 x 18 pixels (the tile and one row above and below), shifted by dx; the
                    // kdx boxes of a stage follow each other (each a whole number of atoms)
                    for (int j = 0; j < kdx; ++j)
                        tc::tma_load_4d(sa + s * P.stage_a + j * kHaloRows * cblk * 2, tmx, &full[s], cb * cblk,
                                        x0 + dx + j - 1, y0 - 1, img);
                    if (!P.wres) {
                        const void* tmw = src ? (const void*)&tm_w1 : (const void*)&tm_w0;
                        const int col = (src ? P.cin[0] : 0) + cb * cblk;
                        for (int dy = 0; dy < 3; ++dy)
                            tc::tma_load_2d(sb + s * P.stage_b + dy * bsub, tmw, &full[s], (3 * dy + dx) * P.ctot + col,
                                            0);
                    }
                }
                __syncwarp();
                if (++cb == (src ? nb1 : nb0)) {
                    cb = 0;
                    if (++src == P.nsrc) { src = 0; dx += kdx; }
                }
                if (++s == NS) { s = 0; ph ^= 1u; }
            }
        }
    } else if (warp == 5) {
        // MMA issuer
        const uint32_t idesc = tc::idesc_bf16_f32(kTileM, (uint32_t)(P.wide ? 3 * P.cout : P.cout));
        // descriptors of stage 0 (A, streamed B) or of the resident weights per input; the
        // descriptor of an address a + 16 j is desc(a) + j (all shared addresses < 256 KB)
        const uint64_t a_base0 = tc::smem_desc(sa, 2u * P.cblk[0]), a_base1 = tc::smem_desc(sa, 2u * P.cblk[1]);
        unsigned char* bb = P.wres ? sw : sb;
        const uint64_t b_base0 = tc::smem_desc(bb, 2u * P.cblk[0]), b_base1 = tc::smem_desc(bb, 2u * P.cblk[1]);
        const uint32_t b_dy_res = (uint32_t)(3 * P.cout * P.ctot) / 8u;  // 3 taps of 2 cout ctot bytes
        int s = 0, it = 0;
        uint32_t ph = 0;
        bool ok = !P.wres || tc::mbar_wait_warp(wready, 0, lane);
        if (!ok && lane == 0) atomicExch(P.err, 1);
        for (int t = blockIdx.x; t < P.tiles && ok; t += gridDim.x, ++it) {
            const int acc = it & 1, use = it >> 1;
            if (it >= 2 && !tc::mbar_wait_warp(&tempty[acc], (uint32_t)(use - 1) & 1u, lane)) {
                if (lane == 0) atomicExch(P.err, 1);
                break;
            }
            tc::tc_fence_after();
            const uint32_t d = tmem + (uint32_t)(acc * P.tmem_cols);
            int dx = 0, src = 0, cb = 0;
            for (int kb = 0; kb < nkb; ++kb) {
                // the stage's producer is the TMA unit (async proxy, completion through the
                // mbarrier): no tcgen05 fence is needed before the MMAs read it
                if (!tc::mbar_wait_warp(&full[s], ph, lane)) {
                    if (lane == 0) atomicExch(P.err, 1);
                    ok = false;
                    break;
                }
                const int cblk = (src ? P.cblk[1] : P.cblk[0]);
                const int col = (src ? P.cin[0] : 0) + cb * cblk;
                // descriptor offsets in 16-byte units.  A: tap dy starts dy rows of the tile
                // (8 pixel rows = one swizzle atom of 8 * 2 cblk bytes) into the halo box.
                // B: the (dy, dx) weight box, resident or in the stage.
                const uint64_t a = (src ? a_base1 : a_base0) + (uint32_t)(s * P.stage_a) / 16u;
                // wide: one image row of the window is 16 pixel rows = two atoms
                const uint32_t a_dy = (uint32_t)(P.wide ? 2 * cblk : cblk);
                uint64_t b;
                uint32_t b_dy;
                if (P.wide) {
                    // the three dx boxes of (dy, column block) are one 3 cout-row operand
                    b = (src ? b_base1 : b_base0) + (uint32_t)(3 * P.cout * col) / 8u;
                    b_dy = b_dy_res;
                } else if (P.wres) {
                    b = (src ? b_base1 : b_base0) + (uint32_t)(P.cout * (dx * P.ctot + col)) / 8u;
                    b_dy = b_dy_res;
                } else {
                    b = (src ? b_base1 : b_base0) + (uint32_t)(s * P.stage_b) / 16u;
                    b_dy = (uint32_t)(P.cout * cblk) / 8u;
                }
                const int nk = cblk / 16;
                // next dx box of the stage: 144 rows of 2 cblk bytes further (A); the weight
                // box of tap dx + 1 is ctot columns further (resident weights only: kdx = 3)
                const uint32_t a_dx = 18u * (uint32_t)cblk, b_dx = (uint32_t)(P.cout * P.ctot) / 8u;
                const int nj = P.wide ? 1 : kdx;  // A boxes in the stage
                if (tc::elect_one()) {
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        if (j < nj)
#pragma unroll
                            for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                                for (int k = 0; k < 4; ++k)
                                    if (k < nk)
                                        tc::mma_bf16(d, a + j * a_dx + dy * a_dy + 2 * k,
                                                     b + j * b_dx + dy * b_dy + 2 * k, idesc,
                                                     (kb | j | dy | k) != 0);
                    tc::mma_commit(&empty[s]);
                }
                __syncwarp();
                if (++cb == (src ? nb1 : nb0)) {
                    cb = 0;
                    if (++src == P.nsrc) { src = 0; dx += kdx; }
                }
                if (++s == NS) { s = 0; ph ^= 1u; }
            }
            // also after a failed wait: tracks the MMAs in flight
            if (tc::elect_one()) tc::mma_commit(&tfull[acc]);
            __syncwarp();
        }
    } else {
        // epilogue: two groups of four warps, group e = warps 0-3 / 6-9 drains accumulator e
        // (the tiles it = e, e + 2, ...); warp w reads tensor-memory lanes 32 (w % 4) + lane,
        // pixel m = that lane
        const int e = warp < 4 ? 0 : 1, quarter = warp & 3;
        if (e == 0) {
            for (int i = threadIdx.x; i < P.cout; i += 128) sbias[i] = P.bias ? P.bias[i] : 0.f;
            if (P.head_w && threadIdx.x <= 32) shead[threadIdx.x] = P.head_w[threadIdx.x];
        }
        asm volatile("bar.sync 1, 256;" ::: "memory");  // the eight epilogue warps
        int it = e;
        for (int t = blockIdx.x + e * gridDim.x; t < P.tiles; t += 2 * gridDim.x, it += 2) {
            const int acc = e, use = it >> 1;
            int ok = 1;
            if (lane == 0) ok = tc::mbar_wait(&tfull[acc], use & 1) ? 1 : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) {
                if (lane == 0) atomicExch(P.err, 1);
                break;
            }
            tc::tc_fence_after();
            int img, x0, y0;
            tile_origin(P, t, img, x0, y0);
            const int m = quarter * 32 + lane;
            // wide: lane m holds the window column m % 16 (input x0 - 1 + m % 16) whose output
            // column is x0 + m % 16 once the shifted partial sums are added; 14 are valid
            const int xx = P.wide ? (m & 15) : m % P.tw, yy = P.wide ? (m >> 4) : m / P.tw;
            const int y = y0 + yy, x = x0 + xx;
            const bool valid = !P.wide || (xx < kWideTileW && x < P.w);
            const size_t pix = ((size_t)img * P.h + y) * P.w + x;
            const size_t ppix = ((size_t)img * (P.h / 2) + y / 2) * (P.w / 2) + x / 2;
            float head = P.head_w ? shead[32] : 0.f;
            const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * P.tmem_cols);
            // whole 32-column chunks (the accumulator has tmem_cols >= the rounded-up cout)
            if (P.wide) {
                // D[x] = (E_0[x] + E_1[x + 1]) + E_2[x + 2], 32 output channels at a time
                for (int c0 = 0; c0 < P.cout; c0 += 32) {
                    uint32_t r[32], e1[32], e2[32];
                    tc::tmem_ld32_nowait(taddr + (uint32_t)c0, r);
                    tc::tmem_ld32_nowait(taddr + (uint32_t)(P.cout + c0), e1);
                    tc::tmem_ld32_nowait(taddr + (uint32_t)(2 * P.cout + c0), e2);
                    tc::tmem_wait_ld();
                    tc::tmem_pin<32>(r);
                    tc::tmem_pin<32>(e1);
                    tc::tmem_pin<32>(e2);
                    if (c0 + 32 >= P.cout) {
                        tc::tc_fence_before();
                        tc::mbar_arrive(&tempty[acc]);
                    }
#pragma unroll
                    for (int i = 0; i < 32; ++i) {
                        const float a = __uint_as_float(r[i]) + __shfl_down_sync(0xffffffffu, __uint_as_float(e1[i]), 1);
                        r[i] = __float_as_uint(a + __shfl_down_sync(0xffffffffu, __uint_as_float(e2[i]), 2));
                    }
                    conv_epilogue_store<32>(P, sbias, shead, pix, ppix, lane, valid, c0, r, P.cout - c0, head);
                }
                if (P.head_w && valid) {
                    P.head_out[pix] = head;
                    if (P.head_x0)
                        P.head_x0[pix] = (double)head * P.head_sigma[img] * P.hsq * P.head_rho[pix];
                }
            } else if (P.cout <= 64) {
                // the whole accumulator in registers: release it before the stores
                uint32_t r[64];
                tc::tmem_ld32_nowait(taddr, r);
                if (P.cout > 32) tc::tmem_ld32_nowait(taddr + 32u, r + 32);
                tc::tmem_wait_ld();
                tc::tmem_pin<64>(r);
                tc::tc_fence_before();
                tc::mbar_arrive(&tempty[acc]);
                conv_epilogue_store<64>(P, sbias, shead, pix, ppix, lane, true, 0, r, P.cout, head);
                if (P.head_w) {
                    P.head_out[pix] = head;
                    if (P.head_x0)
                        P.head_x0[pix] = (double)head * P.head_sigma[img] * P.hsq * P.head_rho[pix];
                }
            } else {
                for (int c0 = 0; c0 < P.cout; c0 += 32) {
                    uint32_t r[32];
                    tc::tmem_ld32_nowait(taddr + (uint32_t)c0, r);
                    tc::tmem_wait_ld();
                    tc::tmem_pin<32>(r);
                    conv_epilogue_store<32>(P, sbias, shead, pix, ppix, lane, true, c0, r, P.cout - c0, head);
                }
                tc::tc_fence_before();
                tc::mbar_arrive(&tempty[acc]);
            }
        }
    }
    __syncwarp();
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, (uint32_t)(2 * P.tmem_cols));
    }
}

}  // namespace unet
}  // namespace lica
