// Learned initial guess of the pressure solve: the convolution primitive of the U-Net on
// the tcgen05 tensor cores and its host plumbing (TMA tensor maps, launch shapes).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "unet_conv.cuh"

extern "C" void lica_count_launches(int64_t n);

using namespace lica;
using namespace lica::unet;

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

CUtensorMapSwizzle swizzle_for(int row_bytes) {
    return row_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                            : (row_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
}

// NHWC BF16 activations (c channels): box = cblk channels x tw x th pixels of one image.
int act_map(CUtensorMap* m, const void* p, int c, int w, int h, int n, int cblk, int tw, int th) {
    auto fn = encode_fn();
    if (!fn) {
        lica_set_last_error("cuTensorMapEncodeTiled", "driver entry point unavailable", __FILE__, __LINE__);
        return LICA_ERR_CUDA;
    }
    cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
    cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)c * w * 2, (cuuint64_t)c * w * h * 2};
    cuuint32_t box[4] = {(cuuint32_t)cblk, (cuuint32_t)tw, (cuuint32_t)th, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(p), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(cblk * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        lica_set_last_error("cuTensorMapEncodeTiled", "activation map rejected", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    return LICA_OK;
}

// Weight matrix cout x ktot (BF16, K contiguous): box = cblk columns x cout rows.
int weight_map(CUtensorMap* m, const void* p, int ktot, int cout, int cblk) {
    auto fn = encode_fn();
    if (!fn) {
        lica_set_last_error("cuTensorMapEncodeTiled", "driver entry point unavailable", __FILE__, __LINE__);
        return LICA_ERR_CUDA;
    }
    cuuint64_t dims[2] = {(cuuint64_t)ktot, (cuuint64_t)cout};
    cuuint64_t strides[1] = {(cuuint64_t)ktot * 2};
    cuuint32_t box[2] = {(cuuint32_t)cblk, (cuuint32_t)cout};
    cuuint32_t es[2] = {1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(p), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(cblk * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        lica_set_last_error("cuTensorMapEncodeTiled", "weight map rejected", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    return LICA_OK;
}

int channel_block(int c) { return (c % 64 == 0) ? 64 : ((c % 32 == 0) ? 32 : 16); }

int tmem_columns(int cout) {
    int c = 32;
    while (c < cout) c *= 2;
    return c;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

constexpr int kConvSmemMax = 227 * 1024;

}  // namespace

namespace lica {
namespace unet {

// Fused consumers of a convolution's BF16 output (see ConvParams).
struct ConvFuse {
    __nv_bfloat16* pool = nullptr;
    const float* head_w = nullptr;
    float* head_out = nullptr;
    double* head_x0 = nullptr;
    const double* head_rho = nullptr;
    const double* head_sigma = nullptr;
    double hsq = 0.0;
};

// out[:, :, :, out_c0 : out_c0 + cout] = conv3x3([x0, x1]) (+ bias, ReLU), NHWC BF16.
int conv3x3(const __nv_bfloat16* x0, int c0, const __nv_bfloat16* x1, int c1, const __nv_bfloat16* w,
            const float* bias, int n, int h, int wd, int cout, int relu, __nv_bfloat16* out, float* out32, int out_c,
            int out_c0, int* err, cudaStream_t s, const ConvFuse* fuse = nullptr) {
    if (n < 1 || h < 1 || wd < 1 || c0 <= 0 || c0 % 16 || c1 < 0 || c1 % 16 || (c1 > 0 && !x1) || cout < 16 ||
        cout > 256 || cout % 16 || out_c0 < 0 || out_c0 % 8 || out_c % 8 || out_c0 + cout > out_c) {
        lica_set_last_error("lica_unet_conv3x3", "unsupported channel counts", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    if (!aligned16(x0) || (x1 && !aligned16(x1)) || !aligned16(w) || (out && !aligned16(out)) ||
        (out32 && !aligned16(out32))) {
        lica_set_last_error("lica_unet_conv3x3", "arrays must be 16-byte aligned", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    const int tw = kTileW, th = kTileH;
    if (wd % tw || h % th) {
        lica_set_last_error("lica_unet_conv3x3", "image width must be a multiple of 8 and height of 16", __FILE__,
                            __LINE__);
        return LICA_BAD_ARG;
    }
    static std::once_flag attr_once;
    static cudaError_t attr_err = cudaSuccess;
    static int num_sms = 148;
    std::call_once(attr_once, [] {
        attr_err = cudaFuncSetAttribute(k_conv3x3_tcp, cudaFuncAttributeMaxDynamicSharedMemorySize, kConvSmemMax);
        int dev = 0;
        if (attr_err == cudaSuccess) attr_err = cudaGetDevice(&dev);
        if (attr_err == cudaSuccess) attr_err = cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    });
    LICA_CUDA_TRY(attr_err);
    ConvParams P{};
    P.n = n; P.h = h; P.w = wd; P.tw = tw; P.th = th;
    P.nsrc = c1 > 0 ? 2 : 1;
    P.cin[0] = c0; P.cin[1] = c1;
    P.cblk[0] = channel_block(c0); P.cblk[1] = c1 > 0 ? channel_block(c1) : 16;
    P.ctot = c0 + c1;
    P.cout = cout;
    P.tmem_cols = tmem_columns(cout);
    P.out_c = out_c; P.out_c0 = out_c0;
    P.relu = relu;
    P.bias = bias;
    P.out = out;
    P.out32 = out32;
    P.err = err;
    if (fuse) {
        if ((fuse->pool || fuse->head_w) && (cout > 64 || out_c0 != 0 || out_c != cout)) {
            lica_set_last_error("lica_unet_conv3x3", "fused pool/head need cout <= 64 and a dense output", __FILE__,
                                __LINE__);
            return LICA_BAD_ARG;
        }
        if (fuse->head_w && (cout != 32 || !fuse->head_out || (fuse->head_x0 && (!fuse->head_rho || !fuse->head_sigma)))) {
            lica_set_last_error("lica_unet_conv3x3", "fused head needs 32 channels and its outputs", __FILE__,
                                __LINE__);
            return LICA_BAD_ARG;
        }
        P.pool = fuse->pool;
        P.head_w = fuse->head_w;
        P.head_out = fuse->head_out;
        P.head_x0 = fuse->head_x0;
        P.head_rho = fuse->head_rho;
        P.head_sigma = fuse->head_sigma;
        P.hsq = fuse->hsq;
    }
    const int cbmax = std::max(P.cblk[0], P.nsrc > 1 ? P.cblk[1] : 0);
    const auto round_kb = [](int b) { return ((b + 1023) / 1024) * 1024; };
    // Resident weights: the whole cout x (9 ctot) matrix (one box per tap, input and
    // channel block) stays in shared memory for all tiles of the CTA when it fits beside
    // the ring and every box starts on its swizzle atom; the ring then carries only the
    // activation boxes.
    const int wres = 18 * cout * P.ctot;
    const int avail = kConvSmemMax - 1024 - kBarBytes - kBiasBytes;
    const auto boxes_aligned = [&](bool wide) {
        for (int tap = 0; tap < 9; ++tap)
            for (int src = 0; src < P.nsrc; ++src)
                for (int c = src ? c0 : 0; c < (src ? P.ctot : c0); c += P.cblk[src]) {
                    const int at = wide ? 3 * (tap / 3) * P.ctot + 3 * c + (tap % 3) * P.cblk[src] : tap * P.ctot + c;
                    if ((2 * cout * at) % (16 * P.cblk[src])) return false;
                }
        return true;
    };
    // wide mode (N = 3 cout): resident weights beside at least two window stages.  Chosen
    // for 32 output channels from at least 64 input channels, where one N = 96 MMA
    // replaces three N = 32 ones and the tile's 9 ctot / 16 of them dominate; for fewer
    // input channels or 64 outputs the 14-column tiles and the shifted-sum epilogue cost
    // more than they save.
    const int stage_w = round_kb(kWideRows * cbmax * 2);
    P.stage_a = round_kb(kHaloRows * cbmax * 2);
    if (cout == 32 && P.ctot >= 64 && wd >= kWideBoxW && h >= kWideBoxH && avail - wres >= 2 * stage_w && boxes_aligned(true)) {
        P.wide = 1;
        P.tw = kWideTileW;
        P.th = kWideTileH;
        P.tmem_cols = tmem_columns(3 * cout);
        P.wres = wres;
        P.stage_a = stage_w;
        P.stage_b = 0;
        P.kdx = 3;
        P.nstages = std::min<int>(kStages, (avail - wres) / stage_w);
    } else if (avail - wres >= 3 * P.stage_a && boxes_aligned(false)) {
        P.wres = wres;
        P.stage_b = 0;
        // all three dx boxes per stage when at least two such stages fit
        const int stage3 = round_kb(3 * kHaloRows * cbmax * 2);
        if ((avail - wres) / stage3 >= 2) {
            P.kdx = 3;
            P.stage_a = stage3;
        } else {
            P.kdx = 1;
        }
        P.nstages = std::min<int>(kStages, (avail - wres) / P.stage_a);
    } else {
        P.wres = 0;
        P.kdx = 1;
        P.stage_b = round_kb(3 * cout * cbmax * 2);
        P.nstages = std::min<int>(kStages, avail / (P.stage_a + P.stage_b));
    }
    const int box_w = P.wide ? kWideBoxW : tw, box_h = P.wide ? kWideBoxH : th + 2;
    CUtensorMap mx0, mx1, mw0, mw1;
    int st;
    if ((st = act_map(&mx0, x0, c0, wd, h, n, P.cblk[0], box_w, box_h))) return st;
    if ((st = weight_map(&mw0, w, 9 * P.ctot, cout, P.cblk[0]))) return st;
    if (P.nsrc > 1) {
        if ((st = act_map(&mx1, x1, c1, wd, h, n, P.cblk[1], box_w, box_h))) return st;
        if ((st = weight_map(&mw1, w, 9 * P.ctot, cout, P.cblk[1]))) return st;
    } else {
        mx1 = mx0;
        mw1 = mw0;
    }
    const int tiles = n * (h / P.th) * ((wd + P.tw - 1) / P.tw);
    P.tiles = tiles;
    if (P.nstages < 1) return LICA_BAD_ARG;
    const size_t smem = conv_p_smem_bytes(P.stage_a, P.stage_b, P.nstages, P.wres);
    // CTAs per SM: shared memory and tensor memory (two accumulators of tmem_cols each)
    int per_sm = 0;
    LICA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv3x3_tcp, kConvThreads, smem));
    per_sm = std::max(1, std::min(per_sm, 512 / (2 * P.tmem_cols)));
    const int grid = std::min(tiles, per_sm * num_sms);
    k_conv3x3_tcp<<<grid, kConvThreads, smem, s>>>(mx0, mx1, mw0, mw1, P);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

}  // namespace unet
}  // namespace lica

extern "C" {

int lica_unet_conv3x3_device(const void* x0, int32_t c0, const void* x1, int32_t c1, const void* w, const float* bias,
                             int32_t n, int32_t h, int32_t wd, int32_t cout, int32_t relu, void* out, float* out32,
                             int32_t out_c, int32_t out_c0, int32_t* err, void* stream) {
    if (!x0 || !w || !err || (!out && !out32)) return LICA_BAD_ARG;
    return lica::unet::conv3x3((const __nv_bfloat16*)x0, c0, (const __nv_bfloat16*)x1, c1,
                               (const __nv_bfloat16*)w, bias, n, h, wd, cout, relu, (__nv_bfloat16*)out, out32, out_c,
                               out_c0, err, (cudaStream_t)stream, nullptr);
}

}  // extern "C"

// ====================================================================================
// The U-Net of the learned initial guess.
//
// Input (per image, h x w): channel 0 = log10(rho) / 3, channel 1 = f / sigma with
// sigma = sqrt(mean f^2); channels 2..15 zero (the tensor-core K step is 16 channels).
// Levels 0, 1, 2 at h x w, h/2 x w/2, h/4 x w/4 with 32, 64, 128 channels:
//   L0 x16 -> e1a   L1 e1a -> e1b            pool -> p1
//   L2 p1 -> e2a    L3 e2a -> e2b            pool -> p2
//   L4 p2 -> e3a    L5 e3a -> e3b            up   -> u2
//   L6 [u2, e2b] -> d2a   L7 d2a -> d2b      up   -> u1
//   L8 [u1, e1b] -> d1a   L9 d1a -> d1b
//   head: out = wh . d1b + bh (1x1), guess x0 = out * sigma * h^2 * rho
// 3x3 convolutions with bias and ReLU, 2x2 average pooling, nearest upsampling.
// Training loss: the guess's relative residual squared, ||f - A x0||^2 / ||f||^2, with A
// the pressure operator of the multigrid solver (averaged over the images).
// ====================================================================================
namespace {

struct LayerDef {
    int cin0, cin1, cout, level;
};
constexpr int kLayers = 10;
constexpr LayerDef kNet[kLayers] = {{16, 0, 32, 0},  {32, 0, 32, 0},   {32, 0, 64, 1},  {64, 0, 64, 1},
                                    {64, 0, 128, 2}, {128, 0, 128, 2}, {128, 64, 64, 1}, {64, 0, 64, 1},
                                    {64, 32, 32, 0}, {32, 0, 32, 0}};
constexpr int kHead = 32;
constexpr int kIn = 16;
constexpr int kNT = 256;

using bf16 = __nv_bfloat16;

// ---------------------------------------------------------------- elementwise kernels
// sigma[n] = sqrt(mean f^2) of each image: kRmsParts blocks per image write partial
// sums, one block per image adds them (fixed order).
constexpr int kRmsParts = 512;
__global__ void k_rms_part(const double* __restrict__ f, double* __restrict__ part, int npix) {
    __shared__ double red[32];
    const double* fi = f + (size_t)blockIdx.y * npix;
    double s = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < npix; k += gridDim.x * blockDim.x) s += fi[k] * fi[k];
    s = block_sum(s, red);
    if (threadIdx.x == 0) part[blockIdx.y * kRmsParts + blockIdx.x] = s;
}
__global__ void k_rms_final(const double* __restrict__ part, double* __restrict__ sigma, int npix) {
    __shared__ double red[32];
    double s = 0.0;
    for (int k = threadIdx.x; k < kRmsParts; k += blockDim.x) s += part[blockIdx.x * kRmsParts + k];
    s = block_sum(s, red);
    if (threadIdx.x == 0) {
        const double m = s / npix;
        sigma[blockIdx.x] = m > 0.0 ? sqrt(m) : 1.0;
    }
}

__global__ void k_input(const double* __restrict__ rho, const double* __restrict__ f, const double* __restrict__ sigma,
                        bf16* __restrict__ x, int npix, int nimg) {
    const size_t total = (size_t)npix * nimg;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
        const int img = (int)(p / npix);
        __align__(16) bf16 v[kIn];
        v[0] = __float2bfloat16_rn((float)(log10(rho[p]) / 3.0));
        v[1] = __float2bfloat16_rn((float)(f[p] / sigma[img]));
#pragma unroll
        for (int c = 2; c < kIn; ++c) v[c] = __float2bfloat16_rn(0.f);
        uint4* d = reinterpret_cast<uint4*>(x + p * kIn);
        d[0] = reinterpret_cast<const uint4*>(v)[0];
        d[1] = reinterpret_cast<const uint4*>(v)[1];
    }
}

// nearest upsampling x2 (H x W the output size): each thread copies one 8-channel group
// of an input pixel to its 2 x 2 output pixels.
__global__ void k_up(const bf16* __restrict__ in, bf16* __restrict__ out, int nimg, int H, int W, int c) {
    const int c8 = c / 8, Hi = H / 2, Wi = W / 2;
    const size_t total = (size_t)nimg * Hi * Wi * c8;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int ch = (int)(q % c8) * 8;
        const size_t r = q / c8;  // input pixel
        const int X = (int)(r % Wi);
        const size_t r2 = r / Wi;
        const int Y = (int)(r2 % Hi);
        const int img = (int)(r2 / Hi);
        const uint4 v = *reinterpret_cast<const uint4*>(in + r * c + ch);
        bf16* o = out + (((size_t)img * H + 2 * Y) * W + 2 * X) * c + ch;
        *reinterpret_cast<uint4*>(o) = v;
        *reinterpret_cast<uint4*>(o + c) = v;
        *reinterpret_cast<uint4*>(o + (size_t)W * c) = v;
        *reinterpret_cast<uint4*>(o + (size_t)W * c + c) = v;
    }
}

__global__ void k_head_bwd(const float* __restrict__ gout, const float* __restrict__ wh, bf16* __restrict__ g,
                           size_t total) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x)
        for (int c = 0; c < kHead; ++c) g[p * kHead + c] = __float2bfloat16_rn(gout[p] * wh[c]);
}

// Per-block partial sums of the head's gradients: part[b][c] = sum gout*d1b[:, c] (c < 32),
// part[b][32] = sum gout, over the pixels of block b (fixed order).
__global__ void k_head_grad_part(const float* __restrict__ gout, const bf16* __restrict__ d, float* __restrict__ part,
                                 size_t total) {
    __shared__ float red[kNT / 32][kHead + 1];
    float acc[kHead + 1];
#pragma unroll
    for (int c = 0; c <= kHead; ++c) acc[c] = 0.f;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
        const float g = gout[p];
#pragma unroll
        for (int c = 0; c < kHead; ++c) acc[c] += g * __bfloat162float(d[p * kHead + c]);
        acc[kHead] += g;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c <= kHead; ++c) {
        float v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][c] = v;
    }
    __syncthreads();
    if (threadIdx.x <= kHead) {
        float v = 0.f;
        for (int w = 0; w < kNT / 32; ++w) v += red[w][threadIdx.x];
        part[(size_t)blockIdx.x * (kHead + 1) + threadIdx.x] = v;
    }
}

// dz = g * (y > 0), g read as a channel slice [g_c0, g_c0 + c) of a tensor with g_cs channels,
// plus (optionally) 0.25 * gp at the parent cell of a half-size tensor (pool backward).
__global__ void k_relu_bwd(const bf16* __restrict__ g, int g_cs, int g_c0, const bf16* __restrict__ gp,
                           const bf16* __restrict__ y, bf16* __restrict__ dz, int nimg, int H, int W, int c) {
    const size_t total = (size_t)nimg * H * W * c;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int ch = (int)(q % c);
        const size_t pix = q / c;
        float v = g ? __bfloat162float(g[pix * g_cs + g_c0 + ch]) : 0.f;
        if (gp) {
            const int x = (int)(pix % W);
            const size_t r = pix / W;
            const int yy = (int)(r % H);
            const int img = (int)(r / H);
            v += 0.25f * __bfloat162float(gp[(((size_t)img * (H / 2) + yy / 2) * (W / 2) + x / 2) * c + ch]);
        }
        dz[q] = __bfloat162float(y[q]) > 0.f ? __float2bfloat16_rn(v) : __float2bfloat16_rn(0.f);
    }
}

// upsampling backward: out[n, Y, X, c] = sum of the 4 children of g (channel slice [g_c0, g_c0 + c)).
__global__ void k_up_bwd(const bf16* __restrict__ g, int g_cs, int g_c0, bf16* __restrict__ out, int nimg, int Ho,
                         int Wo, int c) {
    const size_t total = (size_t)nimg * Ho * Wo * c;
    const int W = 2 * Wo;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int ch = (int)(q % c);
        size_t r = q / c;
        const int X = (int)(r % Wo);
        r /= Wo;
        const int Y = (int)(r % Ho);
        const int img = (int)(r / Ho);
        const size_t b = (((size_t)img * 2 * Ho + 2 * Y) * W + 2 * X) * g_cs + g_c0 + ch;
        const float s = (__bfloat162float(g[b]) + __bfloat162float(g[b + g_cs])) +
                        (__bfloat162float(g[b + (size_t)W * g_cs]) + __bfloat162float(g[b + (size_t)W * g_cs + g_cs]));
        out[q] = __float2bfloat16_rn(s);
    }
}

// Weight gradient of a 3x3 convolution, per pixel chunk:
//   part[chunk][co][tap][ci] = sum_{p in chunk} dz[p, co] * x[p + off(tap), ci]
// (x = [x0, x1] along channels, zero outside the image), and bpart[chunk][co] = sum dz.
// Block: one tap, a 32 x 32 (co, ci) block; 256 threads, 4 outputs each, 32-pixel stages.
constexpr int kDwChunk = 2048;
__global__ void __launch_bounds__(kNT) k_dw_part(const bf16* __restrict__ dz, int cout, const bf16* __restrict__ x0,
                                                 int c0, const bf16* __restrict__ x1, int c1, int nimg, int H, int W,
                                                 float* __restrict__ part, float* __restrict__ bpart) {
    __shared__ float sd[32][33];
    __shared__ float sx[32][33];
    const int ctot = c0 + c1;
    const int tap = blockIdx.y, dy = tap / 3 - 1, dx = tap % 3 - 1;
    const int cob = blockIdx.z % (cout / 32), cib = blockIdx.z / (cout / 32);  // ci blocks of 32 (last one partial)
    const int chunk = blockIdx.x;
    const size_t npix = (size_t)nimg * H * W;
    const size_t p0 = (size_t)chunk * kDwChunk, p1 = min(npix, p0 + kDwChunk);
    const int t = threadIdx.x, co = t >> 3, ci4 = (t & 7) * 4;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    float bacc = 0.f;
    for (size_t pb = p0; pb < p1; pb += 32) {
        // stage dz[32 px][32 co] and x[32 px][32 ci] (4 values per thread each)
        for (int e = t; e < 32 * 32; e += kNT) {
            const int pi = e >> 5, cc = e & 31;
            const size_t p = pb + pi;
            float vd = 0.f, vx = 0.f;
            if (p < p1) {
                vd = __bfloat162float(dz[p * cout + cob * 32 + cc]);
                const int xx = (int)(p % W);
                const size_t r = p / W;
                const int yy = (int)(r % H);
                const int sx_ = xx + dx, sy_ = yy + dy;
                const int ci = cib * 32 + cc;
                if (ci < ctot && sx_ >= 0 && sx_ < W && sy_ >= 0 && sy_ < H) {
                    const size_t q = p + (ptrdiff_t)dy * W + dx;
                    vx = ci < c0 ? __bfloat162float(x0[q * c0 + ci]) : __bfloat162float(x1[q * c1 + (ci - c0)]);
                }
            }
            sd[pi][cc] = vd;
            sx[pi][cc] = vx;
        }
        __syncthreads();
#pragma unroll 8
        for (int pi = 0; pi < 32; ++pi) {
            const float a = sd[pi][co];
            acc[0] += a * sx[pi][ci4];
            acc[1] += a * sx[pi][ci4 + 1];
            acc[2] += a * sx[pi][ci4 + 2];
            acc[3] += a * sx[pi][ci4 + 3];
            if (tap == 0 && cib == 0 && (t & 7) == 0) bacc += a;
        }
        __syncthreads();
    }
    float* dst = part + (size_t)chunk * cout * 9 * ctot;
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (cib * 32 + ci4 + j < ctot) dst[((size_t)(cob * 32 + co) * 9 + tap) * ctot + cib * 32 + ci4 + j] = acc[j];
    if (tap == 0 && cib == 0 && (t & 7) == 0) bpart[(size_t)chunk * cout + cob * 32 + co] = bacc;
}

// grad[k] = sum over chunks of part[chunk][k] (chunk order), for k < n.
__global__ void k_sum_parts(const float* __restrict__ part, int nchunk, size_t n, float* __restrict__ grad) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int c = 0; c < nchunk; ++c) s += part[(size_t)c * n + k];
        grad[k] = s;
    }
}

// Adam (FP32 master weights).
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const float gk = g[k];
        const float mk = b1 * m[k] + (1.f - b1) * gk;
        const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
        m[k] = mk;
        v[k] = vk;
        w[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    }
}

// BF16 copies of a layer's weights: wb[co][tap][ci] = w, and the transposed, tap-flipped
// copy wf[ci][8 - tap][co] that turns the input-gradient into a forward convolution.
__global__ void k_pack(const float* __restrict__ w, bf16* __restrict__ wb, bf16* __restrict__ wf, int cout, int ctot) {
    const size_t n = (size_t)cout * 9 * ctot;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int ci = (int)(k % ctot);
        const size_t r = k / ctot;
        const int tap = (int)(r % 9);
        const int co = (int)(r / 9);
        const bf16 b = __float2bfloat16_rn(w[k]);
        wb[k] = b;
        wf[((size_t)ci * 9 + (8 - tap)) * cout + co] = b;
    }
}

// FP64 pressure operator of the solver: out = s - d*u (x periodic, bottom Neumann, top
// p = 0 on the face), the oracle's apply, for nimg images.
__global__ void k_apply_op(const double* __restrict__ u, const double* __restrict__ bx, const double* __restrict__ by,
                           double* __restrict__ out, int nimg, int ny, int nx, double cx, double cy) {
    const size_t npix = (size_t)nx * ny, total = npix * nimg;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const size_t img = q / npix, k = q - img * npix;
        const int j = (int)(k / nx), i = (int)(k - (size_t)j * nx);
        const double* U = u + img * npix;
        const double* BX = bx + img * npix;
        const double* BY = by + img * (npix + nx);
        const int ip = (i + 1 == nx) ? 0 : i + 1, im = (i == 0) ? nx - 1 : i - 1;
        const double aw = cx * BX[k];
        const double ae = cx * BX[(size_t)j * nx + ip];
        const double as = (j > 0) ? cy * BY[k] : 0.0;
        const double an = (j < ny - 1) ? cy * BY[k + nx] : (2.0 * cy) * BY[k + nx];
        const double us = (j > 0) ? U[k - nx] : 0.0;
        const double un = (j < ny - 1) ? U[k + nx] : 0.0;
        double s = aw * U[(size_t)j * nx + im];
        s += ae * U[(size_t)j * nx + ip];
        s += as * us;
        s += an * un;
        double d = aw;
        d += ae;
        d += as;
        d += an;
        out[q] = s - d * U[k];
    }
}

// r = f - A x0 (in place over ax), and per-image ||r||^2 (one block per image).
// r = f - (A x0) in place and ||r||^2 per image: kRmsParts blocks per image write partial
// sums (k_part_sum adds them in a fixed order).
__global__ void k_residual(const double* __restrict__ f, double* __restrict__ r, double* __restrict__ part,
                           int npix) {
    __shared__ double red[32];
    const size_t off = (size_t)blockIdx.y * npix;
    double s = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < npix; k += gridDim.x * blockDim.x) {
        const double v = f[off + k] - r[off + k];
        r[off + k] = v;
        s += v * v;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) part[blockIdx.y * kRmsParts + blockIdx.x] = s;
}

// out[image] = the sum of its kRmsParts partial sums, in index order (one block per image).
__global__ void k_part_sum(const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double red[32];
    double s = 0.0;
    for (int k = threadIdx.x; k < kRmsParts; k += blockDim.x) s += part[blockIdx.x * kRmsParts + k];
    s = block_sum(s, red);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// dL/dout = -2 (A r) sigma h^2 rho / (nimg ||f||^2), ||f||^2 = sigma^2 npix.
__global__ void k_gout(const double* __restrict__ ar, const double* __restrict__ sigma, const double* __restrict__ rho,
                       double hsq, float* __restrict__ gout, int npix, int nimg) {
    const size_t total = (size_t)npix * nimg;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
        const double sg = sigma[p / npix];
        gout[p] = (float)(-2.0 * ar[p] * hsq * rho[p] / (sg * nimg * (double)npix));
    }
}

// A-norm loss with the solver's solution p*: e = x0 - p* (into x0's buffer), per image
// num = -e.(A e) (ae holds A e), den = -p*.f = p*.(-A p*), as kRmsParts partial sums per
// image (k_part_sum adds them).
__global__ void k_energy(const double* __restrict__ ae, const double* __restrict__ e, const double* __restrict__ ps,
                         const double* __restrict__ f, double* __restrict__ part_num, double* __restrict__ part_den,
                         int npix) {
    __shared__ double red[32];
    const size_t off = (size_t)blockIdx.y * npix;
    double a = 0.0, b = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < npix; k += gridDim.x * blockDim.x) {
        a -= e[off + k] * ae[off + k];
        b -= ps[off + k] * f[off + k];
    }
    a = block_sum(a, red);
    b = block_sum(b, red);
    if (threadIdx.x == 0) {
        part_num[blockIdx.y * kRmsParts + blockIdx.x] = a;
        part_den[blockIdx.y * kRmsParts + blockIdx.x] = b;
    }
}

// dL/dout of L = mean_images num/den: -2 (A e) sigma h^2 rho / (nimg den).
__global__ void k_gout_energy(const double* __restrict__ ae, const double* __restrict__ den,
                              const double* __restrict__ sigma, const double* __restrict__ rho, double hsq,
                              float* __restrict__ gout, int npix, int nimg) {
    const size_t total = (size_t)npix * nimg;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
        const size_t img = p / npix;
        gout[p] = (float)(-2.0 * ae[p] * sigma[img] * hsq * rho[p] / (nimg * den[img]));
    }
}

__global__ void k_sub(double* __restrict__ a, const double* __restrict__ b, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        a[k] -= b[k];
}

// gout from a given dL/dx0 (the gradient check): gout = gx0 * sigma * h^2 * rho
__global__ void k_gout_from_gx(const double* __restrict__ gx, const double* __restrict__ sigma,
                               const double* __restrict__ rho, double hsq, float* __restrict__ gout, int npix,
                               int nimg) {
    const size_t total = (size_t)npix * nimg;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x)
        gout[p] = (float)(gx[p] * sigma[p / npix] * hsq * rho[p]);
}

int grid_for(size_t n) { return (int)std::min<size_t>(4 * 148 * 8, (n + kNT - 1) / kNT); }

// Deterministic normal deviates for the initial weights (splitmix64 + Box-Muller).
struct InitRng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double normal() {
        const double u1 = uniform(), u2 = uniform();
        return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    }
};

}  // namespace

// ---------------------------------------------------------------- host runtime
struct lica_unet {
    int n = 0, h = 0, w = 0;
    size_t nparams = 0;
    size_t woff[kLayers], boff[kLayers], hoff = 0;  // offsets into the FP32 parameter vector
    float* param = nullptr;                         // master weights (device)
    float* grad = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    int adam_t = 0;
    bf16* wb[kLayers] = {};
    bf16* wf[kLayers] = {};
    // activations (NHWC BF16): x16, per layer output, pooled and upsampled tensors
    bf16* x16 = nullptr;
    bf16* y[kLayers] = {};
    bf16 *p1 = nullptr, *p2 = nullptr, *u2 = nullptr, *u1 = nullptr;
    float* out32 = nullptr;
    double* sigma = nullptr;
    double* rms_part = nullptr;
    double* x0 = nullptr;   // guess (training)
    double* ax = nullptr;   // A x0, then r, then A r
    double* rr = nullptr;   // per-image ||r||^2 (or the A-norm loss's numerator)
    double* den = nullptr;  // per-image A-norm of p*
    double* part2 = nullptr;  // the A-norm loss's second set of partial sums (kRmsParts per image)
    // training buffers
    bool train_ready = false;
    float* gout = nullptr;
    bf16* gy = nullptr;      // gradient w.r.t. a layer output / input (largest level-0 tensor)
    bf16* gcat = nullptr;    // input gradient of a layer (up to 192 channels at its level)
    bf16* dz = nullptr;
    bf16* gsave[3] = {};     // skip gradients kept across the backward pass (e1b, e2b) and pool grads
    bf16* gpool = nullptr;
    float* part = nullptr;
    float* bpart = nullptr;
    size_t part_elems = 0;
    float* hpart = nullptr;
    int* err = nullptr;
};

namespace {

size_t level_pixels(const lica_unet* u, int level) { return (size_t)u->n * (u->h >> level) * (u->w >> level); }

template <typename T>
int dev_alloc(T** p, size_t count) {
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1));
    if (e != cudaSuccess) {
        lica_set_last_error("cudaMalloc", cudaGetErrorString(e), __FILE__, __LINE__);
        return LICA_ERR_NOMEM;
    }
    return LICA_OK;
}

int pack_all(lica_unet* u, cudaStream_t s) {
    for (int l = 0; l < kLayers; ++l) {
        const LayerDef& L = kNet[l];
        const size_t n = (size_t)L.cout * 9 * (L.cin0 + L.cin1);
        k_pack<<<grid_for(n), kNT, 0, s>>>(u->param + u->woff[l], u->wb[l], u->wf[l], L.cout, L.cin0 + L.cin1);
        LICA_CUDA_TRY(cudaGetLastError());
    }
    lica_count_launches(kLayers);
    return LICA_OK;
}

int conv_layer(lica_unet* u, int l, const bf16* x0, const bf16* x1, bf16* out, cudaStream_t s,
               const ConvFuse* fuse = nullptr) {
    const LayerDef& L = kNet[l];
    return conv3x3(x0, L.cin0, x1, L.cin1, u->wb[l], u->param + u->boff[l], u->n, u->h >> L.level, u->w >> L.level,
                   L.cout, 1, out, nullptr, L.cout, 0, u->err, s, fuse);
}

template <typename K, typename... A>
int launch(size_t n, cudaStream_t s, K kernel, A... args) {
    kernel<<<grid_for(n), kNT, 0, s>>>(args...);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

// Forward pass: input tensor from (rho, f), every activation kept (the last one, d1b, only
// with keep_last: the head is fused into its convolution), the head output and the guess
// x0 (if given).  The 2x2 poolings are fused into the convolutions that produce e1b and e2b.
int forward(lica_unet* u, const double* rho, const double* f, double hsq, double* x0, cudaStream_t s,
            bool keep_last = true) {
    const int npix = u->h * u->w;
    int st;
    k_rms_part<<<dim3(kRmsParts, u->n), kNT, 0, s>>>(f, u->rms_part, npix);
    k_rms_final<<<u->n, kNT, 0, s>>>(u->rms_part, u->sigma, npix);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(2);
    if ((st = launch(level_pixels(u, 0), s, k_input, rho, f, (const double*)u->sigma, u->x16, npix, u->n))) return st;
    const int h = u->h, w = u->w, n = u->n;
    ConvFuse pool1, pool2, head;
    pool1.pool = u->p1;
    pool2.pool = u->p2;
    head.head_w = u->param + u->hoff;
    head.head_out = u->out32;
    head.head_x0 = x0;
    head.head_rho = rho;
    head.head_sigma = u->sigma;
    head.hsq = hsq;
    if ((st = conv_layer(u, 0, u->x16, nullptr, u->y[0], s))) return st;
    if ((st = conv_layer(u, 1, u->y[0], nullptr, u->y[1], s, &pool1))) return st;
    if ((st = conv_layer(u, 2, u->p1, nullptr, u->y[2], s))) return st;
    if ((st = conv_layer(u, 3, u->y[2], nullptr, u->y[3], s, &pool2))) return st;
    if ((st = conv_layer(u, 4, u->p2, nullptr, u->y[4], s))) return st;
    if ((st = conv_layer(u, 5, u->y[4], nullptr, u->y[5], s))) return st;
    if ((st = launch(level_pixels(u, 2) * 16, s, k_up, (const bf16*)u->y[5], u->u2, n, h / 2, w / 2, 128))) return st;
    if ((st = conv_layer(u, 6, u->u2, u->y[3], u->y[6], s))) return st;
    if ((st = conv_layer(u, 7, u->y[6], nullptr, u->y[7], s))) return st;
    if ((st = launch(level_pixels(u, 1) * 8, s, k_up, (const bf16*)u->y[7], u->u1, n, h, w, 64))) return st;
    if ((st = conv_layer(u, 8, u->u1, u->y[1], u->y[8], s))) return st;
    return conv_layer(u, 9, u->y[8], nullptr, keep_last ? u->y[9] : nullptr, s, &head);
}

int alloc_training(lica_unet* u) {
    if (u->train_ready) return LICA_OK;
    const size_t p0 = level_pixels(u, 0), p1 = level_pixels(u, 1), p2 = level_pixels(u, 2);
    int st;
    if ((st = dev_alloc(&u->grad, u->nparams))) return st;
    if ((st = dev_alloc(&u->adam_m, u->nparams))) return st;
    if ((st = dev_alloc(&u->adam_v, u->nparams))) return st;
    LICA_CUDA_TRY(cudaMemset(u->adam_m, 0, sizeof(float) * u->nparams));
    LICA_CUDA_TRY(cudaMemset(u->adam_v, 0, sizeof(float) * u->nparams));
    const size_t big = std::max({p0 * 96, p1 * 192, p2 * 128});
    if ((st = dev_alloc(&u->gout, p0))) return st;
    if ((st = dev_alloc(&u->gy, big))) return st;
    if ((st = dev_alloc(&u->gcat, big))) return st;
    if ((st = dev_alloc(&u->dz, big))) return st;
    if ((st = dev_alloc(&u->gsave[0], p0 * 32))) return st;   // d(e1b) from the decoder
    if ((st = dev_alloc(&u->gsave[1], p1 * 64))) return st;   // d(e2b) from the decoder
    if ((st = dev_alloc(&u->gpool, big))) return st;
    // weight-gradient partials: the largest layer's chunks x weights
    size_t pe = 0, be = 0;
    for (int l = 0; l < kLayers; ++l) {
        const LayerDef& L = kNet[l];
        const size_t chunks = (level_pixels(u, L.level) + kDwChunk - 1) / kDwChunk;
        pe = std::max(pe, chunks * L.cout * 9 * (L.cin0 + L.cin1));
        be = std::max(be, chunks * L.cout);
    }
    u->part_elems = pe;
    if ((st = dev_alloc(&u->part, pe))) return st;
    if ((st = dev_alloc(&u->bpart, be))) return st;
    if ((st = dev_alloc(&u->hpart, (size_t)grid_for(p0) * (kHead + 1)))) return st;
    u->train_ready = true;
    return LICA_OK;
}

// Weight and bias gradients of layer l from dz (its masked output gradient).
int layer_wgrad(lica_unet* u, int l, const bf16* x0, const bf16* x1, cudaStream_t s) {
    const LayerDef& L = kNet[l];
    const int H = u->h >> L.level, W = u->w >> L.level, ctot = L.cin0 + L.cin1;
    const size_t npix = (size_t)u->n * H * W;
    const int chunks = (int)((npix + kDwChunk - 1) / kDwChunk);
    dim3 grid(chunks, 9, (L.cout / 32) * ((ctot + 31) / 32));
    k_dw_part<<<grid, kNT, 0, s>>>(u->dz, L.cout, x0, L.cin0, x1, L.cin1, u->n, H, W, u->part, u->bpart);
    LICA_CUDA_TRY(cudaGetLastError());
    const size_t nw = (size_t)L.cout * 9 * ctot;
    k_sum_parts<<<grid_for(nw), kNT, 0, s>>>(u->part, chunks, nw, u->grad + u->woff[l]);
    k_sum_parts<<<grid_for(L.cout), kNT, 0, s>>>(u->bpart, chunks, (size_t)L.cout, u->grad + u->boff[l]);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(3);
    return LICA_OK;
}

// Input gradient of layer l: gcat = conv3x3(dz, wf) (channels [x0 | x1]).
int layer_igrad(lica_unet* u, int l, cudaStream_t s) {
    const LayerDef& L = kNet[l];
    const int ctot = L.cin0 + L.cin1;
    return conv3x3(u->dz, L.cout, nullptr, 0, u->wf[l], nullptr, u->n, u->h >> L.level, u->w >> L.level, ctot, 0,
                   u->gcat, nullptr, ctot, 0, u->err, s);
}

// dz = g (channel slice of a tensor) [+ pool backward of gp] masked by the layer's ReLU.
int relu_bwd(lica_unet* u, int l, const bf16* g, int g_cs, int g_c0, const bf16* gp, cudaStream_t s) {
    const LayerDef& L = kNet[l];
    const int H = u->h >> L.level, W = u->w >> L.level;
    return launch(level_pixels(u, L.level) * L.cout, s, k_relu_bwd, g, g_cs, g_c0, gp, (const bf16*)u->y[l], u->dz,
                  u->n, H, W, L.cout);
}

// Backward pass from gout (dL/d out32): every parameter gradient into u->grad.
int backward(lica_unet* u, cudaStream_t s) {
    const int h = u->h, w = u->w, n = u->n;
    const size_t p0 = level_pixels(u, 0);
    int st;
    // head
    const int hb = grid_for(p0);
    k_head_grad_part<<<hb, kNT, 0, s>>>(u->gout, u->y[9], u->hpart, p0);
    k_sum_parts<<<1, kNT, 0, s>>>(u->hpart, hb, (size_t)(kHead + 1), u->grad + u->hoff);
    k_head_bwd<<<grid_for(p0), kNT, 0, s>>>(u->gout, u->param + u->hoff, u->gy, p0);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(3);
    // L9 (input d1a)
    if ((st = relu_bwd(u, 9, u->gy, 32, 0, nullptr, s))) return st;
    if ((st = layer_wgrad(u, 9, u->y[8], nullptr, s))) return st;
    if ((st = layer_igrad(u, 9, s))) return st;  // gcat = d(d1a), 32 ch
    // L8 (inputs [u1 (64), e1b (32)])
    if ((st = relu_bwd(u, 8, u->gcat, 32, 0, nullptr, s))) return st;
    if ((st = layer_wgrad(u, 8, u->u1, u->y[1], s))) return st;
    if ((st = layer_igrad(u, 8, s))) return st;  // gcat = [d(u1) 64 | d(e1b) 32]
    LICA_CUDA_TRY(cudaMemcpy2DAsync(u->gsave[0], 32 * sizeof(bf16), u->gcat + 64, 96 * sizeof(bf16),
                                    32 * sizeof(bf16), p0, cudaMemcpyDeviceToDevice, s));
    if ((st = launch(level_pixels(u, 1) * 64, s, k_up_bwd, (const bf16*)u->gcat, 96, 0, u->gy, n, h / 2, w / 2, 64)))
        return st;  // gy = d(d2b)
    // L7 (input d2a)
    if ((st = relu_bwd(u, 7, u->gy, 64, 0, nullptr, s))) return st;
    if ((st = layer_wgrad(u, 7, u->y[6], nullptr, s))) return st;
    if ((st = layer_igrad(u, 7, s))) return st;  // gcat = d(d2a)
    // L6 (inputs [u2 (128), e2b (64)])
    if ((st = relu_bwd(u, 6, u->gcat, 64, 0, nullptr, s))) return st;
    if ((st = layer_wgrad(u, 6, u->u2, u->y[3], s))) return st;
    if ((st = layer_igrad(u, 6, s))) return st;  // gcat = [d(u2) 128 | d(e2b) 64]
    LICA_CUDA_TRY(cudaMemcpy2DAsync(u->gsave[1], 64 * sizeof(bf16), u->gcat + 128, 192 * sizeof(bf16),
                                    64 * sizeof(bf16), level_pixels(u, 1), cudaMemcpyDeviceToDevice, s));
    if ((st = launch(level_pixels(u, 2) * 128, s, k_up_bwd, (const bf16*)u->gcat, 192, 0, u->gy, n, h / 4, w / 4,
                     128)))
        return st;  // gy = d(e3b)
    // L5 (input e3a)
    if ((st = relu_bwd(u, 5, u->gy, 128, 0, nullptr, s))) return st;
    if ((st = layer_wgrad(u, 5, u->y[4], nullptr, s))) return st;
    if ((st = layer_igrad(u, 5, s))) return st;  // gcat = d(e3a)
    // L4 (input p2)
    if ((st = relu_bwd(u, 4, u->gcat, 128, 0, nullptr, s))) return st;
    if ((st = layer_wgrad(u, 4, u->p2, nullptr, s))) return st;
    if ((st = layer_igrad(u, 4, s))) return st;  // gcat = d(p2), 64 ch at level 2
    LICA_CUDA_TRY(cudaMemcpyAsync(u->gpool, u->gcat, sizeof(bf16) * level_pixels(u, 2) * 64,
                                  cudaMemcpyDeviceToDevice, s));
    // L3 (input e2a): d(e2b) = decoder part + pool backward of d(p2)
    if ((st = relu_bwd(u, 3, u->gsave[1], 64, 0, u->gpool, s))) return st;
    if ((st = layer_wgrad(u, 3, u->y[2], nullptr, s))) return st;
    if ((st = layer_igrad(u, 3, s))) return st;  // gcat = d(e2a)
    // L2 (input p1)
    if ((st = relu_bwd(u, 2, u->gcat, 64, 0, nullptr, s))) return st;
    if ((st = layer_wgrad(u, 2, u->p1, nullptr, s))) return st;
    if ((st = layer_igrad(u, 2, s))) return st;  // gcat = d(p1), 32 ch at level 1
    LICA_CUDA_TRY(cudaMemcpyAsync(u->gpool, u->gcat, sizeof(bf16) * level_pixels(u, 1) * 32,
                                  cudaMemcpyDeviceToDevice, s));
    // L1 (input e1a): d(e1b) = decoder part + pool backward of d(p1)
    if ((st = relu_bwd(u, 1, u->gsave[0], 32, 0, u->gpool, s))) return st;
    if ((st = layer_wgrad(u, 1, u->y[0], nullptr, s))) return st;
    if ((st = layer_igrad(u, 1, s))) return st;  // gcat = d(e1a)
    // L0 (input x16): weights only
    if ((st = relu_bwd(u, 0, u->gcat, 32, 0, nullptr, s))) return st;
    return layer_wgrad(u, 0, u->x16, nullptr, s);
}

int check_err(lica_unet* u, cudaStream_t s) {
    int e = 0;
    LICA_CUDA_TRY(cudaMemcpyAsync(&e, u->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    LICA_CUDA_TRY(cudaStreamSynchronize(s));
    if (e) {
        lica_set_last_error("lica_unet", "a bounded wait in a tensor-core convolution ran out", __FILE__, __LINE__);
        return LICA_ERR_CUDA;
    }
    return LICA_OK;
}

}  // namespace

extern "C" {

int lica_unet_create(lica_unet** out, int32_t n, int32_t h, int32_t w, uint64_t seed) {
    if (!out || n < 1 || h < 64 || w < 64 || h % 64 || w % 64) {
        lica_set_last_error("lica_unet_create", "images must be at least 64 x 64, multiples of 64", __FILE__,
                            __LINE__);
        return LICA_BAD_ARG;
    }
    *out = nullptr;
    lica_unet* u = new lica_unet();
    u->n = n; u->h = h; u->w = w;
    size_t off = 0;
    for (int l = 0; l < kLayers; ++l) {
        const LayerDef& L = kNet[l];
        u->woff[l] = off;
        off += (size_t)L.cout * 9 * (L.cin0 + L.cin1);
        u->boff[l] = off;
        off += L.cout;
    }
    u->hoff = off;
    off += kHead + 1;
    u->nparams = off;
    // He initialisation (deterministic): N(0, 2 / fan_in); input channels 2..15 carry
    // nothing and start at zero; biases zero; head N(0, 1 / 32)
    std::vector<float> host(off, 0.f);
    InitRng rng{seed};
    for (int l = 0; l < kLayers; ++l) {
        const LayerDef& L = kNet[l];
        const int ctot = L.cin0 + L.cin1;
        const int fan = 9 * (l == 0 ? 2 : ctot);
        const double sd = sqrt(2.0 / fan);
        for (int co = 0; co < L.cout; ++co)
            for (int tap = 0; tap < 9; ++tap)
                for (int ci = 0; ci < ctot; ++ci) {
                    const double v = rng.normal() * sd;
                    if (l > 0 || ci < 2) host[u->woff[l] + ((size_t)co * 9 + tap) * ctot + ci] = (float)v;
                }
    }
    for (int c = 0; c < kHead; ++c) host[u->hoff + c] = (float)(rng.normal() * sqrt(1.0 / kHead));
    auto fail = [&](int code) { lica_unet_destroy(u); return code; };
    int st;
    if ((st = dev_alloc(&u->param, off))) return fail(st);
    if (cudaMemcpy(u->param, host.data(), sizeof(float) * off, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(LICA_ERR_CUDA);
    for (int l = 0; l < kLayers; ++l) {
        const LayerDef& L = kNet[l];
        const size_t nw = (size_t)L.cout * 9 * (L.cin0 + L.cin1);
        if ((st = dev_alloc(&u->wb[l], nw)) || (st = dev_alloc(&u->wf[l], nw))) return fail(st);
        if ((st = dev_alloc(&u->y[l], level_pixels(u, L.level) * L.cout))) return fail(st);
    }
    const size_t p0 = level_pixels(u, 0), p1 = level_pixels(u, 1), p2 = level_pixels(u, 2);
    if ((st = dev_alloc(&u->x16, p0 * kIn)) || (st = dev_alloc(&u->p1, p1 * 32)) || (st = dev_alloc(&u->p2, p2 * 64)) ||
        (st = dev_alloc(&u->u2, p1 * 128)) || (st = dev_alloc(&u->u1, p0 * 64)) || (st = dev_alloc(&u->out32, p0)) ||
        (st = dev_alloc(&u->sigma, n)) || (st = dev_alloc(&u->rms_part, (size_t)n * kRmsParts)) ||
        (st = dev_alloc(&u->rr, n)) || (st = dev_alloc(&u->err, 1)))
        return fail(st);
    if (cudaMemset(u->err, 0, sizeof(int)) != cudaSuccess) return fail(LICA_ERR_CUDA);
    if ((st = pack_all(u, 0))) return fail(st);
    if (cudaDeviceSynchronize() != cudaSuccess) return fail(LICA_ERR_CUDA);
    *out = u;
    return LICA_OK;
}

int lica_unet_destroy(lica_unet* u) {
    if (!u) return LICA_OK;
    void* ptrs[] = {u->param, u->grad, u->adam_m, u->adam_v, u->x16, u->p1, u->p2, u->u2, u->u1, u->out32,
                    u->sigma, u->rms_part, u->x0, u->ax, u->rr, u->den, u->part2, u->gout, u->gy, u->gcat, u->dz,
                    u->gsave[0], u->gsave[1], u->gsave[2], u->gpool, u->part, u->bpart, u->hpart, u->err};
    for (void* p : ptrs) cudaFree(p);
    for (int l = 0; l < kLayers; ++l) {
        cudaFree(u->wb[l]);
        cudaFree(u->wf[l]);
        cudaFree(u->y[l]);
    }
    delete u;
    return LICA_OK;
}

int64_t lica_unet_param_count(const lica_unet* u) { return u ? (int64_t)u->nparams : -1; }

int lica_unet_get_params(lica_unet* u, float* host, int64_t count) {
    if (!u || !host || count != (int64_t)u->nparams) return LICA_BAD_ARG;
    LICA_CUDA_TRY(cudaMemcpy(host, u->param, sizeof(float) * u->nparams, cudaMemcpyDeviceToHost));
    return LICA_OK;
}

int lica_unet_set_params(lica_unet* u, const float* host, int64_t count) {
    if (!u || !host || count != (int64_t)u->nparams) return LICA_BAD_ARG;
    LICA_CUDA_TRY(cudaMemcpy(u->param, host, sizeof(float) * u->nparams, cudaMemcpyHostToDevice));
    int st = pack_all(u, 0);
    if (st) return st;
    LICA_CUDA_TRY(cudaDeviceSynchronize());
    u->adam_t = 0;
    if (u->train_ready) {
        LICA_CUDA_TRY(cudaMemset(u->adam_m, 0, sizeof(float) * u->nparams));
        LICA_CUDA_TRY(cudaMemset(u->adam_v, 0, sizeof(float) * u->nparams));
    }
    return LICA_OK;
}

int lica_unet_guess_device(lica_unet* u, const double* rho, const double* f, double hsq, double* x0, void* stream) {
    if (!u || !rho || !f || !x0 || !(hsq > 0)) return LICA_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int st = forward(u, rho, f, hsq, x0, s, false);
    if (st) return st;
    return check_err(u, s);
}

int lica_unet_guess_checked_device(lica_unet* u, const double* rho, const double* f, const double* bx,
                                   const double* by, double hx, double hy, double* x0, double* rel0, void* stream) {
    if (!u || !rho || !f || !bx || !by || !x0 || !rel0 || !(hx > 0) || !(hy > 0)) return LICA_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int st;
    const size_t p0 = level_pixels(u, 0);
    if (!u->ax) {
        if ((st = dev_alloc(&u->ax, p0))) return st;
    }
    if ((st = forward(u, rho, f, hx * hy, x0, s, false))) return st;
    if ((st = launch(p0, s, k_apply_op, (const double*)x0, bx, by, u->ax, u->n, u->h, u->w, 1.0 / (hx * hx),
                     1.0 / (hy * hy))))
        return st;
    const int npix = u->h * u->w;
    k_residual<<<dim3(kRmsParts, u->n), kNT, 0, s>>>(f, u->ax, u->rms_part, npix);
    k_part_sum<<<u->n, kNT, 0, s>>>(u->rms_part, u->rr);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(2);
    std::vector<double> rr(u->n), sg(u->n);
    LICA_CUDA_TRY(cudaMemcpyAsync(rr.data(), u->rr, sizeof(double) * u->n, cudaMemcpyDeviceToHost, s));
    LICA_CUDA_TRY(cudaMemcpyAsync(sg.data(), u->sigma, sizeof(double) * u->n, cudaMemcpyDeviceToHost, s));
    if ((st = check_err(u, s))) return st;
    for (int i = 0; i < u->n; ++i) {
        rel0[i] = sqrt(rr[i] / (sg[i] * sg[i] * npix));
        if (!(rel0[i] < 1.0))  // no better than zero (or not finite): start from zero
            LICA_CUDA_TRY(cudaMemsetAsync(x0 + (size_t)i * npix, 0, sizeof(double) * npix, s));
    }
    return LICA_OK;
}

int lica_unet_grad_device(lica_unet* u, const double* rho, const double* f, double hsq, const double* gx0,
                          float* grad_host, int64_t count, void* stream) {
    if (!u || !rho || !f || !gx0 || !grad_host || count != (int64_t)u->nparams || !(hsq > 0)) return LICA_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int st;
    if ((st = alloc_training(u))) return st;
    if ((st = forward(u, rho, f, hsq, nullptr, s))) return st;
    if ((st = launch(level_pixels(u, 0), s, k_gout_from_gx, gx0, (const double*)u->sigma, rho, hsq, u->gout,
                     u->h * u->w, u->n)))
        return st;
    if ((st = backward(u, s))) return st;
    if ((st = check_err(u, s))) return st;
    LICA_CUDA_TRY(cudaMemcpy(grad_host, u->grad, sizeof(float) * u->nparams, cudaMemcpyDeviceToHost));
    return LICA_OK;
}

int lica_unet_train_step_device(lica_unet* u, const double* rho, const double* f, const double* bx, const double* by,
                                const double* p_star, double hx, double hy, float lr, double* loss, void* stream) {
    if (!u || !rho || !f || !bx || !by || !loss || !(hx > 0) || !(hy > 0) || !(lr > 0)) return LICA_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int st;
    if ((st = alloc_training(u))) return st;
    const size_t p0 = level_pixels(u, 0);
    if ((!u->x0 && (st = dev_alloc(&u->x0, p0))) || (!u->ax && (st = dev_alloc(&u->ax, p0))) ||
        (!u->den && (st = dev_alloc(&u->den, u->n))) ||
        (!u->part2 && (st = dev_alloc(&u->part2, (size_t)u->n * kRmsParts))))
        return st;
    const double hsq = hx * hy;
    const int npix = u->h * u->w;
    if ((st = forward(u, rho, f, hsq, u->x0, s))) return st;
    const double cx = 1.0 / (hx * hx), cy = 1.0 / (hy * hy);
    if (p_star) {
        // e = x0 - p*, A e, loss = -e.(A e) / (-p*.f) per image, dL/dout
        if ((st = launch(p0, s, k_sub, u->x0, p_star, p0))) return st;
        if ((st = launch(p0, s, k_apply_op, (const double*)u->x0, bx, by, u->ax, u->n, u->h, u->w, cx, cy))) return st;
        k_energy<<<dim3(kRmsParts, u->n), kNT, 0, s>>>(u->ax, u->x0, p_star, f, u->rms_part, u->part2, npix);
        k_part_sum<<<u->n, kNT, 0, s>>>(u->rms_part, u->rr);
        k_part_sum<<<u->n, kNT, 0, s>>>(u->part2, u->den);
        LICA_CUDA_TRY(cudaGetLastError());
        lica_count_launches(3);
        if ((st = launch(p0, s, k_gout_energy, (const double*)u->ax, (const double*)u->den, (const double*)u->sigma,
                         rho, hsq, u->gout, npix, u->n)))
            return st;
    } else {
        // r = f - A x0, ||r||^2; then A r into x0's buffer, and dL/dout
        if ((st = launch(p0, s, k_apply_op, (const double*)u->x0, bx, by, u->ax, u->n, u->h, u->w, cx, cy))) return st;
        k_residual<<<dim3(kRmsParts, u->n), kNT, 0, s>>>(f, u->ax, u->rms_part, npix);
        k_part_sum<<<u->n, kNT, 0, s>>>(u->rms_part, u->rr);
        LICA_CUDA_TRY(cudaGetLastError());
        lica_count_launches(2);
        if ((st = launch(p0, s, k_apply_op, (const double*)u->ax, bx, by, u->x0, u->n, u->h, u->w, cx, cy))) return st;
        if ((st = launch(p0, s, k_gout, (const double*)u->x0, (const double*)u->sigma, rho, hsq, u->gout, npix, u->n)))
            return st;
    }
    if ((st = backward(u, s))) return st;
    u->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)u->adam_t), c2 = 1.f - powf(b2, (float)u->adam_t);
    if ((st = launch(u->nparams, s, k_adam, u->param, (const float*)u->grad, u->adam_m, u->adam_v, u->nparams, lr, b1,
                     b2, 1e-8f, c1, c2)))
        return st;
    if ((st = pack_all(u, s))) return st;
    // loss = mean over images of ||r||^2 / ||f||^2, or of the relative A-norm error squared
    std::vector<double> rr(u->n), sg(u->n), dn(u->n);
    LICA_CUDA_TRY(cudaMemcpyAsync(rr.data(), u->rr, sizeof(double) * u->n, cudaMemcpyDeviceToHost, s));
    LICA_CUDA_TRY(cudaMemcpyAsync(sg.data(), u->sigma, sizeof(double) * u->n, cudaMemcpyDeviceToHost, s));
    LICA_CUDA_TRY(cudaMemcpyAsync(dn.data(), u->den, sizeof(double) * u->n, cudaMemcpyDeviceToHost, s));
    if ((st = check_err(u, s))) return st;
    double L = 0.0;
    for (int i = 0; i < u->n; ++i) L += p_star ? rr[i] / dn[i] : rr[i] / (sg[i] * sg[i] * npix);
    *loss = L / u->n;
    return LICA_OK;
}

}  // extern "C"
