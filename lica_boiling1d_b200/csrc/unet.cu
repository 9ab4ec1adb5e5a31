// Learned initial guess of the pressure solve: the convolution primitive of the U-Net on
// the tcgen05 tensor cores and its host plumbing (TMA tensor maps, launch shapes).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

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

}  // namespace

namespace lica {
namespace unet {

// out[:, :, :, out_c0 : out_c0 + cout] = conv3x3([x0, x1]) (+ bias, ReLU), NHWC BF16.
int conv3x3(const __nv_bfloat16* x0, int c0, const __nv_bfloat16* x1, int c1, const __nv_bfloat16* w,
            const float* bias, int n, int h, int wd, int cout, int relu, __nv_bfloat16* out, float* out32, int out_c,
            int out_c0, int* err, cudaStream_t s) {
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
    const int tw = std::min(wd, 128), th = kTileM / tw;
    if (tw * th != kTileM || wd % tw || h % th) {
        lica_set_last_error("lica_unet_conv3x3", "image size does not tile by 128 pixels", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    static std::once_flag attr_once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(attr_once, [] {
        attr_err = cudaFuncSetAttribute(k_conv3x3_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)conv_smem_bytes(256));
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
    CUtensorMap mx0, mx1, mw0, mw1;
    int st;
    if ((st = act_map(&mx0, x0, c0, wd, h, n, P.cblk[0], tw, th))) return st;
    if ((st = weight_map(&mw0, w, 9 * P.ctot, cout, P.cblk[0]))) return st;
    if (P.nsrc > 1) {
        if ((st = act_map(&mx1, x1, c1, wd, h, n, P.cblk[1], tw, th))) return st;
        if ((st = weight_map(&mw1, w, 9 * P.ctot, cout, P.cblk[1]))) return st;
    } else {
        mx1 = mx0;
        mw1 = mw0;
    }
    const int tiles = n * (h / th) * (wd / tw);
    k_conv3x3_tc<<<tiles, 128, conv_smem_bytes(cout), s>>>(mx0, mx1, mw0, mw1, P);
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
                               out_c0, err, (cudaStream_t)stream);
}

}  // extern "C"
