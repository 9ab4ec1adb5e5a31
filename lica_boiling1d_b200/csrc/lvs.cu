// Level-set transport of 1-D boiling columns on the GPU: TRANSPORT (two_phase.f:701-984)
// with TRANSPORT_RK3/HJWENO, REIN_TRIGGER, REINITIALIZATION/GODUNOV, ALPHI_BC,
// BAND_GENERATION, VEL_INTP, CAL_PSIF_MTP, GLOBAL_MASS_CORRECTION and GRID_COUPLING in
// their 1-D form: one flow cell in x and y, the refined level-set grid replicated over
// its 2 x 2 (I,J) cells, so every x/y derivative is exactly zero (two_phase.f:885-892).
//
// Parallel structure and layout:
//   * one warp per column; a batch of columns of equal geometry is stored back to back
//     (phi/layer/mflvs: nf+7 values per column, psif: nf+2, flow faces: n+2);
//   * the narrow band (N_MAX = 11 layers, 1dmodulesX.f:21) lives in a 128-cell shared-
//     memory window that follows it.  TRANSPORT zeroes phi outside the band on entry
//     (two_phase.f:750-767), so a window holding the band and its stencil halo is exact;
//     a band that does not fit returns LICA_BAND_OVERFLOW (the analogue of the band-size
//     STOP, two_phase.f:1989-1994) and leaves that column's state untouched;
//   * the band is kept both as a per-cell layer number (for the per-cell stencil work,
//     spread over the lanes) and as ordered lists per layer, built in the reference's
//     order (S-tube in old-list order, then children parent by parent, lower side first),
//     so that the order-dependent FP64 sums (vapour volume, two_phase.f:6230-6290) are
//     added in the same sequence as the CPU restatement and agree bit for bit.
// Every expression keeps the reference's operation order; the library is compiled without
// FMA contraction.
#include "lvs_device.cuh"

#include <mutex>

extern "C" void lica_count_launches(int64_t n);

namespace lica {
namespace lvs {

__global__ void __launch_bounds__(32 * WARPS)
    k_lvs_transport(int ncol, int n, double length, double* __restrict__ phi, int* __restrict__ layer,
                    double* __restrict__ psif, double* __restrict__ wo, const double* __restrict__ w,
                    const double* __restrict__ mf, double* __restrict__ vol_ori, const double* __restrict__ vol_iphs,
                    double* __restrict__ psi_cn, double* __restrict__ psi_zn, int* __restrict__ status,
                    double* __restrict__ stats, Params P) {
    __shared__ Win win[WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = blockIdx.x * WARPS + warp;
    if (col >= ncol) return;
    const size_t nf = 2 * (size_t)n, sp = nf + 7, sf = nf + 2, sw = (size_t)n + 2;
    const int st = transport_column(&win[warp], lane, n, length, phi + col * sp, layer + col * sp, psif + col * sf,
                                    wo + col * sw, w + col * sw, mf + col * sp, vol_ori + col, vol_iphs[col],
                                    psi_cn + col * sw, psi_zn + col * sw, stats + 4 * (size_t)col, P);
    if (lane == 0) status[col] = st;
}

}  // namespace lvs
}  // namespace lica

using namespace lica;
using namespace lica::lvs;

namespace {

// device copies for the host entry point, grown on demand
struct HostBufs {
    std::mutex mu;
    void* ptr = nullptr;
    size_t bytes = 0;
};
HostBufs& host_bufs() {
    static HostBufs b;
    return b;
}

int check_args(int32_t ncol, int32_t n, double length, const lica_lvs_params* prm) {
    if (ncol < 1 || n < 8 || n > (1 << 24) || !(length > 0.0) || !prm) {
        lica_set_last_error("lica_gpu_lvs_transport", "need ncol >= 1, n >= 8, length > 0 and params", __FILE__,
                            __LINE__);
        return LICA_BAD_ARG;
    }
    return LICA_OK;
}

}  // namespace

extern "C" {

int lica_gpu_lvs_transport_device(int32_t ncol, int32_t n, double length, double* phi, int32_t* layer, double* psif,
                                  double* wo, const double* w, const double* mflvs, double* vol_tot_ori,
                                  const double* vol_tot_iphs, double* psi_cn, double* psi_zn, int32_t* status,
                                  double* stats, const lica_lvs_params* prm, void* stream) {
    int st = check_args(ncol, n, length, prm);
    if (st) return st;
    if (!phi || !layer || !psif || !wo || !w || !mflvs || !vol_tot_ori || !vol_tot_iphs || !psi_cn || !psi_zn ||
        !status || !stats)
        return LICA_BAD_ARG;
    Params P{prm->iphs, prm->first, prm->m_step, prm->mglobal, prm->denr, prm->dtconst};
    const unsigned blocks = (unsigned)((ncol + WARPS - 1) / WARPS);
    k_lvs_transport<<<blocks, 32 * WARPS, 0, (cudaStream_t)stream>>>(ncol, n, length, phi, layer, psif, wo, w, mflvs,
                                                                      vol_tot_ori, vol_tot_iphs, psi_cn, psi_zn,
                                                                      status, stats, P);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

int lica_gpu_lvs_transport(int32_t ncol, int32_t n, double length, double* phi, int32_t* layer, double* psif,
                           double* wo, const double* w, const double* mflvs, double* vol_tot_ori,
                           const double* vol_tot_iphs, double* psi_cn, double* psi_zn, int32_t* status, double* stats,
                           const lica_lvs_params* prm) {
    int st = check_args(ncol, n, length, prm);
    if (st) return st;
    if (!phi || !layer || !psif || !wo || !w || !mflvs || !vol_tot_ori || !vol_tot_iphs || !psi_cn || !psi_zn ||
        !status || !stats)
        return LICA_BAD_ARG;
    const size_t nc = (size_t)ncol, nf = 2 * (size_t)n, sp = nf + 7, sf = nf + 2, sw = (size_t)n + 2;
    // byte offsets of each array in one device allocation (each 256-byte aligned)
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_phi = take(8 * nc * sp), o_lay = take(4 * nc * sp), o_psif = take(8 * nc * sf),
                 o_wo = take(8 * nc * sw), o_w = take(8 * nc * sw), o_mf = take(8 * nc * sp), o_vo = take(8 * nc),
                 o_vi = take(8 * nc), o_cn = take(8 * nc * sw), o_zn = take(8 * nc * sw), o_st = take(4 * nc),
                 o_stats = take(8 * 4 * nc);
    HostBufs& hb = host_bufs();
    std::lock_guard<std::mutex> lk(hb.mu);
    if (off > hb.bytes) {
        if (hb.ptr) cudaFree(hb.ptr);
        hb.ptr = nullptr;
        hb.bytes = 0;
        LICA_CUDA_TRY(cudaMalloc(&hb.ptr, off));
        hb.bytes = off;
    }
    char* base = (char*)hb.ptr;
    struct Cp {
        size_t o;
        const void* h;
        size_t bytes;
    } ins[] = {{o_phi, phi, 8 * nc * sp},    {o_lay, layer, 4 * nc * sp},  {o_psif, psif, 8 * nc * sf},
               {o_wo, wo, 8 * nc * sw},      {o_w, w, 8 * nc * sw},        {o_mf, mflvs, 8 * nc * sp},
               {o_vo, vol_tot_ori, 8 * nc},  {o_vi, vol_tot_iphs, 8 * nc}, {o_cn, psi_cn, 8 * nc * sw},
               {o_zn, psi_zn, 8 * nc * sw},  {o_stats, stats, 8 * 4 * nc}};
    for (const Cp& cp : ins) LICA_CUDA_TRY(cudaMemcpy(base + cp.o, cp.h, cp.bytes, cudaMemcpyHostToDevice));
    st = lica_gpu_lvs_transport_device(ncol, n, length, (double*)(base + o_phi), (int32_t*)(base + o_lay),
                                       (double*)(base + o_psif), (double*)(base + o_wo), (const double*)(base + o_w),
                                       (const double*)(base + o_mf), (double*)(base + o_vo),
                                       (const double*)(base + o_vi), (double*)(base + o_cn), (double*)(base + o_zn),
                                       (int32_t*)(base + o_st), (double*)(base + o_stats), prm, nullptr);
    if (st) return st;
    struct Out {
        void* h;
        size_t o, bytes;
    } outs[] = {{phi, o_phi, 8 * nc * sp},   {layer, o_lay, 4 * nc * sp}, {psif, o_psif, 8 * nc * sf},
                {wo, o_wo, 8 * nc * sw},     {vol_tot_ori, o_vo, 8 * nc}, {psi_cn, o_cn, 8 * nc * sw},
                {psi_zn, o_zn, 8 * nc * sw}, {status, o_st, 4 * nc},      {stats, o_stats, 8 * 4 * nc}};
    for (const Out& cp : outs) LICA_CUDA_TRY(cudaMemcpy(cp.h, base + cp.o, cp.bytes, cudaMemcpyDeviceToHost));
    int worst = LICA_OK;
    for (size_t c = 0; c < nc; ++c)
        if (status[c] != LICA_OK) worst = status[c];
    return worst;
}

}  // extern "C"
