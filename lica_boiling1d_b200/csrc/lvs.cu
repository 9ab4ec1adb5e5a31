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
                    double* __restrict__ stats, Params P, const __grid_constant__ col::ColGeoDev geo,
                    int has_geo) {
    __shared__ Win win[WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = blockIdx.x * WARPS + warp;
    if (col >= ncol) return;
    const size_t nf = 2 * (size_t)n, sp = nf + 7, sf = nf + 2, sw = (size_t)n + 2;
    const int st = transport_column(&win[warp], lane, n, length, phi + col * sp, layer + col * sp, psif + col * sf,
                                    wo + col * sw, w + col * sw, mf + col * sp, vol_ori + col, vol_iphs[col],
                                    psi_cn + col * sw, psi_zn + col * sw, stats + 4 * (size_t)col, P,
                                    has_geo ? &geo : nullptr);
    if (lane == 0) status[col] = st;
}

// REINITIALIZATION(NN1, NN2, ILIMIT) (two_phase.f:2033-2474) of one column per warp: ILIMIT
// SSP-RK3 pseudo-time iterations on band layers 1..NN2 (WENO on 1..NN1); ALPHI_EXT is the
// caller's phi array (the reference's call sites hold it zero off the band); only the
// cells of layers 1..NN2 are written.
__global__ void __launch_bounds__(32 * WARPS)
    k_reinitialization(int ncol, int n, double length, double* __restrict__ phi, const int* __restrict__ layer,
                       int ilimit, int* __restrict__ status) {
    __shared__ Win win[WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = blockIdx.x * WARPS + warp;
    if (col >= ncol) return;
    const size_t sp = 2 * (size_t)n + 7;
    double* ph = phi + col * sp;
    Ctx c;
    c.s = &win[warp];
    const int st = load_band_window(c, lane, n, length, ph, layer + col * sp, false);
    if (st == LICA_OK) {
        reinitialization(c, ilimit);
        for (int i = c.blo + lane; i <= c.bhi; i += 32) {
            const int m = c.s->layer[i];
            if (m >= 1 && m <= NN2) ph[c.w0 + i + 2] = c.s->phi[i];
        }
    }
    if (lane == 0) status[col] = st;
}

// GRID_COUPLING(INI_PSI) (two_phase.f:4863-5118) of one column per CTA.  ini = 1: every flow
// cell; ini = 0: the flow cells KCOUMP_VEL(k) of the refined cells of band layers 1..NN1
// (MASK_GLOBAL) -- the cells k = 2K-4 .. 2K+5 are the only ones that can map to flow cell
// K.  PSI_ZN(K), K >= 2: box mean of PSIF over [ZP(K-1), ZP(K)]; PSI_CN(K) over [Z(K),
// Z(K+1)]; every cell snapped at 1e-3 / 0.999; PSI_CN(0) = PSI_CN(1), PSI_CN(n+1) = PSI_CN(n).
__global__ void __launch_bounds__(128)
    k_grid_coupling(int ncol, int n, double length, int ini, const double* __restrict__ psif,
                    const int* __restrict__ layer, double* __restrict__ psi_cn, double* __restrict__ psi_zn) {
    const int col = blockIdx.x;
    if (col >= ncol) return;
    const int nf = 2 * n;
    const double h = length / n, hf = length / nf;
    const double* pf = psif + col * (size_t)(nf + 2);
    const int* lay = layer + col * (size_t)(nf + 7);
    double* cn = psi_cn + col * (size_t)(n + 2);
    double* zn = psi_zn + col * (size_t)(n + 2);
    for (int kk = 1 + (int)threadIdx.x; kk <= n; kk += (int)blockDim.x) {
        bool mk = ini != 0;
        if (!mk)
            for (int k = max(1, 2 * kk - 4); k <= min(nf, 2 * kk + 5); ++k) {
                const int m = lay[k + 2];
                if (m >= 1 && m <= NN1 && col::kcoump_vel(h, hf, n, k) == kk) {
                    mk = true;
                    break;
                }
            }
        double z = zn[kk];
        if (kk >= 2 && mk) z = col::box_mean(pf, nf, 2 * kk - 2, 2 * kk - 1, col::grid_zp(h, n, kk - 1),
                                             col::grid_zp(h, n, kk), hf);
        if (z < 1e-3) z = 0.0;
        else if (z > 0.999) z = 1.0;
        zn[kk] = z;
        double v = cn[kk];
        if (mk) v = col::box_mean(pf, nf, 2 * kk - 1, 2 * kk, col::grid_z(h, kk), col::grid_z(h, kk + 1), hf);
        if (v < 1e-3) v = 0.0;
        else if (v > 0.999) v = 1.0;
        cn[kk] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        cn[0] = cn[1];
        cn[n + 1] = cn[n];
    }
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

int transport_device(int32_t ncol, int32_t n, double length, double* phi, int32_t* layer, double* psif, double* wo,
                     const double* w, const double* mflvs, double* vol_tot_ori, const double* vol_tot_iphs,
                     double* psi_cn, double* psi_zn, int32_t* status, double* stats, const lica_lvs_params* prm,
                     void* stream, const lica_col_geo* geo) {
    int st = check_args(ncol, n, length, prm);
    if (st) return st;
    if (!phi || !layer || !psif || !wo || !w || !mflvs || !vol_tot_ori || !vol_tot_iphs || !psi_cn || !psi_zn ||
        !status || !stats)
        return LICA_BAD_ARG;
    Params P{prm->iphs, prm->first, prm->m_step, prm->mglobal, prm->denr, prm->dtconst};
    const unsigned blocks = (unsigned)((ncol + WARPS - 1) / WARPS);
    const col::ColGeoDev g = geo ? geo->dev : col::ColGeoDev{};
    k_lvs_transport<<<blocks, 32 * WARPS, 0, (cudaStream_t)stream>>>(ncol, n, length, phi, layer, psif, wo, w, mflvs,
                                                                      vol_tot_ori, vol_tot_iphs, psi_cn, psi_zn,
                                                                      status, stats, P, g, geo ? 1 : 0);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

int transport_host(int32_t ncol, int32_t n, double length, double* phi, int32_t* layer, double* psif, double* wo,
                   const double* w, const double* mflvs, double* vol_tot_ori, const double* vol_tot_iphs,
                   double* psi_cn, double* psi_zn, int32_t* status, double* stats, const lica_lvs_params* prm,
                   const lica_col_geo* geo) {
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
    st = transport_device(ncol, n, length, (double*)(base + o_phi), (int32_t*)(base + o_lay),
                          (double*)(base + o_psif), (double*)(base + o_wo), (const double*)(base + o_w),
                          (const double*)(base + o_mf), (double*)(base + o_vo), (const double*)(base + o_vi),
                          (double*)(base + o_cn), (double*)(base + o_zn), (int32_t*)(base + o_st),
                          (double*)(base + o_stats), prm, nullptr, geo);
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

}  // namespace

extern "C" {

int lica_gpu_lvs_transport_device(int32_t ncol, int32_t n, double length, double* phi, int32_t* layer, double* psif,
                                  double* wo, const double* w, const double* mflvs, double* vol_tot_ori,
                                  const double* vol_tot_iphs, double* psi_cn, double* psi_zn, int32_t* status,
                                  double* stats, const lica_lvs_params* prm, void* stream) {
    return transport_device(ncol, n, length, phi, layer, psif, wo, w, mflvs, vol_tot_ori, vol_tot_iphs, psi_cn, psi_zn,
                            status, stats, prm, stream, nullptr);
}

int lica_gpu_lvs_transport(int32_t ncol, int32_t n, double length, double* phi, int32_t* layer, double* psif,
                           double* wo, const double* w, const double* mflvs, double* vol_tot_ori,
                           const double* vol_tot_iphs, double* psi_cn, double* psi_zn, int32_t* status, double* stats,
                           const lica_lvs_params* prm) {
    return transport_host(ncol, n, length, phi, layer, psif, wo, w, mflvs, vol_tot_ori, vol_tot_iphs, psi_cn, psi_zn,
                          status, stats, prm, nullptr);
}

int lica_gpu_lvs_transport_geometry_device(const lica_col_geo* geo, int32_t ncol, double* phi, int32_t* layer,
                                           double* psif, double* wo, const double* w, const double* mflvs,
                                           double* vol_tot_ori, const double* vol_tot_iphs, double* psi_cn,
                                           double* psi_zn, int32_t* status, double* stats, const lica_lvs_params* prm,
                                           void* stream) {
    if (!geo) return LICA_BAD_ARG;
    return transport_device(ncol, geo->n, geo->length, phi, layer, psif, wo, w, mflvs, vol_tot_ori, vol_tot_iphs,
                            psi_cn, psi_zn, status, stats, prm, stream, geo);
}

int lica_gpu_lvs_transport_geometry(const lica_col_geo* geo, int32_t ncol, double* phi, int32_t* layer, double* psif,
                                    double* wo, const double* w, const double* mflvs, double* vol_tot_ori,
                                    const double* vol_tot_iphs, double* psi_cn, double* psi_zn, int32_t* status,
                                    double* stats, const lica_lvs_params* prm) {
    if (!geo) return LICA_BAD_ARG;
    return transport_host(ncol, geo->n, geo->length, phi, layer, psif, wo, w, mflvs, vol_tot_ori, vol_tot_iphs, psi_cn,
                          psi_zn, status, stats, prm, geo);
}

int lica_gpu_reinitialization_device(int32_t ncol, int32_t n, double length, double* phi, const int32_t* layer,
                                     int32_t ilimit, int32_t* status, void* stream) {
    if (ncol < 1 || n < 8 || n > (1 << 24) || !(length > 0.0) || !phi || !layer || ilimit < 0 || !status) {
        lica_set_last_error("lica_gpu_reinitialization_device", "bad sizes or null pointers", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    const unsigned blocks = (unsigned)((ncol + WARPS - 1) / WARPS);
    k_reinitialization<<<blocks, 32 * WARPS, 0, (cudaStream_t)stream>>>(ncol, n, length, phi, layer, ilimit, status);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

int lica_gpu_reinitialization(int32_t ncol, int32_t n, double length, double* phi, const int32_t* layer,
                              int32_t ilimit, int32_t* status) {
    if (ncol < 1 || n < 8 || n > (1 << 24) || !(length > 0.0) || !phi || !layer || ilimit < 0 || !status) {
        lica_set_last_error("lica_gpu_reinitialization", "bad sizes or null pointers", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    const size_t nc = (size_t)ncol, sp = 2 * (size_t)n + 7;
    double* dphi = nullptr;
    int32_t *dlay = nullptr, *dst = nullptr;
    int rc = LICA_OK;
    auto done = [&](int code) {
        cudaFree(dphi);
        cudaFree(dlay);
        cudaFree(dst);
        return code;
    };
    if (cudaMalloc((void**)&dphi, 8 * nc * sp) != cudaSuccess || cudaMalloc((void**)&dlay, 4 * nc * sp) != cudaSuccess ||
        cudaMalloc((void**)&dst, 4 * nc) != cudaSuccess) {
        lica_set_last_error("cudaMalloc", "lica_gpu_reinitialization buffers", __FILE__, __LINE__);
        return done(LICA_ERR_NOMEM);
    }
    if (cudaMemcpy(dphi, phi, 8 * nc * sp, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dlay, layer, 4 * nc * sp, cudaMemcpyHostToDevice) != cudaSuccess)
        return done(LICA_ERR_CUDA);
    if ((rc = lica_gpu_reinitialization_device(ncol, n, length, dphi, dlay, ilimit, dst, nullptr))) return done(rc);
    if (cudaMemcpy(phi, dphi, 8 * nc * sp, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(status, dst, 4 * nc, cudaMemcpyDeviceToHost) != cudaSuccess)
        return done(LICA_ERR_CUDA);
    int worst = LICA_OK;
    for (size_t c = 0; c < nc; ++c)
        if (status[c] != LICA_OK) worst = status[c];
    return done(worst);
}

int lica_gpu_grid_coupling_device(int32_t ncol, int32_t n, double length, int32_t ini_psi, const double* psif,
                                  const int32_t* layer, double* psi_cn, double* psi_zn, void* stream) {
    if (ncol < 1 || n < 8 || n > (1 << 24) || !(length > 0.0) || !psif || !psi_cn || !psi_zn ||
        (ini_psi == 0 && !layer)) {
        lica_set_last_error("lica_gpu_grid_coupling_device", "bad sizes or null pointers", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    k_grid_coupling<<<ncol, 128, 0, (cudaStream_t)stream>>>(ncol, n, length, ini_psi, psif, layer, psi_cn, psi_zn);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

int lica_gpu_grid_coupling(int32_t ncol, int32_t n, double length, int32_t ini_psi, const double* psif,
                           const int32_t* layer, double* psi_cn, double* psi_zn) {
    if (ncol < 1 || n < 8 || n > (1 << 24) || !(length > 0.0) || !psif || !psi_cn || !psi_zn ||
        (ini_psi == 0 && !layer)) {
        lica_set_last_error("lica_gpu_grid_coupling", "bad sizes or null pointers", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    const size_t nc = (size_t)ncol, sp = 2 * (size_t)n + 7, sq = 2 * (size_t)n + 2, sf = (size_t)n + 2;
    double *dpf = nullptr, *dcn = nullptr, *dzn = nullptr;
    int32_t* dlay = nullptr;
    auto done = [&](int code) {
        cudaFree(dpf);
        cudaFree(dcn);
        cudaFree(dzn);
        cudaFree(dlay);
        return code;
    };
    if (cudaMalloc((void**)&dpf, 8 * nc * sq) != cudaSuccess || cudaMalloc((void**)&dcn, 8 * nc * sf) != cudaSuccess ||
        cudaMalloc((void**)&dzn, 8 * nc * sf) != cudaSuccess ||
        (layer && cudaMalloc((void**)&dlay, 4 * nc * sp) != cudaSuccess)) {
        lica_set_last_error("cudaMalloc", "lica_gpu_grid_coupling buffers", __FILE__, __LINE__);
        return done(LICA_ERR_NOMEM);
    }
    if (cudaMemcpy(dpf, psif, 8 * nc * sq, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dcn, psi_cn, 8 * nc * sf, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dzn, psi_zn, 8 * nc * sf, cudaMemcpyHostToDevice) != cudaSuccess ||
        (layer && cudaMemcpy(dlay, layer, 4 * nc * sp, cudaMemcpyHostToDevice) != cudaSuccess))
        return done(LICA_ERR_CUDA);
    int rc = lica_gpu_grid_coupling_device(ncol, n, length, ini_psi, dpf, dlay, dcn, dzn, nullptr);
    if (rc) return done(rc);
    if (cudaMemcpy(psi_cn, dcn, 8 * nc * sf, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(psi_zn, dzn, 8 * nc * sf, cudaMemcpyDeviceToHost) != cudaSuccess)
        return done(LICA_ERR_CUDA);
    return done(LICA_OK);
}

}  // extern "C"
