// Tridiagonal solvers and the 1-D pressure POISSON of the reference, on the GPU.
//
// TRDIAG3 / TRDIAG3P (1d.f:3783-3983) solve one system per line I, the line index being
// the leading (contiguous) Fortran dimension: one thread per line, so the loads of a
// warp at a given J are coalesced.  The Thomas recurrences keep the reference's
// statement order (BET = 1/B then products) and the library is built without FMA
// contraction, so results are bit-identical to the CPU restatement.  The forward-sweep
// coefficients (GAM, or Q/S/QE for the periodic variant) live in a device scratch
// buffer laid out like the arrays themselves (line index fastest).
#include "common.cuh"

#include <mutex>
#include <vector>

extern "C" void lica_count_launches(int64_t n);

namespace lica {
namespace tri {

__global__ void k_trdiag3(const double* __restrict__ A, const double* __restrict__ B, const double* __restrict__ C,
                          double* R, double* UU, double* __restrict__ gam, int64_t l1, int64_t l2, int64_t ll1,
                          int64_t ll2, int64_t ld) {
    const int64_t i = ll1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i > ll2) return;
    auto at = [ld](int64_t ii, int64_t jj) { return (size_t)((ii - 1) + (jj - 1) * ld); };
    double bet = 1.0 / B[at(i, l1)];
    UU[at(i, l1)] = R[at(i, l1)] * bet;
    for (int64_t j = l1 + 1; j <= l2; ++j) {
        const double g = C[at(i, j - 1)] * bet;
        gam[at(i, j)] = g;
        bet = 1.0 / (B[at(i, j)] - A[at(i, j)] * g);
        UU[at(i, j)] = (R[at(i, j)] - A[at(i, j)] * UU[at(i, j - 1)]) * bet;
    }
    for (int64_t j = l2 - 1; j >= l1; --j) {
        const double u = UU[at(i, j)] - gam[at(i, j + 1)] * UU[at(i, j + 1)];
        UU[at(i, j)] = u;
        R[at(i, j)] = u;
    }
}

__global__ void k_trdiag3p(const double* __restrict__ A, const double* __restrict__ B, const double* __restrict__ C,
                           double* __restrict__ F, double* __restrict__ Q, double* __restrict__ S,
                           double* __restrict__ QE, int64_t j1, int64_t j2, int64_t l1, int64_t l2, int64_t ld) {
    const int64_t k = l1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k > l2) return;
    auto at = [ld](int64_t kk, int64_t jj) { return (size_t)((kk - 1) + (jj - 1) * ld); };
    const int64_t ja = j1 + 1, jj = j1 + j2;
    const double binv = 1.0 / B[at(k, j1)];
    Q[at(k, j1)] = -C[at(k, j1)] * binv;
    S[at(k, j1)] = -A[at(k, j1)] * binv;
    const double fn = F[at(k, j2)];
    F[at(k, j1)] = F[at(k, j1)] * binv;
    for (int64_t j = ja; j <= j2; ++j) {
        const double pn = 1.0 / (B[at(k, j)] + A[at(k, j)] * Q[at(k, j - 1)]);
        Q[at(k, j)] = -C[at(k, j)] * pn;
        S[at(k, j)] = -A[at(k, j)] * S[at(k, j - 1)] * pn;
        F[at(k, j)] = (F[at(k, j)] - A[at(k, j)] * F[at(k, j - 1)]) * pn;
    }
    S[at(k, j2)] = 1.0;
    QE[at(k, j2)] = 0.0;
    for (int64_t ii = ja; ii <= j2; ++ii) {
        const int64_t j = jj - ii;
        S[at(k, j)] = S[at(k, j)] + Q[at(k, j)] * S[at(k, j + 1)];
        QE[at(k, j)] = F[at(k, j)] + Q[at(k, j)] * QE[at(k, j + 1)];
    }
    F[at(k, j2)] = (fn - C[at(k, j2)] * QE[at(k, j1)] - A[at(k, j2)] * QE[at(k, j2 - 1)]) /
                   (C[at(k, j2)] * S[at(k, j1)] + A[at(k, j2)] * S[at(k, j2 - 1)] + B[at(k, j2)]);
    for (int64_t ii = ja; ii <= j2; ++ii) {
        const int64_t j = jj - ii;
        F[at(k, j)] = F[at(k, j2)] * S[at(k, j)] + QE[at(k, j)];
    }
}

// POISSON (1d.f:3492-3578): coefficients, Thomas forward/back substitution, P(1,1,K),
// then the K ghosts for every (I,J) in [1,n1m] x [1,n2m].  One CTA; thread 0 runs the
// recurrence with GAM and UU in shared memory, the ghost copies use every thread.
__global__ void k_poisson1d(int64_t m1, int64_t m2, int64_t n1m, int64_t n2m, int64_t n3m,
                            const double* __restrict__ vvdz, const double* __restrict__ ssdz,
                            const double* __restrict__ fixkl, const int64_t* __restrict__ kpv, double* p,
                            const double* __restrict__ divgsum, const double* __restrict__ denf_zi) {
    extern __shared__ double sh[];
    double* gam = sh;             // n3m + 2
    double* uu = sh + (n3m + 2);  // n3m + 2
    const int64_t s1 = m1 + 1, s2 = (m1 + 1) * (m2 + 1);
    const int64_t d1 = m1 - 1, d2 = (m1 - 1) * (m2 - 1);
    auto f3 = [&](int64_t i, int64_t j, int64_t k) { return (size_t)(i + s1 * j + s2 * k); };
    auto dv = [&](int64_t i, int64_t j, int64_t k) { return (size_t)((i - 1) + d1 * (j - 1) + d2 * (k - 1)); };
    if (threadIdx.x == 0) {
        auto coeffs = [&](int64_t k, double& ak, double& bk, double& ck) {
            const int64_t kp1 = kpv[k];
            ak = vvdz[k - 1] * ssdz[k] * denf_zi[f3(1, 1, k)] * (1.0 - fixkl[k - 1]);
            ck = vvdz[kp1 - 1] * ssdz[k] * denf_zi[f3(1, 1, kp1)];
            bk = -(ak + ck);
        };
        double ak, bk, ck, ck_prev;
        coeffs(1, ak, bk, ck);
        double bet = 1.0 / bk;
        uu[1] = divgsum[dv(1, 1, 1)] * bet;
        ck_prev = ck;
        for (int64_t k = 2; k <= n3m; ++k) {
            coeffs(k, ak, bk, ck);
            const double g = ck_prev * bet;
            gam[k] = g;
            bet = 1.0 / (bk - ak * g);
            uu[k] = (divgsum[dv(1, 1, k)] - ak * uu[k - 1]) * bet;
            ck_prev = ck;
        }
        for (int64_t k = n3m - 1; k >= 1; --k) uu[k] = uu[k] - gam[k + 1] * uu[k + 1];
    }
    __syncthreads();
    for (int64_t k = 1 + threadIdx.x; k <= n3m; k += blockDim.x) p[f3(1, 1, k)] = uu[k];
    __syncthreads();
    for (int64_t t = threadIdx.x; t < n1m * n2m; t += blockDim.x) {
        const int64_t i = 1 + t % n1m, j = 1 + t / n1m;
        p[f3(i, j, 0)] = p[f3(i, j, 1)];
        p[f3(i, j, n3m + 1)] = p[f3(i, j, n3m)];
    }
}

// Grow-only device scratch shared by the tridiagonal entry points of this process.
struct Scratch {
    std::mutex mu;
    double* ptr = nullptr;
    size_t bytes = 0;
};
Scratch& scratch() {
    static Scratch s;
    return s;
}

int get_scratch(size_t bytes, double** out) {
    Scratch& s = scratch();
    if (bytes > s.bytes) {
        if (s.ptr) cudaFree(s.ptr);
        s.ptr = nullptr;
        s.bytes = 0;
        LICA_CUDA_TRY(cudaMalloc((void**)&s.ptr, bytes));
        s.bytes = bytes;
    }
    *out = s.ptr;
    return LICA_OK;
}

struct DevBufs {
    std::vector<void*> ptrs;
    ~DevBufs() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    int alloc_copy(T** d, const T* h, size_t n) {
        void* p = nullptr;
        LICA_CUDA_TRY(cudaMalloc(&p, sizeof(T) * n));
        ptrs.push_back(p);
        if (h) LICA_CUDA_TRY(cudaMemcpy(p, h, sizeof(T) * n, cudaMemcpyHostToDevice));
        *d = (T*)p;
        return LICA_OK;
    }
};

// Fixed scratch for lica_gpu_trdiag3_noalloc_device: 2 MiB of doubles, enough for
// ld * l2 <= 262144 (e.g. 512 lines of 512 unknowns).  Every GPU that loads this library
// holds it until the process exits.  All calls on a device share it.
constexpr size_t kNoAllocScratchDoubles = 262144;
static __device__ __align__(256) double g_trdiag3_noalloc_scratch[kNoAllocScratchDoubles];

// Device address of g_trdiag3_noalloc_scratch per device ordinal, looked up once with the
// device current (host code may not use the symbol itself as a device pointer).
std::mutex g_noalloc_mu;
constexpr int kMaxDevices = 128;
double* g_noalloc_addr[kMaxDevices] = {};

}  // namespace tri
}  // namespace lica

using namespace lica::tri;

extern "C" {

int lica_gpu_trdiag3_device(const double* A, const double* B, const double* C, double* R, double* UU, int64_t l1,
                            int64_t l2, int64_t ll1, int64_t ll2, int64_t ld, void* stream) {
    if (!A || !B || !C || !R || !UU || l2 < l1 || ll2 < ll1 || ll1 < 1 || ld < ll2 || l1 < 1) return LICA_BAD_ARG;
    std::lock_guard<std::mutex> lk(scratch().mu);
    double* gam;
    int st = get_scratch(sizeof(double) * (size_t)ld * (size_t)l2, &gam);
    if (st) return st;
    const int64_t nlines = ll2 - ll1 + 1;
    const int threads = 128;
    const unsigned blocks = (unsigned)((nlines + threads - 1) / threads);
    k_trdiag3<<<blocks, threads, 0, (cudaStream_t)stream>>>(A, B, C, R, UU, gam, l1, l2, ll1, ll2, ld);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    LICA_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return LICA_OK;
}

int lica_gpu_trdiag3p_device(const double* A, const double* B, const double* C, double* F, int64_t j1, int64_t j2,
                             int64_t l1, int64_t l2, int64_t ld, void* stream) {
    if (!A || !B || !C || !F || j2 <= j1 || j1 < 1 || l2 < l1 || l1 < 1 || ld < l2) return LICA_BAD_ARG;
    std::lock_guard<std::mutex> lk(scratch().mu);
    double* sc;
    const size_t plane = (size_t)ld * (size_t)j2;
    int st = get_scratch(sizeof(double) * 3 * plane, &sc);
    if (st) return st;
    const int64_t nlines = l2 - l1 + 1;
    const int threads = 128;
    const unsigned blocks = (unsigned)((nlines + threads - 1) / threads);
    k_trdiag3p<<<blocks, threads, 0, (cudaStream_t)stream>>>(A, B, C, F, sc, sc + plane, sc + 2 * plane, j1, j2, l1,
                                                              l2, ld);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    LICA_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return LICA_OK;
}

// TRDIAG3 on device arrays without allocating: same kernel and results as
// lica_gpu_trdiag3_device, with the forward-sweep coefficients kept in the fixed scratch
// array above instead of cudaMalloc'd memory.  The first call on a device looks up the
// scratch address (cudaGetSymbolAddress) and should come before any stream capture.
// The address is kept per device ordinal for the life of the process: do not call this
// entry point again on a device after cudaDeviceReset (the module may be reloaded at
// another address).  Returns after enqueueing the kernel on `stream` (no synchronisation).  Calls that
// overlap on the GPU (different streams, or different host threads on one device) share
// the scratch and race.  The scratch needs no clearing: each line writes every
// coefficient before it reads it.
int lica_gpu_trdiag3_noalloc_device(const double* A, const double* B, const double* C, double* R, double* UU,
                                    int64_t l1, int64_t l2, int64_t ll1, int64_t ll2, int64_t ld, void* stream) {
    if (!A || !B || !C || !R || !UU || l2 < l1 || ll2 < ll1 || ll1 < 1 || ld < ll2 || l1 < 1) return LICA_BAD_ARG;
    if ((double)ld * (double)l2 > (double)kNoAllocScratchDoubles) {
        lica_set_last_error("lica_gpu_trdiag3_noalloc_device",
                            "ld * l2 exceeds the fixed scratch of 262144 doubles (2 MiB)", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    int dev = -1;
    LICA_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        lica_set_last_error("lica_gpu_trdiag3_noalloc_device", "device ordinal outside 0..127", __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    double* gam = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            void* addr = nullptr;
            LICA_CUDA_TRY(cudaGetSymbolAddress(&addr, g_trdiag3_noalloc_scratch));
            g_noalloc_addr[dev] = static_cast<double*>(addr);
        }
        gam = g_noalloc_addr[dev];
    }
    const int64_t nlines = ll2 - ll1 + 1;
    const int threads = 128;
    const unsigned blocks = (unsigned)((nlines + threads - 1) / threads);
    k_trdiag3<<<blocks, threads, 0, (cudaStream_t)stream>>>(A, B, C, R, UU, gam, l1, l2, ll1, ll2, ld);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    return LICA_OK;
}

int lica_gpu_trdiag3(const double* A, const double* B, const double* C, double* R, double* UU, int64_t l1, int64_t l2,
                     int64_t ll1, int64_t ll2, int64_t ld) {
    if (!A || !B || !C || !R || !UU || l2 < l1 || ll2 < ll1 || ll1 < 1 || ld < ll2 || l1 < 1) return LICA_BAD_ARG;
    const size_t n = (size_t)ld * (size_t)l2;
    DevBufs b;
    double *dA, *dB, *dC, *dR, *dU;
    int st;
    if ((st = b.alloc_copy(&dA, A, n)) || (st = b.alloc_copy(&dB, B, n)) || (st = b.alloc_copy(&dC, C, n)) ||
        (st = b.alloc_copy(&dR, (const double*)R, n)))
        return st;
    const bool alias = (R == UU);
    if (alias) dU = dR;
    else if ((st = b.alloc_copy(&dU, (const double*)UU, n))) return st;
    if ((st = lica_gpu_trdiag3_device(dA, dB, dC, dR, dU, l1, l2, ll1, ll2, ld, nullptr))) return st;
    LICA_CUDA_TRY(cudaMemcpy(R, dR, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (!alias) LICA_CUDA_TRY(cudaMemcpy(UU, dU, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return LICA_OK;
}

int lica_gpu_trdiag3p(const double* A, const double* B, const double* C, double* F, int64_t j1, int64_t j2, int64_t l1,
                      int64_t l2, int64_t ld) {
    if (!A || !B || !C || !F || j2 <= j1 || j1 < 1 || l2 < l1 || l1 < 1 || ld < l2) return LICA_BAD_ARG;
    const size_t n = (size_t)ld * (size_t)j2;
    DevBufs b;
    double *dA, *dB, *dC, *dF;
    int st;
    if ((st = b.alloc_copy(&dA, A, n)) || (st = b.alloc_copy(&dB, B, n)) || (st = b.alloc_copy(&dC, C, n)) ||
        (st = b.alloc_copy(&dF, (const double*)F, n)))
        return st;
    if ((st = lica_gpu_trdiag3p_device(dA, dB, dC, dF, j1, j2, l1, l2, ld, nullptr))) return st;
    LICA_CUDA_TRY(cudaMemcpy(F, dF, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return LICA_OK;
}

int lica_gpu_poisson(int64_t m1, int64_t m2, int64_t m3, int64_t n1m, int64_t n2m, int64_t n3m, const double* vvdz,
                     const double* ssdz, const double* fixkl, const int64_t* kpv, double* p, const double* divgsum,
                     const double* denf_zi) {
    if (!vvdz || !ssdz || !fixkl || !kpv || !p || !divgsum || !denf_zi) return LICA_BAD_ARG;
    if (n1m != 1 || n2m != 1 || n3m < 1 || n3m > m3 - 1 || m1 < 2 || m2 < 2 || n3m > 6000) {
        lica_set_last_error("lica_gpu_poisson", "only the 1-D column (N1M = N2M = 1, N3M <= 6000) is supported",
                            __FILE__, __LINE__);
        return LICA_BAD_ARG;
    }
    for (int64_t k = 1; k <= n3m; ++k)
        if (kpv[k] < 1 || kpv[k] > m3) return LICA_BAD_ARG;
    const size_t n3d = (size_t)(m1 + 1) * (m2 + 1) * (m3 + 1);
    const size_t ndv = (size_t)(m1 - 1) * (m2 - 1) * (m3 - 1);
    DevBufs b;
    double *dvv, *dss, *dfix, *dp, *ddiv, *dden;
    int64_t* dkpv;
    int st;
    if ((st = b.alloc_copy(&dvv, vvdz, (size_t)m3)) || (st = b.alloc_copy(&dss, ssdz, (size_t)m3 + 1)) ||
        (st = b.alloc_copy(&dfix, fixkl, (size_t)m3 - 1)) || (st = b.alloc_copy(&dkpv, kpv, (size_t)m3 + 2)) ||
        (st = b.alloc_copy(&dp, (const double*)p, n3d)) || (st = b.alloc_copy(&ddiv, divgsum, ndv)) ||
        (st = b.alloc_copy(&dden, denf_zi, n3d)))
        return st;
    const size_t smem = sizeof(double) * 2 * (size_t)(n3m + 2);
    if (smem > 48 * 1024)
        LICA_CUDA_TRY(cudaFuncSetAttribute(k_poisson1d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_poisson1d<<<1, 256, smem>>>(m1, m2, n1m, n2m, n3m, dvv, dss, dfix, dkpv, dp, ddiv, dden);
    LICA_CUDA_TRY(cudaGetLastError());
    lica_count_launches(1);
    LICA_CUDA_TRY(cudaMemcpy(p, dp, sizeof(double) * n3d, cudaMemcpyDeviceToHost));
    return LICA_OK;
}

}  // extern "C"
