// pms_material.cu -- batched von Mises return map + consistent tangent (one thread per IP).
//
// Replaces the per-IP virtual calls StressStrainTrait::update_stress / stiffness
// (reference src/material/model_stress_strain.rs:8-43; VonMises src/material/von_mises.rs:124-226;
// LinearElastic src/material/linear_elastic.rs:49-71) by one launch over n IPs.
//
// Layout: structure of arrays, component stride n, so that each warp reads 32 consecutive
// doubles per component (fully coalesced 256-byte transactions).  The tangent is written as
// its upper triangle (21 components in 3D, 10 in plane strain): D is symmetric.
// Roofline: HBM-bound.  Algorithmic bytes per 3D IP: read sigma(6)+z+deps(6)+H = 112 B, write
// sigma(6)+z+lambda+D(21) = 232 B, plus 1 B elastic flag = 345 B; about 200 flop per IP.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <atomic>
#include <mutex>

#include "../../include/pms.h"
#include "pms_device.cuh"

using namespace pms;

namespace {

std::atomic<int64_t> g_launches{0};

__device__ __forceinline__ void report(int32_t* status, int code, int64_t ip) {
    if (status == nullptr || code == OK) return;
    if (atomicCAS(status, 0, code) == 0) {
        status[1] = (int32_t)(ip & 0x7fffffff);
        status[2] = (int32_t)(ip >> 31);
    }
}

template <int NC>
__device__ __forceinline__ void write_tangent(const MatConst& m, double a, double b, const double* s, double* dd,
                                              int64_t i, int64_t n) {
    int k = 0;
#pragma unroll
    for (int r = 0; r < NC; r++) {
#pragma unroll
        for (int c = r; c < NC; c++) {
            double ii = (r < 3 && c < 3) ? m.kk : 0.0;
            dd[(int64_t)k * n + i] = a * psd(r, c) + b * s[r] * s[c] + ii;
            k++;
        }
    }
}

template <int NC, bool UPDATE>
__global__ void __launch_bounds__(256) vm_batch_kernel(MatConst m, int64_t n, double* __restrict__ sig,
                                                       double* __restrict__ z, double* __restrict__ lambda,
                                                       uint8_t* __restrict__ elastic,
                                                       const double* __restrict__ deps,
                                                       const double* __restrict__ hh_ip, double* __restrict__ dd,
                                                       int32_t* status) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double s[NC], de[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) s[c] = sig[(int64_t)c * n + i];
        double hh = hh_ip ? hh_ip[i] : m.hh;
        double lam;
        int el;
        int st = OK;
        if (UPDATE) {
#pragma unroll
            for (int c = 0; c < NC; c++) de[c] = deps[(int64_t)c * n + i];
            double zz = (m.model == 1) ? z[i] : 0.0;
            lam = 0.0;
            el = 1;
            st = ip_update<NC>(m, hh, s, zz, lam, el, de);
#pragma unroll
            for (int c = 0; c < NC; c++) sig[(int64_t)c * n + i] = s[c];
            if (m.model == 1) z[i] = zz;
            lambda[i] = lam;
            elastic[i] = (uint8_t)el;
        } else {
            lam = lambda[i];
            el = elastic[i];
        }
        if (dd) {
            double a, b, dv[NC];
            int st2 = tangent_coefs<NC>(m, hh, s, lam, el, a, b, dv);
            if (st == OK) st = st2;
            write_tangent<NC>(m, a, b, dv, dd, i, n);
        }
        report(status, st, i);
    }
}

// FP64 FMA throughput probe: 8 independent dependent-FMA chains per thread.
__global__ void __launch_bounds__(256) fp64_fma_probe_kernel(int64_t iters, double b, double c, double* out) {
    double a0 = threadIdx.x * 1e-3, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
           a7 = a0 + 7;
    for (int64_t i = 0; i < iters; i++) {
        a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
        a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
    }
    out[(int64_t)blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

int grid_for(int64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t blocks = (n + 255) / 256;
    int64_t cap = (int64_t)sms * 8;  // 8 resident 256-thread blocks per SM, grid-stride beyond
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return (int)blocks;
}

int check_mat(const pms_material* mat, int ndim) {
    if (!mat || (ndim != 2 && ndim != 3)) return PMS_ERR_INVALID;
    if (mat->model != PMS_LINEAR_ELASTIC && mat->model != PMS_VON_MISES) return PMS_ERR_INVALID;
    if (mat->model == PMS_VON_MISES && !(mat->z_ini > F_TOL)) return PMS_ERR_INVALID;
    return PMS_OK;
}

template <bool UPDATE>
int launch(const pms_material* mat, int ndim, int64_t n, double* sig, double* z, double* lambda, uint8_t* elastic,
           const double* deps, const double* hh, double* dd, int32_t* status, cudaStream_t st) {
    int rc = check_mat(mat, ndim);
    if (rc) return rc;
    if (n <= 0) return PMS_OK;
    MatConst m = make_matconst(mat->model, mat->young, mat->poisson, mat->hh, mat->z_ini);
    int grid = grid_for(n);
    if (ndim == 2)
        vm_batch_kernel<4, UPDATE><<<grid, 256, 0, st>>>(m, n, sig, z, lambda, elastic, deps, hh, dd, status);
    else
        vm_batch_kernel<6, UPDATE><<<grid, 256, 0, st>>>(m, n, sig, z, lambda, elastic, deps, hh, dd, status);
    g_launches++;
    return cudaGetLastError() == cudaSuccess ? PMS_OK : PMS_ERR_CUDA;
}

// Device staging for the host-buffer entry point (grown on demand, kept until exit).
struct Staging {
    std::mutex mu;
    void* buf = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
} g_stage;

}  // namespace

extern "C" {

int pms_vm_update_and_stiffness_batch(const pms_material* mat, int32_t ndim, int64_t n, double* sig, double* z,
                                      double* lambda, uint8_t* elastic, const double* deps, const double* hh,
                                      double* dd, int32_t* status, void* stream) {
    return launch<true>(mat, ndim, n, sig, z, lambda, elastic, deps, hh, dd, status, (cudaStream_t)stream);
}

int pms_vm_stiffness_batch(const pms_material* mat, int32_t ndim, int64_t n, const double* sig,
                           const double* lambda, const uint8_t* elastic, const double* hh, double* dd,
                           int32_t* status, void* stream) {
    if (!dd) return PMS_ERR_INVALID;
    return launch<false>(mat, ndim, n, const_cast<double*>(sig), nullptr, const_cast<double*>(lambda),
                         const_cast<uint8_t*>(elastic), nullptr, hh, dd, status, (cudaStream_t)stream);
}

int pms_vm_update_and_stiffness_host(const pms_material* mat, int32_t ndim, int64_t n, double* sig, double* z,
                                     double* lambda, uint8_t* elastic, const double* deps, const double* hh,
                                     double* dd) {
    int rc = check_mat(mat, ndim);
    if (rc) return rc;
    if (n <= 0) return PMS_OK;
    int nc = 2 * ndim, nd = nc * (nc + 1) / 2;
    size_t b_sig = (size_t)nc * n * 8, b_n = (size_t)n * 8;
    size_t need = 2 * b_sig + 3 * b_n + (hh ? b_n : 0) + (dd ? (size_t)nd * n * 8 : 0) + (size_t)n + 64;
    std::lock_guard<std::mutex> lock(g_stage.mu);
    if (!g_stage.stream && cudaStreamCreateWithFlags(&g_stage.stream, cudaStreamNonBlocking) != cudaSuccess)
        return PMS_ERR_CUDA;
    if (g_stage.bytes < need) {
        if (g_stage.buf) cudaFree(g_stage.buf);
        g_stage.buf = nullptr;
        g_stage.bytes = 0;
        if (cudaMalloc(&g_stage.buf, need) != cudaSuccess) return PMS_ERR_NOMEM;
        g_stage.bytes = need;
    }
    char* p = (char*)g_stage.buf;
    int32_t* d_status = (int32_t*)p; p += 64;
    double* d_sig = (double*)p; p += b_sig;
    double* d_deps = (double*)p; p += b_sig;
    double* d_z = (double*)p; p += b_n;
    double* d_lam = (double*)p; p += b_n;
    double* d_hh = nullptr;
    if (hh) { d_hh = (double*)p; p += b_n; }
    double* d_dd = nullptr;
    if (dd) { d_dd = (double*)p; p += (size_t)nd * n * 8; }
    uint8_t* d_el = (uint8_t*)p;
    cudaStream_t s = g_stage.stream;
    cudaMemsetAsync(d_status, 0, 16, s);
    cudaMemcpyAsync(d_sig, sig, b_sig, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_deps, deps, b_sig, cudaMemcpyHostToDevice, s);
    if (mat->model == PMS_VON_MISES) cudaMemcpyAsync(d_z, z, b_n, cudaMemcpyHostToDevice, s);
    if (hh) cudaMemcpyAsync(d_hh, hh, b_n, cudaMemcpyHostToDevice, s);
    rc = launch<true>(mat, ndim, n, d_sig, d_z, d_lam, d_el, d_deps, d_hh, d_dd, d_status, s);
    if (rc) return rc;
    cudaMemcpyAsync(sig, d_sig, b_sig, cudaMemcpyDeviceToHost, s);
    if (mat->model == PMS_VON_MISES && z) cudaMemcpyAsync(z, d_z, b_n, cudaMemcpyDeviceToHost, s);
    if (lambda) cudaMemcpyAsync(lambda, d_lam, b_n, cudaMemcpyDeviceToHost, s);
    if (elastic) cudaMemcpyAsync(elastic, d_el, (size_t)n, cudaMemcpyDeviceToHost, s);
    if (dd) cudaMemcpyAsync(dd, d_dd, (size_t)nd * n * 8, cudaMemcpyDeviceToHost, s);
    int32_t hst[4] = {0, 0, 0, 0};
    cudaMemcpyAsync(hst, d_status, 16, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return PMS_ERR_CUDA;
    return hst[0];
}

int64_t pms_material_launch_count(void) { return g_launches.load(); }

int pms_probe_fp64_fma(int64_t iters, int32_t blocks, double* out, void* stream) {
    if (iters < 1 || blocks < 1 || !out) return PMS_ERR_INVALID;
    fp64_fma_probe_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, 0.999999, 1e-7, out);
    return cudaGetLastError() == cudaSuccess ? PMS_OK : PMS_ERR_CUDA;
}

const char* pms_version(void) { return "pms_b200 0.1.0 (sm_100a, FP64)"; }

// The calling host thread's device (cudaSetDevice / cudaGetDeviceCount), for callers without a CUDA
// runtime binding of their own: handles are created on, and run on, the current device of the thread
// that creates them.
int pms_set_device(int32_t device) {
    return cudaSetDevice(device) == cudaSuccess ? PMS_OK : PMS_ERR_CUDA;
}
int pms_device_count(int32_t* count) {
    int n = 0;
    if (!count) return PMS_ERR_INVALID;
    if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
    *count = n;
    return PMS_OK;
}

}  // extern "C"
