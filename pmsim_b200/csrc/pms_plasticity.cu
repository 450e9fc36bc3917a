// pms_plasticity.cu -- general elastoplastic stress update, batched: one thread per IP.
//
// Replaces Elastoplastic::update_stress (reference src/material/elastoplastic.rs:539-641) with the
// von Mises plasticity model (PlasticityTrait for VonMises, src/material/von_mises.rs:229-282),
// the only model that Elastoplastic::new accepts (elastoplastic.rs:129-135).  Per IP:
//
//   1. yield function f = sigma_d - z (von_mises.rs:236-240) at the start;
//   2. case selection (select_case, elastoplastic.rs:437-499): inside (A) or on/outside (B);
//      going inside when (df/dsigma) : D_e : deps < 0 (going_inside, :379-389); the crossings of
//      the yield surface along the elastic path (intersection_finding, :394-435) give the cases
//      AE, AXB(t), BE, BXP(t), BP with the pseudo-time tolerance 1e-7;
//   3. the elastic part: sigma(t) = sigma0 + t D_e : deps;
//   4. the elastoplastic part: the ODE dsigma/dt = D_ep : deps, dz/dt = Lambda_d H
//      (ode_system_ep, :159-205) from t_int (or 0) to 1.
//
// Two departures from the reference's numerics, both because the B200 path needs no host-side
// solver objects and both exact for this model:
//   * the elastic path is linear in t (linear elasticity), so f(t) = 0 is the root of a quadratic
//     in t, solved in closed form; the reference finds the same roots with a Chebyshev interpolant
//     of f (30 points, truncated at 1e-8) and its companion-matrix root finder;
//   * the ODE is integrated with the Dormand-Prince 5(4) pair (Dormand & Prince 1980, 7 stages,
//     first-same-as-last) and the standard step-size controller (Hairer, Norsett & Wanner, Solving
//     ODEs I, II.4); the reference uses russell_ode's DoPri8.  Along a radial path D_ep : deps is
//     constant and every Runge-Kutta method is exact; elsewhere both are accurate to the tolerance.
//
// The tangent of this model is not built: the reference's Elastoplastic::stiffness returns
// Err("TODO") (elastoplastic.rs:528-537).
// Roofline: HBM-bound for elastic and radial IPs (reads sigma, z, deps: 13 doubles in 3D; writes
// sigma, z, flag); a few thousand FP64 flops per plastic IP otherwise.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/pms.h"
#include "pms_device.cuh"

using namespace pms;

namespace {

constexpr double NUMERATOR_TOL = 1e-8;     // elastoplastic.rs:17
constexpr double PSEUDO_TIME_TOL = 1e-7;   // elastoplastic.rs:23
constexpr double SIGMA_D_SINGULAR = 1e-10;  // df/dsigma is undefined at sigma_d = 0

enum EpErr : int {
    E_DF_DSIGMA = PMS_ERR_DF_DSIGMA,
    E_NUMERATOR = PMS_ERR_NUMERATOR,
    E_ODE = PMS_ERR_ODE,
    E_INTERSECTION = PMS_ERR_INTERSECTION,
};

struct EpConst {
    double rtol, atol, h_ini;
    int max_steps;
};

__device__ __forceinline__ void report(int32_t* status, int code, int64_t ip) {
    if (status == nullptr || code == OK) return;
    if (atomicCAS(status, 0, code) == 0) {
        status[1] = (int32_t)(ip & 0x7fffffff);
        status[2] = (int32_t)(ip >> 31);
    }
}

// deviator of a Mandel vector (the shear components are already deviatoric)
template <int NC>
__device__ __forceinline__ void deviator(const double* v, double* d) {
    const double m = (v[0] + v[1] + v[2]) / 3.0;
    d[0] = v[0] - m;
    d[1] = v[1] - m;
    d[2] = v[2] - m;
#pragma unroll
    for (int i = 3; i < NC; i++) d[i] = v[i];
}

template <int NC>
__device__ __forceinline__ double ddot(const double* a, const double* b) {
    double r = 0.0;
#pragma unroll
    for (int i = 0; i < NC; i++) r = fma(a[i], b[i], r);
    return r;
}

// Right-hand side of the elastoplastic ODE (elastoplastic.rs:159-205) for von Mises:
//   n = df/dsigma = 3/2 s / sigma_d,  df/dz = -1,  H_yf = H  =>  M_p = H,
//   N_p = M_p + n : D_e : n,  dsigma/dt = D_e : deps - (D_e : n)(n : D_e : deps) / N_p,
//   dz/dt = max(0, n : D_e : deps) / N_p * H.
// y = [sigma(NC), z]; dse = D_e : deps (constant: linear elasticity).
template <int NC>
__device__ __forceinline__ int ep_rates(const MatConst& m, const double* y, const double* deps, const double* dse,
                                        double* dy) {
    double s[NC];
    deviator<NC>(y, s);
    const double sd = sqrt(1.5 * ddot<NC>(s, s));
    if (!(sd > SIGMA_D_SINGULAR)) return E_DF_DSIGMA;
    double n[NC], den[NC];
#pragma unroll
    for (int i = 0; i < NC; i++) {
        n[i] = 1.5 * s[i] / sd;
        den[i] = 0.0;
    }
    hooke_add<NC>(m, den, n);  // D_e : n
    const double np = m.hh + ddot<NC>(n, den);
    const double numerator = ddot<NC>(den, deps);  // n : D_e : deps
    if (numerator < -NUMERATOR_TOL) return E_NUMERATOR;
    const double c = numerator / np;
#pragma unroll
    for (int i = 0; i < NC; i++) dy[i] = dse[i] - den[i] * c;
    dy[NC] = fmax(0.0, numerator) / np * m.hh;
    return OK;
}

// Dormand-Prince 5(4) with the standard controller, from t0 to 1.  Returns an Err code; *nstep
// receives the steps taken (accepted and rejected).
template <int NC>
__device__ int ep_integrate(const MatConst& m, const EpConst& e, double t0, double* y, const double* deps,
                            const double* dse, int* nstep) {
    constexpr int D = NC + 1;
    // Butcher tableau (Dormand & Prince 1980); the 5th-order weights equal row 7 (FSAL)
    constexpr double a21 = 1.0 / 5.0;
    constexpr double a31 = 3.0 / 40.0, a32 = 9.0 / 40.0;
    constexpr double a41 = 44.0 / 45.0, a42 = -56.0 / 15.0, a43 = 32.0 / 9.0;
    constexpr double a51 = 19372.0 / 6561.0, a52 = -25360.0 / 2187.0, a53 = 64448.0 / 6561.0, a54 = -212.0 / 729.0;
    constexpr double a61 = 9017.0 / 3168.0, a62 = -355.0 / 33.0, a63 = 46732.0 / 5247.0, a64 = 49.0 / 176.0,
                     a65 = -5103.0 / 18656.0;
    constexpr double b1 = 35.0 / 384.0, b3 = 500.0 / 1113.0, b4 = 125.0 / 192.0, b5 = -2187.0 / 6784.0,
                     b6 = 11.0 / 84.0;
    // error weights: 5th-order minus 4th-order weights
    constexpr double e1 = 71.0 / 57600.0, e3 = -71.0 / 16695.0, e4 = 71.0 / 1920.0, e5 = -17253.0 / 339200.0,
                     e6 = 22.0 / 525.0, e7 = -1.0 / 40.0;
    double k1[D], k2[D], k3[D], k4[D], k5[D], k6[D], k7[D], yt[D], y5[D];
    double t = t0;
    double h = fmin(e.h_ini, 1.0 - t0);
    int rc = ep_rates<NC>(m, y, deps, dse, k1);
    if (rc != OK) return rc;
    bool rejected = false;
    int steps = 0;
    while (t < 1.0) {
        if (steps >= e.max_steps) {
            *nstep = steps;
            return E_ODE;
        }
        steps++;
        const bool last = t + h >= 1.0;
        if (last) h = 1.0 - t;
#pragma unroll
        for (int i = 0; i < D; i++) yt[i] = y[i] + h * (a21 * k1[i]);
        if ((rc = ep_rates<NC>(m, yt, deps, dse, k2)) != OK) break;
#pragma unroll
        for (int i = 0; i < D; i++) yt[i] = y[i] + h * (a31 * k1[i] + a32 * k2[i]);
        if ((rc = ep_rates<NC>(m, yt, deps, dse, k3)) != OK) break;
#pragma unroll
        for (int i = 0; i < D; i++) yt[i] = y[i] + h * (a41 * k1[i] + a42 * k2[i] + a43 * k3[i]);
        if ((rc = ep_rates<NC>(m, yt, deps, dse, k4)) != OK) break;
#pragma unroll
        for (int i = 0; i < D; i++) yt[i] = y[i] + h * (a51 * k1[i] + a52 * k2[i] + a53 * k3[i] + a54 * k4[i]);
        if ((rc = ep_rates<NC>(m, yt, deps, dse, k5)) != OK) break;
#pragma unroll
        for (int i = 0; i < D; i++)
            yt[i] = y[i] + h * (a61 * k1[i] + a62 * k2[i] + a63 * k3[i] + a64 * k4[i] + a65 * k5[i]);
        if ((rc = ep_rates<NC>(m, yt, deps, dse, k6)) != OK) break;
#pragma unroll
        for (int i = 0; i < D; i++)
            y5[i] = y[i] + h * (b1 * k1[i] + b3 * k3[i] + b4 * k4[i] + b5 * k5[i] + b6 * k6[i]);
        if ((rc = ep_rates<NC>(m, y5, deps, dse, k7)) != OK) break;
        double err = 0.0;
#pragma unroll
        for (int i = 0; i < D; i++) {
            const double ei = h * (e1 * k1[i] + e3 * k3[i] + e4 * k4[i] + e5 * k5[i] + e6 * k6[i] + e7 * k7[i]);
            const double sc = e.atol + e.rtol * fmax(fabs(y[i]), fabs(y5[i]));
            err += (ei / sc) * (ei / sc);
        }
        err = sqrt(err / D);
        // new step: h * min(fac_max, max(fac_min, 0.9 err^(-1/5)))
        double fac = err > 0.0 ? 0.9 * pow(err, -0.2) : 10.0;
        if (err <= 1.0) {
            t = last ? 1.0 : t + h;
#pragma unroll
            for (int i = 0; i < D; i++) {
                y[i] = y5[i];
                k1[i] = k7[i];
            }
            fac = fmin(rejected ? 1.0 : 10.0, fmax(0.2, fac));
            rejected = false;
        } else {
            fac = fmin(1.0, fmax(0.2, fac));
            rejected = true;
        }
        h *= fac;
    }
    *nstep = steps;
    return rc;
}

// One IP: returns an Err code; writes sigma, z, the elastic flag and the case.
template <int NC>
__device__ int ep_update_ip(const MatConst& m, const EpConst& e, double* sig, double& z, int& elastic,
                            const double* deps, int& cs, int& nstep) {
    double dse[NC];
#pragma unroll
    for (int i = 0; i < NC; i++) dse[i] = 0.0;
    hooke_add<NC>(m, dse, deps);  // D_e : deps
    double s0[NC], ds[NC];
    deviator<NC>(sig, s0);
    deviator<NC>(dse, ds);
    // along sigma(t) = sigma0 + t dse with z frozen: 3/2 |s0 + t ds|^2 = z^2  <=>
    // a t^2 + 2 b t + cp = 0, a = ds:ds, b = s0:ds, cp = s0:s0 - 2/3 z^2
    const double a = ddot<NC>(ds, ds), b = ddot<NC>(s0, ds), c = ddot<NC>(s0, s0);
    const double cp = c - (2.0 / 3.0) * z * z;
    const double f0 = sqrt(1.5 * c) - z;
    double t_int = 0.0;
    nstep = 0;
    if (f0 < 0.0) {
        // A: inside.  cp < 0, so g(t) = a t^2 + 2 b t + cp has one positive root (a > 0)
        bool root = false;
        if (a > 0.0) {
            const double sq = sqrt(b * b - a * cp);
            t_int = b >= 0.0 ? -cp / (b + sq) : (sq - b) / a;
            root = t_int <= 1.0;
        }
        if (!root) cs = PMS_EP_AE;
        else if (t_int <= PSEUDO_TIME_TOL) cs = PMS_EP_BP;
        else if (t_int >= 1.0 - PSEUDO_TIME_TOL) cs = PMS_EP_AE;
        else cs = PMS_EP_AXB;
    } else {
        // B: on or outside.  going inside: (df/dsigma) : D_e : deps = 3/2 (s0 : dse) / sigma_d < 0
        const double sd0 = f0 + z;
        if (!(sd0 > SIGMA_D_SINGULAR)) return E_DF_DSIGMA;
        // loading tangent to the surface (indicator zero up to rounding, |s0:ds| <= 1e-10 |s0||ds|)
        // is not going inside: the reference's own tangent path (update_stress_von_mises_5) is BP
        const double indicator = 1.5 * b / sd0;
        if (indicator < -1e-10 * 1.5 * sqrt(a * c) / sd0) {
            // b < 0 and cp >= 0 (up to rounding): the smaller root is the start point (counted as
            // a crossing, t1 ~ 0), the larger one is where the path leaves the surface again
            int nroot = 0;
            double t2 = 2.0;
            const double disc = b * b - a * cp;
            if (a > 0.0 && disc >= 0.0) {
                const double q = sqrt(disc) - b;  // > 0
                const double t1 = cp / q;
                t2 = q / a;
                // a second crossing at t = 1 up to rounding still counts (it ends the path on the surface)
                nroot = (t1 <= 1.0 ? 1 : 0) + (t2 >= 0.0 && t2 <= 1.0 + PSEUDO_TIME_TOL ? 1 : 0);
            }
            if (nroot == 2) {
                t_int = t2;
                if (t_int <= PSEUDO_TIME_TOL) cs = PMS_EP_BP;
                else if (t_int >= 1.0 - PSEUDO_TIME_TOL) cs = PMS_EP_BE;
                else cs = PMS_EP_BXP;
            } else {
                // no way back out: the trial point must lie inside (elastoplastic.rs:484)
                const double f1 = sqrt(1.5 * (a + 2.0 * b + c)) - z;
                if (f1 > 0.0) return E_INTERSECTION;
                cs = PMS_EP_BE;
            }
        } else {
            cs = PMS_EP_BP;
        }
    }
    if (cs == PMS_EP_AE || cs == PMS_EP_BE) {
#pragma unroll
        for (int i = 0; i < NC; i++) sig[i] += dse[i];
        elastic = 1;
        return OK;
    }
    double y[NC + 1];
    const double t0 = (cs == PMS_EP_BP) ? 0.0 : t_int;
#pragma unroll
    for (int i = 0; i < NC; i++) y[i] = sig[i] + t0 * dse[i];
    y[NC] = z;
    const int rc = ep_integrate<NC>(m, e, t0, y, deps, dse, &nstep);
    if (rc != OK) return rc;
#pragma unroll
    for (int i = 0; i < NC; i++) sig[i] = y[i];
    z = y[NC];
    elastic = 0;
    return OK;
}

template <int NC>
__global__ void __launch_bounds__(128) ep_update_kernel(MatConst m, EpConst e, int64_t n, double* __restrict__ sig,
                                                        double* __restrict__ z, uint8_t* __restrict__ elastic,
                                                        const double* __restrict__ deps, int32_t* __restrict__ cases,
                                                        int32_t* __restrict__ steps, int32_t* status) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double s[NC], de[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) {
            s[c] = sig[(int64_t)c * n + i];
            de[c] = deps[(int64_t)c * n + i];
        }
        double zi = z[i];
        int el = elastic[i], cs = -1, ns = 0;
        const int rc = ep_update_ip<NC>(m, e, s, zi, el, de, cs, ns);
        if (rc != OK) {
            report(status, rc, i);
        } else {
#pragma unroll
            for (int c = 0; c < NC; c++) sig[(int64_t)c * n + i] = s[c];
            z[i] = zi;
            elastic[i] = (uint8_t)el;
        }
        if (cases) cases[i] = rc == OK ? cs : -1;
        if (steps) steps[i] = ns;
    }
}

}  // namespace

extern "C" int pms_ep_update_stress_batch(const pms_material* mat, int32_t ndim, int64_t n, double* sig, double* z,
                                          uint8_t* elastic, const double* deps, const pms_ep_settings* settings,
                                          int32_t* cases, int32_t* steps, int32_t* status, void* stream) {
    if (!mat || (ndim != 2 && ndim != 3) || n < 0) return PMS_ERR_INVALID;
    if (mat->model != PMS_VON_MISES) return PMS_ERR_INVALID;  // elastoplastic.rs:131-134
    if (!(mat->young > 0.0) || !(mat->poisson > -1.0 && mat->poisson < 0.5) || !(mat->hh >= 0.0))
        return PMS_ERR_INVALID;
    if (n == 0) return PMS_OK;
    if (!sig || !z || !elastic || !deps) return PMS_ERR_INVALID;
    EpConst e;
    e.rtol = settings ? settings->tol_rel : 1e-10;
    e.atol = settings ? settings->tol_abs : 1e-10;
    e.h_ini = settings ? settings->h_ini : 1.0;
    e.max_steps = settings ? settings->max_steps : 1000;
    if (!(e.rtol > 0.0) || !(e.atol > 0.0) || !(e.h_ini > 0.0) || e.max_steps < 1) return PMS_ERR_INVALID;
    const MatConst m = make_matconst(PMS_VON_MISES, mat->young, mat->poisson, mat->hh, mat->z_ini);
    int64_t blocks = (n + 127) / 128;
    if (blocks > 148 * 32) blocks = 148 * 32;
    cudaStream_t st = (cudaStream_t)stream;
    if (ndim == 2)
        ep_update_kernel<4><<<(unsigned)blocks, 128, 0, st>>>(m, e, n, sig, z, elastic, deps, cases, steps, status);
    else
        ep_update_kernel<6><<<(unsigned)blocks, 128, 0, st>>>(m, e, n, sig, z, elastic, deps, cases, steps, status);
    return cudaGetLastError() == cudaSuccess ? PMS_OK : PMS_ERR_CUDA;
}

namespace {
// device staging of the host-buffer entry, grown on demand and kept until exit
struct EpStage {
    std::mutex mu;
    void* buf = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
} g_ep_stage;
}  // namespace

extern "C" int pms_ep_update_stress_host(const pms_material* mat, int32_t ndim, int64_t n, double* sig, double* z,
                                         uint8_t* elastic, const double* deps, const pms_ep_settings* settings,
                                         int32_t* cases, int32_t* steps) {
    if (!mat || (ndim != 2 && ndim != 3) || n < 0) return PMS_ERR_INVALID;
    if (n == 0) return PMS_OK;
    if (!sig || !z || !elastic || !deps) return PMS_ERR_INVALID;
    const size_t nc = 2 * (size_t)ndim, b_sig = nc * n * 8, b_n = (size_t)n * 8, b_i = (size_t)n * 4;
    const size_t need = 64 + 2 * b_sig + b_n + (cases ? b_i : 0) + (steps ? b_i : 0) + (size_t)n;
    std::lock_guard<std::mutex> lock(g_ep_stage.mu);
    if (!g_ep_stage.stream && cudaStreamCreateWithFlags(&g_ep_stage.stream, cudaStreamNonBlocking) != cudaSuccess)
        return PMS_ERR_CUDA;
    if (g_ep_stage.bytes < need) {
        if (g_ep_stage.buf) cudaFree(g_ep_stage.buf);
        g_ep_stage.buf = nullptr;
        g_ep_stage.bytes = 0;
        if (cudaMalloc(&g_ep_stage.buf, need) != cudaSuccess) return PMS_ERR_NOMEM;
        g_ep_stage.bytes = need;
    }
    char* p = (char*)g_ep_stage.buf;
    int32_t* d_status = (int32_t*)p; p += 64;
    double* d_sig = (double*)p; p += b_sig;
    double* d_deps = (double*)p; p += b_sig;
    double* d_z = (double*)p; p += b_n;
    int32_t* d_cases = nullptr;
    if (cases) { d_cases = (int32_t*)p; p += b_i; }
    int32_t* d_steps = nullptr;
    if (steps) { d_steps = (int32_t*)p; p += b_i; }
    uint8_t* d_el = (uint8_t*)p;
    cudaStream_t s = g_ep_stage.stream;
    cudaMemsetAsync(d_status, 0, 16, s);
    cudaMemcpyAsync(d_sig, sig, b_sig, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_deps, deps, b_sig, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_z, z, b_n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_el, elastic, (size_t)n, cudaMemcpyHostToDevice, s);
    int rc = pms_ep_update_stress_batch(mat, ndim, n, d_sig, d_z, d_el, d_deps, settings, d_cases, d_steps,
                                        d_status, s);
    if (rc) {
        cudaStreamSynchronize(s);
        return rc;
    }
    cudaMemcpyAsync(sig, d_sig, b_sig, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(z, d_z, b_n, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(elastic, d_el, (size_t)n, cudaMemcpyDeviceToHost, s);
    if (cases) cudaMemcpyAsync(cases, d_cases, b_i, cudaMemcpyDeviceToHost, s);
    if (steps) cudaMemcpyAsync(steps, d_steps, b_i, cudaMemcpyDeviceToHost, s);
    int32_t hst[4] = {0, 0, 0, 0};
    cudaMemcpyAsync(hst, d_status, 16, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return PMS_ERR_CUDA;
    return hst[0];
}
