// pms_device.cuh -- device arithmetic shared by the material and element kernels.
//
// Mandel (Kelvin) notation, sigma = [xx, yy, zz, sqrt2 xy, sqrt2 yz, sqrt2 xz] (4 components
// in plane strain, 6 in 3D), as the reference stores Tensor2 (compare_results.rs:131-135).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pms {

constexpr double SQRT2 = 1.4142135623730951;
constexpr double INV_SQRT2 = 0.7071067811865476;
constexpr double SQRT_2_BY_3 = 0.816496580927726;
constexpr double F_TOL = 1e-6;  // elastic-regime tolerance on f/z_ini (von_mises.rs:23)

enum Err : int { OK = 0, E_INVALID = 1, E_CUDA = 2, E_ZERO_SIGMA_D = 3, E_ZERO_NORM_S = 4, E_JACOBIAN = 5,
                 E_ORDER = 13 };

// Material constants in the form the kernels use.
struct MatConst {
    int model;       // 0 linear elastic, 1 von Mises
    int plane_stress;  // linear elastic in plane stress (2D): in-plane normal block c(1, nu; nu, 1),
                       // c = E/(1-nu^2), no out-of-plane stress (russell_tensor LinElasticity)
    double kk, gg;   // bulk and shear moduli: K = E/(3(1-2nu)), G = E/(2(1+nu))
    double hh, z_ini;
    double c11, c12, c44;  // Hooke in Mandel form: c(1-nu), c nu, c(1-2nu) with c = E/((1+nu)(1-2nu))
    double ps11, ps12;     // plane stress: E/(1-nu^2), E nu/(1-nu^2) (= the effective Lame lambda*)
};

inline MatConst make_matconst(int model, double young, double poisson, double hh, double z_ini,
                              bool plane_stress = false) {
    MatConst m;
    m.model = model;
    m.plane_stress = plane_stress ? 1 : 0;
    m.ps11 = young / (1.0 - poisson * poisson);
    m.ps12 = m.ps11 * poisson;
    m.kk = young / (3.0 * (1.0 - 2.0 * poisson));
    m.gg = young / (2.0 * (1.0 + poisson));
    m.hh = hh;
    m.z_ini = z_ini;
    double c = young / ((1.0 + poisson) * (1.0 - 2.0 * poisson));
    m.c11 = c * (1.0 - poisson);
    m.c12 = c * poisson;
    m.c44 = c * (1.0 - 2.0 * poisson);
    return m;
}

template <int NC>
__device__ __forceinline__ double sigma_m(const double* v) { return (v[0] + v[1] + v[2]) * (1.0 / 3.0); }

// sigma_d = sqrt(3 J2) = sqrt(3/2 s:s), s = dev(sigma)
template <int NC>
__device__ __forceinline__ double sigma_d(const double* v) {
    double m = (v[0] + v[1] + v[2]) / 3.0;
    double s0 = v[0] - m, s1 = v[1] - m, s2 = v[2] - m;
    double q = s0 * s0 + s1 * s1 + s2 * s2;
#pragma unroll
    for (int i = 3; i < NC; i++) q += v[i] * v[i];
    return sqrt(1.5 * q);
}

// sigma += D_e : deps  (t4_ddot_t2_update with the Hooke modulus)
template <int NC>
__device__ __forceinline__ void hooke_add(const MatConst& m, double* sig, const double* de) {
    if (NC == 4 && m.plane_stress) {  // sigma_zz stays zero
        sig[0] += m.ps11 * de[0] + m.ps12 * de[1];
        sig[1] += m.ps12 * de[0] + m.ps11 * de[1];
        sig[3 % NC] += m.c44 * de[3 % NC];
        return;
    }
    double d0 = m.c11 * de[0] + m.c12 * de[1] + m.c12 * de[2];
    double d1 = m.c12 * de[0] + m.c11 * de[1] + m.c12 * de[2];
    double d2 = m.c12 * de[0] + m.c12 * de[1] + m.c11 * de[2];
    sig[0] += d0;
    sig[1] += d1;
    sig[2] += d2;
#pragma unroll
    for (int i = 3; i < NC; i++) sig[i] += m.c44 * de[i];
}

// VonMises::update_stress (von_mises.rs:170-226) / LinearElastic::update_stress
// (linear_elastic.rs:61-71).  Returns an Err code.  hh is the hardening to use.
template <int NC>
__device__ __forceinline__ int ip_update(const MatConst& m, double hh, double* sig, double& z, double& lambda,
                                         int& elastic, const double* deps) {
    hooke_add<NC>(m, sig, deps);
    if (m.model == 0) return OK;
    elastic = 1;
    lambda = 0.0;
    double sd_trial = sigma_d<NC>(sig);
    double f_trial = sd_trial - z;
    if (f_trial / m.z_ini <= F_TOL) return OK;
    double sm = sigma_m<NC>(sig);
    double lam = f_trial / (3.0 * m.gg + hh);
    double beta = 1.0 - lam * 3.0 * m.gg / sd_trial;
    sig[0] = sm + beta * (sig[0] - sm);
    sig[1] = sm + beta * (sig[1] - sm);
    sig[2] = sm + beta * (sig[2] - sm);
#pragma unroll
    for (int i = 3; i < NC; i++) sig[i] = beta * sig[i];
    int st = OK;
    if (sigma_d<NC>(sig) < 1e-10) st = E_ZERO_SIGMA_D;
    z += hh * lam;
    elastic = 0;
    lambda = lam;
    return st;
}

// Coefficients of the consistent tangent D = a Psd + b s(x)s + K I(x)I
// (VonMises::stiffness, von_mises.rs:124-167); elastic: a = 2G, b = 0.
// s[] receives the deviator.  Returns an Err code.
template <int NC>
__device__ __forceinline__ int tangent_coefs(const MatConst& m, double hh, const double* sig, double lambda,
                                             int elastic, double& a, double& b, double* s) {
    double sm = sigma_m<NC>(sig);
    s[0] = sig[0] - sm;
    s[1] = sig[1] - sm;
    s[2] = sig[2] - sm;
#pragma unroll
    for (int i = 3; i < NC; i++) s[i] = sig[i];
    if (m.model == 0 || elastic) {
        a = 2.0 * m.gg;
        b = 0.0;
        return OK;
    }
    double sd = sigma_d<NC>(sig);
    double sd_trial = sd + lambda * 3.0 * m.gg;
    double norm_s = sd * SQRT_2_BY_3;
    if (norm_s < 1e-10) {
        a = 2.0 * m.gg;
        b = 0.0;
        return E_ZERO_NORM_S;
    }
    double d = 3.0 * m.gg + hh;
    a = 2.0 * m.gg * (1.0 - lambda * 3.0 * m.gg / sd_trial);
    b = 6.0 * m.gg * m.gg * (lambda / sd_trial - 1.0 / d) / (norm_s * norm_s);
    return OK;
}

// Block-Jacobi inverse of the nf x nf free part of a node's diagonal block, held in a[i][0..nf) with
// a[i][nf..2nf) = the identity: Gauss-Jordan without pivoting (the free part of a diagonal block of
// an SPD matrix is SPD), the inverse ends in a[i][nf..2nf).  Returns false at a pivot that is not
// positive (the caller then falls back to the inverse of the diagonal).
__device__ __forceinline__ bool spd_block_inverse(double (&a)[3][6], int nf) {
    for (int k = 0; k < nf; k++) {
        const double piv = a[k][k];
        if (!(piv > 0.0)) return false;
        const double ip = 1.0 / piv;
        for (int j = 0; j < 2 * nf; j++) a[k][j] *= ip;
        for (int i = 0; i < nf; i++)
            if (i != k) {
                const double f = a[i][k];
                for (int j = 0; j < 2 * nf; j++) a[i][j] -= f * a[k][j];
            }
    }
    return true;
}

// Symmetric-deviatoric projector entry in Mandel form
__device__ __forceinline__ double psd(int i, int j) {
    if (i < 3 && j < 3) return (i == j) ? (2.0 / 3.0) : (-1.0 / 3.0);
    return (i == j) ? 1.0 : 0.0;
}

}  // namespace pms
