"""Stress paths of the reference's general-elastoplasticity tests, restated.

The reference tests Elastoplastic::update_stress with the von Mises model on states and targets
given by octahedral invariants (src/material/elastoplastic.rs:655-705 and the tests
update_stress_von_mises_1 .. _5, :861-1424): sample_von_mises parameters (E = 1500, nu = 0.25,
H = 800, z_ini = 9; src/base/parameters.rs:399-406), plane strain (2D Mandel).  The strain
increment is the elastic compliance applied to (sigma_target - sigma_start), as in
update_with_von_mises (:675-705).  The octahedral parametrisation here is any isometry of the
deviatoric plane: the checks use invariants and angles only.
"""
import math

import numpy as np

YOUNG, POISSON, HH, Z_INI = 1500.0, 0.25, 800.0, 9.0
KK = YOUNG / (3.0 * (1.0 - 2.0 * POISSON))
GG = YOUNG / (2.0 * (1.0 + POISSON))

_EA = np.array([2.0, -1.0, -1.0]) / math.sqrt(6.0)
_EB = np.array([0.0, 1.0, -1.0]) / math.sqrt(2.0)


def stress(sig_m, sig_d, alpha, nc=4):
    """Diagonal Mandel stress with mean sig_m, deviatoric invariant sig_d, octahedral angle alpha."""
    r = sig_d * math.sqrt(2.0 / 3.0)
    p = sig_m + r * (math.cos(alpha) * _EA + math.sin(alpha) * _EB)
    v = np.zeros(nc)
    v[:3] = p
    return v


def modulus(nc=4):
    c = YOUNG / ((1.0 + POISSON) * (1.0 - 2.0 * POISSON))
    d = np.zeros((nc, nc))
    d[:3, :3] = c * POISSON
    for i in range(3):
        d[i, i] = c * (1.0 - POISSON)
    for i in range(3, nc):
        d[i, i] = c * (1.0 - 2.0 * POISSON)
    return d


def strain_for(sig0, sig1):
    """deps = C : (sig1 - sig0), C the elastic compliance."""
    return np.linalg.solve(modulus(len(sig0)), sig1 - sig0)


def sigma_m(v):
    return (v[0] + v[1] + v[2]) / 3.0


def sigma_d(v):
    m = sigma_m(v)
    s = np.array(v, dtype=float)
    s[:3] -= m
    return math.sqrt(1.5 * float(s @ s))


def eps_v(e):
    return float(e[0] + e[1] + e[2])


def eps_d(e):
    m = eps_v(e) / 3.0
    d = np.array(e, dtype=float)
    d[:3] -= m
    return math.sqrt(2.0 / 3.0) * math.sqrt(float(d @ d))


def scenarios():
    """(name, sig0, z0, deps, expected case, check) for the reference's test paths; check(sig, z,
    elastic) returns the list of (value, expected) pairs the reference asserts."""
    out = []
    pi = math.pi
    # update_stress_von_mises_1: elastic onto the surface (AE), then elastoplastic (BP), 3 Lode values
    for lode in (-1.0, 0.0, 1.0):
        alpha = pi / 2.0 - math.acos(lode) / 3.0
        s0 = stress(0.0, 0.0, pi / 2.0)
        s1 = stress(1.0, Z_INI, alpha)
        d1 = strain_for(s0, s1)
        out.append((f"vm1_lode{lode:+.0f}_AE", s0, Z_INI, d1, "AE",
                    lambda s, z, el, d=d1: [(sigma_m(s), KK * eps_v(d)), (sigma_d(s), 3 * GG * eps_d(d)),
                                            (z, Z_INI), (el, 1)]))
        s2 = stress(2.0, 2.0 * Z_INI, alpha)
        d2 = strain_for(s1, s2)
        out.append((f"vm1_lode{lode:+.0f}_BP", s1, Z_INI, d2, "BP",
                    lambda s, z, el, d=d2, s1=s1: [
                        (sigma_m(s), sigma_m(s1) + KK * eps_v(d)),
                        (sigma_d(s), sigma_d(s1) + 3 * GG * HH * eps_d(d) / (3 * GG + HH)),
                        (z, sigma_d(s1) + 3 * GG * HH * eps_d(d) / (3 * GG + HH)), (el, 0)]))
    # update_stress_von_mises_2: from zero across the surface (AXB)
    s0 = stress(0.0, 0.0, pi / 3.0)
    d = strain_for(s0, stress(2.0, Z_INI + 9.0, pi / 3.0))

    def check2(s, z, el, d=d):
        sd = Z_INI + 3 * GG * HH * (eps_d(d) - Z_INI / (3 * GG)) / (3 * GG + HH)
        return [(sigma_m(s), KK * eps_v(d)), (sigma_d(s), sd), (z, sd), (el, 0)]
    out.append(("vm2_AXB", s0, Z_INI, d, "AXB", check2))
    # update_stress_von_mises_3a: on the surface, straight through the centre to the other side (BE)
    s0 = stress(0.0, Z_INI, pi / 3.0)
    d = strain_for(s0, stress(2.0, Z_INI, -2.0 * pi / 3.0))
    out.append(("vm3a_BE", s0, Z_INI, d, "BE",
                lambda s, z, el: [(sigma_m(s), 2.0), (sigma_d(s), Z_INI), (z, Z_INI), (el, 1)]))
    # update_stress_von_mises_3c / 3d: chords of the surface at constant mean stress (BE)
    for name, alpha1 in (("vm3c_BE", -pi / 3.0), ("vm3d_BE", pi - pi / 3.0)):
        s0 = stress(1.0, Z_INI, pi / 3.0)
        d = strain_for(s0, stress(1.0, Z_INI, alpha1))
        out.append((name, s0, Z_INI, d, "BE",
                    lambda s, z, el: [(sigma_m(s), 1.0), (sigma_d(s), Z_INI), (z, Z_INI), (el, 1)]))
    # update_stress_von_mises_4: outside by a drift of 1, in through the surface and out again (BXP)
    s0 = stress(0.0, Z_INI + 1.0, pi / 3.0)
    d = strain_for(s0, stress(2.0, 2.5 * Z_INI, -pi / 3.0))
    out.append(("vm4_BXP", s0, Z_INI, d, "BXP", lambda s, z, el: [(el, 0)]))
    # update_stress_von_mises_5: outside by 1e-14, loading outwards (BP)
    s0 = stress(0.0, Z_INI + 1e-14, pi / 3.0)
    d = strain_for(s0, stress(2.0, 2.0 * Z_INI, 0.0))
    out.append(("vm5_BP", s0, Z_INI, d, "BP", lambda s, z, el: [(el, 0)]))
    return out


def random_states(n, ndim, seed):
    """Seeded IP states inside, on and outside the yield surface, with non-radial increments."""
    rng = np.random.default_rng(seed)
    nc = 2 * ndim
    sig = rng.normal(0.0, 1.0, (n, nc))
    for i in range(n):  # scale each deviator to a target sigma_d relative to z
        sd = sigma_d(sig[i])
        ratio = rng.choice([0.0, 0.5, 0.9, 1.0, 1.0 + 1e-3])
        dev = sig[i].copy()
        dev[:3] -= sigma_m(sig[i])
        m = rng.normal(0.0, 5.0)
        sig[i] = dev * (ratio * Z_INI / sd if sd > 0 else 0.0)
        sig[i, :3] += m
    z = np.full(n, Z_INI)
    scale = rng.choice([0.2, 1.0, 3.0], size=(n, 1)) * Z_INI / (2 * GG)
    deps = rng.normal(0.0, 1.0, (n, nc)) * scale
    return sig, z, deps
