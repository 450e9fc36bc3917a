"""K1 parity: batched von Mises return map + consistent tangent on the GPU vs the CPU oracle.

Reference: VonMises::update_stress / stiffness (src/material/von_mises.rs:124-226),
LinearElastic (src/material/linear_elastic.rs:49-71).  Tolerance: relative 1e-12 (FP64).
"""
import numpy as np
import pytest

import oracle
from gpu_util import assert_close

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

E, NU, Z0 = 2e5, 0.3, 250.0


def seeded_batch(ndim, n, seed):
    rng = np.random.default_rng(seed)
    nc = 2 * ndim
    gg = E / (2 * (1 + NU))
    sig = rng.normal(0, 0.15 * Z0, size=(n, nc))
    z = Z0 + rng.uniform(0, 50, n)
    # keep the start state inside the yield surface (as a converged state is)
    m = sig[:, :3].mean(1, keepdims=True)
    s = sig.copy()
    s[:, :3] -= m
    sd = np.sqrt(1.5 * np.sum(s * s, 1))
    scale = np.minimum(1.0, 0.95 * z / np.maximum(sd, 1e-30))
    sig = np.concatenate([m + s[:, :3] * scale[:, None], s[:, 3:] * scale[:, None]], 1)
    deps = rng.normal(0, (0.8 if ndim == 2 else 0.45) * Z0 / (2 * gg), size=(n, nc))
    if ndim == 2:
        deps[:, 2] = 0.0  # plane strain
    hh = rng.uniform(0, 2e3, n)
    return sig, z, deps, hh


def run_oracle(model, ndim, sig, z, deps, hh):
    n, nc = sig.shape
    out_sig = sig.copy()
    ivs = np.stack([z, np.zeros(n)], 1).copy()
    el = np.ones(n, np.uint8)
    dd = np.zeros((n, nc, nc))
    for i in range(n):
        prm = oracle.Params(E, NU, hh[i], Z0)
        st = oracle.model_update_stress(model, prm, ndim, out_sig[i], ivs[i], el[i:i + 1], deps[i])
        assert st == 0
        dd[i] = oracle.model_stiffness(model, prm, ndim, out_sig[i], ivs[i], el[i])
    return out_sig, ivs, el, dd


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("model", ["von_mises", "linear_elastic"])
def test_vm_batch_matches_oracle(ndim, model):
    from pmsim_b200.material import VonMisesBatch, unpack_tangent
    n = 4096
    sig, z, deps, hh = seeded_batch(ndim, n, seed=ndim)
    mi = 1 if model == "von_mises" else 0
    o_sig, o_ivs, o_el, o_dd = run_oracle(mi, ndim, sig, z, deps, hh)
    vm = VonMisesBatch(E, NU, 0.0, Z0, ndim=ndim, model=model)
    dev = torch.device("cuda:0")
    t = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    g_sig = t(sig.T)
    g_z = t(z)
    g_lam = torch.zeros(n, dtype=torch.float64, device=dev)
    g_el = torch.zeros(n, dtype=torch.uint8, device=dev)
    g_dd = torch.zeros((vm.ntan, n), dtype=torch.float64, device=dev)
    status = torch.zeros(4, dtype=torch.int32, device=dev)
    vm.update_and_stiffness(g_sig, g_z, g_lam, g_el, t(deps.T), hh=t(hh), dd=g_dd, status=status)
    torch.cuda.synchronize()
    assert int(status[0]) == 0
    assert_close(g_sig.cpu().numpy().T, o_sig, what="sigma")
    if mi == 1:
        assert_close(g_z.cpu().numpy(), o_ivs[:, 0], what="z")
        assert_close(g_lam.cpu().numpy(), o_ivs[:, 1], what="lambda")
        frac = 1.0 - o_el.mean()
        assert 0.2 < frac < 0.8, frac  # both branches exercised
    assert np.array_equal(g_el.cpu().numpy(), o_el)
    assert_close(unpack_tangent(g_dd.cpu().numpy(), 2 * ndim), o_dd, what="tangent")


def test_vm_host_entry_equals_device_entry():
    from pmsim_b200.material import VonMisesBatch
    n = 1000
    sig, z, deps, hh = seeded_batch(3, n, seed=11)
    vm = VonMisesBatch(E, NU, 0.0, Z0, ndim=3)
    h_sig = np.ascontiguousarray(sig.T)
    h_z = z.copy()
    h_lam = np.zeros(n)
    h_el = np.zeros(n, np.uint8)
    dd = vm.update_and_stiffness_host(h_sig, h_z, h_lam, h_el, np.ascontiguousarray(deps.T), hh=hh)
    dev = torch.device("cuda:0")
    g_sig = torch.tensor(sig.T.copy(), device=dev)
    g_z = torch.tensor(z, device=dev)
    g_lam = torch.zeros(n, dtype=torch.float64, device=dev)
    g_el = torch.zeros(n, dtype=torch.uint8, device=dev)
    g_dd = torch.zeros((21, n), dtype=torch.float64, device=dev)
    vm.update_and_stiffness(g_sig, g_z, g_lam, g_el, torch.tensor(deps.T.copy(), device=dev),
                            hh=torch.tensor(hh, device=dev), dd=g_dd)
    torch.cuda.synchronize()
    assert np.array_equal(g_sig.cpu().numpy(), h_sig)
    assert np.array_equal(g_dd.cpu().numpy(), dd)
    assert np.array_equal(g_el.cpu().numpy(), h_el)


def test_vm_stiffness_kat_2d():
    """src/material/von_mises.rs:418-480 through the GPU path."""
    from pmsim_b200.material import VonMisesBatch, unpack_tangent
    E_, nu, z, H = 1500.0, 0.25, 9.0, 800.0
    dy = z * (1 - nu * nu) / (E_ * np.sqrt(1 - nu + nu * nu))
    ex, ey = dy * nu / (1 - nu), -dy
    vm = VonMisesBatch(E_, nu, H, z, ndim=2)
    sig = np.zeros((4, 1))
    zz = np.array([z])
    lam = np.zeros(1)
    el = np.zeros(1, np.uint8)
    dd = vm.update_and_stiffness_host(sig, zz, lam, el, np.array([[0.9999 * ex], [0.9999 * ey], [0.0], [0.0]]))
    D = unpack_tangent(dd, 4)[0]
    mp = [0, 1, 3]
    spo = np.array([[1800.0, 600.0, 0.0], [600.0, 1800.0, 0.0], [0.0, 0.0, 600.0]])
    for i in range(3):
        for j in range(3):
            assert abs(D[mp[i], mp[j]] - (2.0 if i == j == 2 else 1.0) * spo[i, j]) <= 1e-12
    assert el[0] == 1
    dd = vm.update_and_stiffness_host(sig, zz, lam, el, np.array([[(2 - 0.9999) * ex], [(2 - 0.9999) * ey],
                                                                   [0.0], [0.0]]))
    D = unpack_tangent(dd, 4)[0]
    spo = np.array([[1.389940828402367e03, 9.248520710059172e02, -2.081794007857600e-15],
                    [9.248520710059172e02, 1.262130177514793e03, 2.914511611000640e-15],
                    [-2.081794007857600e-15, 2.914511611000640e-15, 3.923076923076923e02]])
    for i in range(3):
        for j in range(3):
            assert abs(D[mp[i], mp[j]] - (2.0 if i == j == 2 else 1.0) * spo[i, j]) <= 1e-12
    assert el[0] == 0
    assert abs(lam[0] - 3.461538461538463e-03) <= 1e-15


# ---------------------------------------------------------------- general elastoplasticity
def _ep_device(ndim, sig, z, deps, **kw):
    """Runs the device general update on AoS host arrays; returns (sig, z, elastic, cases, steps, status)."""
    import torch
    import ep_cases as E
    from pmsim_b200.material import ElastoplasticBatch
    n = len(z)
    dev = torch.device("cuda:0")
    ts = torch.tensor(np.ascontiguousarray(sig.T), dtype=torch.float64, device=dev)
    tz = torch.tensor(z, dtype=torch.float64, device=dev)
    te = torch.zeros(n, dtype=torch.uint8, device=dev)
    td = torch.tensor(np.ascontiguousarray(deps.T), dtype=torch.float64, device=dev)
    tc = torch.full((n,), -7, dtype=torch.int32, device=dev)
    tn = torch.zeros(n, dtype=torch.int32, device=dev)
    st = torch.zeros(4, dtype=torch.int32, device=dev)
    ElastoplasticBatch(E.YOUNG, E.POISSON, E.HH, E.Z_INI, ndim=ndim, **kw).update_stress(ts, tz, te, td, tc, tn, st)
    torch.cuda.synchronize()
    return (ts.cpu().numpy().T.copy(), tz.cpu().numpy(), te.cpu().numpy(), tc.cpu().numpy(), tn.cpu().numpy(),
            st.cpu().numpy())


@pytest.mark.gpu
def test_elastoplastic_reference_paths_on_device():
    """The reference's general-elastoplasticity test paths (elastoplastic.rs:861-1424) on the
    device: same case keys, and the closed-form invariants the reference asserts (1e-12 absolute)."""
    import ep_cases as E
    from pmsim_b200.material import EP_CASES
    sc = E.scenarios()
    sig = np.array([s[1] for s in sc])
    z = np.array([s[2] for s in sc], dtype=float)
    deps = np.array([s[3] for s in sc])
    s1, z1, el, cases, steps, st = _ep_device(2, sig, z, deps)
    assert st[0] == 0
    for i, (name, _, _, _, case, check) in enumerate(sc):
        assert EP_CASES[cases[i]] == case, (name, cases[i])
        for v, want in check(s1[i], z1[i], int(el[i])):
            assert abs(v - want) <= 1e-12, (name, v, want)


@pytest.mark.gpu
@pytest.mark.parametrize("ndim", [2, 3])
def test_elastoplastic_matches_oracle(ndim):
    """Device vs oracle on 4000 seeded IP states inside, on and outside the yield surface with
    non-radial increments: the same case (up to the inside/on label of states on the surface), the
    same failures (the increments the reference rejects), and stresses within 1e-8 of the largest
    stress (both integrate with the same Dormand-Prince 5(4) controller at 1e-10, in a different
    arithmetic order)."""
    import ep_cases as E
    sig, z, deps = E.random_states(4000, ndim, seed=23 + ndim)
    prm = oracle.Params(E.YOUNG, E.POISSON, E.HH, E.Z_INI)
    osig, oz, oel = sig.copy(), z.copy(), np.zeros(len(z), dtype=np.uint8)
    ost, ocases, osteps, obad = oracle.ep_update(prm, ndim, osig, oz, oel, deps)
    s1, z1, el, cases, steps, st = _ep_device(ndim, sig, z, deps)
    # a state on the surface up to rounding (|f0| <= 1e-12 z) starts "inside" or "on" depending on
    # the last bit of f0, as in the reference: AXB/BXP and AE/BE then describe the same update
    f0 = np.array([E.sigma_d(v) for v in sig]) - z
    pairs = {(1, 3), (3, 1), (0, 2), (2, 0)}
    agree = (cases == ocases) | ((np.abs(f0) <= 1e-12 * z) &
                                 np.array([(int(c), int(o)) in pairs for c, o in zip(cases, ocases)]))
    assert agree.all(), np.flatnonzero(~agree)[:10]
    assert np.array_equal(cases < 0, ocases < 0)
    same = (cases >= 0) & (ocases >= 0)
    assert same.sum() >= 0.9 * len(z)
    assert np.array_equal(el[same], oel[same])
    scale = np.abs(osig[same]).max()
    assert np.abs(s1[same] - osig[same]).max() <= 1e-8 * scale
    assert np.abs(z1[same] - oz[same]).max() <= 1e-8 * scale
    assert (st[0] == 0) == (ost == 0)
    # failed IPs keep their state
    failed = cases < 0
    assert np.array_equal(s1[failed], sig[failed]) and np.array_equal(z1[failed], z[failed])


@pytest.mark.gpu
def test_elastoplastic_host_entry_equals_device_entry():
    """pms_ep_update_stress_host (host buffers, staged through the device) gives the same bits as
    the device entry, and returns the code of the first failing IP (the increments the reference
    rejects) as its status."""
    import ep_cases as E
    from pmsim_b200.material import ElastoplasticBatch
    sig, z, deps = E.random_states(3000, 3, seed=77)
    s1, z1, el1, c1, n1, st = _ep_device(3, sig, z, deps)
    hs, hz, he = np.ascontiguousarray(sig.T), z.copy(), np.zeros(len(z), dtype=np.uint8)
    rc, c2, n2 = ElastoplasticBatch(E.YOUNG, E.POISSON, E.HH, E.Z_INI, ndim=3).update_stress_host(
        hs, hz, he, np.ascontiguousarray(deps.T))
    assert rc == st[0]
    assert np.array_equal(hs.T, s1) and np.array_equal(hz, z1) and np.array_equal(he, el1)
    assert np.array_equal(c2, c1) and np.array_equal(n2, n1)
