"""Benchmark of the pmsim solid hot path on B200.

Default workload (one GPU): the single large 3D problem -- a 64x64x32 block of Hex20 cells with
27 Gauss points (131,072 cells, 3,538,944 IPs, 1,647,555 DOF, CSR nnz 279,514,377), von Mises
E=2e5, nu=0.3, z0=250, H=1e3.  One step = one Newton iteration of the element hot path:
stress update (radial return) at every IP from the step-start state, F_int = sum B^T sigma,
consistent tangent K = sum B^T D_ep B, deterministic gather of K into CSR and of F_int into R.
The displacement increment is a seeded synthetic footing indentation of the block's top
(mid-load), so that plastic and elastic IPs mix.  Metric: IP stress-update+tangent per second.

Also measured in the same run: the stand-alone von Mises batch kernel on 16,777,216 IPs
(``k1_microbench``), the general (ODE-based) elastoplastic update on 4,194,304 IPs
(``ep_microbench``), the FP64 FMA peak of the GPU (``fp64_peak``), and the CPU restatement of
the reference (oracle port, all host cores) on a bounded sample (``cpu_baseline``).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--size small|medium|full]
Multi-GPU (torchrun): every rank processes its own block (weak scaling, no data-path
collective); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

E, NU, Z0, HH = 2e5, 0.3, 250.0, 1e3
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", default="full", choices=["small", "medium", "full"],
                    help="Hex20 block 16x16x8 / 32x32x16 (profiling captures) / 64x64x32")
    ap.add_argument("--no-k1", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-cells", type=int, default=0)
    ap.add_argument("--batched", type=int, default=512, help="footing problems in the batched solve (0: skip)")
    ap.add_argument("--alone-sample", type=int, default=32, help="problems solved one at a time for the ratio")
    ap.add_argument("--served", type=int, default=64, help="requests in the served run (0: skip)")
    ap.add_argument("--rate", type=float, default=200.0, help="Poisson arrival rate of the served run (req/s)")
    ap.add_argument("--no-c0", action="store_true")
    ap.add_argument("--no-qua8", action="store_true")
    ap.add_argument("--qua8-n", type=int, default=1024, help="Qua8 mesh of n x n cells for the memory-bound step")
    ap.add_argument("--served-detail", default="", help="write per-request served records (JSON) to this file")
    ap.add_argument("--pcg-time", nargs="+", default=None, metavar="ARG",
                    help="only time the PCG engines on one problem: ENGINE PROBLEM DIMS... with ENGINE team|wide "
                         "and PROBLEM foot (nx ny Qua8 footing) | hex (nx ny nz Hex8 block)")
    ap.add_argument("--pcg-chunks", type=int, default=0, help="--pcg-time: 128-node chunks per team CTA (0: all fit)")
    ap.add_argument("--pcg-threads", type=int, default=1024, help="--pcg-time: threads per team CTA")
    ap.add_argument("--pcg-iterations", type=int, default=64, help="--pcg-time: PCG iterations timed")
    return ap.parse_args()


def workload_dims(size):
    return {"small": (16, 16, 8), "medium": (32, 32, 16), "full": (64, 64, 32)}[size]


def make_problem(size):
    from pmsim_b200 import mesh as M
    nx, ny, nz = workload_dims(size)
    m = M.structured_3d(M.HEX20, nx, ny, nz, float(nx), float(ny), float(nz))
    return m


def synthetic_ddu(m, size, seed=20241203):
    """Seeded mid-load increment of the footing indentation: the central quarter of the top face is
    pushed down (prescribed uz), decaying with depth and across the footing edge, plus noise."""
    nx, ny, nz = workload_dims(size)
    x, y, z = m.coords[:, 0], m.coords[:, 1], m.coords[:, 2]
    cx, cy = nx / 2.0, ny / 2.0
    hx, hy = nx / 4.0, ny / 4.0
    # smooth plateau under the footing: 1 inside |x-cx|<=hx, |y-cy|<=hy, tanh decay outside
    fx = 0.5 * (np.tanh((hx - np.abs(x - cx)) / 2.0) + 1.0)
    fy = 0.5 * (np.tanh((hy - np.abs(y - cy)) / 2.0) + 1.0)
    depth = np.exp(-(nz - z) / (0.5 * nz))
    delta = 0.005 * nz * 0.35  # 35% of the total indentation (0.5% of the height)
    u = np.zeros_like(m.coords)
    u[:, 2] = -delta * fx * fy * depth
    u[:, 0] = 0.15 * delta * (x - cx) / nx * fy * depth
    u[:, 1] = 0.15 * delta * (y - cy) / ny * fx * depth
    rng = np.random.default_rng(seed)
    u += rng.normal(0.0, 2e-4, size=u.shape)
    return u.reshape(-1).copy()


def flops_per_ip_sparse_b(nd, nn):
    """Algorithmic FP64 FLOPs per IP of update + F_int + tangent in the sparse-B formulation with a
    symmetric K_e (FMA = 2): D G_b for every node (nd * ncomp * nd * nn FMA), G_a^T (D G_b) for the
    node pairs a <= b (nd^3 * nn(nn+1)/2 FMA), the Jacobian J = X^T dN and the gradients G = dN J^-1
    (nn * nd^2 FMA each).  Hex20 (nd 3, 6 Mandel components, 20 nodes): 2 * (1080 + 5670 + 360) =
    14,220 per IP, the count of the roofline the element kernel is reported against."""
    nc = 2 * nd
    fma = nd * nc * nd * nn + nd ** 3 * nn * (nn + 1) // 2 + 2 * nn * nd * nd
    return 2 * fma


def flops_per_ip_hex20(plastic):
    """Algorithmic FP64 FLOPs of the fused element kernel per Hex20 IP (FMA = 2) when a fraction
    `plastic` of the IPs is plastic.  Every IP: J, J^-T dN, strain and B^T sigma (20 nodes x 9 FMA
    each), alpha g (20 x 3 MUL) and X_ab += alpha g_a g_b^T (210 node pairs x 9 FMA); once per cell,
    K_ab = X_ab^T + c X_ab + tr(X_ab) 1 (210 x 9 FMA + 5 ADD), spread over the 27 IPs; every plastic
    IP also h = S g (20 x 9 FMA), kappa g and beta h (20 x 6 MUL) and 210 x 18 FMA."""
    fma = 20 * 9 * 4 + 210 * 9 + 210 * 9 / 27 + plastic * (20 * 9 + 210 * 18)
    other = 20 * 3 + 210 * 5 / 27 + plastic * 20 * 6
    return 2 * fma + other


# DRAM bytes (read + write) per cell of one launch of the element kernel element_kernel<3,20,...>
# (gather assembly: upper element-matrix blocks out) from an ncu capture of a smaller block (traffic
# grows with the cell count, so a launch over n cells moves n times this).
ELEMENT_DRAM_BYTES_PER_CELL = 15798  # 258.8 MB over 16,384 cells (32x32x16 block)


def algorithmic_bytes_step(m, ng, nnz):
    """Bytes a fused implementation must move per Newton iteration: coordinates, connectivity,
    dU (read once), IP state read (sigma, z: 56 B) and written (sigma, z, lambda: 64 B + flag),
    R (8 ndof) and the CSR values written once (8 nnz)."""
    nip = m.ncell * ng
    return (m.npoint * 24 + m.ncell * m.nnode * 4 + m.ndof * 8 + nip * 56 + nip * 65 + m.ndof * 8 + nnz * 8)


class Clocks:
    """SM clock and clock-event reasons sampled every ~2 ms by an NVML polling thread (read-only
    queries); ``mark()`` brackets the timed region and only samples inside it are reported.
    Falls back to one ``nvidia-smi`` reading when NVML is unavailable."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, device):
        import threading
        self.samples, self.t0, self.t1, self.h, self.nv = [], None, None, None, None
        try:
            import pynvml as nv
            nv.nvmlInit()
            props = __import__("torch").cuda.get_device_properties(device)
            bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
            self.h = nv.nvmlDeviceGetHandleByPciBusId(bus)
            self.nv = nv
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
        except Exception:
            self.h = None
        self.stop_flag = threading.Event()
        self.th = None
        if self.h is not None:
            self.th = threading.Thread(target=self._poll, daemon=True)
            self.th.start()

    def _poll(self):
        nv = self.nv
        while not self.stop_flag.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.samples.append((time.perf_counter(), mhz, rs))
            except Exception:
                pass
            time.sleep(0.002)

    def mark(self, start=True):
        if start:
            self.t0 = time.perf_counter()
        else:
            self.t1 = time.perf_counter()

    def stop(self):
        if self.th is None:
            return _smi_clocks()
        self.stop_flag.set()
        self.th.join(timeout=5)
        t1 = self.t1 if self.t1 is not None else float("inf")
        rows = [(m, r) for t, m, r in self.samples if (self.t0 is None or t >= self.t0) and t <= t1]
        if not rows:
            return None
        reasons = sorted({name for _, r in rows for bit, name in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(m for m, _ in rows), "sm_max_mhz": self.max_mhz,
                "sm_min_mhz": min(m for m, _ in rows), "reasons": reasons, "samples": len(rows), "source": "nvml"}


def _smi_clocks():
    try:
        out = subprocess.run(["nvidia-smi", "--query-gpu=clocks.sm,clocks.max.sm", "--format=csv,noheader,nounits"],
                             capture_output=True, text=True, timeout=20).stdout.split("\n")[0].split(",")
        return {"sm_mhz": float(out[0]), "sm_max_mhz": float(out[1]), "reasons": [], "samples": 1,
                "source": "nvidia-smi after the timed region"}
    except Exception:
        return None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def fp64_peak(torch, L, stream):
    out = torch.empty(148 * 8 * 256, dtype=torch.float64, device="cuda")
    iters = 20000
    for _ in range(2):
        L.pms_probe_fp64_fma(1000, 148 * 8, out.data_ptr(), stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    L.pms_probe_fp64_fma(iters, 148 * 8, out.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    flops = 148 * 8 * 256 * 8 * iters * 2
    return flops / (ms * 1e-3) / 1e12


def k1_scale_for_yield(fraction):
    """Factor on the configured deviation 1.5 z0/(2G) that makes the given fraction of the IPs yield.
    With sigma0 = 0 and i.i.d. Mandel components of deviation s, the trial sigma_d is
    sqrt(3/2) 2G s chi_5 (chi with 5 degrees of freedom: the deviator of the strain), so the fraction
    that yields is P(chi_5 > z0 / (sqrt(3/2) 2G s))."""
    from scipy.stats import chi
    return 1.0 / (1.5 * np.sqrt(1.5) * chi.ppf(1.0 - fraction, 5))


def run_k1(torch, stream, steps, warmup, scale=1.0):
    """Stand-alone von Mises batch on 16,777,216 IPs (3D, SoA), sigma0 = 0, z0 = 250,
    deps ~ N(0, (scale * 1.5 z0/(2G))^2), H ~ U[0, 2e3]; K1 reads 112 B and writes 233 B per IP."""
    from pmsim_b200.material import VonMisesBatch
    n = 16_777_216
    gg = E / (2 * (1 + NU))
    g = torch.Generator(device="cuda").manual_seed(1234)
    deps = torch.randn((6, n), generator=g, device="cuda", dtype=torch.float64) * (scale * 1.5 * Z0 / (2 * gg))
    hh = torch.rand(n, generator=g, device="cuda", dtype=torch.float64) * 2e3
    sig = torch.zeros((6, n), device="cuda", dtype=torch.float64)
    z = torch.full((n,), Z0, device="cuda", dtype=torch.float64)
    lam = torch.zeros(n, device="cuda", dtype=torch.float64)
    el = torch.zeros(n, device="cuda", dtype=torch.uint8)
    dd = torch.empty((21, n), device="cuda", dtype=torch.float64)
    vm = VonMisesBatch(E, NU, 0.0, Z0, ndim=3)
    times = []
    with torch.cuda.stream(stream):
        for i in range(warmup + steps):
            sig.zero_()
            z.fill_(Z0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            vm.update_and_stiffness(sig, z, lam, el, deps, hh=hh, dd=dd, stream=stream)
            e1.record(stream)
            if i >= warmup:
                times.append((e0, e1))
    torch.cuda.synchronize()
    ms = statistics.mean(a.elapsed_time(b) for a, b in times)
    yielded = float(1.0 - el.double().mean().item())
    bytes_ip = 112 + 233
    return {"ips": n, "ms": ms, "ip_per_s": n / (ms * 1e-3), "gbs": n * bytes_ip / (ms * 1e-3) / 1e9,
            "bytes_per_ip": bytes_ip, "yield_fraction": yielded, "deps_scale": scale}


def run_ep(torch, stream, steps, warmup, n=4_194_304, cpu_sample=20_000):
    """General elastoplastic update (Elastoplastic::update_stress with von Mises: yield-surface
    crossing + Dormand-Prince 5(4) integration of the elastoplastic rates) on n 3D IPs: half start
    on the yield surface (random deviatoric direction, random mean stress), half at zero stress;
    deps ~ N(0, (1.5 z0/(2G))^2) per Mandel component, H = 1e3.  Also times the oracle (C++
    restatement, one thread) on the first cpu_sample IPs."""
    import oracle
    from pmsim_b200.material import EP_CASES, ElastoplasticBatch
    gg = E / (2 * (1 + NU))
    g = torch.Generator(device="cuda").manual_seed(4321)
    sig0 = torch.randn((6, n), generator=g, device="cuda", dtype=torch.float64)
    mean = sig0[:3].mean(0)
    dev = sig0.clone()
    dev[:3] -= mean
    sd = torch.sqrt(1.5 * (dev * dev).sum(0))
    sig0 = dev * (Z0 / sd)
    sig0[:3] += torch.randn(n, generator=g, device="cuda", dtype=torch.float64) * 50.0
    sig0[:, n // 2:] = 0.0
    deps = torch.randn((6, n), generator=g, device="cuda", dtype=torch.float64) * (1.5 * Z0 / (2 * gg))
    sig = torch.empty_like(sig0)
    z = torch.empty(n, device="cuda", dtype=torch.float64)
    el = torch.zeros(n, device="cuda", dtype=torch.uint8)
    cases = torch.empty(n, device="cuda", dtype=torch.int32)
    nst = torch.empty(n, device="cuda", dtype=torch.int32)
    status = torch.zeros(4, device="cuda", dtype=torch.int32)
    ep = ElastoplasticBatch(E, NU, 1e3, Z0, ndim=3)
    times = []
    with torch.cuda.stream(stream):
        for i in range(warmup + steps):
            sig.copy_(sig0)
            z.fill_(Z0)
            status.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ep.update_stress(sig, z, el, deps, cases, nst, status, stream=stream)
            e1.record(stream)
            if i >= warmup:
                times.append((e0, e1))
    torch.cuda.synchronize()
    ms = statistics.mean(a.elapsed_time(b) for a, b in times)
    cnt = torch.bincount((cases + 1).long(), minlength=6).cpu().tolist()
    mix = {"failed": cnt[0] / n, **{c: cnt[k + 1] / n for k, c in enumerate(EP_CASES)}}
    ok = cases >= 0
    mean_steps = float(nst[ok & (el == 0)].double().mean().item())
    # oracle on a sample, one thread
    m = cpu_sample
    osig = sig0[:, :m].T.contiguous().cpu().numpy().copy()
    odeps = deps[:, :m].T.contiguous().cpu().numpy().copy()
    oz = np.full(m, Z0)
    oel = np.zeros(m, dtype=np.uint8)
    t0 = time.perf_counter()
    oracle.ep_update(oracle.Params(E, NU, 1e3, Z0), 3, osig, oz, oel, odeps)
    t_cpu = time.perf_counter() - t0
    return {"ips": n, "ms": ms, "ip_per_s": n / (ms * 1e-3), "case_fraction": mix,
            "mean_ode_steps_plastic": mean_steps, "tol_rel": 1e-10,
            "cpu_oracle_1thread_ip_per_s": m / t_cpu, "cpu_sample_ips": m,
            "workload": "3D, half on the yield surface (random direction), half at zero stress, "
                        "deps ~ N(0, (1.5 z0/2G)^2), E=2e5, nu=0.3, z0=250, H=1e3"}


def run_qua8_step(torch, stream, steps, warmup, hbm_peak, n=1024):
    """The fused Newton iteration on a large 2D mesh, where it is memory-bound: n x n Qua8 cells
    (9 IP) of the footing material (E=1e4, nu=0.3, z0=9, H=0) under a seeded smooth increment that
    leaves a mix of elastic and plastic IPs.  Reports the step's algorithmic bytes per second
    against the measured HBM peak, with the default (gather) assembly, and the same step with the
    direct assembly for comparison."""
    from pmsim_b200 import _lib
    from pmsim_b200 import mesh as M
    from pmsim_b200.elements import Elements, Material
    L = _lib.load()
    m = M.structured_2d(M.QUA8, n, n, float(n), float(n))
    x, y = m.coords[:, 0] / n, m.coords[:, 1] / n
    rng = np.random.default_rng(99)
    u = np.zeros_like(m.coords)
    u[:, 0] = 1.5e-3 * n * np.sin(3.0 * x) * np.cos(2.0 * y) / 3.0
    u[:, 1] = -2.0e-3 * n * y * (1.0 + 0.5 * np.sin(5.0 * x)) / 1.0
    u += rng.normal(0.0, 1e-4, u.shape)
    el = Elements(m, Material.von_mises(1e4, 0.3, 0.0, 9.0), ngauss=9)
    el.set_stream(stream)
    dev = torch.device("cuda", torch.cuda.current_device())
    d_ddu = torch.tensor(u.reshape(-1), device=dev)
    d_ff = torch.empty(el.ndof, device=dev, dtype=torch.float64)
    d_csr = torch.empty(el.nnz, device=dev, dtype=torch.float64)
    el.initialize_internal_values()
    el.backup_secondary_values()
    for _ in range(warmup):
        el.update_and_assemble(d_ddu, d_ff, d_csr)
    el.sync()
    plastic = float(1.0 - el.get_state()[2].mean())
    ms = time_steps(torch, el, stream, steps, d_ddu, d_ff, d_csr)
    L.pms_elements_set_timing(el.h, 1)
    L.pms_elements_kernel_times(el.h, None, None)
    for _ in range(steps):
        el.update_and_assemble(d_ddu, d_ff, d_csr)
    kt = np.zeros(3)
    kc = np.zeros(3, np.int64)
    L.pms_elements_kernel_times(el.h, _lib.ptr(kt), _lib.ptr(kc))
    L.pms_elements_set_timing(el.h, 0)
    ab = assembly_ab(torch, L, el, stream, steps, warmup, d_ddu, d_ff, d_csr)
    ng, nip = 9, m.ncell * 9
    # the fused step's algorithmic bytes in 2D: coordinates, connectivity, dU, IP state read (sigma 4 +
    # z) and written (sigma 4 + z + lambda + flag), R and the CSR values once
    step_bytes = (m.npoint * 16 + m.ncell * 8 * 4 + m.ndof * 8 + nip * 40 + nip * 49 + m.ndof * 8
                  + int(el.nnz) * 8)
    del d_csr
    el.close()
    gbs_step = step_bytes / (ms * 1e-3) / 1e9
    return {"workload": f"qua8 {n}x{n} footing material, 9 IP, one fused Newton iteration", "ncell": m.ncell,
            "nip": nip, "nnz": int(el.nnz), "plastic_fraction": plastic, "ms_per_step": ms,
            "kernels": "element2d_kernel<8,10,UPD_BACKUP,F,K> (update + F_int + upper K_e blocks), f_gather, "
                       "kk_gather<2,8> (rows summed in ascending cell order)",
            "kernels_ms_per_step": kernel_ms(kt, kc),
            "assembly_ab": ab,
            "step_roofline": {"bound": "hbm", "achieved": gbs_step, "peak": hbm_peak, "unit": "GB/s",
                              "frac": gbs_step / hbm_peak, "algorithmic_bytes_per_step": step_bytes}}


def time_steps(torch, el, stream, steps, d_ddu, d_ff, d_csr):
    """Mean device time (ms, CUDA events on the handle's stream) of `steps` fused Newton iterations."""
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        el.update_and_assemble(d_ddu, d_ff, d_csr)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def assembly_ab(torch, L, el, stream, steps, warmup, d_ddu, d_ff, d_csr, other="direct", default="gather"):
    """The same step with the other assembly, timed per kernel, beside the default's step.  Gather:
    the element kernel writes each cell's upper element-matrix blocks, row gathers sum them in
    ascending cell order.  Direct: the element kernel adds the blocks straight into the CSR values
    (ordered, no element matrices).  Both sum every entry in a fixed order."""
    from pmsim_b200 import _lib
    el.set_assembly(other)
    for _ in range(max(2, warmup)):
        el.update_and_assemble(d_ddu, d_ff, d_csr)
    ms_o = time_steps(torch, el, stream, steps, d_ddu, d_ff, d_csr)
    L.pms_elements_set_timing(el.h, 1)
    L.pms_elements_kernel_times(el.h, None, None)
    for _ in range(steps):
        el.update_and_assemble(d_ddu, d_ff, d_csr)
    kt = np.zeros(3)
    kc = np.zeros(3, np.int64)
    L.pms_elements_kernel_times(el.h, _lib.ptr(kt), _lib.ptr(kc))
    L.pms_elements_set_timing(el.h, 0)
    el.set_assembly(default)
    el.update_and_assemble(d_ddu, d_ff, d_csr)
    el.sync()
    return {"default": default, "other": other, "other_ms_per_step": ms_o,
            "other_kernels_ms_per_step": kernel_ms(kt, kc)}


def lower_triangle_step(torch, L, el, stream, steps, warmup, d_ddu, d_ff):
    """The same device-resident step with K stored as its lower triangle (Sym::YesLower): the row
    gather skips the blocks above the diagonal and writes about half the CSR values."""
    from pmsim_b200 import _lib
    el.set_symmetry("lower")
    d_low = torch.empty(el.nnz, device=d_ddu.device, dtype=torch.float64)
    for _ in range(max(2, warmup)):
        el.update_and_assemble(d_ddu, d_ff, d_low)
    ms = time_steps(torch, el, stream, steps, d_ddu, d_ff, d_low)
    L.pms_elements_set_timing(el.h, 1)
    L.pms_elements_kernel_times(el.h, None, None)
    for _ in range(steps):
        el.update_and_assemble(d_ddu, d_ff, d_low)
    kt = np.zeros(3)
    kc = np.zeros(3, np.int64)
    L.pms_elements_kernel_times(el.h, _lib.ptr(kt), _lib.ptr(kc))
    L.pms_elements_set_timing(el.h, 0)
    nnz = el.nnz
    el.set_symmetry("full")
    del d_low
    return {"nnz": nnz, "ms_per_step": ms, "kernels_ms_per_step": kernel_ms(kt, kc)}


def kernel_ms(kt, kc):
    """Per-step times of the element kernel and the two gathers (absent under the direct assembly)."""
    out = {"element": kt[0] / max(kc[0], 1)}
    if kc[1]:
        out["f_gather"] = kt[1] / kc[1]
    if kc[2]:
        out["kk_gather"] = kt[2] / kc[2]
    return out


def run_batched(nprob, nalone, seed=2024):
    """Batched footing solves (the 512-problem configuration): every problem through its 10 load
    steps to max|R| <= 1e-10 on the device (one element launch and one batched PCG per Newton
    iteration), against the same device solver one problem at a time and the drop-in path with the
    host direct solve, on a seeded sample of the same population."""
    import torch
    from pmsim_b200.batch import BatchSolver
    from pmsim_b200.elements import Elements
    from pmsim_b200.footing import population
    from pmsim_b200.solver import SolverImplicit
    probs = population(nprob, seed=seed)
    t0 = time.perf_counter()
    bs = BatchSolver(probs, n_max_iterations=20, pcg_max_iterations=5000)
    t_setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    tuning = bs.autotune()
    t_tune = time.perf_counter() - t0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bs.solve_independent(on_fail="drop")
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    nfail = len(bs.failed)
    nconv = nprob - nfail
    import ctypes
    pcg_t = ctypes.c_int64()
    bs.L.pms_batch_counters(bs.h, ctypes.byref(pcg_t))
    newton = [sum(h) for i, h in enumerate(bs.history) if i not in bs.failed]
    ndof = int(bs.mesh.ndof)
    syncs_ticks = bs.host_syncs()
    newton_all = int(sum(sum(h) for h in bs.history))
    bs.close()
    del bs
    # the same population in lock-step load steps with the Newton loop resident on the device (one
    # CUDA graph launch and one host wait per load step; the same bits per problem as the ticks)
    bg = BatchSolver(probs, n_max_iterations=20, pcg_max_iterations=5000)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bg.solve(on_fail="drop", device_loop=True)
    torch.cuda.synchronize()
    t_graph = time.perf_counter() - t0
    graph_conv = nprob - len(bg.failed)
    graph_newton = int(sum(sum(h) for h in bg.history))
    graph = {"seconds": t_graph, "solves_per_s": graph_conv / t_graph, "converged": graph_conv,
             "host_syncs": bg.host_syncs(), "newton_iterations_total": graph_newton,
             "host_syncs_per_newton_iteration": bg.host_syncs() / max(graph_newton, 1),
             "note": "lock-step load steps, Newton loop in one CUDA graph per step (conditional WHILE nodes), "
                     "batch-wide PCG engine"}
    bg.close()
    del bg
    rng = np.random.default_rng(seed + 1)
    sample = sorted(rng.choice(nprob, size=min(nalone, nprob), replace=False).tolist())
    t_alone, ok_alone = 0.0, 0
    for i in sample:
        b1 = BatchSolver([probs[i]], n_max_iterations=20, pcg_max_iterations=5000)
        t0 = time.perf_counter()
        b1.autotune()  # its own best launch shapes, timed with the solve
        b1.solve_independent(on_fail="drop")
        torch.cuda.synchronize()
        t_alone += time.perf_counter() - t0
        ok_alone += 0 if b1.failed else 1
        b1.close()
    t_direct, ok_direct = 0.0, 0
    for i in sample[: max(1, len(sample) // 2)]:
        p = probs[i]
        el = Elements(p.mesh, p.material, ngauss=9)
        sol = SolverImplicit(el, p.essential, n_max_iterations=20, t_fin=float(p.nsteps))
        t0 = time.perf_counter()
        try:
            sol.solve()
            ok_direct += 1
        except Exception:
            pass
        t_direct += time.perf_counter() - t0
        el.close()
    n_direct = max(1, len(sample) // 2)
    # converged solves per second on both sides (failures cost time but do not count)
    batched = nconv / t_batch
    alone = ok_alone / t_alone
    direct = ok_direct / t_direct
    return {"problems": nprob, "converged": nconv, "failed": nfail, "ndof_total": ndof,
            "seconds": t_batch, "setup_seconds": t_setup, "autotune_seconds": t_tune, "tuning": tuning,
            "solves_per_s": batched,
            "newton_iterations_total": int(sum(newton)), "pcg_iterations_total": int(pcg_t.value),
            "host_syncs_per_newton_iteration": syncs_ticks / max(newton_all, 1), "device_loop": graph,
            "attempts_per_s": nprob / t_batch, "alone_attempts_per_s": len(sample) / t_alone,
            "alone_sample": len(sample), "alone_converged": ok_alone, "alone_solves_per_s": alone,
            "ratio_vs_alone": batched / alone if alone > 0 else None,
            "direct_sample": n_direct, "direct_converged": ok_direct, "direct_solves_per_s": direct,
            "ratio_vs_direct": batched / direct if direct > 0 else None,
            "note": "solves/s counts converged problems (max|R| <= 1e-10); failures are Newton divergence "
                    "of the reference scheme on the finest meshes (the CPU oracle fails them too)"}


def run_c0():
    """The reference's CPU-runnable case: the 20x10 Qua8 strip footing (9 IP, 1322 DOF, 10 steps)
    solved end to end by (a) the drop-in path (device element calls + host sparse LU), (b) the
    device Newton/PCG solver, (c) the CPU oracle (C++ restatement, one thread, SuperLU), with the
    Newton iteration counts of every step."""
    import oracle
    import torch
    from oracle.driver import OracleSolver
    from pmsim_b200.batch import BatchSolver
    from pmsim_b200.elements import Elements
    from pmsim_b200.footing import footing_problem
    from pmsim_b200.solver import SolverImplicit
    p = footing_problem(20, 10, 1e4, 9.0, 1.0, nsteps=10)
    el = Elements(p.mesh, p.material, ngauss=9)
    sol = SolverImplicit(el, p.essential, n_max_iterations=20, t_fin=10.0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sol.solve()
    t_dropin = time.perf_counter() - t0
    it_dropin = [len(h) for h in sol.history]
    el.close()
    bs = BatchSolver([p], n_max_iterations=20)
    t0 = time.perf_counter()
    bs.solve_independent(on_fail="raise")
    torch.cuda.synchronize()
    t_dev = time.perf_counter() - t0
    it_dev = list(bs.history[0])
    bs.close()
    mt = p.material
    oel = oracle.OracleElements(p.mesh, 1, oracle.Params(mt.young, mt.poisson, mt.hh, mt.z_ini), ngauss=9,
                                sym_tol=-1.0, nthreads=1)
    osol = OracleSolver(oel, p.mesh.ndof, p.essential, n_max_iterations=20, t_fin=10.0)
    t0 = time.perf_counter()
    osol.solve()
    t_cpu = time.perf_counter() - t0
    it_cpu = [len(h) for h in osol.history]
    return {"workload": "footing 20x10 Qua8, 9 IP, 1322 DOF, 10 steps (LMM)", "dropin_s": t_dropin,
            "device_newton_pcg_s": t_dev, "oracle_cpu_1thread_s": t_cpu, "iterations_dropin": it_dropin,
            "iterations_device": it_dev, "iterations_oracle": it_cpu,
            "dropin_elements_s": sol.timing["elements"], "dropin_solve_s": sol.timing["solve"]}


def run_served(nreq, rate, nalone, seed=7, detail_file="", nplain=32, plain_cap=3.0, plain_max3d=60000,
               sweep_rates=(2.0, 4.0, 8.0, 16.0), nsweep=24):
    """Served configuration: Poisson arrivals (rate req/s) of footing (70%, 1k-50k DOF) and Hex8
    block (30%, up to 206,763 DOF) requests, 10 load steps each, admitted under a 120 GB device
    budget into device batches that overlap on the GPU (continuous batching); throughput and
    latency percentiles; the same requests solved one at a time by the device solver, and a sample
    of the smaller ones by the plain drop-in path, for the ratios."""
    import torch
    from pmsim_b200.batch import BatchSolver
    from pmsim_b200.footing import request_population
    from pmsim_b200.serve import Request, Server, poisson_arrivals, summarize
    probs = request_population(nreq, seed=seed)
    arr = poisson_arrivals(nreq, rate, seed=seed + 1)
    reqs = [Request(i, p, float(a)) for i, (p, a) in enumerate(zip(probs, arr))]
    srv = Server(budget_bytes=120e9, n_max_iterations=20, pcg_max_iterations=5000)
    torch.cuda.synchronize()
    srv.serve(reqs)
    torch.cuda.synchronize()
    out = summarize(reqs)
    out.update({"rate_req_per_s": rate, "batches": srv.batches, "peak_concurrent_batches": srv.peak_concurrent,
                "peak_admitted_bytes": srv.peak_in_use, "budget_bytes": 120e9,
                "ndof_min": int(min(p.mesh.ndof for p in probs)), "ndof_max": int(max(p.mesh.ndof for p in probs))})
    rng = np.random.default_rng(seed + 2)
    sample = sorted(rng.choice(nreq, size=min(nalone, nreq), replace=False).tolist())
    t_alone, ok = 0.0, 0
    for i in sample:
        b1 = BatchSolver([probs[i]], n_max_iterations=20, pcg_max_iterations=5000)
        t0 = time.perf_counter()
        b1.autotune()  # its own best launch shapes, timed with the solve
        b1.solve_independent(on_fail="drop")
        torch.cuda.synchronize()
        t_alone += time.perf_counter() - t0
        ok += 0 if b1.failed else 1
        b1.close()
    # the plain GPU path -- the drop-in path (device element calls + host sparse LU) one request
    # at a time -- on a seeded sample of the smaller requests (<= 20,000 DOF).  Larger
    # requests only take longer on it, so the ratio is a lower bound; a request still running
    # after the load step that passes 20 s is stopped and counted as converged at that time (again
    # in the plain path's favour).
    from pmsim_b200.elements import Elements
    from pmsim_b200.solver import SolverImplicit

    class _Cap(Exception):
        pass

    # a sample stratified over the whole DOF range (every nreq/nplain-th request by size); each run
    # stops at plain_cap seconds (checked after every Newton iteration) and counts as converged at
    # that time, and 3D requests whose single host factorisation alone would take far longer than the
    # cap (above plain_max3d DOF) count as capped without running: both favour the plain path, so
    # the ratio is a lower bound, and the capped share is reported
    order = sorted(range(nreq), key=lambda i: probs[i].mesh.ndof)
    nplain = min(nplain, nreq)
    psample = sorted({order[int(k * (nreq - 1) / max(nplain - 1, 1))] for k in range(nplain)})
    t_plain, ok_plain, capped, skipped = 0.0, 0, 0, 0
    for i in psample:
        p = probs[i]
        if p.mesh.ndim == 3 and p.mesh.ndof > plain_max3d:
            t_plain += plain_cap
            ok_plain += 1
            skipped += 1
            continue
        el = Elements(p.mesh, p.material, ngauss=p.ngauss)
        sol = SolverImplicit(el, p.essential, n_max_iterations=20, t_fin=float(p.nsteps))
        t0 = time.perf_counter()

        def cap(step, it, t0=t0):
            if time.perf_counter() - t0 > plain_cap:
                raise _Cap()
        try:
            sol.solve(on_iteration=cap)
            ok_plain += 1
        except _Cap:
            ok_plain += 1
            capped += 1
        except Exception:
            pass
        t_plain += time.perf_counter() - t0
        el.close()
    if detail_file:
        with open(detail_file, "w") as f:
            json.dump([{"rid": r.rid, "kind": r.problem.mesh.kind, "ndof": int(r.problem.mesh.ndof),
                        "arrival": r.arrival, "admitted": r.admitted, "finished": r.finished, "error": r.error,
                        **r.meta} for r in reqs], f)
    # arrival-rate sweep: the highest rate the server keeps up with (completions per second at least
    # 3/4 of the arrival rate over a stream of nsweep requests), with the latency there
    sweep = []
    for lam in sweep_rates:
        probs2 = request_population(nsweep, seed=seed + 10)
        arr2 = poisson_arrivals(nsweep, lam, seed=seed + 11)
        reqs2 = [Request(i, p, float(a)) for i, (p, a) in enumerate(zip(probs2, arr2))]
        srv2 = Server(budget_bytes=120e9, n_max_iterations=20, pcg_max_iterations=5000)
        srv2.serve(reqs2)
        torch.cuda.synchronize()
        s2 = summarize(reqs2)
        done_rate = s2["requests"] / s2["seconds"]
        sweep.append({"rate_req_per_s": lam, "requests": nsweep, "completions_per_s": done_rate,
                      "solves_per_s": s2["solves_per_s"], "latency_p50_s": s2["latency_p50_s"],
                      "latency_p99_s": s2["latency_p99_s"], "kept_up": bool(done_rate >= 0.75 * lam)})
    kept = [x for x in sweep if x["kept_up"]]
    out["rate_sweep"] = sweep
    out["highest_sustained_rate_req_per_s"] = max((x["rate_req_per_s"] for x in kept), default=None)
    out["alone_sample"] = len(sample)
    out["alone_solves_per_s"] = ok / t_alone if t_alone > 0 else None
    out["ratio_vs_alone"] = (out["solves_per_s"] / out["alone_solves_per_s"]) if ok else None
    plain = ok_plain / t_plain if t_plain > 0 else None
    out.update({"plain_sample": len(psample), "plain_sample_ndof": [int(probs[i].mesh.ndof) for i in psample],
                "plain_cap_s": plain_cap, "plain_capped": capped, "plain_not_run_3d_above_ndof": plain_max3d,
                "plain_not_run": skipped, "plain_capped_share": (capped + skipped) / max(len(psample), 1),
                "plain_solves_per_s": plain,
                "ratio_vs_plain": (out["solves_per_s"] / plain) if plain else None,
                "plain_note": "drop-in path (device elements + host SuperLU) one request at a time on a sample "
                              "stratified over the DOF range; capped or not-run requests count as converged "
                              "at the cap: a lower bound of the ratio"})
    return out


def cpu_sample(m, ddu, ncell_sample, nthreads):
    """The oracle (C++ restatement of pmsim's element/material path, structured like the reference:
    per-cell dense B^T D B, COO triplets with duplicates, sort/sum to CSR) on the first
    ncell_sample cells.  Returns seconds for update + F_int + K(COO) + CSR, the IP count and the
    oracle's results (elements with their IP state, F_int over all DOFs, CSR of the sample)."""
    import oracle
    from pmsim_b200 import mesh as M
    sub = M.Mesh(3, m.coords, m.cells[:ncell_sample], m.kind)
    el = oracle.OracleElements(sub, oracle.MODEL_VON_MISES, oracle.Params(E, NU, HH, Z0), sym_tol=-1.0,
                               nthreads=nthreads)
    el.initialize()
    t = [time.perf_counter()]
    el.update_secondary_values(ddu)
    t.append(time.perf_counter())
    ff = el.assemble_f_int()
    t.append(time.perf_counter())
    rows, cols, vals = el.assemble_kk_coo()
    t.append(time.perf_counter())
    csr = oracle.coo_to_csr(m.ndof, rows, cols, vals)
    t.append(time.perf_counter())
    cpu_sample.phases = dict(zip(("update_secondary", "f_int", "k_coo", "csr_sum"),
                                 (t[i + 1] - t[i] for i in range(4))))
    return t[-1] - t[0], ncell_sample * el.ngauss, (el, ff, csr)


def parity_sample(m, ncs, state, ff, csr_values, indptr, indices, ref, tol=1e-12):
    """The GPU step against the oracle on the first ncs cells of the same mesh and increment.

    state = (sig, ivs, elastic) of the GPU (all IPs), ff its F_int, csr_values/indptr/indices its K;
    ref = (oracle elements over the first ncs cells, their F_int over all DOFs, their CSR).  Compared:
    the IP state of the sample's IPs; every R entry and every CSR row of the nodes whose incident
    cells all lie in the sample (the rows the sample computes completely).  Relative normwise 1e-12;
    elastic flags and column indices must be identical."""
    oel, off, (oip, oix, odata) = ref
    ng = oel.ngauss
    nip = ncs * ng
    sig, ivs, el = state
    out = {"sample_cells": int(ncs), "sample_ips": int(nip), "tol_rel": tol}

    def rel(a, b):
        scale = float(np.max(np.abs(b))) if b.size else 0.0
        return float(np.max(np.abs(a - b))) / max(scale, 1e-300) if b.size else 0.0

    errs = {"sigma": rel(sig[:nip], oel.sig), "z_lambda": rel(ivs[:nip], oel.ivs)}
    flags_ok = bool(np.array_equal(el[:nip], oel.elastic))
    n_all = np.bincount(m.cells.ravel(), minlength=m.npoint)
    n_in = np.bincount(m.cells[:ncs].ravel(), minlength=m.npoint)
    inside = np.flatnonzero((n_all == n_in) & (n_in > 0))
    rows = (inside[:, None] * m.ndim + np.arange(m.ndim)).ravel()
    errs["f_int_rows"] = rel(ff[rows], off[rows])
    lo, hi = indptr[rows], indptr[rows + 1]
    olo, ohi = oip[rows], oip[rows + 1]
    pattern_ok = bool(np.array_equal(hi - lo, ohi - olo))
    if pattern_ok and rows.size:
        take = np.concatenate([np.arange(x, y) for x, y in zip(lo, hi)])
        otake = np.concatenate([np.arange(x, y) for x, y in zip(olo, ohi)])
        pattern_ok = bool(np.array_equal(indices[take], oix[otake]))
        errs["csr_rows"] = rel(csr_values[take], odata[otake])
        out["csr_values_compared"] = int(take.size)
    out.update({"rows_compared": int(rows.size), "max_rel_err": errs, "elastic_flags_equal": flags_ok,
                "pattern_equal": pattern_ok})
    out["ok"] = bool(flags_ok and pattern_ok and rows.size > 0 and all(v <= tol for v in errs.values()))
    return out


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def pcg_time(args):
    """--pcg-time: device time per PCG iteration of one problem on its initial tangent (unit
    right-hand side), with the team engine (a thread-block cluster per problem) or the batch-wide
    engine (pms_batch_time_pcg); the launch shapes of profile captures of the PCG kernels."""
    import ctypes
    from pmsim_b200 import _lib
    from pmsim_b200.batch import BatchSolver
    from pmsim_b200.footing import block_problem, footing_problem
    engine, problem, dims = args.pcg_time[0], args.pcg_time[1], [int(v) for v in args.pcg_time[2:]]
    if engine not in ("team", "wide") or problem not in ("foot", "hex"):
        raise SystemExit("--pcg-time ENGINE PROBLEM DIMS: ENGINE team|wide, PROBLEM foot|hex")
    p = footing_problem(*dims[:2]) if problem == "foot" else block_problem(*dims[:3])
    bs = BatchSolver([p])
    t = _lib.BatchTuning_(10 ** 12 if engine == "team" else 0, args.pcg_threads, args.pcg_chunks, 128, 8)
    ms = ctypes.c_double()
    rc = bs.L.pms_batch_time_pcg(bs.h, ctypes.byref(t), args.pcg_iterations, ctypes.byref(ms))
    if rc != 0:
        raise _lib.PmsError(rc)
    print(f"{engine} {problem} {dims} ndof {p.mesh.ndof}: {ms.value / args.pcg_iterations * 1e3:.2f} us per iteration")
    bs.close()


def reference_arm(args, rank):
    """--impl reference: the reference's CPU path (oracle port; the Rust reference cannot be built
    here) on the host cores, same metric and workload, each step a bounded sample."""
    if rank != 0:
        return
    import oracle
    m = make_problem(args.size)
    ddu = synthetic_ddu(m, args.size)
    nthreads = oracle.lib().orc_max_threads()
    ncs = args.cpu_cells or (512 if args.size == "small" else 4096)
    cpu_sample(m, ddu, min(ncs, 256), nthreads)  # warm-up (page-in, thread pool)
    tot, ips = 0.0, 0
    for _ in range(args.steps):
        dt, n, _ = cpu_sample(m, ddu, ncs, nthreads)
        tot += dt
        ips += n
    value = ips / tot
    nx, ny, nz = workload_dims(args.size)
    line = {
        "impl": "reference", "metric": "IP stress-update+tangent/s FP64", "value": value, "unit": "IP/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"hex20 {nx}x{ny}x{nz} block, 27 IP, von Mises (one Newton iteration)",
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "IP/s", "cores": nthreads, "kind": "port",
                         "sample": f"first {ncs} cells ({ncs * 27} IPs) per step: update + F_int + K COO + CSR",
                         "cpu_model": cpu_model(), "nproc": os.cpu_count()},
        "e2e": {"value": value, "unit": "IP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    if args.pcg_time:
        pcg_time(args)
        return
    import torch
    from pmsim_b200 import dist
    if world > 1:
        torch.cuda.set_device(local)
        dist.init("nccl", timeout_s=120)
    from pmsim_b200 import _lib
    from pmsim_b200.elements import Elements, Material
    L = _lib.load()
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)

    m = make_problem(args.size)
    ddu_h = synthetic_ddu(m, args.size, seed=20241203 + rank)
    el = Elements(m, Material.von_mises(E, NU, HH, Z0))
    el.set_stream(stream)
    ng, nnz, ndof = el.ngauss, el.nnz, el.ndof
    d_ddu = torch.tensor(ddu_h, device=dev)
    d_ff = torch.empty(ndof, device=dev, dtype=torch.float64)
    d_csr = torch.empty(nnz, device=dev, dtype=torch.float64)
    el.initialize_internal_values()
    el.backup_secondary_values()

    barrier = dist.barrier

    # warm-up
    for _ in range(args.warmup):
        el.update_and_assemble(d_ddu, d_ff, d_csr)
    el.sync()
    torch.cuda.synchronize(dev)
    sig, ivs, elastic = el.get_state()
    plastic = float(1.0 - elastic.mean())

    # timed region: device-resident inputs (every buffer is far larger than the 126 MB L2)
    L.pms_elements_set_timing(el.h, 1)
    L.pms_elements_kernel_times(el.h, None, None)
    clocks = Clocks(dev)
    launches0 = el.launch_count()
    barrier()
    torch.cuda.synchronize(dev)
    clocks.mark(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        el.update_and_assemble(d_ddu, d_ff, d_csr)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clocks.mark(False)
    barrier()
    clk = clocks.stop()
    launches = el.launch_count() - launches0
    ms = e0.elapsed_time(e1) / args.steps
    kt = np.zeros(3)
    kc = np.zeros(3, np.int64)
    L.pms_elements_kernel_times(el.h, _lib.ptr(kt), _lib.ptr(kc))
    L.pms_elements_set_timing(el.h, 0)
    el.sync()
    ms_max = dist.max_over_ranks(ms, dev)
    nip = m.ncell * ng
    value = world * nip / (ms_max * 1e-3)
    # the step's results, kept for the parity check against the oracle (rank 0, with the CPU leg)
    gpu_state = gpu_ff = gpu_csr = el_pattern = None
    if rank == 0 and not args.no_cpu:
        gpu_state = el.get_state()
        gpu_ff = d_ff.cpu().numpy()
        gpu_csr = d_csr.cpu().numpy()
        el_pattern = el.csr_pattern()

    # the same step with the direct assembly, for the A/B of the two assemblies
    ab = assembly_ab(torch, L, el, stream, min(args.steps, 10), args.warmup, d_ddu, d_ff, d_csr)
    ab["lower_triangle"] = lower_triangle_step(torch, L, el, stream, min(args.steps, 10), args.warmup, d_ddu, d_ff)

    # e2e through the C ABI with host buffers (pinned): dU in, R and CSR values out, every step
    e2e = None
    if not args.no_e2e:
        h_ddu = torch.tensor(ddu_h).pin_memory().numpy()
        h_ff = torch.empty(ndof, dtype=torch.float64).pin_memory().numpy()
        h_csr = torch.empty(nnz, dtype=torch.float64).pin_memory().numpy()
        el.update_and_assemble(h_ddu, h_ff, h_csr)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            el.update_and_assemble(h_ddu, h_ff, h_csr)
        t_e2e = dist.max_over_ranks((time.perf_counter() - t0) / args.steps, dev)
        e2e = {"value": world * nip / t_e2e, "unit": "IP/s", "h2d_bytes_per_step": ndof * 8,
               "d2h_bytes_per_step": (ndof + nnz) * 8, "ms_per_step": t_e2e * 1e3}
        del h_csr
        # the same call with K stored as its lower triangle (Sym::YesLower, pmsim's storage when the
        # linear solver is MUMPS); the headline above keeps both triangles (pmsim's default, UMFPACK)
        el.set_symmetry("lower")
        nnz_lower = el.nnz
        h_csr = torch.empty(nnz_lower, dtype=torch.float64).pin_memory().numpy()
        el.update_and_assemble(h_ddu, h_ff, h_csr)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            el.update_and_assemble(h_ddu, h_ff, h_csr)
        t_low = dist.max_over_ranks((time.perf_counter() - t0) / args.steps, dev)
        el.set_symmetry("full")
        e2e["lower_triangle"] = {"value": world * nip / t_low, "unit": "IP/s", "h2d_bytes_per_step": ndof * 8,
                                 "d2h_bytes_per_step": (ndof + nnz_lower) * 8, "ms_per_step": t_low * 1e3}
        del h_csr

    if world > 1:
        dist.finalize()
    if rank != 0:
        return

    peaks, peaks_kind = measured_peaks()
    probe_clk = Clocks(dev)
    probe_clk.mark(True)
    fp64 = fp64_peak(torch, L, stream)
    probe_clk.mark(False)
    fp64_clocks = probe_clk.stop()
    k1 = None
    ep = None
    if not args.no_k1 and args.size == "full":
        del d_csr
        torch.cuda.empty_cache()
        k1 = run_k1(torch, stream, max(3, args.steps), args.warmup)
        # the ~40% yielding mix the configuration quotes (the configured deviation yields almost all IPs)
        k1["at_40pct_yield"] = run_k1(torch, stream, max(3, args.steps), args.warmup, scale=k1_scale_for_yield(0.4))
        ep = run_ep(torch, stream, 3, args.warmup)
        k1["roofline"] = {"bound": "hbm", "achieved": k1["gbs"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
                          "frac": k1["gbs"] / peaks["hbm_gbs"], "peak_source": peaks_kind}

    qua8 = None
    if not args.no_qua8:
        torch.cuda.empty_cache()
        qua8 = run_qua8_step(torch, stream, max(3, min(args.steps, 10)), args.warmup, peaks["hbm_gbs"], n=args.qua8_n)

    batched = None
    if args.batched > 0 and args.size == "full":
        torch.cuda.empty_cache()
        batched = run_batched(args.batched, args.alone_sample)
    c0 = None
    if not args.no_c0 and args.size == "full":
        c0 = run_c0()
    served = None
    if args.served > 0 and args.size == "full":
        torch.cuda.empty_cache()
        served = run_served(args.served, args.rate, min(args.alone_sample, 16), detail_file=args.served_detail)
    ms_elem = kt[0] / max(kc[0], 1)  # the element kernel (the gathers are memory-bound, separate kernels)
    fl_ip = flops_per_ip_hex20(plastic)
    achieved_tf = nip * fl_ip / (ms_elem * 1e-3) / 1e12
    fl_alg = flops_per_ip_sparse_b(3, 20)
    alg_tf = nip * fl_alg / (ms_elem * 1e-3) / 1e12
    alg_bytes = algorithmic_bytes_step(m, ng, nnz)
    step_gbs = alg_bytes / (ms * 1e-3) / 1e9
    cpu = None
    parity = None
    if not args.no_cpu:
        import oracle
        nthreads = oracle.lib().orc_max_threads()
        ncs = args.cpu_cells or (512 if args.size == "small" else 4096)
        cpu_sample(m, ddu_h, 256, nthreads)
        dt, n, ref = cpu_sample(m, ddu_h, ncs, nthreads)
        phases = {k: v / n * 1e6 for k, v in cpu_sample.phases.items()}
        dt1, n1, _ = cpu_sample(m, ddu_h, max(ncs // 8, 64), 1)
        cpu = {"value": n / dt, "unit": "IP/s", "cores": nthreads, "kind": "port",
               "sample": f"first {ncs} cells ({n} IPs): update + F_int + K COO + CSR sum, all threads",
               "single_thread_ip_per_s": n1 / dt1, "us_per_ip_by_phase": phases,
               "cpu_model": cpu_model(), "nproc": os.cpu_count()}
        indptr, indices = el_pattern
        parity = parity_sample(m, ncs, gpu_state, gpu_ff, gpu_csr, indptr, indices, ref)
        parity["what"] = ("GPU step vs the oracle on the first cells: IP state of their IPs, R entries and CSR "
                          "rows of the nodes whose cells all lie in the sample")
    nx, ny, nz = workload_dims(args.size)
    line = {
        "metric": "IP stress-update+tangent/s FP64",
        "value": value, "unit": "IP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"hex20 {nx}x{ny}x{nz} block, 27 IP, von Mises E=2e5 nu=0.3 z0=250 H=1e3: "
                               f"one fused Newton iteration (update + F_int + K + CSR)",
                   "ncell": m.ncell, "nip": nip, "ndof": ndof, "nnz": nnz,
                   "plastic_fraction": plastic, "l2": "inputs larger than L2 (no flush)",
                   "parallelism": f"replica per GPU x{world}"},
        "roofline": {"bound": "fp64", "achieved": alg_tf, "peak": fp64, "unit": "TFLOP/s",
                     "frac": alg_tf / fp64,
                     "traffic": ELEMENT_DRAM_BYTES_PER_CELL * m.ncell if ELEMENT_DRAM_BYTES_PER_CELL else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch on a "
                                       "smaller block, scaled by cells to this launch",
                     "kernel": "element_kernel<3,20,UPD_BACKUP,F,K> (fused update + B^T sigma + B^T D B, "
                               "upper element-matrix blocks out)",
                     "flop_per_ip": fl_alg, "flop_count": "algorithmic, sparse-B formulation with a symmetric K_e "
                                                          "(D G_b, G_a^T D G_b for a <= b, J and G)",
                     "peak_source": "FP64 FMA probe measured in this run",
                     "kernel_flops": {
                         "flop_per_ip": fl_ip, "achieved": achieved_tf, "frac": achieved_tf / fp64,
                         "note": "the FLOPs the kernel executes: the two-pass node-pair form (X_ab = sum alpha g_a "
                                 "g_b^T at every IP, 18 FMA more per node pair at plastic IPs only) at this "
                                 "step's plastic fraction, fewer than the algorithmic count"}},
        "roofline_hbm": {"bound": "hbm", "achieved": step_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": step_gbs / peaks["hbm_gbs"], "algorithmic_bytes_per_step": alg_bytes,
                         "peak_source": peaks_kind},
        "kernels_ms_per_step": kernel_ms(kt, kc),
        "assembly_ab": ab,
        "gpu_launches": int(launches),
        "e2e": e2e, "cpu_baseline": cpu, "parity": parity, "k1_microbench": k1, "ep_microbench": ep, "qua8_step": qua8, "batched": batched, "served": served, "c0_footing": c0, "fp64_peak_tflops": fp64, "fp64_peak_clocks": fp64_clocks,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    if parity is not None and not parity["ok"]:
        sys.exit("parity check against the oracle failed: " + json.dumps(parity))


if __name__ == "__main__":
    main()
