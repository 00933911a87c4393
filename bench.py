"""Benchmark: projected energy + orbital gradient throughput (grid points per second).

Workload (one step = one full energy + gradient evaluation, as one call of PHF.py's EandG):
  c5 (default): n = 200 spatial orbitals (M = 400 spin orbitals), N = 100 electrons, L = 1000
      Cholesky vectors, grid = Lebedev 50 x 16 gamma x 4 C2v operations = 3200 points, J/K from the
      Cholesky vectors without an n^4 tensor (the streamed exchange form); seeded synthetic h, B_L
      and determinant (no molecular input is available offline).
  c2 / c3: n = 64 (L = 400, 3200 points) / n = 128 (L = 800, 800 points), exchange matrix stored.
  c4: 256 independent instances of uneven size in one batched evaluation.

Arms:
  --impl ours       the GPU path.  `value` is device time of the evaluation with C resident in
                    HBM (CUDA events on the launching stream, max over ranks); `e2e` is the same
                    metric through the C ABI with host buffers: phf_plan_buildhsg with the plan
                    (Hamiltonian and grid on the device) created once, per call the host -> device
                    copy of the determinant and the device -> host copy of Hmat, Smat, Gradmat,
                    Rdmmat inside the timed region; e2e.one_shot is the drop-in phf_buildhsg_chol,
                    which also uploads h, B, Ref and the grid and builds the plan in every call.
  --impl reference  the reference algorithm on the host cores: the C/OpenMP restatement of
                    PHF_fort/PHFTools.f90 BuildHSG timed on a bounded sample of grid points (the
                    reference Fortran cannot be compiled here): MakeGamma over the dense HTwo where it
                    fits in host memory (n = 64: 4.3 GB), else the same Gamma from the spatial Cholesky
                    vectors (the dense HTwo would be 69 GB at n = 128 and 410 GB at n = 200).

Multi-GPU (torchrun, one process per GPU): every rank evaluates its own independent instance
(weak scaling, no collective on the data path); value = points of all ranks / max rank time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "projected E+grad grid-pts/s, split-prec vs FP64 GPU @|ΔE|≤1e-8 Eh; vs host CPU"
UNIT = "grid-pts/s"


def _json_default(o):
    """numpy scalars (bools, floats, ints) in the bench line as their Python values."""
    if isinstance(o, np.generic):
        return o.item()
    raise TypeError(f"{type(o).__name__} is not JSON serializable")


def _peak_source(peaks, what):
    """Where the bf16 denominator came from: the measured file, or the fallback figure."""
    if peaks.get("fallback"):
        return f"{what} the fallback bf16 burst of 1.59 PFLOP/s (MEASURED_PEAKS.json absent; of fallback)"
    return f"{what} the measured bf16 burst of MEASURED_PEAKS.json (of measured)"


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "fallback": True}


class NvmlClockSampler:
    """SM clock, power and clock-event reasons read through NVML every 2 ms during the timed
    region (read-only queries; nothing is changed on the GPU)."""

    def __init__(self, index: int):
        import pynvml

        self.nv = pynvml
        pynvml.nvmlInit()
        self.h = None
        try:  # NVML numbers all GPUs of the node; find this process's device by its PCI address
            import torch

            pr = torch.cuda.get_device_properties(index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
        self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        self.samples = []
        self._stop = threading.Event()

    def _read(self):
        nv = self.nv
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self._stop.is_set():
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)),
                                     int(get_reasons(self.h)), nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0))
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        self._stop.clear()
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=5)

    def summary(self):
        nv = self.nv
        bits = {"hw_slowdown": nv.nvmlClocksThrottleReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksThrottleReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksThrottleReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksThrottleReasonSwPowerCap}
        reasons = sorted({nm for _, r, _ in self.samples for nm, b in bits.items() if r & b})
        sm = [c for c, _, _ in self.samples]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax, "reasons": reasons,
                "samples": len(sm), "power_w_max": max((w for _, _, w in self.samples), default=None),
                "source": "NVML, 2 ms period"}


def clock_sampler(index: int):
    """NVML sampler when pynvml works, else nvidia-smi."""
    try:
        return NvmlClockSampler(index)
    except Exception:
        return ClockSampler(index)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def problem_for(name: str, seed: int, ngrid=None):
    """The configuration's problem; ``ngrid`` (Lebedev points, gamma points) replaces its grid, for
    profiling a configuration's kernels on a smaller grid."""
    from phf_pcc_b200 import synth
    if not ngrid:
        return synth.config_problem(name, seed=seed)
    c = synth.CONFIGS[name]
    return synth.make_problem(c["n"], c["N"], c["L"], ngrid=tuple(ngrid), seed=seed, pg=c["pg"])


def api_kwargs(p):
    kw = p.grid_kwargs()
    return dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
                r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
                roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])


def jk_form_of(p):
    """The library's automatic J/K form: the stored exchange matrix up to n = 128, above it the
    streamed form (exchange rows regenerated from the Cholesky vectors panel by panel, no n^4
    tensor), as the n = 200 workload asks."""
    return "eri" if p.n <= 128 else "streamed"


def sym_active(p, form, precision, sym="auto"):
    """Whether the library runs the streamed form with the exchange symmetry (pairs i <= k against the
    symmetric half of each density, i < k against the antisymmetric half): on by default in FP64 and,
    for n > 64, in the tensor-core precisions."""
    return form == "streamed" and sym != "off" and (precision == "fp64" or p.n > 64)


def choose_ipanel(n):
    """Spatial indices per exchange panel of the streamed form, as the library chooses them: at most
    8192 exchange rows, fewest 128-row padded rows over all panels, ties to the larger panel."""
    best, best_rows = 1, -1
    for I in range(1, n + 1):
        if I * n > max(8192, n):
            break
        rows = (n // I) * (-(-I * n // 128) * 128) + ((-(-(n % I) * n // 128) * 128) if n % I else 0)
        if best_rows < 0 or rows <= best_rows:
            best, best_rows = I, rows
    return best


def sym_panels(n, ipanel=0):
    """Panels (i0, indices) of the symmetric form: a panel starting at i0 takes max(1, ipanel n / (n - i0))
    indices, so that its Gram block (indices x n rows, (n - i0) n columns) stays within ipanel n x n^2."""
    budget = (ipanel or choose_ipanel(n)) * n
    out, i0 = [], 0
    while i0 < n:
        ip = max(1, min(n - i0, budget // (n - i0)))
        out.append((i0, ip))
        i0 += ip
    return out


def jk_flops_per_point(p, form, sym=False, precision="ozaki_i8"):
    """Algorithmic real flops of the exchange/Coulomb contraction per grid point.

    eri / streamed:  K = EK (n^2 x n^2, real) times 4 complex density columns: 16 n^4, and the
                     Coulomb term d = B vec P, J = B^T d: 8 L n^2 (the streamed form also
                     regenerates EK once per chunk: jk_regen_flops, counted as executed work)
    streamed with the exchange symmetry: the pair rows times 8 real columns, 16 (p_le^2 + p_lt^2) with
                     p_le = n(n+1)/2 and p_lt = n(n-1)/2 (about 8 n^4); in the tensor-core forms the
                     Coulomb d runs over the pairs too: 4 L (p_le + n^2)
    factorized form: T = V^H X (8 L N^2 M), Q = X T' (8 L N^2 M), GX = sum_L B_L Q_L (8 L n^2 N)"""
    n, N, M, L = p.n, p.N, p.M, p.L
    if form == "streamed" and sym:
        ple, plt = n * (n + 1) / 2, n * (n - 1) / 2
        coul = 8.0 * L * n * n if precision == "fp64" else 4.0 * L * (ple + n * n)
        return 16.0 * (ple * ple + plt * plt) + coul
    if form in ("eri", "streamed"):
        return 16.0 * n ** 4 + 8.0 * L * n * n
    return 8.0 * L * N * N * M * 2 + 8.0 * L * n * n * N


def jk_regen_flops(p, form, chunks, sym=False, ipanel=0):
    """Flops of the streamed form's exchange-row regeneration per evaluation: the Gram products
    B^T B (n^2 x n^2, k = L) once per chunk; with the exchange symmetry each panel's Gram block keeps
    only the columns k >= i0 (panel indices x n rows, (n - i0) n columns)."""
    if form != "streamed":
        return 0.0
    if sym:
        n = p.n
        return 2.0 * p.L * chunks * sum(ip * n * (n - i0) * n for i0, ip in sym_panels(n, ipanel))
    return 2.0 * p.n ** 4 * p.L * chunks


def tc_reps(precision, slices):
    """Tensor-core products per FP64-equivalent product: S(S+1)/2 int8 slice products, three BF16
    products for bf16x3, one TF32 product for tf32."""
    if precision == "ozaki_i8":
        return slices * (slices + 1) / 2
    return 3.0 if precision == "bf16x3" else 1.0


def tc_ops_per_step(p, precision, slices, form, chunks, sym=False, ipanel=0):
    """Executed tensor-core operations of the J/K contraction per evaluation (2 per multiply-add)."""
    return tc_reps(precision, slices) * (jk_flops_per_point(p, form, sym, precision) * p.grid.npoints +
                                         jk_regen_flops(p, form, chunks, sym, ipanel))


def tc_ops_per_point(p, precision, slices):
    """Executed tensor-core operations per grid point of the stored-exchange-matrix contractions."""
    return tc_reps(precision, slices) * (16.0 * p.n ** 4 + 8.0 * p.L * p.n ** 2)


def quoted_flops_per_point(p):
    """Per-point work figure of the benchmark description: 32 L n^3 + 8 L n^2 (J/K) plus
    16 M^2 N + 16 M N^2 + 8 N^3 + 16 M^3 (small algebra)."""
    n, N, M, L = p.n, p.N, p.M, p.L
    return 32.0 * L * n ** 3 + 8.0 * L * n ** 2 + 16.0 * M * M * N + 16.0 * M * N * N + 8.0 * N ** 3 + 16.0 * M ** 3


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of the dominant exchange launch, from
# ncu captures of these workloads, with the note that says what was captured.
TRAFFIC = {
    ("c2", "ozaki_i8"): (2.412e9 + 0.820e9,
                         "DRAM read + write of the K launch (4096 x 25600 x 4096, the whole 3200-point chunk, wide "
                         "MMA issue) from an ncu capture of this workload; algorithmic bytes of that "
                         "launch: A slices 84 MB + B slices 524 MB + FP64 output 839 MB = 1.45e9"),
    ("c5", "ozaki_i8"): (39.0e9,
                         "DRAM read + write of the first panel's symmetric exchange GEMM (7059 pair rows x 25600 x "
                         "20100, the exchange symmetry's largest launch), scaled by the columns (points) from an ncu "
                         "capture of the same panel on a 384-point grid (4.68 GB for 7059 x 3072 x 20100; an upper "
                         "estimate, the A-slice reads do not grow with the columns); algorithmic bytes of the full "
                         "launch: A slices 0.71 GB + B slices 2.58 GB + FP64 output at both mirror positions "
                         "2.89 GB = 6.2e9"),
}


def measure_int8_peak(torch, dev):
    """cuBLASLt int8 GEMM throughput (TOP/s, 8192^3, best of 5), or None if unavailable."""
    try:
        a = torch.randint(-127, 127, (8192, 8192), dtype=torch.int8, device=dev)
        b = torch.randint(-127, 127, (8192, 8192), dtype=torch.int8, device=dev).t()
        torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 0.0
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch._int_mm(a, b)
            e.record()
            e.synchronize()
            best = max(best, 2 * 8192 ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
        return best
    except Exception:
        return None


def measure_fp64_peak(torch, dev):
    """cuBLAS DGEMM throughput (TFLOP/s) as the FP64 roofline denominator (best of 5, 8192^3)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * 8192 ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


def cpu_model():
    """The host CPU's model name (from /proc/cpuinfo), or None."""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


def oracle_setup(p):
    """Inputs of the C oracle for problem p and the name of its Gamma form: the dense antisymmetrised
    HTwo of the reference's MakeGamma where it fits in 8 GB of host memory (Ref = I, the determinant in
    Thouless form Z = C_vir C_occ^-1), else the spatial Cholesky vectors (Ref = the unitary whose
    first N columns are C, Z = 0: the same determinant)."""
    from oracle import phf_oracle as orc

    M, N = p.M, p.N
    kw = p.grid_kwargs()
    if 16.0 * M ** 4 <= 8e9:
        Z = p.C[N:] @ np.linalg.inv(p.C[:N])
        H2 = orc.dense_htwo_from_chol(p.B).astype(np.complex128)
        return dict(HOne=p.hone_ao(), HTwo=H2, Ref=np.eye(M), Z=Z, **kw), "dense HTwo MakeGamma", True
    Ref, Z = p.ref_and_z()
    return (dict(HOne=orc.mo_transform_1(p.hone_ao(), Ref), HTwo=None, Ref=Ref, Z=Z, Bs=p.B, **kw),
            "spatial Cholesky MakeGamma", False)


def sample_start(p):
    """First grid point of the CPU sample: the beta = 0 Lebedev point (overlaps near one), so that the
    sample's partial sums give a well-conditioned energy for the parity figure."""
    g = p.grid
    il = int(np.argmin(np.abs(np.asarray(g.rootb))))
    return il * g.ngrid[1] * g.npg


def cpu_sample(p, seconds_target=15.0, nthreads=0, setup=None, npts=None):
    """Time the C oracle (the reference's algorithm) on a bounded block of grid points.

    Dense form: the points run in parallel, one per thread; Cholesky form: one point at a time, its
    work split over the threads (a point costs ~45 core-seconds at n = 200).  The block starts at the
    beta = 0 point.  Returns (points/s, threads, description, (w0, w1), oracle sums of the block)."""
    from oracle import phf_oracle_c as corc

    okw, form, dense = setup if setup is not None else oracle_setup(p)
    nth = nthreads or os.cpu_count() or 1
    w0 = sample_start(p)
    avail = p.grid.npoints - w0

    def run(k):
        t0 = time.perf_counter()
        out = corc.buildhsg(omega_list=np.arange(w0, w0 + k), nthreads=nth, **okw)
        return time.perf_counter() - t0, out

    how = "points in parallel" if dense else "each point split over the threads"
    if npts is None:
        k0 = min(avail, nth if dense else 1)
        t1, out = run(k0)
        if t1 >= 0.5 * seconds_target:
            return k0 / t1, nth, f"{k0} of {p.grid.npoints} grid points ({form}, M={p.M}, {how}), {t1:.1f} s", \
                (w0, w0 + k0), out
        k = int(seconds_target / (t1 / k0))
        k = max(k0, (k // nth) * nth if dense else k)
        npts = min(avail, k)
    t2, out = run(npts)
    return npts / t2, nth, f"{npts} of {p.grid.npoints} grid points ({form}, M={p.M}, {how}), {t2:.1f} s", \
        (w0, w0 + npts), out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.config == "c4":  # the batch's rate on its first instance
        from phf_pcc_b200 import synth
        p = synth.batch_problems(args.batch, seed=1000)[0]
    else:
        p = problem_for(args.config, seed=0, ngrid=args.ngrid)
    nth = os.cpu_count() or 1
    setup = oracle_setup(p)
    # size the per-step sample once (about --cpu-seconds of CPU work), then time every step on it
    _, _, _, (w0, w1), _ = cpu_sample(p, seconds_target=args.cpu_seconds, nthreads=nth, setup=setup)
    vals = []
    desc = ""
    for i in range(args.warmup + args.steps):
        v, nth, desc, _, _ = cpu_sample(p, nthreads=nth, setup=setup, npts=w1 - w0)
        if i >= args.warmup:
            vals.append(v)
    v = statistics.median(vals)
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * p.grid.npoints / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "impl": "reference",
            "config": {"workload": workload_name(p), "points_per_step": p.grid.npoints},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nth, "cpu_model": cpu_model(), "kind": "port",
                             "sample": desc + "; rate scaled to the full grid (per-point work is independent)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line, default=_json_default), flush=True)
    return 0


def workload_name(p):
    g = p.grid
    return (f"n={p.n} M={p.M} N={p.N} L={p.L}, grid {g.ngrid[0]}x{g.ngrid[1]}x{g.npg} = {g.npoints} points "
            f"({'C2v' if g.npg == 4 else 'no PG'}), FP64-accurate E+grad")


def time_plan(torch, plan, C, stream, steps, warmup, flush, lib, sampler=None):
    """Device time (ms) per energy+gradient step (the plan replays its captured CUDA graph), then
    the per-class event profile from the same number of steps launched kernel by kernel."""
    from phf_pcc_b200.autograd import energy_and_gradient

    for _ in range(warmup):
        E, G = energy_and_gradient(C, plan)
    torch.cuda.synchronize()
    launches0 = lib.kernel_launches()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if sampler:
        sampler.__enter__()
    try:
        torch.cuda.synchronize()
        for i in range(steps):
            flush.zero_()                        # L2 flush between timed steps (not timed)
            ev[i][0].record(stream)
            E, G = energy_and_gradient(C, plan)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
    finally:
        if sampler:
            sampler.__exit__(None, None, None)
    launches = lib.kernel_launches() - launches0
    step_ms = sum(s.elapsed_time(e) for s, e in ev) / steps
    E, G = E.clone(), G.clone()  # the plan's output buffers are reused by later evaluations
    lib.profile_enable(True)
    for _ in range(steps):
        flush.zero_()
        energy_and_gradient(C, plan)
    torch.cuda.synchronize()
    prof = {c: lib.profile_read(c) for c in range(4)}
    lib.profile_enable(False)
    return step_ms, E, G, launches, prof


def block_energy_gradient(p, H, S, G, R, localg):
    """E = Re H / |Re S| and the LocalG gradient G[N:, :N] of (partial) sums, nci = 1."""
    e = H[0, 0].real / abs(S[0, 0].real)
    g = localg(G, R, S, e, [1.0 / np.sqrt(abs(S[0, 0].real))], [1.0], [1.0], 1)
    return e, g[p.N:, :p.N]


def oracle_parity(p, okw, block, ora, plan_kw_list):
    """The GPU forms on the CPU sample's block of grid points against the oracle's sums of the same
    block: max |difference| of Hmat, Smat, Gradmat, Rdmmat relative to the largest element of each,
    and |dE|, max |dG| of the block's energy and gradient."""
    from oracle import phf_oracle_c as corc
    from phf_pcc_b200 import api

    e_o, g_o = block_energy_gradient(p, *ora, lambda G, R, S, e, a, b, c, cc: corc.localg(G, R, S, e, a, b, c, cc, p.M,
                                                                                          1, 1, 1))
    res = {"points": list(block), "energy_of_block": e_o}
    for label, kw in plan_kw_list:
        with api.Plan(ref=okw["Ref"], point_range=block, **kw) as plan:
            out = plan.buildhsg(okw["Z"], check_hermitian=False)
        rel = max(float(np.abs(x - y).max()) / max(float(np.abs(y).max()), 1e-300) for x, y in zip(out, ora))
        e, g = block_energy_gradient(p, *out, api.localg)
        res[label] = {"abs_dE_vs_oracle": abs(e - e_o), "max_abs_dgrad_vs_oracle": float(np.abs(g - g_o).max()),
                      "max_rel_dHSGR_vs_oracle": rel, "meets_1e-8_Eh": abs(e - e_o) <= 1e-8,
                      "meets_1e-7_grad": float(np.abs(g - g_o).max()) <= 1e-7}
    return res


def run_ours(args):
    import torch

    from phf_pcc_b200 import _lib, api

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    p = problem_for(args.config, seed=1000 + rank, ngrid=args.ngrid)
    Ref, Z = p.ref_and_z()
    kw = api_kwargs(p)
    form = jk_form_of(p) if args.jk_form == "auto" else args.jk_form
    C = torch.from_numpy(p.C).to(dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(int(256e6) // 4, dtype=torch.float32, device=dev)  # > L2 (126 MB)
    slices = args.slices or 5

    tune = not args.no_autotune
    xs = {"auto": "auto", "on": True, "off": False}[args.exchange_symmetry]
    sym = sym_active(p, form, args.precision, args.exchange_symmetry)
    plan = api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision=args.precision, slices=args.slices, jk_form=form,
                    autotune=tune, exchange_panel=args.exchange_panel, exchange_symmetry=xs, **kw)
    clk = clock_sampler(local)
    step_ms, E, G, launches, prof = time_plan(torch, plan, C, stream, args.steps, args.warmup, flush, _lib, clk)
    t = torch.tensor([step_ms], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms = float(t.item())
    value = world * p.grid.npoints / (step_ms * 1e-3)
    chunk = plan.chunk
    chunks = -(-p.grid.npoints // chunk)
    plan.close()
    torch.cuda.empty_cache()

    # (measured right after the device timing, so that both run under the same thermal and power state;
    # the FP64 comparison runs below heat the GPU, which then clocks lower under the power cap)
    # end to end with host buffers: (1) the plan API an optimiser loop uses (Hamiltonian set up once;
    # per call: Z host -> device, the grid pass, Hmat/Smat/Gradmat/Rdmmat device -> host, and the
    # energy and LocalG gradient); (2) the one-shot drop-in call, which also rebuilds the
    # Hamiltonian-side plan every call.  Ref is the unitary whose first N columns are the benchmark's
    # determinant, so Z = 0 is the same state as `value`'s (the energies are reported side by side).
    e2e_vals, e2e_once = [], []
    h2d = d2h = h2d_once = 0
    e2e_energy = None
    e2e_steps = args.steps if args.e2e_steps is None else args.e2e_steps
    if e2e_steps > 0:
        z0 = np.zeros((p.M - p.N, p.N), dtype=np.complex128)
        planh = api.Plan(ref=Ref, h=p.h, B=p.B, precision=args.precision, slices=args.slices, jk_form=form,
                         autotune=tune, exchange_panel=args.exchange_panel, exchange_symmetry=xs, **kw)
        for i in range(1 + e2e_steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = planh.buildhsg(z0, check_hermitian=False)
            e2e_energy, _ = block_energy_gradient(p, *out, api.localg)
            t1 = time.perf_counter()
            if i > 0:
                e2e_vals.append(p.grid.npoints / (t1 - t0))
        planh.close()
        torch.cuda.empty_cache()
        # per call the plan uploads newMO and its conjugate (the AO vectors are formed on the device)
        h2d = 2 * p.M * p.N * 16
        d2h = sum(x.nbytes for x in out)
        for i in range(1 + min(e2e_steps, 2)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = api.buildhsg_chol(p.h, p.B, Ref, z0, precision=args.precision, check_hermitian=False, **kw)
            t1 = time.perf_counter()
            if i > 0:
                e2e_once.append(p.grid.npoints / (t1 - t0))
        torch.cuda.empty_cache()
        h2d_once = (p.h.nbytes + p.B.nbytes + Ref.nbytes + z0.nbytes + kw["r1"].nbytes + kw["r2"].nbytes +
                    kw["rpg"].nbytes + kw["weightsp"].nbytes + kw["weightpg"].nbytes)
    # the plain FP64 forms on the same problem (comparison and error reference): the exchange-matrix
    # form of the benchmark workload (stored for n <= 128, streamed above) with this library's FP64
    # GEMM kernels and with cuBLAS DGEMM for the exchange products; the speed-up is taken against the
    # faster of the two.  --fp64-all adds the stored-matrix form above n = 128 and the factorized form.
    fp64 = None
    ref64 = None
    if args.precision != "fp64" and not args.no_fp64:
        fp64 = {}
        forms = [("cublas_exchange", True, form), ("own_kernels", False, form)]
        if args.fp64_all:
            if form == "streamed":
                forms.append(("cublas_stored_eri", True, "eri"))
            forms.append(("factorized", False, "factorized"))
        for label, lib_gemm, jf in forms:
            plan64 = api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision="fp64", fp64_library_gemm=lib_gemm,
                              jk_form=jf, autotune=tune, exchange_panel=args.exchange_panel, exchange_symmetry=xs,
                              **kw)
            n64 = 1 if jf == "factorized" else max(1, min(args.steps, 3))
            ms64, E64, G64, _, prof64 = time_plan(torch, plan64, C, stream, n64, 1, flush, _lib)
            plan64.close()
            torch.cuda.empty_cache()
            if ref64 is None:
                ref64 = (E64, G64)
            dE = abs(E.item() - E64.item())
            dG = float((G - G64).abs().max().item())
            fp64[label] = {"value": p.grid.npoints / (ms64 * 1e-3), "ms_per_step": ms64, "energy": E64.item(),
                           "jk_form": jf, "exchange_ms_per_step": prof64[0][0] / n64,
                           "abs_dE_vs_fp64": dE, "max_abs_dgrad_vs_fp64": dG, "speedup": ms64 / step_ms,
                           "meets_1e-8_Eh": dE <= 1e-8}
        same = [k for k in fp64 if fp64[k]["jk_form"] == form]
        best = min(same, key=lambda k: fp64[k]["ms_per_step"])
        fp64["speedup_reference"] = {"form": best, "jk_form": form, "speedup": fp64[best]["speedup"],
                                  "meets_4x": fp64[best]["speedup"] >= 4.0,
                                  "note": "the faster FP64 GPU form of the same J/K algorithm"}

    # precision study: the other tensor-core precisions on the same problem, timed the same way,
    # with their energy and gradient errors against the FP64 form
    study = None
    if (args.study or args.config == "c3") and ref64 is not None:
        study = {args.precision: {"ms_per_step": step_ms, "value": p.grid.npoints / (step_ms * 1e-3),
                                  "abs_dE_vs_fp64": abs(E.item() - ref64[0].item()),
                                  "max_abs_dgrad_vs_fp64": float((G - ref64[1]).abs().max().item()),
                                  "jk_ms_per_step": prof[0][0] / args.steps}}
        for prec in ("ozaki_i8", "bf16x3", "tf32"):
            if prec == args.precision:
                continue
            plan_s = api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision=prec, slices=args.slices, jk_form=form,
                              exchange_panel=args.exchange_panel, exchange_symmetry=xs, **kw)
            ms_s, E_s, G_s, _, prof_s = time_plan(torch, plan_s, C, stream, max(1, min(args.steps, 3)), 2, flush,
                                                  _lib)
            plan_s.close()
            torch.cuda.empty_cache()
            study[prec] = {"ms_per_step": ms_s, "value": p.grid.npoints / (ms_s * 1e-3),
                           "abs_dE_vs_fp64": abs(E_s.item() - ref64[0].item()),
                           "max_abs_dgrad_vs_fp64": float((G_s - ref64[1]).abs().max().item()),
                           "jk_ms_per_step": prof_s[0][0] / max(1, min(args.steps, 3))}
        for prec, r in study.items():
            r["meets_1e-8_Eh"] = r["abs_dE_vs_fp64"] <= 1e-8
            r["meets_1e-7_grad"] = r["max_abs_dgrad_vs_fp64"] <= 1e-7
            r["tc_tops"] = tc_ops_per_step(p, prec, slices, form, chunks, sym_active(p, form, prec, args.exchange_symmetry),
                                           args.exchange_panel) / (r["jk_ms_per_step"] * 1e-3) / 1e12

    e2e_val = statistics.median(e2e_vals) * world if e2e_vals else None
    e2e_once_val = statistics.median(e2e_once) * world if e2e_once else None

    if rank == 0:
        peaks = _peaks()
        jk_ms, jk_n = prof[0]
        all_ms = sum(v[0] for v in prof.values())
        alg = jk_flops_per_point(p, form, sym, args.precision)
        regen = jk_regen_flops(p, form, chunks, sym, args.exchange_panel)
        fp64_peak = measure_fp64_peak(torch, dev)
        if args.precision == "fp64":
            achieved = (alg * p.grid.npoints + regen) * args.steps / (jk_ms * 1e-3) / 1e12
            roof = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                    "frac": achieved / fp64_peak, "traffic": None,
                    "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
                    "kernel": "zgemm_kernel<true> (exchange GEMM)"}
        else:
            i8 = measure_int8_peak(torch, dev)
            bf16 = peaks.get("bf16_tflops")
            peak = 2.0 * bf16 if bf16 else i8
            if args.precision != "ozaki_i8":  # dense bf16 rate; TF32 runs at half of it
                peak = bf16 * (0.5 if args.precision == "tf32" else 1.0) if bf16 else None
            achieved = (tc_ops_per_step(p, args.precision, slices, form, chunks, sym, args.exchange_panel) * args.steps
                        / (jk_ms * 1e-3) / 1e12)
            unit = {"ozaki_i8": "TOP/s (int8)", "bf16x3": "TFLOP/s (bf16)", "tf32": "TFLOP/s (tf32)"}[args.precision]
            traffic = TRAFFIC.get((args.config, args.precision))
            roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": unit,
                    "frac": achieved / peak if peak else None,
                    "traffic": traffic[0] if traffic else None,
                    "traffic_note": traffic[1] if traffic else "no ncu capture of this workload's exchange launch",
                    "peak_source": (_peak_source(peaks, {"ozaki_i8": "2 x (dense int8 rate = 2 x bf16 on B200)",
                                                         "bf16x3": "1 x", "tf32": "0.5 x (dense TF32 rate)"}
                                                 [args.precision])
                                    if bf16 else "cuBLASLt int8 GEMM 8192^3 measured in this run"),
                    "int8_cublaslt_tops_measured": i8,
                    "frac_of_cublaslt_int8": achieved / i8 if i8 else None,
                    "bf16_tflops_measured": bf16,
                    "kernel": "ozaki_i8_gemm_kernel (tcgen05 kind::%s, exchange, exchange-row regeneration and "
                              "Coulomb GEMMs)" % {"ozaki_i8": "i8", "bf16x3": "f16 (bf16)", "tf32": "tf32"}[args.precision],
                    "fp64_equivalent_tflops": (alg * p.grid.npoints + regen) * args.steps
                                              / (jk_ms * 1e-3) / 1e12,
                    "fp64_dgemm_peak_tflops": fp64_peak}
        roof.update({"jk_form": form, "jk_launches": jk_n, "jk_ms_per_step": jk_ms / args.steps,
                     "jk_share_of_device_time": jk_ms / all_ms if all_ms else None,
                     "device_ms_by_class": {k: v[0] / args.steps for k, v in
                                            zip(("jk", "other_gemm", "overlap_inverse", "memory"), prof.values())},
                     "exchange_symmetry": sym,
                     "alg_flops_per_point": alg, "regen_flops_per_step": regen,
                     "quoted_flops_per_point": quoted_flops_per_point(p)})
        cpu = None
        parity = None
        if not args.no_cpu:
            setup = oracle_setup(p)
            v, nth, desc, block, ora = cpu_sample(p, seconds_target=args.cpu_seconds, setup=setup)
            cpu = {"value": v, "unit": UNIT, "cores": nth, "cpu_model": cpu_model(), "kind": "port",
                   "sample": desc + "; rate scaled to the full grid (per-point work is independent)"}
            pk = dict(h=p.h, B=p.B, **kw)
            xk = dict(exchange_panel=args.exchange_panel, exchange_symmetry=xs)
            plist = [(args.precision, dict(pk, precision=args.precision, slices=args.slices, jk_form=form, **xk))]
            if args.precision != "fp64":
                plist.append(("fp64_cublas_exchange", dict(pk, precision="fp64", jk_form=form, fp64_library_gemm=True,
                                                           **xk)))
            parity = oracle_parity(p, setup[0], block, ora, plist)
            parity["oracle"] = setup[1]
            del setup
        dtype = {"fp64": "f64", "ozaki_i8": f"int8 x{slices} slices (FP64-accurate emulation) + f64",
                 "bf16x3": "bf16 hi+lo x3 products, f32 accumulation + f64",
                 "tf32": "tf32, f32 accumulation + f64"}[args.precision]
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded h, B_L, determinant)",
                "config": {"workload": workload_name(p), "precision": args.precision, "jk_form": form,
                           "exchange_symmetry": sym,
                           "points_per_step": p.grid.npoints, "chunk": chunk, "autotune": tune,
                           "l2": "flushed (256 MB write) between timed steps",
                           "parallelism": f"{world} independent instance(s), one per GPU"},
                "energy": float(E.item()), "fp64_gpu": fp64, "precision_study": study,
                "oracle_parity": parity, "roofline": roof, "cpu_baseline": cpu,
                "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "steps": e2e_steps, "energy": e2e_energy,
                        "abs_dE_vs_value_path": abs(e2e_energy - float(E.item())) if e2e_energy is not None else None,
                        "path": "phf_plan_buildhsg (C ABI, host Z in, host Hmat/Smat/Gradmat/Rdmmat out, energy and "
                                "LocalG gradient; plan created once before timing)",
                        "one_shot": {"value": e2e_once_val, "h2d_bytes_per_step": h2d_once,
                                     "d2h_bytes_per_step": d2h,
                                     "path": "phf_buildhsg_chol (plan set-up from h, B, Ref and the grid "
                                             "inside every call)"}},
                "gpu_launches": launches, "clocks": clk.summary()}
        print(json.dumps(line, default=_json_default), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batch(args):
    """Configuration 4: independent instances of uneven size evaluated together (phf_eval_batch:
    one CUDA graph over concurrent branches).  value = grid points of all instances / device time
    of one batch evaluation; the FP64 and split-BF16 forms are the same batch with FP64 and BF16x3
    plans."""
    import torch

    from phf_pcc_b200 import _lib, api, synth
    from phf_pcc_b200.autograd import _combine

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    probs = synth.batch_problems(args.batch, seed=1000 + rank)
    pts = sum(p.grid.npoints for p in probs)
    ws = 512 << 20

    def make(prec, tune=not args.no_autotune):
        return [api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision=prec, slices=args.slices, jk_form="eri",
                         workspace_bytes=ws, autotune=tune, **api_kwargs(p)) for p in probs]

    def energies(outs):
        res = []
        for p, (hs, yg, yr) in zip(probs, outs):
            E, G = _combine(hs, yg, yr, 1, 1, 1)
            res.append((float(E.item()), G))
        return res

    Cs = [torch.from_numpy(p.C).to(dev) for p in probs]
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(int(256e6) // 4, dtype=torch.float32, device=dev)

    def time_batch(plans, steps, warmup, sampler=None):
        outs = api.eval_batch(plans, Cs)  # captures (and tunes) the batch graph
        for _ in range(max(0, warmup - 1)):
            api.eval_batch(plans, Cs, outs)
        torch.cuda.synchronize()
        l0 = _lib.kernel_launches()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        if sampler:
            sampler.__enter__()
        try:
            for i in range(steps):
                flush.zero_()
                ev[i][0].record(stream)
                api.eval_batch(plans, Cs, outs)
                ev[i][1].record(stream)
            torch.cuda.synchronize()
        finally:
            if sampler:
                sampler.__exit__(None, None, None)
        launches = _lib.kernel_launches() - l0
        return sum(a.elapsed_time(b) for a, b in ev) / steps, outs, launches

    plans = make(args.precision)
    clk = clock_sampler(local)
    t_tune = time.perf_counter()
    tuned0 = int(_lib.load().phf_tuned_shapes())
    api.eval_batch(plans, Cs)  # first call: tunes the plans' GEMM shapes (autotune) and captures the graph
    torch.cuda.synchronize()
    t_tune = time.perf_counter() - t_tune
    tuned = int(_lib.load().phf_tuned_shapes()) - tuned0
    step_ms, outs, launches = time_batch(plans, args.steps, args.warmup, clk)
    # per-class device time, kernel by kernel
    _lib.profile_enable(True)
    api.eval_batch(plans, Cs, outs)
    torch.cuda.synchronize()
    prof = {c: _lib.profile_read(c) for c in range(4)}
    _lib.profile_enable(False)
    res = energies(outs)
    branches = int(_lib.load().phf_batch_branches())
    # end to end: determinants host -> device, the batch, all accumulators device -> host
    host_C = [c.cpu().pin_memory() for c in Cs]
    host_out = [tuple(t.cpu().pin_memory() for t in o) for o in outs]
    e2e = []
    for i in range(1 + (args.steps if args.e2e_steps is None else args.e2e_steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for hc, dc in zip(host_C, Cs):
            dc.copy_(hc, non_blocking=True)
        api.eval_batch(plans, Cs, outs)
        for ho, do in zip(host_out, outs):
            for a, b in zip(ho, do):
                a.copy_(b, non_blocking=True)
        torch.cuda.synchronize()
        if i > 0:
            e2e.append(pts / (time.perf_counter() - t0))
    h2d = sum(c.numel() * 16 for c in Cs)
    d2h = sum(sum(t.numel() * 16 for t in o) for o in outs)
    for pl in plans:
        pl.close()
    torch.cuda.empty_cache()
    fp64 = None
    ref64 = None
    if args.precision != "fp64" and not args.no_fp64:
        plans64 = make("fp64")
        ms64, outs64, _ = time_batch(plans64, max(1, min(args.steps, 3)), 1)
        res64 = energies(outs64)
        for pl in plans64:
            pl.close()
        torch.cuda.empty_cache()
        dE = max(abs(a[0] - b[0]) for a, b in zip(res, res64))
        dG = max(float((a[1] - b[1]).abs().max().item()) for a, b in zip(res, res64))
        fp64 = {"own_kernels": {"value": pts / (ms64 * 1e-3), "ms_per_step": ms64, "speedup": ms64 / step_ms,
                                "max_abs_dE_vs_fp64": dE, "max_abs_dgrad_vs_fp64": dG, "meets_1e-8_Eh": dE <= 1e-8}}
        # the split-BF16 form of the same batch (three BF16 products, FP32 accumulation, FP64 segment sums)
        if args.precision != "bf16x3":
            plansb = make("bf16x3")
            msb, outsb, _ = time_batch(plansb, max(1, min(args.steps, 3)), 1)
            resb = energies(outsb)
            for pl in plansb:
                pl.close()
            torch.cuda.empty_cache()
            fp64["split_bf16"] = {
                "value": pts / (msb * 1e-3), "ms_per_step": msb, "speedup_vs_fp64": ms64 / msb,
                "max_abs_dE_vs_fp64": max(abs(a[0] - b[0]) for a, b in zip(resb, res64)),
                "max_rel_dE_vs_fp64": max(abs(a[0] - b[0]) / abs(b[0]) for a, b in zip(resb, res64)),
                "max_abs_dgrad_vs_fp64": max(float((a[1] - b[1]).abs().max().item()) for a, b in zip(resb, res64))}
    t = torch.tensor([step_ms], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms = float(t.item())
    if rank == 0:
        peaks = _peaks()
        jk_ms = prof[0][0]
        slices = args.slices or 5
        ops = sum(tc_ops_per_point(p, args.precision, slices) * p.grid.npoints for p in probs)
        bf16 = peaks.get("bf16_tflops")
        peak = 2.0 * bf16 if bf16 else None
        achieved = ops / (jk_ms * 1e-3) / 1e12 if args.precision != "fp64" else None
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TOP/s (int8)",
                "frac": (achieved / peak) if (achieved and peak) else None, "traffic": None,
                "peak_source": _peak_source(peaks, "2 x (dense int8 rate = 2 x bf16 on B200)"),
                "device_ms_by_class": {k: v[0] for k, v in zip(("jk", "other_gemm", "overlap_inverse", "memory"),
                                                               prof.values())},
                "kernel": "ozaki_i8_gemm_kernel (all instances' exchange and Coulomb GEMMs)"}
        cpu = None
        if not args.no_cpu:
            v, nth, desc, _, _ = cpu_sample(probs[0], seconds_target=args.cpu_seconds)
            cpu = {"value": v, "unit": UNIT, "cores": nth, "cpu_model": cpu_model(), "kind": "port",
                   "sample": f"instance 0: {desc}"}
        sizes = sorted({p.n for p in probs})
        line = {"metric": METRIC, "value": world * pts / (step_ms * 1e-3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else f"int8 x{slices} slices (FP64-accurate emulation) + f64",
                "data": "synthetic (seeded h, B_L, determinants per instance)",
                "config": {"workload": f"{len(probs)} independent instances, n in {sizes}, N = n/2, L = 4n, "
                                       f"grids 112 / 800 points alternating, {pts} points in all",
                           "precision": args.precision, "jk_form": "eri", "points_per_step": pts,
                           "batch_branches": branches, "autotune": not args.no_autotune,
                           "tuned_shapes": tuned, "tune_and_capture_s": t_tune,
                           "l2": "flushed (256 MB write) between timed steps",
                           "parallelism": f"{world} independent batch(es), one per GPU"},
                "max_abs_dE_vs_fp64": fp64["own_kernels"]["max_abs_dE_vs_fp64"] if fp64 else None,
                "fp64_gpu": fp64, "roofline": roof, "cpu_baseline": cpu,
                "e2e": {"value": statistics.median(e2e) * world if e2e else None, "unit": UNIT,
                        "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "path": "pinned host determinants -> device, phf_eval_batch, accumulators -> pinned host"},
                "gpu_launches": launches, "clocks": clk.summary()}
        print(json.dumps(line, default=_json_default), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


PCC_METRIC = "projected-CCSD grid kernel (PbarHbarOlap) grid-pts/s, FP64 on the GPU; vs host CPU"


def pcc_call_args(p):
    """PbarHbarOlap's inputs after its outputs, in the Fortran order (SUCCSD_Boson_cmplx/FPUCC.f90:14-17)."""
    M, o = p["HOne"].shape[0], p["NOcc"]
    return (p["HOne"], p["HTwo"], None, p["T1"], p["T2"], o, M // 2, M, p["ENuc"], p["QJ"], p["SP"], p["NPoints"],
            p["Npg"], len(p["fsp"]), len(p["fpg"]), p["ncik"], p["R1"], p["R2"], p["Rpg"], p["Rk"], p["Roota"],
            p["Rootb"], p["Rooty"], p["Weightsp"], p["Weightpg"], p["fsp"], p["fpg"], p["fk"], p["TrunODE"])


def pcc_workload(trunode=1):
    from phf_pcc_b200 import synth

    c = synth.PCC_CONFIG
    p = synth.make_pcc_problem(c["n"], c["N"], c["L"], ngrid=c["ngrid"], seed=0)
    p.pop("MO")
    p["TrunODE"] = trunode
    M, o = p["HOne"].shape[0], p["NOcc"]
    npts = p["NPoints"][0] * p["NPoints"][1] * p["Npg"]
    name = (f"projected CCSD grid kernel: n={c['n']} M={M} NOcc={o}, dense <pq||rs>, grid "
            f"{p['NPoints'][0]}x{p['NPoints'][1]}x{p['Npg']} = {npts} points, TrunODE {trunode}")
    return p, npts, name


def pcc_cpu_sample(p, seconds_target):
    """Time the numpy oracle of PbarHbarOlap (all host threads through BLAS) on a bounded block of grid
    points; returns (points/s, threads, description, (w0, w1), oracle sums of the block)."""
    from oracle import phf_pcc as pcc

    nth = os.cpu_count() or 1
    npts = p["NPoints"][0] * p["NPoints"][1] * p["Npg"]
    t0 = time.perf_counter()
    out = pcc.pbarhbarolap(**p, points=[0])
    t1 = time.perf_counter() - t0
    k = int(max(1, min(npts, seconds_target / max(t1, 1e-3))))
    t0 = time.perf_counter()
    out = pcc.pbarhbarolap(**p, points=list(range(k)))
    t2 = time.perf_counter() - t0
    return k / t2, nth, f"{k} of {npts} grid points (numpy oracle, BLAS threads = host cores), {t2:.1f} s", \
        (0, k), out


def run_pcc_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    p, npts, name = pcc_workload(args.trunode)
    _, _, _, (w0, w1), _ = pcc_cpu_sample(p, args.cpu_seconds)
    from oracle import phf_pcc as pcc

    vals = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        pcc.pbarhbarolap(**p, points=list(range(w0, w1)))
        if i >= args.warmup:
            vals.append((w1 - w0) / (time.perf_counter() - t0))
    v = statistics.median(vals)
    nth = os.cpu_count() or 1
    line = {"metric": PCC_METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * npts / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": name, "points_per_step": npts},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nth, "cpu_model": cpu_model(), "kind": "port",
                             "sample": f"{w1 - w0} of {npts} grid points per step (numpy oracle); rate scaled to "
                                       "the full grid"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line, default=_json_default), flush=True)
    return 0


def run_pcc(args):
    import torch

    from phf_pcc_b200 import _lib, api

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    p, npts, name = pcc_workload(args.trunode)
    cargs = pcc_call_args(p)
    lib = _lib.load()
    flush = torch.empty(int(256e6) // 4, dtype=torch.float32, device=dev)  # > L2 (126 MB)
    ms, fl = ctypes.c_double(), ctypes.c_double()
    for _ in range(args.warmup):
        out = api.pbarhbarolap(*cargs)
    torch.cuda.synchronize()
    dev_ms, wall, flops = [], [], 0.0
    launches0 = lib.phf_kernel_launches()
    clk = clock_sampler(local)
    clk.__enter__()
    try:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = api.pbarhbarolap(*cargs)       # host arrays in, host sums out (synchronous)
            wall.append(time.perf_counter() - t0)
            lib.phf_pbarhbarolap_stats(ctypes.byref(ms), ctypes.byref(fl))
            dev_ms.append(ms.value)
            flops = fl.value
    finally:
        clk.__exit__(None, None, None)
    launches = (lib.phf_kernel_launches() - launches0) // max(1, args.steps)
    t = torch.tensor([sum(dev_ms) / len(dev_ms), sum(wall) / len(wall)], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms, wall_s = float(t[0]), float(t[1])
    value = world * npts / (step_ms * 1e-3)
    if rank == 0:
        fp64_peak = measure_fp64_peak(torch, dev)
        achieved = flops / (step_ms * 1e-3) / 1e12
        h2d = sum(np.asarray(x).nbytes for x in cargs if isinstance(x, np.ndarray))
        d2h = 2 * 16 + sum(np.asarray(x).nbytes for x in (out[1], out[2], out[4], out[5]))
        roof = {"bound": "fp64 tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak, "traffic": None,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
                "kernel": "zgemm_kernel (all contractions of the pipeline, FP64 mma.sync m8n8k4)",
                "note": "achieved = FP64 flops the pipeline's GEMMs executed (8 m n k per complex product) / "
                        "device time of the whole pipeline (elementwise kernels and inverses included)",
                "gemm_flops_per_step": flops}
        cpu, parity = None, None
        if not args.no_cpu:
            v, nth, desc, (w0, w1), ora = pcc_cpu_sample(p, args.cpu_seconds)
            cpu = {"value": v, "unit": UNIT, "cores": nth, "cpu_model": cpu_model(), "kind": "port",
                   "sample": desc + "; rate scaled to the full grid (per-point work is independent)"}
            # the same block on the GPU: the first w1 gamma points of the first Lebedev point
            k = min(w1, p["NPoints"][1])
            if k < w1:
                from oracle import phf_pcc as pcc
                ora = pcc.pbarhbarolap(**p, points=list(range(k)))
            q = dict(p)
            q.update(R1=p["R1"][:1], R2=p["R2"][:k], NPoints=(1, k), Roota=p["Roota"][:1], Rootb=p["Rootb"][:1],
                     Rooty=p["Rooty"][:k], Weightsp=p["Weightsp"][:1, :k])
            got = api.pbarhbarolap(*pcc_call_args(q))
            rel = max(float(np.abs(np.asarray(g) - np.asarray(r)).max() / max(np.abs(np.asarray(r)).max(), 1e-300))
                      for g, r in zip(got, ora))
            e_g, e_o = got[3] / got[0], ora[3] / ora[0]
            parity = {"points": [0, k], "max_rel_diff_of_sums": rel, "energy_of_block": e_o.real,
                      "abs_dE_vs_oracle": abs(e_g - e_o), "oracle": "numpy restatement of PbarHbarOlap"}
        line = {"metric": PCC_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded h, B_L, amplitudes)",
                "config": {"workload": name, "points_per_step": npts,
                           "l2": "flushed (256 MB write) between timed steps",
                           "timing": "device time of the grid pipeline inside each call (CUDA events on its "
                                     "stream, inputs uploaded before the first event)",
                           "parallelism": f"{world} independent instance(s), one per GPU"},
                "energy_ratio": (out[3] / out[0]).real, "oracle_parity": parity, "roofline": roof,
                "cpu_baseline": cpu,
                "e2e": {"value": world * npts / wall_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h,
                        "path": "phf_pbarhbarolap through PUCC_X2-style api.pbarhbarolap: host arrays in (device "
                                "buffers allocated and filled inside the call), host sums out"},
                "gpu_launches": launches, "clocks": clk.summary()}
        print(json.dumps(line, default=_json_default), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", default="c5", choices=["c1", "c2", "c3", "c4", "c5", "pcc"])
    ap.add_argument("--batch", type=int, default=256, help="instances for --config c4")
    ap.add_argument("--precision", default="ozaki_i8", choices=["fp64", "ozaki_i8", "bf16x3", "tf32"])
    ap.add_argument("--study", action="store_true",
                    help="also run the other tensor-core precisions and report their errors against FP64 "
                         "(on by default for --config c3)")
    ap.add_argument("--slices", type=int, default=0, help="int8 slices per operand (0 = library default)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-form comparison run")
    ap.add_argument("--no-autotune", action="store_true", help="plans without the launch tuner")
    ap.add_argument("--narrow-mma", action="store_true",
                    help="int8 GEMMs with one MMA per slice pair instead of the wide issue (same results)")
    ap.add_argument("--jk-form", default="auto", choices=["auto", "eri", "streamed"],
                    help="J/K form (auto: stored exchange matrix up to n = 128, streamed above)")
    ap.add_argument("--fp64-all", action="store_true",
                    help="also time the stored-exchange-matrix FP64 form above n = 128 and the factorized FP64 form")
    ap.add_argument("--e2e-steps", type=int, default=None, help="end-to-end steps (default: --steps)")
    ap.add_argument("--ngrid", type=lambda t: [int(v) for v in t.split(",")], default=None,
                    help="Lebedev,gamma points replacing the configuration's grid (profiling on a smaller grid)")
    ap.add_argument("--exchange-symmetry", choices=("auto", "on", "off"), default="auto",
                    help="streamed form: run the exchange over index pairs with the symmetric and antisymmetric "
                         "density halves (auto: wherever the library offers it), or over the full rows (off)")
    ap.add_argument("--exchange-panel", type=int, default=0,
                    help="streamed form: spatial indices per exchange panel (0 = the plan's choice)")
    ap.add_argument("--trunode", type=int, default=1, choices=[1, 2, 3],
                    help="--config pcc: TrunODE of the grid kernel (3 adds the (T) energy at every point)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_pcc_reference(args) if args.config == "pcc" else run_reference(args)
    if args.config == "pcc":
        return run_pcc(args)
    if args.narrow_mma:
        from phf_pcc_b200 import _lib

        _lib.load().phf_int8_wide_mma(0)
    if args.config == "c4":
        return run_batch(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
