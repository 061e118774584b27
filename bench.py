"""Benchmark: Car-Parrinello steps per second of the WAVES hot path.

Workload: Si64 (2x2x2 supercell of cubic diamond Si, a=20.52 bohr, seeded
+-0.05 bohr displacements), Gamma point, 128 bands (64 super wave functions),
30/60 Ry, 64^3 FFT grid, NVE CP steps with dt=10 a.u. and m=1000 a.u., atoms
moving.  Synthetic setups, V_loc and DH (no dataset is involved).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--system NAME] [--no-mixed] [--no-precision] [--no-serving] ...

One JSON line is printed by rank 0.  `value` is whole-job steps/s with every
array resident in HBM (N independent replicas with --gpus N: the path does
not shard, one system per GPU); `e2e` is the same metric through the C ABI
with per-step host buffers (V(r), DH and positions uploaded from pinned host
memory, energies and forces read back).  --impl reference times the CPU
restatement of the reference (the reference itself cannot be compiled in this
image: no Fortran compiler, FFTW or LAPACK) on all host cores, its ZGEMMs on the
OpenBLAS that scipy bundles where the reference calls BLAS.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cp-paw_b200"))

METRIC = "CP steps/s Si64"
WORKLOAD = "Si64 Gamma 128 bands 30/60 Ry 64^3 grid, NVE CP (dt=10, m=1000), moving atoms"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(vals, world, device="cuda"):
    """Element-wise maximum of every rank's timings (ms) over all ranks: the
    job's time is that of its slowest replica.  One collective, taken by every
    rank in the same order."""
    if world == 1:
        return [float(v) for v in vals]
    import torch

    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(x) for x in t]


class ClockSampler:
    """SM clock and clock-event (throttle) reasons during the timed region:
    NVML read every 10 ms from a thread (read-only queries), else
    nvidia-smi every 200 ms."""

    NAMES = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
             ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
             ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
             ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, index: int):
        self.index = index
        self.samples = []  # (sm_mhz, max_mhz, [reasons])
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            import torch

            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:  # noqa: BLE001 (fall back to the index)
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.nvml = (nv, h)
            self.thread = threading.Thread(target=self._poll_nvml, daemon=True)
            self.thread.start()
            return self
        except Exception:  # noqa: BLE001
            self.nvml = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read_smi, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _poll_nvml(self):
        nv, h = self.nvml
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                rs = [n for n, c in self.NAMES if bits & getattr(nv, c, 0)]
                self.samples.append((float(sm), float(mx), rs))
            except Exception:  # noqa: BLE001
                break
            self.stop.wait(0.01)

    def _read_smi(self):
        for line in self.proc.stdout:
            s = [x.strip() for x in line.split(",")]
            if len(s) < 9 or not s[1].replace(".", "").isdigit():
                continue
            rs = [n for k, (n, _) in enumerate(self.NAMES) if s[5 + k].lower().startswith("active")]
            self.samples.append((float(s[1]), float(s[2]), rs))

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml:
            self.thread.join(timeout=2)
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:  # noqa: BLE001
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        import statistics

        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = sorted({r for _, _, rs in self.samples for r in rs})
        return {"sm_mhz": statistics.median(x[0] for x in self.samples), "sm_max_mhz": max(x[1] for x in self.samples),
                "reasons": reasons, "samples": len(self.samples),
                "source": "nvml (10 ms)" if self.nvml else "nvidia-smi (200 ms)"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "MEASURED_PEAKS.json"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def fp64_peak_tflops(torch):
    """FP64 tensor throughput measured here: cuBLAS DGEMM via torch.matmul
    (MEASURED_PEAKS.json has HBM and BF16 only)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) * 1e-3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def tf32_peak_tflops(torch):
    """TF32 tensor throughput measured here: cuBLAS SGEMM with TF32 allowed
    (torch.matmul float32, 8192^3), the denominator of the mixed path's
    tensor-core roofline (MEASURED_PEAKS.json has BF16 only)."""
    n = 8192
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    try:
        a = torch.randn(n, n, dtype=torch.float32, device="cuda")
        b = torch.randn(n, n, dtype=torch.float32, device="cuda")
        for _ in range(2):
            torch.matmul(a, b)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch.matmul(a, b)
            e.record()
            e.synchronize()
            best = min(best, s.elapsed_time(e) * 1e-3)
        del a, b
        torch.cuda.empty_cache()
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return 2.0 * n ** 3 / best / 1e12


def fft_roofline(t_ms, fft_bytes, peaks, peak_src):
    """HBM roofline of the V.psi transforms: one full-grid read and write per
    transform (two transforms per super wave function), over the phase time."""
    if not t_ms or t_ms <= 0:
        return None
    achieved = fft_bytes / (t_ms * 1e-3) / 1e9
    peak = peaks.get("hbm_gbs")
    return {"bound": "hbm", "kernels": "k_gtor_plane + k_zcol_v64 + k_rtog_plane", "achieved": round(achieved, 1),
            "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4) if peak else None,
            "peak_source": f"{peak_src} hbm_gbs (of measured)" if peak_src != "fallback" else "fallback",
            "bytes_per_step": fft_bytes, "traffic": None}


def load_ncu_traffic():
    """Per-launch DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum,
    bytes) of the dominant FP64 kernels, from the committed ncu summaries: a
    line `traffic_bytes_per_launch: <phase> <bytes>` in profiles/*.md."""
    out = {}
    d = os.path.join(ROOT, "profiles")
    try:
        names = sorted(os.listdir(d))
    except OSError:
        return out
    for n in names:
        if not n.endswith(".md"):
            continue
        with open(os.path.join(d, n)) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    parts = line.split()
                    if len(parts) == 3:
                        out[parts[1]] = float(parts[2])
    return out


def make_inputs(name="Si64"):
    from cuwaves import systems

    return systems.build_inputs(systems.named_system(name))


def flops_model(inp):
    """Algorithmic work per step (real flops / bytes), as used for the roofline."""
    ngl, nbh, npro = inp["ngl"], inp["nbh"], None
    npro = sum(sum(2 * l + 1 for l in inp["lox"][s - 1]) for s in inp["isp"].tolist())
    nr = inp["grid"][0] * inp["grid"][1] * inp["grid"][2]
    contr = 8.0 * ngl * npro * nbh
    return {
        "addpro_propagate_flops": 2 * contr,      # H and O back-projection (one fused kernel)
        "projections_flops": 2 * contr,           # <p|psibar>, <p|O psi0> at R(+) (one fused kernel)
        "forces_flops": contr,
        "gram_flops": 6 * 8.0 * ngl * nbh * nbh,
        "fft_bytes": 2 * nbh * 2 * nr * 16.0,     # two transforms per band, grid read+write
        "npro": npro,
    }


def phase_pass(w, steps):
    """Device time per phase of the step, from CUDA events at the phase
    boundaries, over untimed steps after the timed region (the events need
    launches from the host, so these steps are not replayed as graphs)."""
    w.set_timing(True)
    for _ in range(max(3, min(steps, 10))):
        w.cp_step(move_atoms=True)
    phases, _, nsteps = w.get_timing()
    w.set_timing(False)
    return phases, nsteps


def run_cuda(args, rank, world, local):
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    import cuwaves

    inp = make_inputs(args.system)
    w = cuwaves.open_waves(inp, precision=cuwaves.CUW_PREC_FP64).setup().initialize()
    tuned = w.autotune() if not args.no_autotune else None
    stream = torch.cuda.ExternalStream(w.stream())
    for _ in range(args.warmup):
        w.cp_step(move_atoms=True)
    # ---- timed region, device-resident ---------------------------------------
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    _, l0, _ = w.get_timing()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            out, f = w.cp_step(move_atoms=True)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ms = ev0.elapsed_time(ev1)
    _, l1, _ = w.get_timing()
    launches = l1 - l0
    graphs = w.graph_stats()
    phases, nsteps = phase_pass(w, args.steps)
    # ---- e2e: per-step host inputs from pinned memory -------------------------
    v_h = torch.from_numpy(np.ascontiguousarray(inp["v"])).pin_memory()
    dh_h = torch.from_numpy(np.ascontiguousarray(inp["dh"]).view(np.float64)).pin_memory()
    r_h = torch.from_numpy(np.ascontiguousarray(inp["r0"])).pin_memory()
    out_h = torch.zeros(8, dtype=torch.float64).pin_memory()
    f_h = torch.zeros((inp["nat"], 3), dtype=torch.float64).pin_memory()
    m_h = torch.from_numpy(np.ascontiguousarray(inp["masses"])).pin_memory()
    import ctypes as C

    D = C.POINTER(C.c_double)
    fns = w._f
    lmnxx = inp["dh"].shape[-1]
    torch.cuda.synchronize()
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    for _ in range(args.steps):
        fns["set_potential"](w.h, C.cast(v_h.data_ptr(), D))
        fns["set_dh"](w.h, lmnxx, C.cast(dh_h.data_ptr(), D))
        fns["set_atoms"](w.h, C.cast(r_h.data_ptr(), D), None)
        rc = fns["cp_step"](w.h, 1, C.cast(m_h.data_ptr(), D), 200, 1e-8, C.cast(out_h.data_ptr(), D),
                            C.cast(f_h.data_ptr(), D))
        if rc:
            w._chk(rc, "TIMESTEP")
    ev3.record(stream)
    ev3.synchronize()
    ms_e2e = ev2.elapsed_time(ev3)
    h2d = v_h.numel() * 8 + dh_h.numel() * 8 + r_h.numel() * 8 + m_h.numel() * 8
    d2h = out_h.numel() * 8 // 8 * 5 + f_h.numel() * 8
    ms, ms_e2e = max_over_ranks([ms, ms_e2e], world)
    # roofline of the dominant phase
    fm = flops_model(inp)
    peaks, peak_src = measured_peaks()
    result = {"phases_ms_per_step": {k: v / max(1, nsteps) for k, v in phases.items()},
              "launches": launches, "ms": ms, "ms_e2e": ms_e2e, "h2d": h2d, "d2h": d2h,
              "clocks": clk.summary(), "fm": fm, "iters_last": float(out[4]), "etot_last": float(out[0]),
              "ortho": w.ortho_stats(), "graphs": {"held": graphs[0], "replays": graphs[1]}, "autotune": tuned}
    if rank == 0:
        p64 = fp64_peak_tflops(torch)
        result["fp64_peak"] = p64
        result["peak_src"] = peak_src
    w.close()
    return result


def run_mixed(args, local):
    """The same workload on the mixed-precision path (FP32 FFTs, tf32x3
    tensor-core contractions, FP64 constraint solve and sums): device-timed
    steps/s and phase split, and the largest deviation of energy and forces
    from the FP64 path over the first steps from an identical state.  (CP
    trajectories from random wave functions separate chaotically over tens of
    steps, so later differences measure the dynamics, not the precision.)"""
    import numpy as np
    import torch
    import cuwaves

    inp = make_inputs(args.system)
    ref = cuwaves.open_waves(inp, precision=cuwaves.CUW_PREC_FP64).setup().initialize()
    w = cuwaves.open_waves(inp, precision=cuwaves.CUW_PREC_MIXED).setup()
    copy_state(ref, w)
    tuned = w.autotune() if not args.no_autotune else None
    de = df = 0.0
    nacc = 5
    for _ in range(nacc):
        o_r, f_r = ref.cp_step(move_atoms=True)
        o_m, f_m = w.cp_step(move_atoms=True)
        de = max(de, abs(float(o_m[0]) - float(o_r[0])) / inp["nat"])
        df = max(df, float(np.abs(f_m - f_r).max()))
    ref.close()
    stream = torch.cuda.ExternalStream(w.stream())
    for _ in range(args.warmup):
        w.cp_step(move_atoms=True)
    torch.cuda.synchronize()
    _, l0, _ = w.get_timing()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        w.cp_step(move_atoms=True)
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    _, l1, _ = w.get_timing()
    phases, nsteps = phase_pass(w, args.steps)
    w.close()
    ph = {k: v / max(1, nsteps) for k, v in phases.items()}
    # tensor-core roofline of the dominant tcgen05 phase: the split products
    # issue three TF32 MMAs (hi*hi + hi*lo + lo*hi) per product of the model
    fm = flops_model(inp)
    cand = {"addpro_propagate": (ph.get("addpro_propagate", 0.0), fm["addpro_propagate_flops"], "k_tc_addpro<FUSED>"),
            "projections": (ph.get("projections", 0.0), fm["projections_flops"], "k_tc_proj")}
    name = max(cand, key=lambda k: cand[k][0])
    t_ms, flops, kern = cand[name]
    p32 = tf32_peak_tflops(torch)
    tensor = 3.0 * flops / (t_ms * 1e-3) / 1e12 if t_ms > 0 else None
    peaks, peak_src = measured_peaks()
    return {"value": round(args.steps / (ms * 1e-3), 4), "unit": "steps/s", "ms_per_step": round(ms / args.steps, 4),
            "dtype": "f32 FFT / tf32x3 tensor cores / f64 solve and sums",
            f"max_dE_per_atom_vs_fp64_{nacc}_steps": de, f"max_dF_vs_fp64_{nacc}_steps": df,
            "gpu_launches": l1 - l0, "autotune": tuned,
            "roofline": {"bound": "tensor", "kernel": kern, "phase": name,
                         "achieved": round(tensor, 3) if tensor else None, "peak": round(p32, 3), "unit": "TFLOP/s",
                         "frac": round(tensor / p32, 4) if tensor else None,
                         "peak_source": "TF32 cuBLAS (torch.matmul float32 8192^3, TF32 allowed) measured in this run",
                         "tensor_flops_per_step": 3.0 * flops, "model_flops_per_step": flops,
                         "model_tflops": round(flops / (t_ms * 1e-3) / 1e12, 3) if t_ms > 0 else None,
                         "traffic": load_ncu_traffic().get("tc_" + name)},
            "roofline_fft": fft_roofline(ph.get("fft_vpsi"), fm["fft_bytes"] / 2, peaks, peak_src),
            "phase_ms_per_step": {k: round(v, 4) for k, v in ph.items()}}


def copy_state(src, dst):
    """PSI0, PSIM, PROJ and RLAM0 of one handle into another."""
    import cuwaves

    for which in (cuwaves.CUW_PSI0, cuwaves.CUW_PSIM):
        dst.upload_psi(which, src.download_psi(which))
    dst.set_proj(src.get_proj())
    dst.set_rlam0(src.get_rlam0())


AU_TIME_PS = 2.4188843265857e-5  # one atomic unit of time in ps


def run_precision(args):
    """Errors of the mixed path against the FP64 path, per system (Si64 at
    64^3, 30/60 Ry, and 32 H2O at 72^3, 40/80 Ry):
    - energy per atom and forces over the first 5 CP steps (moving nuclei) from
      one state;
    - orthonormality residual max|<psi_i|O|psi_j> - delta_ij| of PSI0 after every
      step, formed in FP64 with projections computed afresh (the test of
      WAVES$ORTHOGONALIZE, src/paw_waves2.f90:421-460, whose bound is 1e-4);
    - NVE drift: the wave functions are first relaxed with friction (ANNEE)
      at fixed nuclei, then both paths run `drift_steps` frictionless CP steps
      with moving nuclei from rest; the conserved energy is assembled as the
      reference's 'CONSTANT ENERGY' (src/paw_driver.f90:481-535): total energy
      + wave-function (fictitious) kinetic energy + ionic kinetic energy.  The
      drift is the least-squares slope of that energy per atom in Ha/atom/ps,
      with its largest excursion from the start."""
    import numpy as np
    import cuwaves

    out = {}
    for name in args.precision_systems.split(","):
        inp = make_inputs(name)
        nat = inp["nat"]
        ref = cuwaves.open_waves(inp, precision=cuwaves.CUW_PREC_FP64).setup().initialize()
        mix = cuwaves.open_waves(inp, precision=cuwaves.CUW_PREC_MIXED).setup()
        copy_state(ref, mix)
        de = df = 0.0
        ores = {"fp64": 0.0, "mixed": 0.0}
        for _ in range(5):
            o_r, f_r = ref.cp_step(move_atoms=True)
            o_m, f_m = mix.cp_step(move_atoms=True)
            de = max(de, abs(float(o_m[0]) - float(o_r[0])) / nat)
            df = max(df, float(np.abs(f_m - f_r).max()))
            ores["fp64"] = max(ores["fp64"], ref.overlap_check()[1])
            ores["mixed"] = max(ores["mixed"], mix.overlap_check()[1])
        # relax the wave functions at fixed nuclei (damped CP), FP64
        ref.reset_atoms(inp["r0"])
        ref.set_dynamics(inp["delt"], args.quench_friction)
        for _ in range(args.quench_steps):
            ref.cp_step(move_atoms=False)
        ref.set_dynamics(inp["delt"], 0.0)
        ref.reset_atoms(inp["r0"])
        mix.set_dynamics(inp["delt"], 0.0)
        mix.reset_atoms(inp["r0"])
        copy_state(ref, mix)
        drift = {}
        for tag, w in (("fp64", ref), ("mixed", mix)):
            econs = []
            worst = 0.0
            for k in range(args.drift_steps):
                o, _ = w.cp_step(move_atoms=True, want_force=False)
                econs.append(float(o[0] + o[2] + o[3]))
                if k % 50 == 49:
                    worst = max(worst, w.overlap_check()[1])
            e = np.asarray(econs) / nat
            t_ps = np.arange(len(e)) * inp["delt"] * AU_TIME_PS
            slope = float(np.polyfit(t_ps, e, 1)[0])
            drift[tag] = {"slope_ha_per_atom_per_ps": slope,
                          "max_excursion_ha_per_atom": float(np.abs(e - e[0]).max()),
                          "orthonormality_residual_max": worst,
                          "econs_start_ha": float(econs[0]), "econs_end_ha": float(econs[-1])}
        ref.close()
        mix.close()
        out[name] = {
            "grid": "x".join(map(str, inp["grid"])), "bands": inp["nb"], "atoms": nat,
            "max_dE_per_atom_vs_fp64_5_steps": de, "max_dF_vs_fp64_5_steps": df,
            "orthonormality_residual_5_steps": ores,
            "nve": {"steps": args.drift_steps, "dt_au": inp["delt"], "quench_steps": args.quench_steps,
                    "quench_friction": args.quench_friction, **drift},
        }
    return out


def _serve_stream(pool, kinds, rate, nreq, workers, budget_gb, seed):
    """One seeded Poisson stream through a fresh server; per-request latency is
    measured by the server from submission to completion."""
    import numpy as np
    import cuwaves
    from cuwaves.serve import Server

    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=nreq))
    plan = []
    for _ in range(nreq):
        kind, n = kinds[int(rng.integers(0, len(kinds)))]
        plan.append(((kind, n, int(rng.integers(1, 3))), 0 if rng.random() < 0.5 else 20))
    srv = Server(hbm_budget=budget_gb << 30, workers=workers)
    ids = []
    t0 = time.perf_counter()
    for (key, nsteps), ta in zip(plan, arrivals):
        dt = ta - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        ids.append((srv.submit(pool[key], nsteps=nsteps, move_atoms=nsteps > 0, precision=cuwaves.CUW_PREC_MIXED,
                               borrow=True), nsteps))
    srv.wait_all()
    st = srv.stats()
    lat = {0: [], 20: []}
    failed = 0
    for rid, nsteps in ids:
        r = srv.poll(rid)
        if r[0]:
            failed += 1
        else:
            lat[nsteps].append(r[3])
    srv.close()
    pct = lambda v, q: round(float(np.percentile(v, q)), 3) if v else None  # noqa: E731
    return {"requests": nreq, "offered_rate_per_s": round(rate, 3), "completed": int(st["completed"]),
            "failed": failed, "solves_per_s": round(st["throughput_per_s"], 3), "p50_ms": round(st["p50_ms"], 3),
            "p99_ms": round(st["p99_ms"], 3), "max_ms": round(st["max_ms"], 3),
            "single_point_p50_ms": pct(lat[0], 50), "single_point_p99_ms": pct(lat[0], 99),
            "cp20_p50_ms": pct(lat[20], 50), "cp20_p99_ms": pct(lat[20], 99),
            "peak_admitted_gb": round(st["peak_bytes"] / 2 ** 30, 3), "mean_admitted_sets": round(st["mean_admitted"], 2)}


def run_serving(args):
    """Serving workload: seeded Poisson streams of single-point solves and
    20-step CP runs of perturbed bulk Si_n and water clusters, submitted in
    real time to the device-resident server (HBM-budget admission, continuous
    batching).  The stream at the nominal rate (200 requests/s) overloads one
    GPU, so it measures the capacity (solves/s); a second stream offered at
    50% of that capacity gives the latency at sustained throughput."""
    import cuwaves
    from cuwaves import systems
    from cuwaves.serve import Server

    kinds = [("Si", n) for n in sorted(systems.SERVING_SI)] + [("W", n) for n in systems.SERVING_WATER]
    pool = {}
    for kind, n in kinds:
        for seed in (1, 2):
            inp = systems.build_inputs(systems.serving_system(kind, n, seed))
            inp["annee"] = 0.05  # friction on the wave functions: a damped (relaxing) run
            pool[(kind, n, seed)] = inp
    # warm-up outside the streams: one request of every kind
    srv = Server(hbm_budget=args.serve_budget_gb << 30, workers=args.serve_workers)
    for kind, n in kinds:
        srv.submit(pool[(kind, n, 1)], nsteps=1, move_atoms=True, precision=cuwaves.CUW_PREC_MIXED, borrow=True)
    srv.wait_all()
    srv.close()
    peak = _serve_stream(pool, kinds, args.serve_rate, args.serve_requests, args.serve_workers, args.serve_budget_gb, 7)
    cap = max(peak["solves_per_s"], 0.1)
    rate = 0.5 * cap
    nreq = max(10, min(args.serve_requests, int(rate * args.serve_seconds)))
    sustained = _serve_stream(pool, kinds, rate, nreq, args.serve_workers, args.serve_budget_gb, 8)
    return {"at_nominal_rate": peak, "sustained_at_50pct_capacity": sustained,
            "p50_ms": sustained["p50_ms"], "p99_ms": sustained["p99_ms"], "solves_per_s": peak["solves_per_s"],
            "hbm_budget_gb": args.serve_budget_gb, "workers": args.serve_workers, "precision": "mixed",
            "workload": "Poisson streams, 50% single points (energy+forces) and 50% 20-step damped CP runs with "
                        "moving nuclei; Si8/16/32/64/128 (+-0.05 bohr, 30 Ry) and (H2O)1/2/4/8/16 clusters (40 Ry, "
                        "8 bohr vacuum), two seeds each; latency from submission to completion; solves_per_s is the "
                        "capacity measured under the nominal 200 requests/s stream, p50/p99 are at 50% of it"}


def run_batched(args):
    """Batched workloads, mixed precision (and FP64 for the Si64 cells), every
    batch advanced by one CUDA graph launch per two CP steps of all its sets
    (cuwaves_batch_step: the sets' kernels run concurrently on the device, the
    host issues one launch and reads the energies back per call):
    (1) `batched_si64` independent Si64 cells (different seeded displacements);
    (2) 64 independent small systems of uneven size: bulk Si2-Si16 cells and
        Si2 / H2O molecules in 20-bohr boxes, 4-32 bands, grids 18^3 to 36^3
        (the smallest holding each wave-function sphere), 30 Ry;
        beside the same systems stepped one at a time.
    Aggregate CP steps/s between synchronised start and end of the timed
    batch calls (after warm-up calls that capture the graphs)."""
    import cuwaves
    from cuwaves import systems

    def timed_batch(ws, calls):
        for w in ws:
            w.cp_step(move_atoms=True)  # eigenbasis and Lagrange history
        batch = cuwaves.Batch(ws)
        for _ in range(max(2, args.warmup)):
            batch.step(move_atoms=True)
        t0 = time.perf_counter()
        for _ in range(calls):
            batch.step(move_atoms=True)
        dt = time.perf_counter() - t0
        batch.close()
        return len(ws) * 2 * calls / dt

    import torch

    nsm = torch.cuda.get_device_properties(0).multi_processor_count

    def share(nsets):
        # SMs each set's launch shapes assume (CUW_OPT_SM_SHARE): the sets of
        # a batch share the device, so each launches fewer split-K blocks; in
        # measurements, max(16, SMs / sets) did best for 8 Si64 cells (18) and
        # for the 64 small systems (16), 3 % and 16 % above the whole device
        return max(16, nsm // max(1, nsets))

    res = {}
    calls = max(1, args.steps // 2)
    for prec, tag in ((cuwaves.CUW_PREC_MIXED, "mixed"), (cuwaves.CUW_PREC_FP64, "fp64")):
        ws = []
        for i in range(args.batched_si64):
            inp = systems.build_inputs(systems.si_cell(2, a=10.26, disp=0.05, seed=1 + i, grid=(64, 64, 64),
                                                       name="Si64"))
            ws.append(cuwaves.open_waves(inp, precision=prec).setup().initialize())
            ws[-1].set_option(cuwaves.CUW_OPT_SM_SHARE, share(args.batched_si64))
            if not args.no_autotune:
                ws[-1].autotune()
        res[tag] = timed_batch(ws, calls)
        for w in ws:
            w.close()
    inps = [systems.build_inputs(s) for s in systems.config_batch_mix(64)]
    ws = [cuwaves.open_waves(inp, precision=cuwaves.CUW_PREC_MIXED).setup().initialize() for inp in inps]
    for w in ws:
        w.set_option(cuwaves.CUW_OPT_SM_SHARE, share(len(ws)))
    tiles = []
    if not args.no_autotune:
        # launch shapes and contraction tile family per shape (the table keeps
        # one choice per shape, so repeated shapes are not timed again)
        tiles = [w.autotune()["dmma_tiles"] for w in ws]
    small = timed_batch(ws, args.batched_steps // 2)
    # the same sets one at a time (each step a graph replay of its own), each
    # with the whole device again
    for w in ws:
        w.set_option(cuwaves.CUW_OPT_SM_SHARE, 0)
        w.cp_step(move_atoms=True)
    t0 = time.perf_counter()
    nsteps = max(2, args.batched_steps // 2)
    for w in ws:
        for _ in range(nsteps):
            w.cp_step(move_atoms=True)
    alone = len(ws) * nsteps / (time.perf_counter() - t0)
    for w in ws:
        w.close()
    return {"value": round(res["mixed"], 2), "unit": "CP steps/s (all Si64 cells)", "precision": "mixed",
            "si64_cells": args.batched_si64, "fp64_same_batch": round(res["fp64"], 2),
            "sm_share_per_set": share(args.batched_si64),
            "timing": "one CUDA graph launch per two CP steps of every set (cuwaves_batch_step), synchronised; "
                      "wall clock over the timed calls after graph capture and warm-up",
            "small_systems": {"value": round(small, 2), "unit": "CP steps/s (all systems)", "systems": len(ws),
                              "one_at_a_time_value": round(alone, 2), "precision": "mixed",
                              "dmma_tile_sets": int(sum(tiles)) if tiles else None,
                              "sm_share_per_set": share(len(ws)),
                              "sizes": "Si2-Si16 bulk (4-32 bands, 18^3 and 18x18x36 grids), Si2 and H2O molecules "
                                       "in 20-bohr boxes (4 bands, 36^3), 30 Ry"}}


def emit_cuda(args, res, world):
    ph = res["phases_ms_per_step"]
    fm = res["fm"]
    ms_step = res["ms"] / args.steps
    value = world * args.steps / (res["ms"] * 1e-3)
    e2e = world * args.steps / (res["ms_e2e"] * 1e-3)
    # dominant kernel: the larger of the two fused FP64 contractions
    cand = {"addpro_propagate": (ph["addpro_propagate"], fm["addpro_propagate_flops"]),
            "projections": (ph["projections"], fm["projections_flops"])}
    name = max(cand, key=lambda k: cand[k][0])
    t_ms, flops = cand[name]
    achieved = flops / (t_ms * 1e-3) / 1e12 if t_ms > 0 else None
    peak = res.get("fp64_peak")
    traffic = load_ncu_traffic().get(name)
    cpu = cpu_baseline(args) if not args.no_cpu else None
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Si64 cell, synthetic setups, V_loc and DH)",
        "config": {"workload": WORKLOAD, "system": args.system, "precision": "fp64",
                   "parallelism": f"replicas{world}", "bands": 128, "grid": "64^3",
                   "l2": "working set (~0.3 GB: psi0/psim/hpsi/opsi 24 MB each, FFT grid, EIGR) exceeds the 126 MB L2"},
        "e2e": {"value": round(e2e, 4), "unit": "steps/s", "h2d_bytes_per_step": res["h2d"],
                "d2h_bytes_per_step": res["d2h"]},
        "gpu_launches": res["launches"],
        "roofline": {"bound": "tensor", "kernel": f"k_{'addpro<FUSED>' if name == 'addpro_propagate' else 'proj<DUAL>'}",
                     "achieved": round(achieved, 3) if achieved else None, "peak": round(peak, 3) if peak else None,
                     "unit": "TFLOP/s", "frac": round(achieved / peak, 4) if achieved and peak else None,
                     "peak_source": "FP64 cuBLAS DGEMM (torch.matmul float64 8192^3) measured in this run; "
                                    "MEASURED_PEAKS.json has no FP64 figure",
                     "traffic": traffic, "flops_per_launch": flops},
        "roofline_fft": fft_roofline(ph.get("fft_vpsi"), fm["fft_bytes"], *measured_peaks()),
        "phase_ms_per_step": {k: round(v, 4) for k, v in ph.items()},
        "ortho_solve": res.get("ortho"),
        "step_graphs": res.get("graphs"),
        "autotune": res.get("autotune"),
        "mixed": res.get("mixed"),
        "precision": res.get("precision"),
        "serving": res.get("serving"),
        "batched": res.get("batched"),
        "clocks": res["clocks"],
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(args):
    """The oracle (C++ restatement of the reference, OpenMP) on the host cores,
    over a bounded sample of the same workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import binding

    binding.build()
    inp = make_inputs(args.system)
    threads = binding.library().orc_max_threads()
    w = binding.open_oracle(inp).setup().initialize()
    w.cp_step(move_atoms=True)  # warm caches
    n = 0
    t0 = time.perf_counter()
    while True:
        w.cp_step(move_atoms=True)
        n += 1
        if time.perf_counter() - t0 > args.cpu_seconds or n >= args.cpu_steps:
            break
    dt = time.perf_counter() - t0
    w.close()
    gemm = "ZGEMM on the bundled OpenBLAS" if binding.blas_in_use() else "GEMMs as OpenMP loops"
    return {"value": round(n / dt, 5), "unit": "steps/s", "cores": threads, "kind": "port",
            "sample": f"{n} CP steps of {args.system} after one warm-up step ({dt:.1f} s); {gemm}"}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import binding

    binding.build()
    inp = make_inputs(args.system)
    threads = binding.library().orc_max_threads()
    w = binding.open_oracle(inp).setup().initialize()
    for _ in range(args.warmup):
        w.cp_step(move_atoms=True)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        w.cp_step(move_atoms=True)
    dt = time.perf_counter() - t0
    w.close()
    v = args.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 5), "unit": "steps/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Si64 cell, synthetic setups, V_loc and DH)",
            "config": {"workload": WORKLOAD, "system": args.system, "precision": "fp64",
                       "parallelism": "host cores"},
            "cpu_baseline": {"value": round(v, 5), "unit": "steps/s", "cores": threads, "kind": "port",
                             "sample": f"{args.steps} CP steps of {args.system} after {args.warmup} warm-up steps; "
                                       "the CPU restatement of the reference (the Fortran reference cannot be "
                                       "built here: no Fortran compiler, FFTW or LAPACK); "
                                       + ("its ZGEMMs on the OpenBLAS bundled with scipy, as the reference's "
                                          "BLAS calls" if binding.blas_in_use() else "GEMMs as OpenMP loops")},
            "e2e": {"value": round(v, 5), "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--system", default="Si64")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--cpu-steps", type=int, default=8)
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision run")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--no-precision", action="store_true", help="skip the precision (error and drift) runs")
    ap.add_argument("--precision-systems", default="Si64,H2O32")
    ap.add_argument("--drift-steps", type=int, default=500)
    ap.add_argument("--quench-steps", type=int, default=300)
    ap.add_argument("--quench-friction", type=float, default=0.1)
    ap.add_argument("--no-serving", action="store_true", help="skip the serving and batched runs")
    ap.add_argument("--no-serving-stream", action="store_true", help="skip the serving streams, keep the batched runs")
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-workers", type=int, default=8)
    ap.add_argument("--serve-budget-gb", type=int, default=48)
    ap.add_argument("--serve-seconds", type=float, default=25.0, help="arrival window of the sustained stream")
    ap.add_argument("--batched-steps", type=int, default=20)
    ap.add_argument("--batched-workers", type=int, default=16)
    ap.add_argument("--batched-si64", type=int, default=8)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "cuda" else args.warmup
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local = dist_env()
    if world > 1:
        import torch

        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    res = run_cuda(args, rank, world, local)
    if not args.no_mixed:
        res["mixed"] = run_mixed(args, local)
        if world == 1 and not args.no_precision:
            res["precision"] = run_precision(args)
    if not args.no_serving and world == 1:
        res["serving"] = None if args.no_serving_stream else run_serving(args)
        res["batched"] = run_batched(args)
    if rank == 0:
        if world > 1 or args.no_cpu:
            args.no_cpu = args.no_cpu or rank != 0
        emit_cuda(args, res, world)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
