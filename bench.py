"""Benchmark of the B200 KMM channel timestep (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl kmm|reference] [--config cfg2]

Workload (default, the configuration the headline metric is quoted on): the Re_tau = 180 channel on
128 x 129 x 128 (Lx = 4 pi, Lz = 4 pi/3, dt = 0.005), log-law mean profile + 10 % rms divergence-
free noise (seed 1), passive scalar (Sc = 1, uniform source, Dirichlet walls) and 100,000 tracers
(seed 2, RK3), FP64.  A "step" is one iteration of the reference's time loop (main_dns.f90:198-811).
Inputs are synthetic and seeded.  The working set (~0.8 GB) is far larger than L2 (126 MB), so no
L2 flush is inserted between steps.

--impl kmm (default): value = steps/s of the device-resident run (CUDA events on the library's
    stream, max over ranks); e2e = the same steps through the C ABI with the restart state held on
    the host (kmm_bind_host + kmm_run_host): every step uploads the prognostic state from pinned
    memory, steps, and downloads it, one step's downloads overlapping the next step's uploads;
    e2e.single_calls = the same copies as kmm_upload / kmm_step / kmm_download calls.
--impl reference: the CPU restatement of the reference (oracle/, OpenMP over all host cores) on a
    bounded sample of the same workload (rank 0 only).
Multi-GPU: replicas only (the reference's ensemble is independent runs); each rank runs its own
    channel on its GPU, value = total steps of all ranks / max elapsed time.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "timesteps/s at 128x129x128: FP64 drop-in vs mixed-prec; ensemble steps/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d, "measured"
    except Exception:
        return PEAKS_FALLBACK, "fallback"


# --grid N: the cfg2 / cfg3 workload at N x (N+1) x N (small cases for single-kernel profiles)
GRID_OVERRIDE = None


def make_config(name, precision=0):
    from polymer_dns_b200 import configs
    return configs.make(name, precision, grid=GRID_OVERRIDE if name in ("cfg2", "cfg3") else None)


def build_inputs(p, init, name):
    from polymer_dns_b200 import configs
    return configs.build_inputs(p, init, name)


def load(ctx, f, extra, setter):
    from polymer_dns_b200 import configs
    configs.load(f, extra, setter)


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled every ~2 ms through NVML while the timed
    region runs (read-only queries; nothing is set).  Falls back to nvidia-smi at 100 ms when NVML
    is unavailable."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, gpu, period_s=0.002):
        self.gpu = gpu
        self.period = period_s
        self.rows = []          # (sm_mhz, max_mhz, set of reason names)
        self.stop = threading.Event()
        self.t = None
        self.proc = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = None
            try:   # the CUDA ordinal's NVML handle through its PCI address (CUDA_VISIBLE_DEVICES renumbers)
                import torch
                pr = torch.cuda.get_device_properties(self.gpu)
                bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
                self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            except Exception:
                self.h = None
            if self.h is None:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.maxmhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.t = threading.Thread(target=self._poll_nvml, daemon=True)
            self.t.start()
        except Exception:
            self.nv = None
            try:
                self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=clocks.sm,clocks.max.sm,"
                                              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                                              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                                              "--format=csv,noheader,nounits", "-lms", "100"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.t = threading.Thread(target=self._read_smi, daemon=True)
                self.t.start()
            except Exception:
                self.proc = None
        return self

    def _poll_nvml(self):
        nv = self.nv
        while not self.stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                rs = {n for n, attr in self.REASONS if bits & getattr(nv, attr)}
                self.rows.append((float(mhz), float(self.maxmhz), rs))
            except Exception:
                return
            time.sleep(self.period)

    def _read_smi(self):
        names = [n for n, _ in self.REASONS]
        for line in self.proc.stdout:
            c = [x.strip() for x in line.split(",")]
            try:
                self.rows.append((float(c[0]), float(c[1]), {n for n, v in zip(names, c[2:]) if v.lower() == "active"}))
            except Exception:
                pass

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        if self.nv:
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [r[0] for r in self.rows]
        reasons = set()
        for r in self.rows:
            reasons |= r[2]
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(r[1] for r in self.rows),
                "sm_mhz_min": min(sm), "reasons": sorted(reasons), "samples": len(self.rows),
                "source": "nvml" if self.nv else "nvidia-smi"}


# per-stage algorithmic bytes per launch (each operand read or written once)
def stage_bytes(p, nin, nout):
    nyp, nz, nxh, mx, mz = p.ny + 1, p.nz, p.nx // 2, 3 * p.nx // 2, 3 * p.nz // 2
    spec = nyp * nz * nxh * 16
    q = nyp * mz * nxh * 16
    phys = nyp * mz * mx * 8
    return {
        "dct_fwd": 2 * nin * spec,
        "zfft_bwd": nin * (spec + q),
        "xphys": nin * q + nout * phys + 3 * phys,
        "xfwd": nout * (phys + q),
        "zfft_fwd": nout * (q + spec),
        "dct_bwd": 2 * nout * spec,
    }


def fused_stage_bytes(p):
    """Algorithmic bytes per step of each stage of the fused step (each operand read or written
    once): complex state fields 16 B, intermediates 16 B (FP64) or 8 B (mixed), tracer copies 8 B."""
    nyp, nz, nxh, mx, mz = p.ny + 1, p.nz, p.nx // 2, 3 * p.nx // 2, 3 * p.nz // 2
    spec, qn, phys = nyp * nz * nxh, nyp * mz * nxh, nyp * mz * mx
    cb = 8 if p.precision == 1 else 16
    sc = 1 if p.scalar_on else 0
    n_yp, nq, nr = 6 + 2 * sc, 6 + 3 * sc, 3 + sc
    # column kernels: reads (scalar 3, omega_y 3, v 5, u/w 2), state writes (scalar, omega_y, v), y-physical writes
    col = ((3 * sc + 3 + 5 + 2) + (sc + 2)) * spec * 16 + n_yp * spec * cb
    return {
        "column": col,
        "zfft_bwd": n_yp * spec * cb + nq * qn * cb,
        "xphys": (nq + nr) * qn * cb + (3 * phys * 8 if p.npart else 0),
        "zfft_fwd": nr * (qn + spec) * cb,
        "post": nr * spec * (cb + 16),
    }


# kernels of each fused stage (ncu names at 128x129x128, FP64)
STAGE_KERNELS = {
    "column": ["k_bcol_scl<8,double2>", "k_bcol_omy<8,double2>", "k_bcol_v<8,double2>", "k_bcol_uw<8,double2>"],
    "zfft_bwd": ["k_zb_tma<192>"], "xphys": ["k_fx2<192,double2>"], "zfft_fwd": ["k_zf_tma<192>"],
    "post": ["k_bcol_bwd<8,double2>"],
}


def profiled_traffic(p, stage):
    """DRAM bytes per step of a stage's kernels from the committed ncu summary (FP64 128x129x128
    only), or None when a kernel was not captured."""
    if not (p.nx == 128 and p.ny == 128 and p.nz == 128 and p.precision == 0):
        return None
    try:
        tab = {}
        with open(os.path.join(ROOT, "profiles", "kmm_fused_fp64_128x129x128_traffic.txt")) as f:
            for line in f:
                if line.strip() and not line.startswith("#"):
                    k, v = line.split("\t")
                    tab[k.strip()] = int(v)
        return sum(tab[k] for k in STAGE_KERNELS[stage])
    except Exception:
        return None


def fused_model_bytes(p):
    """Fused-minimum bytes per step (field passes x 16 B): velocity 28, scalar +13, polymer +108,
    tracers 264 B/particle, IB 52 B per solid cell."""
    nyp, nz, nxh = p.ny + 1, p.nz, p.nx // 2
    P = nyp * nz * nxh
    passes = 28 + (13 if p.scalar_on else 0) + (108 if p.polymer_on else 0)
    return passes * 16 * P + 264 * p.npart


def run_kmm(a, rank, world, local_rank):
    import torch
    from polymer_dns_b200 import runtime
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    p, init, desc = make_config(a.config, a.precision)
    f, extra = build_inputs(p, init, a.config)
    ctx = runtime.KmmContext(p, device=local_rank)
    if a.ztma is not None:
        ctx.call("set_option", 4, a.ztma)
    if a.tc_dct is not None:
        ctx.call("set_option", 7, a.tc_dct)
    load(ctx, f, extra, ctx.upload)
    ctx.initial()
    for _ in range(a.warmup):
        ctx.step()
    ctx.call("sync")

    def barrier():
        if dist is not None:
            dist.barrier()
        ctx.call("sync")

    # device-resident timed region (the fused step replays its captured CUDA graphs)
    barrier()
    launches0 = ctx.launch_count()
    with ClockSampler(local_rank) as clk:
        ctx.event_record(0)
        for _ in range(a.steps):
            ctx.step()
        ctx.event_record(1)
        ms = ctx.event_elapsed(0, 1)
    barrier()
    launches = ctx.launch_count() - launches0
    # per-stage breakdown: a separate pass with stage events, kernel by kernel
    ctx.set_timing(1)
    for _ in range(min(a.steps, 10)):
        ctx.step()
    stages = ctx.stage_times()
    ctx.set_timing(0)
    nstage = min(a.steps, 10)
    from polymer_dns_b200 import replicas
    ms, value = replicas.job_throughput(dist, ms, a.steps, world, "cuda")
    ms_per_step = ms / a.steps

    # end-to-end through the C ABI with the restart state on the host (pinned buffers)
    state = ["V", "FN", "FNM1", "OMY", "GN", "GNM1", "U0", "H1N", "H1NM1", "W0", "H3N", "H3NM1"]
    if p.scalar_on:
        state += ["SCALAR", "SCN", "SCNM1"]
    if p.npart:
        state += ["XPART", "YPART", "ZPART", "UPART", "VPART", "WPART"]
    if p.polymer_on:   # the c-restart records (restart.py)
        comp = ["11", "12", "13", "22", "23", "33"]
        state += ["C11", "C12", "C13", "C21", "C22", "C23", "C31", "C32", "C33"]
        state += ["C%sN" % c for c in comp] + ["C%sNM1" % c for c in comp]
        state += ["STR%sN" % c for c in comp] + ["STR%sNM1" % c for c in comp]
    host = {}
    for n in state:
        arr = ctx.download(n)
        buf = torch.empty(arr.nbytes, dtype=torch.uint8, pin_memory=True)
        buf.numpy()[:] = np.frombuffer(arr.tobytes(order="F"), dtype=np.uint8)
        host[n] = buf
    nbytes = sum(int(b.numel()) for b in host.values())
    e2e_steps = max(2, min(a.steps, 10))
    # (1) kmm_run_host: the state bound to the host arrays; every step uploads all of it, steps and
    # downloads all of it, one step's downloads overlapping the next step's uploads
    for n, b in host.items():
        ctx.bind_host(n, b.data_ptr(), int(b.numel()))
    barrier()
    ctx.event_record(2)
    ctx.run_host(e2e_steps)
    ctx.event_record(3)
    e2e_ms = ctx.event_elapsed(2, 3)
    ctx.unbind_host()
    # (2) the same copies as single calls: kmm_upload per field, kmm_step, kmm_download per field
    barrier()
    ctx.event_record(2)
    for _ in range(e2e_steps):
        for n, b in host.items():
            ctx.upload_ptr(n, b.data_ptr(), int(b.numel()))
        ctx.step()
        for n, b in host.items():
            ctx.download_ptr(n, b.data_ptr(), int(b.numel()))
    ctx.event_record(3)
    calls_ms = ctx.event_elapsed(2, 3)
    barrier()
    e2e_ms, e2e_value = replicas.job_throughput(dist, e2e_ms, e2e_steps, world, "cuda")
    calls_ms, calls_value = replicas.job_throughput(dist, calls_ms, e2e_steps, world, "cuda")

    result = None
    if rank == 0:
        peaks, peaks_kind = load_peaks()
        fused = stages.get("dct_fwd", (0, 0))[1] == 0   # the fused step records no separate DCT stages
        if fused:
            sb = fused_stage_bytes(p)
        else:
            nin = 6 + (4 if p.scalar_on else 0) + (45 if p.polymer_on else 0)
            nout = 3 + (1 if p.scalar_on else 0) + (18 if p.polymer_on else 0)
            sb = stage_bytes(p, nin, nout)
        vc_stages = {k: v for k, v in stages.items() if k in sb and v[1] > 0}
        dom = max(vc_stages, key=lambda k: vc_stages[k][0]) if vc_stages else None
        total_stage_ms = sum(v[0] for v in stages.values())
        roof = None
        peak = float(peaks.get("hbm_gbs", 6650.0))
        per_stage = {}
        for k, v in vc_stages.items():
            per_stage[k] = round(sb[k] / (v[0] / v[1] / 1e3) / 1e9 / peak, 4)
        if dom:
            avg_ms = vc_stages[dom][0] / vc_stages[dom][1]
            ach = sb[dom] / (avg_ms / 1e3) / 1e9
            kern = ", ".join(STAGE_KERNELS[dom]) if fused else dom
            roof = {"bound": "hbm", "kernel": kern, "stage": dom, "achieved": round(ach, 1), "peak": peak,
                    "peak_kind": peaks_kind, "unit": "GB/s", "frac": round(ach / peak, 4),
                    "avg_launch_ms": round(avg_ms, 4), "algorithmic_bytes_per_launch": sb[dom],
                    "traffic": profiled_traffic(p, dom) if fused else None,
                    "frac_by_stage": per_stage,
                    "note": "column stage = 3-4 launches per step, counted together"}
        model = fused_model_bytes(p)
        result = {
            "metric": METRIC, "value": round(value, 3), "unit": "timesteps/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if p.precision == 0 else "mixed",
            "data": "synthetic (seeded log-law + noise, uniform tracers)",
            "config": {"workload": desc, "grid": [p.nx, p.ny + 1, p.nz], "dt": p.dt, "npart": p.npart,
                       "precision": "fp64 drop-in" if p.precision == 0 else "mixed",
                       "parallelism": "replicas x%d" % world,
                       "l2": "inputs larger than L2 (state ~%d MB), no flush" % int(model / 1e6),
                       "grid_point_steps_per_s": round(value * p.nx * (p.ny + 1) * p.nz, 1),
                       "fused_model_bytes_per_step": model,
                       "step_frac_of_hbm": round(model / (ms_per_step / 1e3) / 1e9 / float(peaks.get("hbm_gbs", 6650.0)), 4),
                       "stage_ms_per_step": {k: round(v[0] / max(1, nstage), 4) for k, v in stages.items()},
                       "stage_note": "stage times from a separate %d-step pass launched kernel by kernel" % nstage,
                       "stage_share": {k: round(v[0] / total_stage_ms, 4) for k, v in stages.items()} if total_stage_ms else {}},
            "roofline": roof,
            "e2e": {"value": round(e2e_value, 3), "unit": "timesteps/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "steps": e2e_steps, "call": "kmm_bind_host + kmm_run_host",
                    "single_calls": {"value": round(calls_value, 3), "unit": "timesteps/s",
                                     "call": "kmm_upload per field, kmm_step, kmm_download per field"}},
            "gpu_launches": int(launches),
            "clocks": dict(clk.summary(), **({"ms_per_step_x_median_mhz": round(ms_per_step * clk.summary()["sm_mhz"], 2)}
                                             if clk.summary().get("sm_mhz") else {})),
        }
        if p.precision == 0 and not a.no_mixed and a.config in ("cfg1", "cfg2"):
            result["mixed"] = mixed_report(a, f, extra, local_rank, ms_per_step)
        if a.config == "cfg2" and not a.no_ensemble:
            result["ensemble"] = ensemble_report(a, local_rank)
        if a.config == "cfg2" and not a.no_polymer and world == 1:
            result["polymer"] = polymer_report(a, local_rank)
        if a.config == "cfg2" and not a.no_cfg5 and world == 1:
            result["cfg5"] = cfg5_report(a, local_rank)
        if not a.no_cpu_baseline and world == 1:
            result["cpu_baseline"] = cpu_baseline(a.config, a.cpu_steps, one_thread_steps=2)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return result


def mixed_report(a, f, extra, local_rank, fp64_ms):
    """The mixed-precision form (FP32 transforms and products, FP64 solves) on the same workload:
    its device-resident speed, and its error against the FP64 drop-in from the same initial state
    after 10 and 1000 steps (relative max-norm error of u, v, w and the scalar; bulk kinetic
    energy and wall shear from kmm_flowstats)."""
    from polymer_dns_b200 import runtime
    p32, _, _ = make_config(a.config, 1)
    p64, _, _ = make_config(a.config, 0)
    c32 = runtime.KmmContext(p32, device=local_rank)
    load(c32, f, extra, c32.upload)
    c32.initial()
    for _ in range(a.warmup):
        c32.step()
    c32.call("sync")
    c32.event_record(0)
    for _ in range(a.steps):
        c32.step()
    c32.event_record(1)
    ms = c32.event_elapsed(0, 1) / a.steps
    c32.close()
    # accuracy: both forms from the same state
    ctx = {}
    for prec, pp in ((0, p64), (1, p32)):
        c = runtime.KmmContext(pp, device=local_rank)
        load(c, f, extra, c.upload)
        c.initial()
        ctx[prec] = c
    names = {"u": "U", "v": "V", "w": "W"}
    if p64.scalar_on:
        names["scalar"] = "SCALAR"
    _, s0 = ctx[0].flowstats()
    errs = {}
    done = 0
    for mark in (10, 1000):
        for c in ctx.values():
            c.run(mark - done)
        done = mark
        st = {prec: c.flowstats() for prec, c in ctx.items()}   # runs veloc: u, w current
        e = {}
        for k, n in names.items():
            x, y = ctx[1].download(n), ctx[0].download(n)
            e[k] = float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-300))
        (_, s64), (_, s32) = st[0], st[1]
        e["bulk_ke"] = float(abs(s32[3] - s64[3]) / abs(s64[3]))
        e["wall_shear"] = float(max(abs(s32[1] - s64[1]), abs(s32[2] - s64[2])) / max(abs(s64[1]), abs(s64[2])))
        errs[str(mark)] = {k: float("%.3e" % v) for k, v in e.items()}
    _, s64 = ctx[0].flowstats()
    drift = {"bulk_ke_fp64": float("%.4e" % ((s64[3] - s0[3]) / s0[3])),
             "wall_shear_top_fp64": float("%.4e" % ((s64[1] - s0[1]) / s0[1]))}
    for c in ctx.values():
        c.close()
    return {"value": round(1e3 / ms, 3), "unit": "timesteps/s", "ms_per_step": round(ms, 4),
            "speedup_vs_fp64": round(fp64_ms / ms, 3), "dtype": "fp32 transforms/products, fp64 solves",
            "rel_err_vs_fp64": errs, "drift_over_1000_steps": drift}


def polymer_report(a, local_rank):
    """The polymer + immersed-boundary configuration (the Re_tau = 180 case with FENE-P Wi = 20,
    beta = 0.9, L^2 = 900 and the Goldstein force on the cylinder; routine path): FP64 and
    mixed-precision steps/s; the mixed form's relative error against FP64 from the same state after
    10, 100 and 1000 steps (u, v, w, scalar, the six conformation-tensor components, bulk kinetic
    energy, wall shear) or up to the step where a run stops; the same for the reference's spreading
    test (cylinder inert) over 1000 steps; the oracle on the host cores."""
    from polymer_dns_b200 import runtime
    p64, init, desc = make_config("cfg3", 0)
    f, extra = build_inputs(p64, init, "cfg3")
    nst = 5
    ms = {}
    for prec in (0, 1):
        p, _, _ = make_config("cfg3", prec)
        c = runtime.KmmContext(p, device=local_rank)
        load(c, f, extra, c.upload)
        c.initial()
        for _ in range(3):
            c.step()
        c.call("sync")
        c.event_record(0)
        for _ in range(nst):
            c.step()
        c.event_record(1)
        ms[prec] = c.event_elapsed(0, 1) / nst
        c.close()
    from polymer_dns_b200 import abi, configs
    names = {"u": "U", "v": "V", "w": "W", "scalar": "SCALAR", "c11": "C11", "c12": "C12", "c13": "C13",
             "c22": "C22", "c23": "C23", "c33": "C33"}

    def accuracy_run(marks, **over):
        """FP64 and mixed from the same state: relative max-norm errors at each mark, the bulk
        kinetic energy and wall shear, where a run stopped (if one did) and the largest trace of
        the conformation tensor seen on the 3/2 grid's spectral means at that point."""
        ctx = {}
        for prec in (0, 1):
            p, _, _ = configs.make("cfg3", prec, **over)
            c = runtime.KmmContext(p, device=local_rank)
            load(c, f, extra, c.upload)
            c.initial()
            ctx[prec] = c
        errs, done, stopped = {}, 0, None
        for mark in marks:
            for step in range(done + 1, mark + 1):
                sts = [c.call("step", allow=(abi.ERR_CFL, abi.ERR_NAN)) for c in ctx.values()]
                if any(sts):
                    c11 = max(np.abs(c.download("C11")).max() for c in ctx.values())
                    stopped = ("step %d: %s (CFL %.2f; max |C11| coefficient %.1f against L^2 = %.0f)" % (
                        step, ", ".join(abi.STATUS_NAMES.get(x, str(x)) for x in sts),
                        max(c.stats().cflmax for c in ctx.values()), c11, p64.zlmax ** 2))
                    break
            if stopped:
                break
            done = mark
            st = {prec: c.flowstats() for prec, c in ctx.items()}   # runs veloc: u, w current
            e = {}
            for k, n in names.items():
                x, y = ctx[1].download(n), ctx[0].download(n)
                e[k] = float("%.3e" % (np.abs(x - y).max() / max(np.abs(y).max(), 1e-300)))
            (_, s64), (_, s32) = st[0], st[1]
            e["bulk_ke"] = float("%.3e" % (abs(s32[3] - s64[3]) / abs(s64[3])))
            e["wall_shear"] = float("%.3e" % (max(abs(s32[1] - s64[1]), abs(s32[2] - s64[2])) /
                                              max(abs(s64[1]), abs(s64[2]))))
            errs[str(mark)] = e
        for c in ctx.values():
            c.close()
        return errs, stopped or "both forms ran %d steps" % marks[-1]

    errs, stopped = accuracy_run((10, 100, 1000))
    # the same workload with the reference's spreading test, under which the cylinder's planes get
    # no force (kmaxsurf is an x index): the polymer-laden channel itself over 1000 steps
    errs_ref, stopped_ref = accuracy_run((10, 1000), ib_spread_all=0)
    cpu = cpu_baseline("cfg3", a.cpu_steps, one_thread_steps=1) if not a.no_cpu_baseline else None
    return {"workload": desc, "fp64": {"value": round(1e3 / ms[0], 3), "unit": "timesteps/s",
                                       "ms_per_step": round(ms[0], 4)},
            "mixed": {"value": round(1e3 / ms[1], 3), "unit": "timesteps/s", "ms_per_step": round(ms[1], 4),
                      "speedup_vs_fp64": round(ms[0] / ms[1], 3)},
            "mixed_rel_err_vs_fp64": errs, "long_run": stopped,
            "reference_spreading": {"note": "ib_spread_all = 0: the reference's i <= kmaxsurf test, the cylinder inert",
                                    "mixed_rel_err_vs_fp64": errs_ref, "long_run": stopped_ref},
            "cpu_baseline": cpu}


def cfg5_report(a, local_rank, nsteps=5, mark=10):
    """The large single run (384 x 257 x 384, Re_tau = 395, polymer + scalar + IB cylinder + 1 M RK3
    tracers) on the routine path, FP64 and mixed in turn (one context at a time: the FP64 form holds
    about 158 GB): steps/s, device memory held, size-independent checks after the timed steps
    (continuity of the spectral velocity, finite CFL, tracer cells in range), and the mixed form's
    relative error against FP64 from the same inputs after `mark` steps (u, v, w, scalar, the six
    conformation components, bulk kinetic energy, wall shear).  1000 steps of this workload take
    about five minutes per form and are left out of the default run."""
    import torch
    from polymer_dns_b200 import abi, configs, runtime
    torch.cuda.set_device(local_rank)
    p64, init, desc = configs.make("cfg5", 0)
    f, extra = configs.build_inputs(p64, init, "cfg5")
    names = {"u": "U", "v": "V", "w": "W", "scalar": "SCALAR", "c11": "C11", "c12": "C12", "c13": "C13",
             "c22": "C22", "c23": "C23", "c33": "C33"}
    out = {"workload": desc, "grid": [p64.nx, p64.ny + 1, p64.nz], "npart": p64.npart}
    fields, flow = {}, {}
    for prec in (0, 1):
        key = "fp64" if prec == 0 else "mixed"
        p, _, _ = configs.make("cfg5", prec)
        free0, total = torch.cuda.mem_get_info()
        c = runtime.KmmContext(p, device=local_rank)
        try:
            configs.load(f, extra, c.upload)
            st = c.call("initial", allow=(abi.ERR_CFL, abi.ERR_NOMEM, abi.ERR_UNSUPPORTED))
            if st:
                out[key] = abi.STATUS_NAMES.get(st, st) + ": " + c.error()
                continue
            bad = None
            for _ in range(2):
                st = c.call("step", allow=(abi.ERR_CFL, abi.ERR_NAN, abi.ERR_NOMEM, abi.ERR_UNSUPPORTED))
                if st:
                    bad = abi.STATUS_NAMES.get(st, st) + " in warm-up: " + c.error()
                    break
            if bad:
                out[key] = bad
                continue
            c.call("sync")
            free1, _ = torch.cuda.mem_get_info()
            c.event_record(0)
            sts = [c.call("step", allow=(abi.ERR_CFL, abi.ERR_NAN)) for _ in range(nsteps)]
            c.event_record(1)
            ms = c.event_elapsed(0, 1) / nsteps
            for _ in range(mark - 2 - nsteps):
                sts.append(c.call("step", allow=(abi.ERR_CFL, abi.ERR_NAN)))
            flow[prec] = c.flowstats()   # runs veloc: u, w current
            fields[prec] = {k: c.download(n) for k, n in names.items()}
            u, w = fields[prec]["u"], fields[prec]["w"]
            c.call("cderiv", "V", "WRKC")
            dv = c.download("WRKC")
            kx = np.arange(p.nx // 2) * 2 * math.pi / p.xl
            kz = np.fft.fftfreq(p.nz, 1.0 / p.nz) * 2 * math.pi / p.zl
            div = 1j * kx[None, None, :] * u + dv + 1j * kz[None, :, None] * w
            cells = c.tracer_cells()
            out[key] = {"value": round(1e3 / ms, 3), "unit": "timesteps/s", "ms_per_step": round(ms, 3),
                        "grid_point_steps_per_s": round(1e3 / ms * p.nx * (p.ny + 1) * p.nz, 1),
                        "fused_model_bytes_per_step": fused_model_bytes(p),
                        "frac_of_hbm": round(fused_model_bytes(p) / (ms / 1e3) / 1e9 /
                                             float(load_peaks()[0].get("hbm_gbs", 6650.0)), 4),
                        "timed_steps": nsteps, "steps_run": mark, "status": sorted({abi.STATUS_NAMES.get(x, x) for x in sts}),
                        "device_memory_gb": round((free0 - free1) / 1e9, 2),
                        "checks": {"max_divergence_rel": float("%.3e" % (np.abs(div).max() / np.abs(u).max())),
                                   "cflmax": round(c.stats().cflmax, 5),
                                   "tracer_cells_in_range": bool(cells.min() >= 1)}}
            out["device_total_gb"] = round(total / 1e9, 1)
        finally:
            c.close()
    if 0 in fields and 1 in fields:
        e = {}
        for k in names:
            x, y = fields[1][k], fields[0][k]
            e[k] = float("%.3e" % (np.abs(x - y).max() / max(np.abs(y).max(), 1e-300)))
        (_, s64), (_, s32) = flow[0], flow[1]
        e["bulk_ke"] = float("%.3e" % (abs(s32[3] - s64[3]) / abs(s64[3])))
        e["wall_shear"] = float("%.3e" % (max(abs(s32[1] - s64[1]), abs(s32[2] - s64[2])) /
                                          max(abs(s64[1]), abs(s64[2]))))
        out["mixed_rel_err_vs_fp64"] = {str(mark): e}
        out["mixed"]["speedup_vs_fp64"] = round(out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"], 3)
    out["status"] = "ok" if isinstance(out.get("fp64"), dict) and isinstance(out.get("mixed"), dict) else "incomplete"
    return out


ENSEMBLE_GRIDS = [(64, 64, 64)] * 4 + [(96, 96, 96)] * 4 + [(128, 128, 96)] * 4 + [(128, 128, 128)] * 4


def ensemble_members(precision):
    """The 16-member uneven-grid ensemble: 4 each of 64x65x64, 96x97x96, 128x129x96, 128x129x128,
    Re_tau cycling 120 / 150 / 180, seeds 10..25, each with a scalar and 20,000 RK3 tracers, in the
    Re_tau = 180 box (Lx = 4 pi, Lz = 4 pi / 3, dt = 0.005, re = 2800)."""
    from polymer_dns_b200 import abi
    out = []
    for m, (nx, ny, nz) in enumerate(ENSEMBLE_GRIDS):
        p = abi.default_params(nx=nx, ny=ny, nz=nz, dt=0.005, re=2800.0, r_tau=(120.0, 150.0, 180.0)[m % 3],
                               xl=4 * math.pi, zl=4 * math.pi / 3, scalar_on=1, diff=1.0, scalar_bc=1,
                               scalar_q=1.0, npart=20000, ap=1e-3, tracer_scheme=1, precision=precision)
        out.append((p, dict(profile="loglaw", amp=0.1, kmax=8, seed=10 + m)))
    return out


def ensemble_report(a, local_rank):
    """Ensemble steps/s of the 16 members advanced together (kmm_ensemble_run), FP64 and mixed.
    Timed with CUDA events on a stream ordered after a device-wide synchronisation (start) and
    recorded after every member has finished (end), so host launch gaps are included."""
    import torch
    from polymer_dns_b200 import runtime, inputs
    torch.cuda.set_device(local_rank)
    res = {"members": len(ENSEMBLE_GRIDS), "grids": ["%dx%dx%d" % (g[0], g[1] + 1, g[2]) for g in ENSEMBLE_GRIDS]}
    member_inputs = []
    for p, init in ensemble_members(0):
        f = inputs.channel_initial(p.nx, p.ny, p.nz, p.xl, p.yl, p.zl, p.re, p.r_tau, init["profile"],
                                   init["amp"], init["kmax"], init["seed"])
        extra = {"INITSCL": np.zeros_like(f[0])}
        x, y, z = inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, init["seed"])
        extra.update(XPART=x, YPART=y, ZPART=z)
        member_inputs.append((f, extra))
    from polymer_dns_b200 import autotune
    for prec in (0, 1):
        ctxs, model = [], 0
        tuned = {}
        for (p, init), (f, extra) in zip(ensemble_members(prec), member_inputs):
            # the runtime variants of each member shape, picked by timing them once per shape
            best, timings = autotune.tune(runtime, p, lambda cc, f=f, extra=extra: load(cc, f, extra, cc.upload),
                                          device=local_rank)
            tuned["%dx%dx%d" % (p.nx, p.ny + 1, p.nz)] = {"chosen": autotune.describe(best), "ms_per_step": timings}
            c = runtime.KmmContext(p, device=local_rank)
            autotune.apply(c, best)
            load(c, f, extra, c.upload)
            c.initial()
            ctxs.append(c)
            model += fused_model_bytes(p)
        runtime.ensemble_run(ctxs, a.warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = runtime.ensemble_run(ctxs, a.steps)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / a.steps
        pts = sum(p.nx * (p.ny + 1) * p.nz for p, _ in ensemble_members(prec))
        peak = float(load_peaks()[0].get("hbm_gbs", 6650.0))
        res["fp64" if prec == 0 else "mixed"] = {
            "value": round(1e3 / ms, 3), "unit": "ensemble steps/s", "ms_per_ensemble_step": round(ms, 4),
            "member_steps_per_s": round(len(ctxs) * 1e3 / ms, 2),
            "grid_point_steps_per_s": round(pts * 1e3 / ms, 1),
            "fused_model_bytes_per_ensemble_step": model,
            "frac_of_hbm": round(model / (ms / 1e3) / 1e9 / peak, 4),
            "autotune": tuned,
            "status": "ok" if all(s == 0 for s in st) else "member status %s" % st}
        for c in ctxs:
            c.close()
    return res


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def cpu_baseline(config, nsteps, one_thread_steps=1, skip=10):
    """The oracle (C restatement of the reference, OpenMP over y-planes / kx slabs) on the host cores,
    timed like the reference's cadence timer (main_dns.f90:797-809): steps 1..skip run untimed
    (setup, first-touch, the start-up transient), then steps skip+1 .. skip+nsteps are timed with all
    host cores, then `one_thread_steps` further steps with one thread."""
    from oracle import pyoracle
    p, init, desc = make_config(config)
    f, extra = build_inputs(p, init, config)
    cores = pyoracle.set_threads(0)
    o = pyoracle.Oracle(p)
    load(o, f, extra, o.set)
    o.initial()
    for _ in range(skip):
        o.step()
    t0 = time.perf_counter()
    for _ in range(nsteps):
        o.step()
    dt = time.perf_counter() - t0
    one = None
    if one_thread_steps > 0:
        pyoracle.set_threads(1)
        t1 = time.perf_counter()
        for _ in range(one_thread_steps):
            o.step()
        d1 = time.perf_counter() - t1
        pyoracle.set_threads(0)
        one = {"value": round(one_thread_steps / d1, 5), "unit": "timesteps/s", "cores": 1,
               "sample": "step%s %s (%.1f s)" % ("s" if one_thread_steps > 1 else "",
                                                 "%d..%d" % (skip + nsteps + 1, skip + nsteps + one_thread_steps)
                                                 if one_thread_steps > 1 else str(skip + nsteps + 1), d1)}
    o.close()
    return {"value": round(nsteps / dt, 5), "unit": "timesteps/s", "cores": cores, "kind": "port",
            "cpu_model": cpu_model(), "nproc": os.cpu_count(),
            "sample": "steps %d..%d of the same workload after %d untimed steps (%.1f s)" % (
                skip + 1, skip + nsteps, skip, dt),
            "one_thread": one}


def run_reference(a, rank, world):
    if rank != 0:
        return None
    p, init, desc = make_config(a.config)
    steps = max(1, min(a.steps, a.cpu_steps))
    cb = cpu_baseline(a.config, steps, one_thread_steps=0)
    return {"metric": METRIC, "value": cb["value"], "unit": "timesteps/s", "n_gpus": world, "steps": steps,
            "warmup": 10, "ms_per_step": round(1e3 / cb["value"], 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": desc, "grid": [p.nx, p.ny + 1, p.nz], "npart": p.npart},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kmm", choices=["kmm", "reference"])
    ap.add_argument("--config", default="cfg2", choices=["cfg1", "cfg2", "cfg3", "cfg5"])
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--cpu-steps", type=int, default=5, help="timed oracle steps after the 10 untimed ones")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision speed / error report")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 16-member ensemble measurement")
    ap.add_argument("--no-polymer", action="store_true", help="skip the polymer + IB (FP64 / mixed) measurement")
    ap.add_argument("--no-cfg5", action="store_true", help="skip the 384x257x384 polymer + IB + 1M tracer run")
    ap.add_argument("--ztma", type=int, default=None, choices=[0, 1],
                    help="inverse z transform with TMA tile copies (1, the library default) or plain loads (0)")
    ap.add_argument("--tc-dct", type=int, default=None, choices=[0, 1],
                    help="mixed routine path: y transforms on the tensor cores (1) or as FP32 FFTs (0)")
    ap.add_argument("--grid", type=int, default=None,
                    help="run the cfg2 / cfg3 workload at N x (N+1) x N instead of 128 x 129 x 128 (profiling)")
    a = ap.parse_args()
    global GRID_OVERRIDE
    GRID_OVERRIDE = a.grid
    if a.warmup < 3:
        a.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if a.impl == "reference":
        res = run_reference(a, rank, world)
    else:
        res = run_kmm(a, rank, world, local_rank)
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
