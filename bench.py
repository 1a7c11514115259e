"""Benchmark: seconds to solve the 3D punched-lattice recovery on B200.

One step = one complete interior-point solve (csipm_solve) of the workload,
from A^T z0 to beta on the device.  Workload (default): 320^3 grid, 0.5%
log-normal(0,1) nonzeros with random signs, balls of radius 3 punched on a
period-16 lattice (~3% missing), sigma = 0.01, lambda = 0.05 ||A^T y||_inf,
seeded synthetic data (the reference's crystallography volumes are not
available).  Multi-GPU: one independent replica per rank (weak scaling, no
collective on the path); times are the max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload 3d320|3d256|3d160|3d128|2d1024|1d16384] [--precision fp64|mixed]

Beside the headline solve the line carries: the FP64 path at the same
settings, the other measured configurations (1D 2^14, 2D 1024^2, 3D 256^3 in
FP64) as legs, the serving stream, and one complete FP64 CPU-twin solve of
the headline problem (the accuracy oracle and the CPU baseline).  The
reference arm (--impl reference) runs that CPU solve alone, measured end to
end.

Prints ONE JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "compressedsensingipm.jl_b200")
sys.path.insert(0, PKG)

WORKLOADS = {
    "3d320": dict(kind="3d", dims=(320, 320, 320)),
    "3d256": dict(kind="3d", dims=(256, 256, 256)),
    "3d160": dict(kind="3d", dims=(160, 160, 160)),
    "3d128": dict(kind="3d", dims=(128, 128, 128)),
    "2d1024": dict(kind="2d", dims=(1024, 1024)),
    "1d16384": dict(kind="1d", dims=(16384,)),
}
METRIC = "s-to-solve 3D 320^3 (beta 1e-6 vs FP64)"
ORACLE_TOL, ORACLE_CG_RTOL = 1e-12, 1e-10     # the FP64 device accuracy oracle
LEGS = ("1d16384", "2d1024", "3d256")          # the other measured configurations (FP64)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="3d320", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                    help="mixed (the headline): FP32 CG products with FP64 residuals/refinement; "
                         "the FP64 solve of the same problem is timed beside it as the accuracy oracle")
    ap.add_argument("--tol", type=float, default=1e-10, help="IPM stop (relative duality gap / scaled KKT error)")
    ap.add_argument("--cg-rtol", type=float, default=1e-2,
                    help="relative tolerance of each Newton solve (inexact Newton; the library default is 1e-8)")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU-twin solve of the headline problem (accuracy vs the CPU twin and the CPU "
                         "baseline; about three minutes of host time at 320^3)")
    ap.add_argument("--no-legs", action="store_true", help="skip the 1D / 2D / 3D-256 FP64 legs")
    ap.add_argument("--clock-log", default=None,
                    help="CSV file for the clock samples of the timed region (default: a temporary file)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--serve-requests", type=int, default=2000,
                    help="requests of the serving stream measured beside the headline solve (0: skip)")
    ap.add_argument("--serve-slots", type=int, default=16, help="concurrent solves of the serving loop")
    ap.add_argument("--serve-batch", type=int, default=32,
                    help="requests of one batch class a slot solves together in the batched closed run (<= 1: skip)")
    ap.add_argument("--serve-batch-slots", type=int, default=16, help="slots of the batched closed run")
    ap.add_argument("--serve-batch-max-n", type=int, default=1 << 16,
                    help="batched closed run: requests of more samples are solved alone (0: no limit)")
    ap.add_argument("--serve-only", action="store_true",
                    help="run only the serving leg and print its JSON object (slot-count experiments)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="plain kernel launches instead of CUDA graphs (launch-list profiling sees every kernel)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="default pass variants instead of the per-size autotuner (profilers distort its timings)")
    ap.add_argument("--solves-only", action="store_true",
                    help="run the warm-up and timed headline solves only, print their time and exit (the command "
                         "for launch lists)")
    ap.add_argument("--passes-only", action="store_true",
                    help="build the handle, launch each pass of one CG product twice (csipm_profile_passes, "
                         "reps=1), print the pass list and exit: the small command for kernel captures")
    return ap.parse_args()


def workload_config(args, wl):
    return {
        "workload": f"{wl['kind']}-{'x'.join(map(str, wl['dims']))}-punched-{args.precision}",
        "grid": list(wl["dims"]),
        "precision": args.precision,
        "generator": "seeded synthetic (numpy default_rng), rank r uses seed r",
        "missing": {"3d": "balls r=3 on a period-16 lattice", "2d": "disks r=4 period 32 + 5% random",
                    "1d": "20 random gaps, 15%"}[wl["kind"]],
        "lambda": {"3d": "0.05*||A^T y||_inf", "2d": "0.1*||A^T y||_inf", "1d": "0.1*||A^T y||_inf"}[wl["kind"]],
        "stop": f"relative LASSO duality gap {args.tol:g} (or scaled KKT error {args.tol:g})",
        "newton_cg_rtol": args.cg_rtol,
        "l2": "no flush needed: the solve streams a multi-GB working set (> 126 MB L2) every CG iteration",
        "parallelism": f"replicas x{args.gpus}",
    }


# ----------------------------------------------------------------------- dist
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Dist:
    def __init__(self, world, rank, local, use_gpu=True):
        self.world, self.rank, self.local = world, rank, local
        self.pg = None
        if world > 1:
            import datetime
            import torch.distributed as dist
            backend = "nccl" if use_gpu else "gloo"
            # short: ranks that wait for a dead peer end with an error, not a hang
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.dist = dist

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, v):
        if self.world == 1:
            return v
        import torch
        t = torch.tensor([float(v)], device="cuda" if self.dist.get_backend() == "nccl" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


# ----------------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock, power and clock-event reasons sampled during the timed region.

    NVML read queries every 5 ms from a thread (three headline solves last
    about 0.16 s, shorter than the 200 ms period of `nvidia-smi -lms`); when
    NVML cannot be opened, `nvidia-smi -lms 200`.  Both only read the GPU's
    state."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                   ("sw_power_cap", 0x4))
    PERIOD_S = 0.005

    def __init__(self, index, path=None):
        self.index = index
        self.proc = None
        self.thread = None
        self.path = path or os.path.join(tempfile.gettempdir(), f"csipm_clocks_{os.getpid()}_gpu{index}.csv")

    def _nvml_handle(self):
        import pynvml as N
        N.nvmlInit()
        try:
            import torch
            u = str(torch.cuda.get_device_properties(self.index).uuid)
            return N, N.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
        except Exception:
            return N, N.nvmlDeviceGetHandleByIndex(self.index)

    def _start_nvml(self):
        import threading
        N, h = self._nvml_handle()
        reasons = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or N.nvmlDeviceGetCurrentClocksThrottleReasons
        self.max_mhz = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))
        self.samples = []
        self.halt = threading.Event()

        def run():
            while not self.halt.is_set():
                try:
                    self.samples.append((float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)), int(reasons(h)),
                                         N.nvmlDeviceGetPowerUsage(h) / 1000.0))
                except Exception:
                    pass
                self.halt.wait(self.PERIOD_S)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def _stop_nvml(self):
        self.halt.set()
        self.thread.join(timeout=5)
        if not self.samples:
            return None
        found = set()
        with open(self.path, "w") as fh:
            fh.write("# NVML every %g ms: sm_mhz, max_sm_mhz, power_w, event_reasons_hex\n" % (1e3 * self.PERIOD_S))
            for sm, rs, pw in self.samples:
                fh.write(f"{sm:.0f}, {self.max_mhz:.0f}, {pw:.1f}, {rs:#x}\n")
                for nm, bit in self.REASON_BITS:
                    if rs & bit:
                        found.add(nm)
        return {"sm_mhz": statistics.median(s[0] for s in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(found), "samples": len(self.samples), "source": "nvml"}

    def start(self):
        try:
            self._start_nvml()
            return
        except Exception:
            self.thread = None
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            return self._stop_nvml()
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for nm, val in zip(names, p[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvidia-smi"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(workload, precision, kernel):
    """DRAM bytes (read + write) per launch of `kernel` from the committed ncu
    summary (profiles/dram_traffic.json), scaled to this workload, or None."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        d = json.load(open(p))
        e = d.get(f"{workload}/{precision}", {}).get(kernel)
        return None if e is None else e["bytes_per_launch"]
    except Exception:
        return None


def profile_passes(L, nlp, N, reps):
    """csipm_profile_passes: each pass of one CG product timed alone with CUDA events."""
    import torch
    from csipm import _native
    ms_p = (ctypes.c_double * 8)()
    by_p = (ctypes.c_double * 8)()
    names = ctypes.create_string_buffer(8 * 32)
    npass = ctypes.c_int()
    xr = torch.randn(N, dtype=torch.float64, device="cuda")
    _native.check(L.csipm_profile_passes(nlp.handle, ctypes.c_void_p(xr.data_ptr()), reps, ms_p, by_p, names,
                                         ctypes.byref(npass)), nlp.handle)
    passes = []
    for k in range(npass.value):
        nm = names.raw[32 * k:32 * k + 32].split(b"\0")[0].decode()
        passes.append({"kernel": nm, "ms": ms_p[k], "bytes": by_p[k], "GBps": by_p[k] / ms_p[k] / 1e6})
    return passes


# ----------------------------------------------------------------------- problem
def build_problem(wl, seed):
    """Seeded problem, synthesised with the library's own (unmasked) operator."""
    import torch
    import csipm
    import csipm.problems as P
    spec = P.make_spec(wl["kind"], dims=wl["dims"], seed=seed)
    N = spec.N
    zeros = torch.zeros(N, dtype=torch.float64, device="cuda")
    op_full = csipm.FFTOperator(csipm.FFTParameters(len(spec.size), spec.size, zeros, 0.0, None))
    x = op_full.M_perp_beta(torch.tensor(spec.beta_true, device="cuda")).cpu().numpy()
    keep = spec.keep
    z0 = np.where(keep, x + spec.noise, 0.0)
    b = op_full.M_perpt_z(torch.tensor(z0, device="cuda"))
    lam = float(spec.lam_factor * b.abs().max().item())
    op_full.close()
    del zeros, b
    missing = np.flatnonzero(~keep).astype(np.int64)
    return spec, z0, lam, missing


# ----------------------------------------------------------------------- ours
def run_ours(args):
    import torch
    import csipm
    from csipm import _native
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    D = Dist(world, rank, local)
    if args.serve_only:
        out = run_serving(args, args.serve_requests, args.serve_slots, rank)
        D.close()
        if rank == 0:
            print(json.dumps(out), flush=True)
        return
    wl = WORKLOADS[args.workload]
    spec, z0_host, lam, missing = build_problem(wl, seed=rank)
    N = spec.N
    L = csipm.lib()

    # resident problem
    z0_dev = torch.tensor(z0_host, device="cuda")
    params = csipm.FFTParameters(len(spec.size), spec.size, z0_dev, lam, missing)
    kw = dict(tol=args.tol)
    if args.cg_rtol is not None:
        kw["ipm_cg_rtol"] = args.cg_rtol
    if args.no_graphs:
        kw["cuda_graphs"] = False
    if args.no_autotune:
        kw["autotune"] = False
    nlp = csipm.FFTNLPModel(params, rdft=True, precision=args.precision, **kw)
    stream = torch.cuda.current_stream()
    if args.passes_only:
        print(json.dumps({"workload": args.workload, "precision": args.precision,
                          "passes": profile_passes(L, nlp, N, reps=1)}), flush=True)
        D.close()
        return
    sol = torch.empty(2 * N, dtype=torch.float64, device="cuda")
    st = _native.Stats()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def solve(model):
        s = L.csipm_solve(model.handle, ctypes.c_void_p(sol.data_ptr()), ctypes.c_void_p(sol.data_ptr() + 8 * N),
                          ctypes.byref(st))
        if s != 0:
            _native.check(s, model.handle)
        return st.as_dict()

    def timed(model, steps, warmup, sample_clocks):
        for _ in range(warmup):
            solve(model)
        stats = []
        clocks = ClockSampler(local, args.clock_log) if sample_clocks else None
        D.barrier()
        torch.cuda.synchronize()
        if clocks:
            clocks.start()
        e0.record(stream)
        for _ in range(steps):
            stats.append(solve(model))
        e1.record(stream)
        torch.cuda.synchronize()
        clk = clocks.stop() if clocks else None
        D.barrier()
        # the residual pass over the timed steps (CUDA events around each
        # launch on the solve's stream, inside the timed region)
        rp = {k: sum(s_[k] for s_ in stats) for k in ("resid_pass_ms", "resid_pass_bytes", "resid_pass_launches")}
        return D.max(e0.elapsed_time(e1) / steps), stats[-1], clk, rp

    ms, last, clk, rp = timed(nlp, args.steps, args.warmup, args.solves_only is False)
    if args.solves_only:
        if rank == 0:
            print(json.dumps({"workload": args.workload, "precision": args.precision, "ms_per_solve": round(ms, 3),
                              "ipm_iter": last["ipm_iter"], "cg_iter": last["cg_iter"], "launches": last["launches"]}),
                  flush=True)
        nlp.op_fft.close()
        D.close()
        return
    beta_main = sol[:N].clone()

    # ---- accuracy oracle: a tight FP64 device solve of the same problem
    # (untimed), and the FP64 path timed beside the headline solve at the
    # same settings (the CPU-twin comparison comes at the end)
    def rel(a, b_):
        return float(torch.linalg.vector_norm(a - b_) / torch.linalg.vector_norm(b_))

    oracle_kw = dict(tol=ORACLE_TOL, ipm_cg_rtol=ORACLE_CG_RTOL)
    nlp_o = csipm.FFTNLPModel(params, rdft=True, precision="fp64", **oracle_kw)
    last_o = solve(nlp_o)
    beta_o = sol[:N].clone()
    nlp_o.op_fft.close()
    accuracy = {
        "oracle": f"FP64 device solve, tol {ORACLE_TOL:g}, Newton rtol {ORACLE_CG_RTOL:g}",
        "beta_rel_err": rel(beta_main, beta_o),
        "lasso_obj_rel_err": abs(last["lasso_obj"] - last_o["lasso_obj"]) / abs(last_o["lasso_obj"]),
        "ipm_iter": last["ipm_iter"], "ipm_iter_oracle": last_o["ipm_iter"],
    }
    accuracy["within_1e-6"] = accuracy["beta_rel_err"] <= 1e-6
    fp64 = None
    if args.precision == "mixed":
        # the plain FP64 GPU path on the same problem at the same settings
        nlp64 = csipm.FFTNLPModel(params, rdft=True, precision="fp64", **kw)
        ms64, last64, _, _ = timed(nlp64, args.steps, args.warmup, False)
        fp64 = {"value": round(ms64 / 1000.0, 5), "tol": args.tol, "newton_cg_rtol": args.cg_rtol,
                "ipm_iter": last64["ipm_iter"], "cg_iter": last64["cg_iter"], "matvecs": last64["matvecs"],
                "beta_rel_err": rel(sol[:N], beta_o), "speedup_mixed_vs_fp64": round(ms64 / ms, 3),
                "what": "FP64 device solve of the same problem with the same options (tol, Newton rtol, forcing)"}
        nlp64.op_fft.close()
    beta_main_host = beta_main.cpu().numpy()
    del beta_main, beta_o

    # ---- end to end through the C ABI with host buffers (pinned), per step:
    # H2D z0, csipm_create (mask from host indices, plans, A^T z0), csipm_solve,
    # D2H beta, csipm_destroy
    z0_pin = torch.tensor(z0_host).pin_memory()
    beta_pin = torch.empty(N, dtype=torch.float64).pin_memory()
    z0_e2e = torch.empty(N, dtype=torch.float64, device="cuda")
    sol_e2e = torch.empty(2 * N, dtype=torch.float64, device="cuda")
    miss = np.ascontiguousarray(missing)

    def e2e_step():
        z0_e2e.copy_(z0_pin, non_blocking=True)
        prob = _native.Problem()
        prob.dim = len(spec.size)
        for d in range(3):
            prob.size[d] = spec.size[d] if d < len(spec.size) else 1
        prob.lam = lam
        prob.z0 = z0_e2e.data_ptr()
        prob.host_missing = miss.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        prob.n_missing = int(miss.size)
        opt = csipm._options(rdft=True, precision=args.precision, **kw)
        h = ctypes.c_void_p()
        _native.check(L.csipm_create(ctypes.byref(prob), ctypes.byref(opt), ctypes.byref(h)))
        s2 = _native.Stats()
        _native.check(L.csipm_solve(h, ctypes.c_void_p(sol_e2e.data_ptr()), None, ctypes.byref(s2)), h)
        beta_pin.copy_(sol_e2e[:N], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        L.csipm_destroy(h)

    e2e_ms = float("nan")
    if not args.no_e2e:
        e2e_step()   # warm
        D.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = D.max(e0.elapsed_time(e1) / args.steps)

    # ---- roofline of the dominant kernel: the residual pass (largest share of
    # the solve in the ncu launch list), timed live inside the timed region;
    # beside it each pass of one CG product timed alone (CUDA events)
    passes = profile_passes(L, nlp, N, reps=10)
    peak, peak_kind = measured_peaks()
    matvec_ms = sum(p["ms"] for p in passes)
    matvec_bytes = sum(p["bytes"] for p in passes)
    rp_launches = max(1, int(rp["resid_pass_launches"]))
    rp_ms = D.max(rp["resid_pass_ms"] / rp_launches)
    rp_bytes = rp["resid_pass_bytes"] / rp_launches
    rp_gbs = rp_bytes / rp_ms / 1e6
    roofline = {
        "bound": "hbm",
        "kernel": "ipm_resdiag_kernel (residual pass: pending step, residual, barrier diagonals, predictor rhs)",
        "achieved": round(rp_gbs, 1),
        "peak": peak,
        "peak_kind": f"{peak_kind} copy bandwidth (the kernel is timed inside the solve)",
        "unit": "GB/s",
        "frac": round(rp_gbs / peak, 4),
        "traffic": ncu_traffic(args.workload, args.precision, "ipm_resdiag_kernel"),
        "algorithmic_bytes_per_launch": round(rp_bytes),
        "ms_per_launch": round(rp_ms, 4),
        "launches_timed": rp_launches,
        "matvec": {"ms": round(matvec_ms, 4), "GBps": round(matvec_bytes / matvec_ms / 1e6, 1),
                   "frac": round(matvec_bytes / matvec_ms / 1e6 / peak, 4),
                   "note": "one CG product, each pass timed alone with CUDA events after the timed region"},
        "passes": [{k: (round(v, 5) if isinstance(v, float) else v) for k, v in p.items()} for p in passes],
    }

    launches = int(last["launches"]) * args.steps
    out = {
        "metric": METRIC if args.workload == "3d320" else f"s-to-solve {args.workload}",
        "value": round(ms / 1000.0, 5),
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 3),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-matvec/f64-ipm",
        "data": "synthetic",
        "config": workload_config(args, wl),
        "e2e": {"value": round(e2e_ms / 1000.0, 5), "unit": "s", "h2d_bytes_per_step": int(8 * N + 8 * miss.size),
                "d2h_bytes_per_step": int(8 * N),
                "includes": "H2D z0 + csipm_create (mask, plans, A^T z0) + csipm_solve + D2H beta + destroy"},
        "solve": {"ipm_iter": last["ipm_iter"], "cg_iter": last["cg_iter"], "matvecs": last["matvecs"],
                  "refinements": last["refinements"], "fallbacks": last["fallbacks"], "gap": last["gap"], "obj": last["obj"],
                  "status": last["status"]},
        "roofline": roofline,
        "accuracy": accuracy,
        "fp64": fp64,
        "gpu_launches": launches,
        "clocks": clk,
    }
    nlp.op_fft.close()
    del z0_dev, sol, sol_e2e, z0_e2e
    torch.cuda.empty_cache()
    if not args.no_legs:
        out["legs"] = {name: run_leg(args, name, rank) for name in LEGS if name != args.workload}
    if args.serve_requests > 0:
        out["serving"] = run_serving(args, args.serve_requests, args.serve_slots, rank)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        twin = cpu_twin_solve(spec.size, spec.keep, z0_host, lam, args.tol, args.cg_rtol)
        out["cpu_baseline"] = twin["cpu_baseline"]
        out["accuracy"]["vs_cpu_twin"] = twin_accuracy(twin, beta_main_host, last, z0_host, lam)
    D.close()
    if rank == 0:
        print(json.dumps(out), flush=True)


# ----------------------------------------------------------------------- legs
def run_leg(args, name, rank):
    """One more measured configuration, FP64, at the headline's settings: the
    solve timed with CUDA events (a few steps), its counts, the residual pass
    and each pass of one CG product (roofline), and beta against the CPU twin
    (1D, 2D) or a tight FP64 device solve (3D 256^3: the twin would take
    minutes)."""
    import torch
    import csipm
    from csipm import _native
    wl = WORKLOADS[name]
    spec, z0_host, lam, missing = build_problem(wl, seed=rank)
    N = spec.N
    L = csipm.lib()
    z0_dev = torch.tensor(z0_host, device="cuda")
    params = csipm.FFTParameters(len(spec.size), spec.size, z0_dev, lam, missing)
    nlp = csipm.FFTNLPModel(params, rdft=True, precision="fp64", tol=args.tol, ipm_cg_rtol=args.cg_rtol)
    sol = torch.empty(N, dtype=torch.float64, device="cuda")
    st = _native.Stats()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def solve(model):
        _native.check(L.csipm_solve(model.handle, ctypes.c_void_p(sol.data_ptr()), None, ctypes.byref(st)),
                      model.handle)
        return st.as_dict()

    steps = max(1, min(args.steps, 5))
    for _ in range(max(1, min(args.warmup, 3))):
        solve(nlp)
    stats = []
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        stats.append(solve(nlp))
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    last = stats[-1]
    beta = sol.cpu().numpy()
    peak, peak_kind = measured_peaks()
    rp_ms = sum(x["resid_pass_ms"] for x in stats) / max(1, sum(x["resid_pass_launches"] for x in stats))
    rp_bytes = sum(x["resid_pass_bytes"] for x in stats) / max(1, sum(x["resid_pass_launches"] for x in stats))
    passes = profile_passes(L, nlp, N, reps=10)
    mv_ms = sum(p["ms"] for p in passes)
    mv_bytes = sum(p["bytes"] for p in passes)
    leg = {
        "workload": workload_config(args, wl)["workload"].replace(args.precision, "fp64"),
        "value": round(ms / 1000.0, 6), "unit": "s", "steps": steps, "precision": "fp64",
        "ipm_iter": last["ipm_iter"], "cg_iter": last["cg_iter"], "matvecs": last["matvecs"], "gap": last["gap"],
        "roofline": {
            "resid_pass": {"ms": round(rp_ms, 5), "GBps": round(rp_bytes / rp_ms / 1e6, 1),
                           "frac": round(rp_bytes / rp_ms / 1e6 / peak, 4)},
            "cg_product": {"ms": round(mv_ms, 5), "GBps": round(mv_bytes / mv_ms / 1e6, 1),
                           "frac": round(mv_bytes / mv_ms / 1e6 / peak, 4),
                           "passes": [{k: (round(v, 5) if isinstance(v, float) else v) for k, v in p.items()}
                                      for p in passes]},
            "peak": peak, "peak_kind": peak_kind,
            "note": "small grids stream from L2 (126 MB): fractions of the HBM copy rate above 1 are L2 reads"},
    }
    if wl["kind"] in ("1d", "2d"):
        twin = cpu_twin_solve(spec.size, spec.keep, z0_host, lam, args.tol, args.cg_rtol)
        leg["accuracy"] = twin_accuracy(twin, beta, last, z0_host, lam)
        leg["cpu_baseline"] = twin["cpu_baseline"]
    else:
        o = csipm.FFTNLPModel(params, rdft=True, precision="fp64", tol=ORACLE_TOL, ipm_cg_rtol=ORACLE_CG_RTOL)
        solve(o)
        bo = sol.cpu().numpy()
        leg["accuracy"] = {"oracle": f"FP64 device solve, tol {ORACLE_TOL:g}, Newton rtol {ORACLE_CG_RTOL:g}",
                           "beta_rel_err": float(np.linalg.norm(beta - bo) / np.linalg.norm(bo))}
        o.op_fft.close()
    nlp.op_fft.close()
    del z0_dev, sol
    torch.cuda.empty_cache()
    return leg


# ----------------------------------------------------------------------- serving
MAX_1D = 2 ** 20
SERVE_CG_RTOL = 1e-3


def serving_problems(n, seed0=1000):
    """The serving stream's requests: seeded specs (csipm.problems.serving_spec),
    synthesised and scaled with the library's own unmasked operator."""
    import torch
    import csipm
    import csipm.problems as P
    out = []
    for k in range(n):
        spec, precision = P.serving_spec(seed0 + k, max_1d=MAX_1D)
        zeros = torch.zeros(spec.N, dtype=torch.float64, device="cuda")
        op = csipm.FFTOperator(csipm.FFTParameters(len(spec.size), spec.size, zeros, 0.0, None))
        x = op.M_perp_beta(torch.tensor(spec.beta_true, device="cuda")).cpu().numpy()
        z0 = np.where(spec.keep, x + spec.noise, 0.0)
        lam = float(spec.lam_factor * op.M_perpt_z(torch.tensor(z0, device="cuda")).abs().max().item())
        op.close()
        out.append(dict(size=spec.size, z0=z0, lam=lam, missing=np.flatnonzero(~spec.keep).astype(np.int64),
                        precision=precision, kind=spec.name))
    return out


def run_serving(args, n_req, slots, rank):
    """Sequential plain solves of the stream (one request at a time through the
    C ABI from host buffers: create, solve, D2H, destroy) against the serving
    loop: closed runs (all requests at t=0: capacity) with each request's
    iterations as plain launches and as one graph launch, then a Poisson run
    of the faster mode at 80% of its closed capacity (latency under a load the
    loop sustains)."""
    import torch
    import csipm
    from csipm import _native
    from csipm.serving import Server
    reqs = serving_problems(n_req, seed0=1000 + 100000 * rank)
    L = csipm.lib()
    # every request is solved to a relative duality gap of 1e-8; the serving
    # loop uses inexact Newton solves (CG rtol 1e-3), robust on this mix; the
    # stream's sizes hardly repeat, so per-size autotuning could not amortise
    opts = dict(tol=1e-8, ipm_cg_rtol=SERVE_CG_RTOL, autotune=False)

    def sequential(kw):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        status = []
        per_kind = {"1d": 0.0, "2d": 0.0, "3d": 0.0}
        for r in reqs:
            t1 = time.perf_counter()
            n = int(np.prod(r["size"]))
            z0d = torch.tensor(r["z0"], device="cuda")
            beta = torch.empty(n, dtype=torch.float64, device="cuda")
            params = csipm.FFTParameters(len(r["size"]), r["size"], z0d, r["lam"], r["missing"])
            nlp = csipm.FFTNLPModel(params, rdft=True, precision=r["precision"], **kw)
            st = _native.Stats()
            status.append(L.csipm_solve(nlp.handle, ctypes.c_void_p(beta.data_ptr()), None, ctypes.byref(st)))
            beta.cpu()
            nlp.op_fft.close()
            per_kind[r["kind"]] += time.perf_counter() - t1
        torch.cuda.synchronize()
        total = time.perf_counter() - t0
        return n_req / total, int(sum(s != 0 for s in status)), {k: round(v / total, 3) for k, v in per_kind.items()}

    # the sequential baseline: each request solved alone, with and without the
    # whole-iteration graph (captured per request); the faster is the baseline
    seq_graph_rate, seq_graph_failed, seq_graph_share = sequential(dict(opts, cuda_graphs=True))
    seq_plain_rate, seq_plain_failed, seq_plain_share = sequential(dict(opts, cuda_graphs=False))
    seq_rate = max(seq_graph_rate, seq_plain_rate)

    def serve(rate, graphs, batch=1, nslots=slots, batch_max_n=0):
        rng = np.random.default_rng(7)
        gaps = rng.exponential(1.0 / rate, size=n_req) if rate else np.zeros(n_req)
        arrivals = np.cumsum(gaps) - gaps[0]
        res = []
        with Server(slots=nslots, cuda_graphs=graphs, batch=batch, batch_max_n=batch_max_n) as srv:
            t_start = time.perf_counter()
            for k, r in enumerate(reqs):
                while True:
                    wait = arrivals[k] - (time.perf_counter() - t_start)
                    if wait <= 0:
                        break
                    res.extend(srv.poll(timeout_ms=0))
                    time.sleep(min(wait, 0.002))
                srv.submit(r["size"], r["z0"], r["lam"], r["missing"], tag=k, precision=r["precision"], **opts)
            res.extend(srv.drain())
            t_end = time.perf_counter()
        lat = np.array([x.latency_ms for x in res])
        # slot time (admission to result) by kind, as a share of all slot time
        busy = {k: sum(x.latency_ms - x.queue_ms for x in res if reqs[x.tag]["kind"] == k) for k in ("1d", "2d", "3d")}
        tot = max(1e-9, sum(busy.values()))
        return {"solves_per_s": round(n_req / (t_end - t_start), 2),
                "p50_ms": round(float(np.percentile(lat, 50)), 2), "p99_ms": round(float(np.percentile(lat, 99)), 2),
                "failed": int(sum(x.status != 0 for x in res)),
                "failures": sorted({x.message for x in res if x.status != 0})[:3],
                "mean_group": round(float(np.mean([x.group for x in res])), 2),
                "slot_time_share": {k: round(v / tot, 3) for k, v in busy.items()}}

    # untimed: the first slots' worth of requests through the server, one at
    # a time and batched (device memory pool and kernel set-up warm, as in a
    # running service)
    batch = int(getattr(args, "serve_batch", 1))
    bslots = int(getattr(args, "serve_batch_slots", slots))
    bmax = int(getattr(args, "serve_batch_max_n", 0))
    for warm_batch, warm_slots in (((1, slots), (batch, bslots)) if batch > 1 else ((1, slots),)):
        with Server(slots=warm_slots, batch=warm_batch) as srv:
            for k, r in enumerate(reqs[:max(warm_slots, 4 * warm_batch)]):
                srv.submit(r["size"], r["z0"], r["lam"], r["missing"], tag=k, precision=r["precision"], **opts)
            srv.drain()
    closed_plain = serve(0.0, False)
    closed_graphs = serve(0.0, True)
    closed_batched = None
    if batch > 1:
        # untimed: one closed pass of the whole stream in batches first (the
        # one-at-a-time modes are warm from the sequential runs: every kernel
        # loaded, the memory pool grown to what their peak holds; batches hold
        # more handles at once)
        serve(0.0, False, batch, bslots, bmax)
        closed_batched = serve(0.0, False, batch, bslots, bmax)
    # the fastest closed mode sets the Poisson run's mode and offered rate
    modes = [(closed_plain, False, 1, slots, 0), (closed_graphs, True, 1, slots, 0)]
    if closed_batched:
        modes.append((closed_batched, False, batch, bslots, bmax))
    closed, graphs, pbatch, pslots, pbmax = max(modes, key=lambda m: m[0]["solves_per_s"])
    offered = 0.8 * closed["solves_per_s"]
    poisson = serve(offered, graphs, pbatch, pslots, pbmax)
    kinds = {k: sum(1 for r in reqs if r["kind"] == k) for k in ("1d", "2d", "3d")}
    return {
        "requests": n_req, "slots": slots, "mix": kinds,
        "sizes": "1D N in [2^12, %d], 2D sides in [128, 1024], 3D sides in [32, 128], log-uniform, factors 2/3/5; "
                 "0.5-5%% sparsity; 5-20%% missing; FP64 or mixed per request; relative gap 1e-8" % MAX_1D,
        "newton_cg_rtol": SERVE_CG_RTOL,
        "sequential_plain": {"solves_per_s": round(seq_rate, 2),
                             "failed": seq_graph_failed if seq_graph_rate >= seq_plain_rate else seq_plain_failed,
                             "what": "one request at a time through create/solve/D2H/destroy, same options; the "
                                     "faster of plain launches and the per-request iteration graph",
                             "graph_launches": {"solves_per_s": round(seq_graph_rate, 2), "time_share": seq_graph_share},
                             "plain_launches": {"solves_per_s": round(seq_plain_rate, 2), "time_share": seq_plain_share}},
        "batched_closed": dict(closed, cuda_graphs=graphs, batch=pbatch, slots=pslots),
        "batched_closed_plain_launches": closed_plain,
        "batched_closed_graph_launches": closed_graphs,
        "batched_closed_solve_batch": (dict(closed_batched, batch=batch, slots=bslots, batch_max_n=bmax,
                                            what="each slot solves up to `batch` admitted requests of one batch "
                                                 "class together (csipm_solve_batch, FP64); requests above "
                                                 "batch_max_n samples alone")
                                       if closed_batched else None),
        "batched_poisson": dict(poisson, offered_per_s=round(offered, 2), cuda_graphs=graphs, batch=pbatch,
                                slots=pslots),
        "speedup_vs_sequential": round(closed["solves_per_s"] / seq_rate, 2),
    }


# ----------------------------------------------------------------------- CPU twin (oracle)
def cpu_twin_solve(size, keep, z0, lam, tol, cg_rtol, on_iter=None):
    """One complete FP64 CPU solve of the problem with the oracle's twin of the
    device method (oracle_ipm.ipm: numpy elementwise work, scipy.fft pocketfft
    products with one worker per host core), timed end to end from A^T z0 to
    beta.  Returns beta, the twin's info and the cpu_baseline object."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import oracle_ipm as OI
    cores = os.cpu_count() or 1
    op = O.Operator(size, keep, True, workers=cores)
    op.AtA(np.zeros(int(np.prod(size))))   # pocketfft plan set-up, untimed
    op.n_matvec, op.t_matvec = 0, 0.0
    t0 = time.perf_counter()
    b = op.At(z0)
    beta, _, info = OI.ipm(op, b, lam, float(z0 @ z0), tol=tol, cg_rtol=cg_rtol, on_iter=on_iter)
    total = time.perf_counter() - t0
    t_cg_vec = info["t_newton"] - info["t_newton_products"]
    grid = "x".join(map(str, size))
    return {
        "beta": beta, "info": info, "op": op, "seconds": total,
        "cpu_baseline": {
            "value": round(total, 3), "unit": "s", "cores": cores, "kind": "port",
            "sample": (f"one complete FP64 CPU solve of the same {grid} problem, measured end to end (not "
                       f"extrapolated): the oracle's twin of the device method (numpy elementwise work on one "
                       f"core, scipy.fft pocketfft products with workers={cores}) at the same tol {tol:g}, "
                       f"Newton rtol {cg_rtol:g} and forcing term; {info['ipm_iter']} IPM iterations, "
                       f"{info['cg_iter']} CG iterations, {op.n_matvec} products ({op.t_matvec:.1f} s), CG vector "
                       f"work {t_cg_vec:.1f} s, IPM elementwise work {total - op.t_matvec - t_cg_vec:.1f} s"),
            "status": info["status"],
        },
    }


def twin_accuracy(twin, beta_gpu, stats, z0, lam):
    """beta, the LASSO objective and the iteration count of a device solve
    against the CPU twin of the same problem."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_ipm as OI
    bc = twin["beta"]
    Fg = OI.lasso_value(twin["op"], beta_gpu, z0, lam)
    Fc = OI.lasso_value(twin["op"], bc, z0, lam)
    rel = float(np.linalg.norm(beta_gpu - bc) / np.linalg.norm(bc))
    return {"oracle": "FP64 CPU twin solve of the same problem (oracle_ipm.ipm), same settings",
            "beta_rel_err": rel, "lasso_obj_rel_err": abs(Fg - Fc) / abs(Fc),
            "ipm_iter": stats["ipm_iter"], "ipm_iter_twin": twin["info"]["ipm_iter"],
            "within_1e-6": rel <= 1e-6}


def run_reference(args):
    """The reference arm: the reference's path on the host cores.  Julia,
    MadNLP and FFTW are not installed, so it is the oracle's FP64 twin of the
    path (same maps, operator, condensed KKT and IPM algorithm) on the same
    workload and settings as the GPU arm.  The warm-up builds the problem and
    sets up the FFT plans; then ONE complete solve is measured end to end,
    one IPM iteration per step (a solve that needs more iterations than
    --steps runs them all; each iteration's seconds are listed), so `value`
    is a measured s-to-solve, not an extrapolation."""
    world, rank, local = dist_setup(args)
    if rank != 0:
        return
    wl = WORKLOADS[args.workload]
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import csipm.problems as P
    cores = os.cpu_count() or 1
    spec = P.make_spec(wl["kind"], dims=wl["dims"], seed=0)
    opf = O.Operator(spec.size, None, True, workers=cores)
    prob = P.finalize(spec, opf.A, opf.At)
    del opf
    marks = []
    t_start = [None]

    def on_iter(k, gap):
        marks.append(time.perf_counter())

    t_start[0] = time.perf_counter()
    twin = cpu_twin_solve(spec.size, spec.keep, prob.z0, prob.lam, args.tol, args.cg_rtol, on_iter=on_iter)
    v = twin["seconds"]
    # seconds of each step: A'z0 + warm start + the first stop test, then one IPM iteration each
    iters = [round(b_ - a_, 3) for a_, b_ in zip([t_start[0]] + marks[:-1], marks)]
    out = {
        "impl": "reference",
        "metric": METRIC if args.workload == "3d320" else f"s-to-solve {args.workload}",
        "value": round(v, 3),
        "unit": "s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1000.0 * v / max(1, len(iters)), 1),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(args, wl),
        "measured": {"what": "one complete CPU solve, one IPM iteration per step (step 1 also holds A^T z0 and "
                             "the warm start); value = the whole solve",
                     "solve_steps": len(iters), "step_s": iters, "ipm_iter": twin["info"]["ipm_iter"],
                     "cg_iter": twin["info"]["cg_iter"], "products": twin["op"].n_matvec,
                     "status": twin["info"]["status"]},
        "cpu_baseline": twin["cpu_baseline"],
        "e2e": {"value": round(v, 3), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
