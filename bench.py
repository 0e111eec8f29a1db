"""Benchmark of the RK3 step of the 2-D MHD solver on B200.

Metric: cell-updates/s (nx*ny*steps / s; one update = one full RK3 step:
three stages including the compact/spectral filter), FP64.

Default workload: Alfvenic turbulence on a 4096 x 4096 periodic grid
(box 20pi x 20pi, rho = 1, B0 = 1 along x, beta = 0.5, d_i = 0.1,
eta = nu = 2e-4, dt = 2e-4), the configuration the reference's headline metric
is quoted on; synthetic seeded initial condition (seed 1).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one process per GPU, each advancing its own
replica of the domain (the whole domain lives on one GPU: replicas only, no
collective on the data path); the timing is the max over ranks.

`--impl reference` times the reference's own C implementation of the path
(compiled from its sources into oracle/_ref/mhd_ref) on the host cores, on the
same grid: P concurrent independent single-rank processes (P = min(cores,
--steps, what host memory holds at ~8.6 GB per 4096^2 process)), each timing
one RK3 step of the full grid; the same sample is the GPU arm's cpu_baseline.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s"
UNIT = "cell-updates/s"
DT = 2e-4


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while the
    timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        rows = [ln.split(",") for ln in self.out.read().splitlines() if ln.strip()]
        os.unlink(self.out.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# the reference's CPU path (oracle/_ref/mhd_ref) on the bench workload itself
# ---------------------------------------------------------------------------
def host_mem_available():
    """MemAvailable of /proc/meminfo in bytes (None where unreadable)."""
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return None


def ref_process_bytes(nx, ny):
    """Host bytes of one single-rank reference process on an nx x ny grid:
    about 62 field-sized arrays (initialize.c:216-320 with eta, nu > 0) plus
    the state it reads, rounded up to 64 fields."""
    return 64 * nx * ny * 8 + (nx * ny * 8 * 8)


def cpu_processes(nx, ny, want=None):
    """Concurrent reference processes: one per host core, at most `want`,
    and no more than 75 % of the available host memory holds."""
    n = os.cpu_count() or 1
    if want is not None:
        n = min(n, want)
    mem = host_mem_available()
    if mem is not None:
        n = min(n, int(0.75 * mem // ref_process_bytes(nx, ny)))
    return max(1, n)


def workload(args, nx, ny):
    """(params, state, dt, name) of the bench workload at nx x ny."""
    from mhd2dcfdfftw_open_b200 import ic
    if args.workload == "parametric":  # parametric decay of an Alfven pump, dt 5e-4
        p, uu = ic.parametric_decay(nx, ny)
        return p, uu, 5e-4, "parametric_decay"
    p, uu = ic.alfvenic_turbulence(nx, ny)  # Alfvenic turbulence, dt 2e-4
    return p, uu, DT, "alfvenic_turbulence"


def run_reference_sample(args, nproc, nsteps=1, timeout=1800):
    """`nproc` concurrent single-rank processes of the reference's C code,
    each on the bench workload's full nx x ny grid from the same initial
    state: set-up and state load untimed, then `nsteps` timed RK3 steps,
    started together (a go file releases every process once all are ready).
    Returns (aggregate cell-updates/s, slowest process's seconds, results)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref  # the checker's build of the reference (test infrastructure)
    from mhd2dcfdfftw_open_b200.dumpio import write_state

    if not os.path.exists(ref.BIN_PATH):
        raise RuntimeError("oracle/_ref/mhd_ref is not built")
    nx, ny = args.nx, args.ny
    p, uu, dt, _ = workload(args, nx, ny)
    with tempfile.TemporaryDirectory(prefix="mhdcpu_") as wd:
        p.write(os.path.join(wd, "input"))
        icp = os.path.join(wd, "ic.dat")
        write_state(icp, uu)
        del uu
        go = os.path.join(wd, "go")
        procs = [subprocess.Popen([ref.BIN_PATH, wd, icp, str(nsteps), repr(dt), "-", "0", go],
                                  stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                 for _ in range(nproc)]
        try:
            t_end = time.time() + timeout
            for pr in procs:  # every process has set up and loaded the state
                while True:  # the reference prints a banner of its own first
                    line = pr.stdout.readline()
                    if not line or time.time() > t_end:
                        raise RuntimeError("a reference process did not get ready")
                    if line.strip() == "READY":
                        break
            open(go, "w").close()
            res = []
            for pr in procs:
                out, _ = pr.communicate(timeout=max(1.0, t_end - time.time()))
                line = [ln for ln in out.splitlines() if ln.startswith("{")][-1]
                res.append(json.loads(line))
        finally:
            for pr in procs:
                if pr.poll() is None:
                    pr.kill()
    tmax = max(r["seconds"] for r in res)
    agg = nproc * nx * ny * nsteps / tmax
    return agg, tmax, res


def reference_sample_text(args, nproc, tmax, nsteps=1):
    name = workload_name(args)
    return (f"{name} {args.nx}x{args.ny} (the full bench grid), {nsteps} RK3 step in each of "
            f"{nproc} concurrent independent single-rank processes of the reference's C code "
            f"(oracle/_ref/mhd_ref), started together; slowest process {tmax:.1f} s per step; "
            f"set-up untimed; no warm-up step, the stage arrays' pages written once before "
            f"timing instead (a first step's page faults excluded); FP64")


def workload_name(args):
    return "parametric_decay" if args.workload == "parametric" else "alfvenic_turbulence"


def arm_config(args, world):
    """The `config` object both arms print for the same workload."""
    cells = float(args.nx) * args.ny
    name = workload_name(args)
    return {"workload": f"{name}_{args.nx}x{args.ny}_{'mixed' if args.precision == 'mixed' else 'fp64'}",
            "nx": args.nx, "ny": args.ny, "precision": args.precision,
            "dt": 5e-4 if args.workload == "parametric" else DT, "path": args.path,
            "parallelism": f"replicas{world}",
            "l2": f"inputs larger than L2 (state alone is {8 * cells * 8 / 1e9:.2f} GB)"}


def data_label(args):
    return ("synthetic (seeded parametric-decay IC, seed 3)" if args.workload == "parametric"
            else "synthetic (seeded Alfvenic turbulence IC, seed 1)")


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def algorithmic_model_bytes():
    """Minimal-pass FP64 traffic model of one cell-update (one RK3 step):
    per stage, x pass 8 read + 16 written, y pass 32 read + 16 written, x and
    y filters 16 each: 104 doubles = 832 B per stage, 2496 B per step."""
    return 2496.0


def traffic_per_launch(kclass):
    """DRAM bytes per launch of a kernel class at the bench workload, from the
    committed ncu summary profiles/ncu_traffic.txt (lines `class bytes`), or
    None when it has no figure for the class."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and parts[0] == kclass:
                    return float(parts[1])
    except OSError:
        pass
    return None


def max_over_ranks(x, dist, device):
    """The largest of the ranks' values of x (every rank calls it, in the
    same order); x itself without a process group."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, cells, steps, seconds):
    """Whole-job cell-updates/s of `world` independent replicas of `cells`
    cells advanced `steps` steps, timed by the slowest rank (seconds)."""
    return world * cells * steps / seconds


def run_ours(args):
    rank, local, world = env_rank()
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from mhd2dcfdfftw_open_b200 import ic
    from mhd2dcfdfftw_open_b200.solver import Domain

    nx, ny = args.nx, args.ny
    p, uu, dt, _ = workload(args, nx, ny)
    fused = args.path == "fused"
    dom = Domain(p, uu, device=local)
    mixed = args.precision == "mixed"
    if mixed:
        dom.set_precision(True)
    stream = torch.cuda.ExternalStream(dom.stream_handle(), device=local)

    def barrier():
        if dist is not None:
            dist.barrier()

    # warm-up steps (untimed)
    dom.steps(args.warmup, dt, fused=fused)
    barrier()
    torch.cuda.synchronize()
    dom.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    dom.profile(True)
    l0 = dom.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dom.steps(args.steps, dt, fused=fused)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    launches = dom.launch_count() - l0
    ms = e0.elapsed_time(e1)
    prof = dom.profile_read()
    dom.profile(False)
    ms = max_over_ranks(ms, dist, f"cuda:{local}")
    cells = float(nx) * ny
    value = replica_value(world, cells, args.steps, ms / 1e3)

    # end to end through the C ABI with host buffers: every step uploads the
    # state from pinned host memory, advances one RK3 step and reads the state
    # back into pinned host memory.  The fused path streams the steps' states
    # through mhdgpu_steps_fused_stream, which overlaps the upload of the next
    # state and the download of the previous one with the current step.
    ke = max(1, min(args.steps, args.e2e_steps))
    h_in = torch.from_numpy(np.ascontiguousarray(dom.get("uu"))).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    nin, nout = h_in.numpy(), h_out.numpy()
    if fused:
        dom.steps_stream([nin], [nout], 1, dt)
    else:
        dom.set("uu", nin)
        dom.steps(1, dt, fused=fused)
    barrier()
    t0 = time.perf_counter()
    if fused:
        dom.steps_stream([nin] * ke, [nout] * ke, 1, dt)
    else:
        for _ in range(ke):
            dom.set("uu", nin)
            dom.steps(1, dt, fused=fused)
            dom.get("uu", out=nout)
    t_e2e = time.perf_counter() - t0
    t_e2e = max_over_ranks(t_e2e, dist, f"cuda:{local}")
    e2e = replica_value(world, cells, ke, t_e2e)
    nbytes = nin.nbytes
    dom.close()

    # mixed precision: its error against the FP64 steps from the same state
    mixed_error = None
    if mixed:
        runs = []
        for mx in (False, True):
            with Domain(p, uu, device=local) as d:
                d.set_precision(mx)
                d.steps(args.warmup + args.steps, dt, fused=fused)
                runs.append(d.get("uu"))
        ref, mix = runs
        per = []
        for v in range(ref.shape[0]):
            den = float(np.linalg.norm(ref[v]))
            if den < 1e-8 * float(np.linalg.norm(ref)):
                den = float(np.linalg.norm(ref))
            per.append(float(np.linalg.norm(mix[v] - ref[v]) / den))
        tot = float(np.linalg.norm(ref))
        per_state = [float(np.linalg.norm(mix[v] - ref[v]) / tot) for v in range(ref.shape[0])]
        mixed_error = {"rel_l2_per_field": per, "rel_l2_max": max(per),
                       "l2_vs_state_norm_per_field": per_state,
                       "steps": args.warmup + args.steps,
                       "against": "FP64 fused steps on the GPU (which match the reference to 1e-12)"}

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    peak, peak_kind = measured_peaks()
    dom_cls = max(prof, key=lambda k: prof[k][0])
    tot_ms, nl, byts = prof[dom_cls]
    achieved = byts / (tot_ms / 1e3) / 1e9 if tot_ms > 0 else 0.0
    tr = traffic_per_launch(dom_cls)
    roofline = {"kernel": dom_cls, "bound": "hbm", "achieved": round(achieved, 1),
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "traffic": tr,
                "algorithmic_bytes_per_launch": byts / max(nl, 1),
                "avg_launch_ms": tot_ms / max(nl, 1), "launches": nl,
                "share_of_step": round(tot_ms / ms, 3)}
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 sweeps/FFT/fluxes, f64 state" if mixed else "f64",
        "data": data_label(args),
        "config": arm_config(args, world),
        "roofline": roofline,
        "model_fraction": {"bytes_per_cell_update": algorithmic_model_bytes(),
                           "frac": round(value / world * algorithmic_model_bytes() / (peak * 1e9), 4)},
        "kernel_classes": {k: {"ms": round(v[0], 3), "launches": v[1]} for k, v in prof.items() if v[1]},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes, "steps": ke,
                "mode": ("mhdgpu_steps_fused_stream: each step a state uploaded from pinned host "
                         "memory, stepped once and downloaded; transfers overlap the "
                         "neighbouring states' steps") if fused else
                        "mhdgpu_set_array, mhdgpu_steps, mhdgpu_get_array per step"},
        "gpu_launches": launches,
        **({"mixed_error": mixed_error} if mixed_error else {}),
        "clocks": clocks,
    }
    if world == 1 and not args.no_cpu_baseline:
        try:
            nproc = cpu_processes(nx, ny, want=args.cpu_procs)
            agg, tmax, _ = run_reference_sample(args, nproc)
            out["cpu_baseline"] = {"value": agg, "unit": UNIT, "cores": nproc, "kind": "reference",
                                   "sample": reference_sample_text(args, nproc, tmax)}
        except Exception as e:  # reported, not hidden
            out["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def run_reference(args):
    """The reference's CPU implementation of the path on the bench workload's
    own grid: min(cores, --steps, memory) concurrent processes, one timed RK3
    step of the full grid each (the --steps requested full-grid steps would
    take about a minute each on one core)."""
    rank, _, world = env_rank()
    if rank != 0:
        return
    nproc = cpu_processes(args.nx, args.ny, want=min(args.steps, args.cpu_procs or 1 << 30))
    agg, tmax, _ = run_reference_sample(args, nproc)
    out = {
        "metric": METRIC, "value": agg, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tmax * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": data_label(args),
        "config": arm_config(args, world),
        "impl": "reference",
        "timed": {"processes": nproc, "steps_per_process": 1, "warmup_steps": 0,
                  "grid": [args.nx, args.ny], "same_config": True},
        "cpu_baseline": {"value": agg, "unit": UNIT, "cores": nproc, "kind": "reference",
                         "sample": reference_sample_text(args, nproc, tmax)},
        "e2e": {"value": agg, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--path", choices=["fused", "operators"], default="fused")
    ap.add_argument("--nx", type=int, default=4096)
    ap.add_argument("--ny", type=int, default=4096)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--workload", choices=["turbulence", "parametric"], default="turbulence")
    ap.add_argument("--cpu-procs", type=int, default=None,
                    help="at most this many concurrent reference processes on the host")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
