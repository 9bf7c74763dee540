#!/usr/bin/env python
"""Benchmark of the SL-BDF2 channel step (slchannel_b200) on B200s.

Workload: slChannel's plain float64 SL-BDF2 step at 256^3 -- staggered MAC
channel 4pi x 2pi x 2, tanh gamma = 2.0, Re_b = 2792.8 (nu = 1/2792.8), bulk
velocity 1, triquintic (order 6), fixed dt = 0.01 -- from a seeded synthetic
field: Poiseuille 1.5 z (2 - z) plus the curl of a seeded random vector
potential (|k| <= 8, damped by z^2 (2-z)^2, u'_rms = 0.1), bulk-rescaled and
projected; one BDF1 bootstrap step precedes the timed BDF2 steps.

    python bench.py [--gpus N --steps K --warmup W]      # this implementation
    python bench.py --impl reference [...]               # CPU reference arm

Multi-GPU: the single-channel step does not shard (replicas only): each rank
advances its own channel; value = total steps over all ranks / max rank time.

One JSON line on rank 0 (see the fields below).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "SL steps/s at 256^3: mixed vs FP64 form at stated error; gather HBM GB/s"
UNIT = "steps/s"
LX, LY, LZ = 4 * math.pi, 2 * math.pi, 2.0
GAMMA = 2.0
RE_B = 2792.8
DT = 0.01
MIXED_ERROR_STEPS = 20


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n", "--size", dest="n", type=int, default=256,
                    help="grid points per direction (--size is the same option, for launchers "
                         "such as torchrun whose own options --n abbreviates)")
    ap.add_argument("--order", type=int, default=6)
    ap.add_argument("--e2e-steps", type=int, default=30)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision form")
    ap.add_argument("--mixed-error-steps", type=int, default=20)
    ap.add_argument("--no-other-order", action="store_true",
                    help="skip the FP64 step at the other interpolation order (4 <-> 6)")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 48-channel ensemble form")
    ap.add_argument("--ensemble-n", type=int, default=48)
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint rollout check")
    ap.add_argument("--no-schemes", action="store_true",
                    help="skip the SL vs Eulerian per-time-unit comparison")
    ap.add_argument("--adjoint-fd-dirs", type=int, default=16)
    ap.add_argument("--mixed-report", action="store_true",
                    help="instead of the bench line: the mixed form against the FP64 form over "
                         "--report-steps steps on --report-grid (JSON lines)")
    ap.add_argument("--report-grid", type=int, nargs=3, default=[512, 384, 384])
    ap.add_argument("--report-steps", type=int, default=1000)
    ap.add_argument("--report-every", type=int, default=100)
    ap.add_argument("--report-re", type=float, default=2800.0, help="Re key (nu = 1/Re)")
    ap.add_argument("--report-dt", type=float, default=0.005)
    ap.add_argument("--report-urms", type=float, default=0.12)
    ap.add_argument("--gather-compare", action="store_true",
                    help="instead of the bench line: time the L1 trace+gather "
                         "(slc_trace_gather_bdf2) against the TMA-staged one "
                         "(slc_trace_gather_bdf2_staged) on the --n^3 benchmark state and on a "
                         "128^3 channel at trajectory CFL 3 (JSON lines)")
    ap.add_argument("--gather-probe", action="store_true",
                    help="instead of the bench line: the order-6 FP32 gather by one thread per "
                         "point against the tensor-core (mma.sync FP16x3) formulation on a "
                         "synthetic --n^3 problem (slc_gather_probe; JSON line)")
    ap.add_argument("--cpu-budget-s", type=float, default=20.0,
                    help="CPU seconds the cpu_baseline sample aims for")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (replicas: no collective on the data path)
# ---------------------------------------------------------------------------

def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def dist_init(world, backend):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist

    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
    return dist


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        try:
            import tempfile

            fd, self.path = tempfile.mkstemp(prefix="slc_clocks_", suffix=".csv")
            os.close(fd)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                   "-lms", "200"]
            if self.gpu_id is not None:
                cmd += ["-i", str(self.gpu_id)]
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "samples": len(sm),
                "power_w_max": max(power) if power else None, "reasons": sorted(reasons)}


def gpu_smi_id(dev_index):
    import torch

    try:
        p = torch.cuda.get_device_properties(dev_index)
        return f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v for v in vis.split(",") if v.strip()]
        return ids[dev_index] if dev_index < len(ids) else None


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------

def config(n, order, precision="fp64"):
    return {
        "grid": {"nx": n, "ny": n, "nz": n},
        "domain": {"Lx": LX, "Ly": LY, "Lz": LZ, "stretching_type": "symmetric"},
        "flow": {"Re": RE_B, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": GAMMA},
        "boundary_conditions": {"top_wall": {"type": "dirichlet"}},
        "initialization": {"type": "parabolic"},
        "time": {"dt": DT, "dt_update_interval": 0},
        "compute": {"device": "cuda"},
        "sl": {"interp_order": order, "n_traj_iters": 2, "interp_dtype": precision},
    }


def bench_config(n, order, world):
    """The `config` object of the JSON line -- the same for both arms."""
    return {"workload": f"SL-BDF2 step {n}^3 (4pi x 2pi x 2), Re_b {RE_B}, dt {DT}, order {order}, "
                        f"FP64, seeded synthetic field (u'_rms 0.1)",
            "grid": [n, n, n], "order": order, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (state ~1.8 GB at 256^3), no flush"}


def initial_field(n, z_f, z_c, seed=0):
    from slchannel_b200.fields import synthetic_channel_field

    return synthetic_channel_field(n, n, n, LX, LY, LZ, z_f, z_c, urms=0.1, seed=seed)


def build_flow(n, order, precision="fp64", seed=0):
    import torch

    from slchannel_b200.solver import SLChannelFlow
    from slchannel_b200.utils import compute_bulk_velocity

    flow = SLChannelFlow(config=config(n, order, precision))
    u, v, w = initial_field(n, flow.z_f.cpu().numpy(), flow.z_c.cpu().numpy(), seed)
    flow.set_state(*(torch.from_numpy(a) for a in (u, v, w)))
    ub = float(compute_bulk_velocity(flow.u, flow.cell_vol_ratio, flow.total_volume))
    flow.u *= 1.0 / ub
    flow._save_and_project_initial()
    flow.step_sl_bdf2(DT)  # BDF1 bootstrap; timed steps are BDF2
    return flow


def field_bytes(n):
    u = (n + 1) * (n + 2) * (n + 2)
    w = (n + 2) * (n + 2) * (n + 1)
    return 8 * u, 8 * u, 8 * w, 8 * (n + 2) ** 3


def sl_algorithmic(n, order):
    """Per step, the fused trace+gather+BDF2 kernels (3 launches): compulsory
    HBM bytes = read V^n, V^{n-1}, U* (9 ghost-shaped fields) + write u_hat
    (3 interiors); FLOPs per arrival point both feet (FMA = 2): trace 3
    trilinear sample points x (3 x 8-point samples + locate) ~ 3 x 100,
    weights 2 x (3 x ~(5 order) products + order-6 z table), contraction
    2 x 2 (O^3 + O^2 + O)."""
    bu, bv, bw, _ = field_bytes(n)
    n_u = n * n * n
    n_w = n * n * (n - 1)
    reads = 3 * (bu + bv + bw)
    writes = 8 * (2 * n_u + n_w)
    pts = 2 * n_u + n_w
    contraction = 2 * (order**3 + order**2 + order)
    weights = 3 * (4 * order) + 20
    trace = 3 * 100
    flops_pt = trace + 2 * (weights + contraction)
    return reads + writes, flops_pt * pts, pts


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic_per_point(profile="k_sl_bdf2_o6_fp64.txt"):
    """DRAM bytes per arrival point of a trace+gather kernel, from its ncu
    summary committed in profiles/ (line 'dram_bytes_per_point: X')."""
    path = os.path.join(REPO, "profiles", profile)
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_point:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# CPU side: the oracle port timed on this host's cores
# ---------------------------------------------------------------------------

def cpu_step_sample(n, order, budget_s, seed=0):
    """Time the oracle (the CPU restatement of the reference's float64 path)
    on a bounded sample of one 256^3 BDF2 step and extrapolate to a whole
    step.  Returns (seconds per full step, description, threads)."""
    import oracle.slbdf2 as O

    z_f, z_c, dz_f, dz_c = O.generate_grid(GAMMA, n, LZ)
    u, v, w = initial_field(n, z_f, z_c, seed)
    ch = O.OracleChannel(n, n, n, LX, LY, LZ, GAMMA, 1.0 / RE_B, u, v, w, order=order, z_f=z_f, z_c=z_c)
    adv = ch.sl
    fb = {c: adv.fill(c, f) for c, f in zip("uvw", (ch.u, ch.v, ch.w))}
    mid = fb  # U* = 2 V^n - V^{n-1} with V^{n-1} = V^n: the cost does not depend on the values
    threads = O.max_threads()
    # calibrate: seconds per arrival point for one component, both feet
    nzi = {"u": n, "v": n, "w": n - 1}
    probe = n * nzi["u"]  # one x-plane
    t0 = time.perf_counter()
    adv.advect_comp("u", fb["u"], mid, 2 * DT, 0, probe)
    adv.advect_comp("u", fb["u"], mid, DT, 0, probe)
    per_pt = (time.perf_counter() - t0) / probe
    total_pts = sum(n * n * nzi[c] for c in "uvw")
    # sample: as many x-planes per component as fit the budget (at least one)
    planes = max(1, min(n, int(budget_s * 0.7 / (per_pt * 3 * n * n))))
    t_sl = 0.0
    pts_done = 0
    for c in "uvw":
        npl = planes * n * nzi[c]
        t0 = time.perf_counter()
        adv.advect_comp(c, fb[c], mid, 2 * DT, 0, npl)  # far foot (depth 2 dt)
        adv.advect_comp(c, fb[c], mid, DT, 0, npl)      # near foot
        t_sl += time.perf_counter() - t0
        pts_done += npl
    t_sl_full = t_sl * total_pts / pts_done
    # z-solve (PCR, as the reference) on the same fraction of columns
    ncol = max(1, planes * n)
    t0 = time.perf_counter()
    a, b, cc = O.zsolve_coefficients("u", (2.0 / 3.0) * DT, n, dz_c, dz_f, 1.0 / RE_B)
    d = ch.u[1 : 1 + planes, 1 : n + 1, 1 : n + 1].reshape(ncol, n)
    for _ in range(3):
        O.pcr_solve(a, b, cc, d)
    t_z = (time.perf_counter() - t0) * (n * n) / ncol
    # divergence + FFT Poisson + projection + bulk shift at full size
    t0 = time.perf_counter()
    div = ch.divergence()
    phi = O.solve_poisson_fft(div / ((2.0 / 3.0) * DT), ch.fft)
    O.project_velocity(ch.u, ch.v, ch.w, phi, n, n, n, ch.dx, ch.dy, ch.dz_c, ch.dz_f, (2.0 / 3.0) * DT)
    ch.bulk_velocity()
    t_p = time.perf_counter() - t0
    t_step = t_sl_full + t_z + t_p
    desc = (f"oracle (C trace+gather on {threads} threads, numpy rest): trace+gather of both feet on "
            f"{planes} of {n} x-planes per component ({pts_done} of {total_pts} arrival points) "
            f"scaled x{total_pts / pts_done:.1f}; PCR z-solve on {ncol} of {n * n} columns scaled; "
            f"divergence + FFT Poisson + projection + bulk at full size once "
            f"(trace+gather {t_sl_full:.1f} s, z-solve {t_z:.2f} s, projection {t_p:.2f} s per step)")
    return t_step, desc, threads


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's float64 path
    (the oracle port: C trace+gather on all host threads, numpy elsewhere)
    stepping the same 256^3 workload as the GPU arm -- one BDF1 bootstrap,
    `--warmup` untimed BDF2 steps, then `--steps` timed whole BDF2 steps, each
    timed by the wall clock.  Rank 0 only; other ranks exit 0."""
    world, rank, local = dist_env()
    if rank != 0:
        return 0
    n, order = args.n, args.order
    import oracle.slbdf2 as O

    z_f, z_c, dz_f, dz_c = O.generate_grid(GAMMA, n, LZ)
    u, v, w = initial_field(n, z_f, z_c, 0)
    ch = O.OracleChannel(n, n, n, LX, LY, LZ, GAMMA, 1.0 / RE_B, u, v, w, order=order, z_f=z_f, z_c=z_c)
    del u, v, w
    ch.u *= 1.0 / ch.bulk_velocity()
    ch.project_initial()
    threads = O.max_threads()
    ch.step_bdf2(DT)  # BDF1 bootstrap: the timed steps are BDF2, as in the GPU arm
    for _ in range(args.warmup):
        ch.step_bdf2(DT)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ch.step_bdf2(DT)
        times.append(time.perf_counter() - t0)
    t_step = float(np.mean(times))
    value = 1.0 / t_step
    sample = (f"oracle port: the CPU restatement of the reference's float64 SL-BDF2 step (C "
              f"trace+gather on {threads} threads, numpy PCR z-solve, FFT Poisson, projection and "
              f"bulk shift); {args.steps} whole {n}^3 BDF2 steps timed after a BDF1 bootstrap and "
              f"{args.warmup} warm-up steps, {min(times):.2f}-{max(times):.2f} s per step.  The "
              f"reference's own eager torch path is slower still (about 294 s per step at 256^3, "
              f"order 6, on 8 cores), so the ratio against this port is conservative")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * t_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": bench_config(n, order, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

STATE = ("u", "v", "w", "u_nm1", "v_nm1", "w_nm1", "p")


def copy_state(dst, src):
    for name in STATE:
        getattr(dst, name).copy_(getattr(src, name))
    dst._dt_prev_step = src._dt_prev_step


def measure_mixed(flow64, n, order, K, W, dist):
    """The mixed-precision form on the same workload and state: device-timed
    steps/s, and its velocity error against the FP64 form after a number of
    free-running steps from a common state."""
    import torch

    from slchannel_b200.solver import SLChannelFlow
    from slchannel_b200.utils import compute_divergence

    flow32 = SLChannelFlow(config=config(n, order, "mixed"), allocate_fields=True)
    flow32.set_state(flow64.u, flow64.v, flow64.w, flow64.p)
    flow32.step_sl_bdf2(DT)  # allocates the history; then adopt the FP64 history
    copy_state(flow32, flow64)
    for _ in range(W):
        flow32.step_sl_bdf2(DT)
    from slchannel_b200 import _native as N

    flow32._grid.timing(True)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    gstats = (ctypes.c_int64 * 4)()
    N.check(N.lib().slc_gather_stats(flow32._grid.handle, gstats, 1), flow32._grid.handle)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(K):
        flow32.step_sl_bdf2(DT)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    phases = flow32._grid.timing_read()
    flow32._grid.timing(False)
    N.check(N.lib().slc_gather_stats(flow32._grid.handle, gstats, 1), flow32._grid.handle)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    world = dist.get_world_size() if dist else 1
    # error against the FP64 form from a common state
    copy_state(flow32, flow64)
    S = MIXED_ERROR_STEPS
    errs = []
    for _ in range(S):
        flow64.step_sl_bdf2(DT)
        flow32.step_sl_bdf2(DT)
    for c in "uvw":
        a, b = getattr(flow32, c), getattr(flow64, c)
        scale = b.abs().max()
        errs.append(((a - b).abs().max() / scale).item())
    l2 = math.sqrt(sum(((getattr(flow32, c) - getattr(flow64, c)) ** 2).sum().item() for c in "uvw")
                   / sum((getattr(flow64, c) ** 2).sum().item() for c in "uvw"))
    div = compute_divergence(flow32.u, flow32.v, flow32.w, n, n, n, flow32.dx, flow32.dy, flow32.dz_f)
    sl_ms, sl_cnt = phases["sl"]
    _, flops_alg, pts = sl_algorithmic(n, order)
    t_sl = sl_ms / 1000.0 / max(sl_cnt, 1)
    fp32_peak = N.fma_peak_gflops(False)
    return {"value": world * K / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms / K,
            "sl_kernel_ms_per_step": sl_ms / max(sl_cnt, 1),
            "fp32_pipe": {"achieved": flops_alg / t_sl / 1e9, "peak": fp32_peak, "unit": "GFLOP/s",
                          "frac": flops_alg / t_sl / 1e9 / fp32_peak,
                          "peak_source": "measured on this GPU: slc_fma_peak (FP32 FMA chains, "
                                         "best of 3); the gather's arithmetic is mostly FP32"},
            "phase_ms": {p: v[0] / max(v[1], 1) for p, v in phases.items() if v[1]},
            "staged_gather": {"blocks": gstats[1], "near_boxes_staged": gstats[2],
                              "far_boxes_staged": gstats[3], "timeouts": gstats[0]},
            "vs_fp64_after_steps": S, "rel_linf_err_vs_fp64": max(errs), "rel_l2_err_vs_fp64": l2,
            "max_div": float(div.abs().max()),
            "form": "FP32 fluctuation about FP64 plane means in trace+gather; rest FP64"}


def measure_other_order(n, order, K, W):
    """The plain FP64 step at the other interpolation order (tricubic when the
    headline is triquintic) on the same workload: its own seeded state, BDF1
    bootstrap, W warm-up steps, K device-timed steps."""
    import torch

    from slchannel_b200.utils import compute_divergence

    other = 4 if order == 6 else 6
    flow = build_flow(n, other)
    for _ in range(W):
        flow.step_sl_bdf2(DT)
    flow._grid.timing(True)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(K):
        flow.step_sl_bdf2(DT)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    phases = flow._grid.timing_read()
    flow._grid.timing(False)
    div = compute_divergence(flow.u, flow.v, flow.w, n, n, n, flow.dx, flow.dy, flow.dz_f)
    sl_ms, sl_cnt = phases["sl"]
    _, flops_alg, pts = sl_algorithmic(n, other)
    t_sl = sl_ms / 1000.0 / max(sl_cnt, 1)
    out = {"order": other, "value": K / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms / K,
           "sl_kernel_ms_per_step": sl_ms / max(sl_cnt, 1),
           "fp64_gflops": flops_alg / t_sl / 1e9,
           "phase_ms": {p: v[0] / max(v[1], 1) for p, v in phases.items() if v[1]},
           "max_div": float(div.abs().max()),
           "workload": f"SL-BDF2 step {n}^3 (4pi x 2pi x 2), Re_b {RE_B}, dt {DT}, order {other}, "
                       f"FP64, {K} steps after {W} warm-up"}
    del flow
    torch.cuda.empty_cache()
    return out


def measure_ensemble(n_inst, K, precision="fp64", world=1, rank=0):
    """The ensemble form: n_inst seeded channels (per-axis sizes from
    {32, 48, 64, 96, 128}, gamma in [1.6, 2.2], Re_b in [2000, 5000], dt at
    trajectory CFL 3, order 6) partitioned over the ranks by point count
    (one rank: all of them); each rank advances its instances with one
    CUDA-graph step per time level and no collective on the step path, and
    the per-instance bulk velocity and forcing are gathered every 10 steps.
    The time is the maximum over ranks.  On one GPU the loop over the same
    channels' single-channel solvers is timed beside it."""
    import torch

    from slchannel_b200.ensemble import (CudaStopwatch, EnsembleShard, drive_sharded,
                                         ensemble_specs, loop_step)

    specs = ensemble_specs(n_inst, seed=4)
    held = {}

    def make(indices):
        held["shard"] = EnsembleShard(specs, indices, order=6, precision=precision)
        return held["shard"]

    k = max(3, min(K, 20))
    dev = torch.device("cuda", torch.cuda.current_device())
    mine, reports, secs = drive_sharded(specs, rank, world, k, 10, make, CudaStopwatch, warmup=3,
                                        device=dev)
    shard = held["shard"]
    ms_graph = secs * 1000.0 / k
    pts = sum(s["nx"] * s["ny"] * s["nz"] for s in specs)
    final = reports[max(reports)]
    ub_dev = max(abs(d[0] - 1.0) for d in final.values())
    out = {"value": 1000.0 / ms_graph, "unit": "ensemble steps/s", "ms_per_step": ms_graph,
           "instances": n_inst, "points": pts, "ranks": world,
           "instances_per_rank_max": max(len(p) for p in partition_instances_for(specs, world)),
           "mpoint_updates_per_s": 3 * pts / (ms_graph / 1000.0) / 1e6,
           "max_abs_bulk_minus_1": ub_dev, "reports_at_steps": sorted(reports),
           "workload": f"{n_inst} channels, sizes from {{32,48,64,96,128}} per axis, 2pi x pi x 2, "
                       f"gamma U[1.6,2.2], Re_b U[2000,5000], dt at trajectory CFL 3, order 6, "
                       f"{precision}; instances partitioned over {world} rank(s), no collective on "
                       f"the step path, diagnostics gathered every 10 steps; max-rank time"}
    if world == 1 and shard.ens is not None:
        def timed(fn, kk):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(kk):
                fn()
            b.record()
            torch.cuda.synchronize()
            return a.elapsed_time(b) / kk

        ms_loop = timed(lambda: loop_step(shard.flows, shard.dts), max(3, k // 2))
        tiles = {}
        for shape, (tk, _) in (shard.ens.tune_ms or {}).items():
            tiles[str(tk)] = tiles.get(str(tk), 0) + 1
        out.update(loop_ms_per_step=ms_loop, speedup_vs_loop=ms_loop / ms_graph,
                   autotuned_tile_z_extents=tiles)
    shard.close()
    del shard, held
    torch.cuda.empty_cache()
    return out


def partition_instances_for(specs, world):
    from slchannel_b200.ensemble import partition_instances

    return partition_instances(specs, world)


def measure_adjoint(n_dirs):
    """The adjoint form on 128 x 96 x 128 (2pi x pi x 2, Re_b 2800, dt 0.01,
    order 6, FP64): 50-step rollout from the seeded synthetic field, loss =
    kinetic energy of the final velocity weighted by a seeded smooth mask in
    (0, 1), gradient w.r.t. the initial velocity through the hand-written
    adjoint with checkpoints every 10 steps, checked against central finite
    differences (h = 1e-6) in n_dirs seeded smooth directions."""
    import torch

    from slchannel_b200 import adjoint as A
    from slchannel_b200.fields import synthetic_channel_field
    from slchannel_b200.solver import SLChannelFlow
    from slchannel_b200.utils import compute_bulk_velocity

    nx, ny, nz, Lx, Ly, dt, steps, K = 128, 96, 128, 2 * math.pi, math.pi, 0.01, 50, 10
    cfg = {"grid": {"nx": nx, "ny": ny, "nz": nz},
           "domain": {"Lx": Lx, "Ly": Ly, "Lz": LZ, "stretching_type": "symmetric"},
           "flow": {"Re": 2800.0, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": GAMMA},
           "initialization": {"type": "parabolic"}, "time": {"dt": dt},
           "compute": {"device": "cuda"},
           "sl": {"interp_order": 6, "n_traj_iters": 2, "interp_dtype": "fp64"}}
    flow = SLChannelFlow(config=cfg)
    u, v, w = synthetic_channel_field(nx, ny, nz, Lx, Ly, LZ, flow.z_f.cpu().numpy(),
                                      flow.z_c.cpu().numpy(), urms=0.1, seed=5)
    flow.set_state(*(torch.from_numpy(a) for a in (u, v, w)))
    flow.apply_bc_uvw()
    flow.u *= 1.0 / float(compute_bulk_velocity(flow.u, flow.cell_vol_ratio, flow.total_volume))
    flow._save_and_project_initial()
    V0 = tuple(t.clone() for t in (flow.u, flow.v, flow.w))
    mask = A.smooth_mask(flow, seed=6)

    def timed(fn):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        r = fn()
        b.record()
        torch.cuda.synchronize()
        return r, a.elapsed_time(b)

    # warm-up with the timed configuration: workspaces, plans and the caching
    # allocator's blocks for the checkpoints are in place before timing
    A.gradient(flow, V0, dt, steps, mask, checkpoint_every=K)
    _, ms_fwd = timed(lambda: A.loss_of(flow, V0, dt, steps, mask))
    (J, grad), ms_grad = timed(lambda: A.gradient(flow, V0, dt, steps, mask, checkpoint_every=K))
    errs, worst = [], 0.0
    for i in range(n_dirs):
        d = A.random_direction(flow, seed=1000 + i)
        fd = A.central_fd(flow, V0, d, 1e-6, dt, steps, mask)
        ad = A.dot(grad, d)
        e = abs(fd - ad) / max(abs(fd), 0.1)
        errs.append(e)
        worst = max(worst, e)
    out = {"grid": [nx, ny, nz], "steps": steps, "checkpoint_every": K, "loss": J,
           "forward_ms": ms_fwd, "gradient_ms": ms_grad,
           "adjoint_ms_per_step": (ms_grad - ms_fwd) / steps,
           "backward_over_forward": (ms_grad - ms_fwd) / ms_fwd,
           "fd_directions": n_dirs, "fd_h": 1e-6, "fd_max_rel_err": worst if errs else None,
           "fd_median_rel_err": sorted(errs)[len(errs) // 2] if errs else None,
           "workload": "128x96x128, 2pi x pi x 2, Re_b 2800, dt 0.01, order 6, FP64, 50 steps, "
                       "checkpoints every 10, loss = masked kinetic energy of V^50"}
    del flow, V0, grad
    torch.cuda.empty_cache()
    return out


def plane_stats(flow):
    """Plane-averaged U and the rms / uw profiles of the interior fields
    (u, v at centres; w averaged to centres)."""
    nx, ny, nz = flow.nx, flow.ny, flow.nz
    u = flow.u[1:nx + 1, 1:ny + 1, 1:nz + 1]
    v = flow.v[1:nx + 1, 1:ny + 1, 1:nz + 1]
    w = 0.5 * (flow.w[1:nx + 1, 1:ny + 1, 0:nz] + flow.w[1:nx + 1, 1:ny + 1, 1:nz + 1])
    U = u.mean(dim=(0, 1))
    up, vp, wp = u - U, v - v.mean(dim=(0, 1)), w - w.mean(dim=(0, 1))
    return {"U": U, "urms": up.pow(2).mean((0, 1)).sqrt(), "vrms": vp.pow(2).mean((0, 1)).sqrt(),
            "wrms": wp.pow(2).mean((0, 1)).sqrt(), "uw": (up * wp).mean((0, 1))}


def run_mixed_report(args):
    """The mixed form and the FP64 form free-running side by side from one
    seeded initial field (both with their own BDF1 bootstrap); every
    `report_every` steps one JSON line with the mixed form's relative
    velocity errors (L2 and Linf over the three components), its max|div|
    and bulk velocity, and the drift of its plane-averaged U, u'_rms, v'_rms,
    w'_rms and uw profiles (max relative difference to the FP64 profiles)."""
    import torch

    from slchannel_b200.fields import synthetic_channel_field
    from slchannel_b200.solver import SLChannelFlow
    from slchannel_b200.utils import compute_bulk_velocity, compute_divergence

    nx, ny, nz = args.report_grid
    cfg = lambda prec: {  # noqa: E731
        "grid": {"nx": nx, "ny": ny, "nz": nz},
        "domain": {"Lx": LX, "Ly": LY, "Lz": LZ, "stretching_type": "symmetric"},
        "flow": {"Re": args.report_re, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": GAMMA},
        "initialization": {"type": "parabolic"}, "time": {"dt": args.report_dt},
        "compute": {"device": "cuda"},
        "sl": {"interp_order": 6, "n_traj_iters": 2, "interp_dtype": prec}}
    f64 = SLChannelFlow(config=cfg("fp64"))
    u, v, w = synthetic_channel_field(nx, ny, nz, LX, LY, LZ, f64.z_f.cpu().numpy(),
                                      f64.z_c.cpu().numpy(), urms=args.report_urms, seed=12)
    f64.set_state(*(torch.from_numpy(a) for a in (u, v, w)))
    f64.apply_bc_uvw()
    f64.u *= 1.0 / float(compute_bulk_velocity(f64.u, f64.cell_vol_ratio, f64.total_volume))
    f64._save_and_project_initial()
    f32 = SLChannelFlow(config=cfg("mixed"))
    f32.set_state(f64.u, f64.v, f64.w, f64.p)
    print(json.dumps({"report": "mixed vs FP64", "grid": [nx, ny, nz], "Lx": LX, "Ly": LY,
                      "nu": 1.0 / args.report_re, "dt": args.report_dt, "urms": args.report_urms,
                      "order": 6, "steps": args.report_steps}), flush=True)
    t0 = time.time()
    for n in range(1, args.report_steps + 1):
        f64.step_sl_bdf2(args.report_dt)
        ub32, _ = f32.step_sl_bdf2(args.report_dt)
        if n % args.report_every and n != args.report_steps:
            continue
        num2 = den2 = 0.0
        linf = 0.0
        for c in "uvw":
            a, b = getattr(f32, c), getattr(f64, c)
            d = a - b
            num2 += float((d * d).sum())
            den2 += float((b * b).sum())
            linf = max(linf, float(d.abs().max() / b.abs().max()))
        s32, s64 = plane_stats(f32), plane_stats(f64)
        drift = {k: float((s32[k] - s64[k]).abs().max() / (s64[k].abs().max() or 1.0)) for k in s64}
        div = compute_divergence(f32.u, f32.v, f32.w, nx, ny, nz, f32.dx, f32.dy, f32.dz_f)
        print(json.dumps({"step": n, "rel_l2": math.sqrt(num2 / den2), "rel_linf": linf,
                          "max_div_mixed": float(div.abs().max()), "u_bulk_mixed": float(ub32),
                          "stats_drift": drift, "wall_s": time.time() - t0}), flush=True)
    return 0


def measure_schemes():
    """The reference's scheme comparison (benchmarks/bench_step.py, case
    re180): 256^3, 4pi x 2pi x 2, Re_b 2792.8, gamma 1.6, vortex initial
    field; the Eulerian IMEX step at its advective-CFL dt 0.0057 against the
    SL-BDF2 step at dt 0.0215 (tricubic and triquintic, the mixed form as the
    reference's fp32_accum64 runs it, and the FP64 form); wall-clock per
    simulated time unit.  3 warm-up and 10 timed steps each, CUDA events."""
    import torch

    from slchannel_b200.solver import SLChannelFlow

    dt_e, dt_sl = 0.0057, 0.0215

    def cfg(scheme, order, prec):
        return {"grid": {"nx": 256, "ny": 256, "nz": 256},
                "domain": {"Lx": LX, "Ly": LY, "Lz": LZ},
                "flow": {"Re": RE_B, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": 1.6},
                "advection": {"scheme": scheme},
                "sl": {"interp_order": order, "traj_interp_order": 2, "n_traj_iters": 2,
                       "interp_dtype": prec},
                "initialization": {"type": "vortices", "perturbation_intensity": 0.05, "n_vortices": 4},
                "time": {"dt": dt_e}, "compute": {"device": "cuda"}}

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(10):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / 10

    ms = {}
    flow = SLChannelFlow(config=cfg("eulerian", 4, "fp64"))
    ms["step_eulerian"] = timed(lambda: flow.step_imex(dt_e))
    del flow
    for order, name in ((4, "cubic"), (6, "quintic")):
        for prec in ("fp32_accum64", "fp64"):
            flow = SLChannelFlow(config=cfg("sl", order, prec))
            ms[f"step_sl_{name}_{'mixed' if prec != 'fp64' else 'fp64'}"] = timed(lambda f=flow: f.step_sl_bdf2(dt_sl))
            del flow
            torch.cuda.empty_cache()
    cost_e = ms["step_eulerian"] / dt_e / 1000.0
    per_unit = {k: v / (dt_sl if k.startswith("step_sl") else dt_e) / 1000.0 for k, v in ms.items()}
    return {"case": "re180 (benchmarks/bench_step.py): 256^3, 4pi x 2pi x 2, Re_b 2792.8, gamma 1.6",
            "dt_eulerian": dt_e, "dt_sl": dt_sl, "step_ms": ms, "seconds_per_time_unit": per_unit,
            "sl_speedup_per_time_unit": {k.replace("step_sl_", ""): cost_e / per_unit[k]
                                         for k in ms if k.startswith("step_sl")}}


def run_gather_compare(args):
    """The two FP64 trace+gather entry points on the same inputs: the L1
    gather (the step's) and the TMA-staged gather, each launched
    `--warmup` + `--steps` times on the BDF2 state of (a) the benchmark
    workload at --n^3 and (b) a 128^3 channel of the ensemble's recipe
    (2pi x pi x 2, gamma 1.9, Re_b 3500) at trajectory CFL 3; device time
    per call, staged-box counters, and the largest difference."""
    import torch

    from slchannel_b200 import _native as N
    from slchannel_b200.ensemble import make_flow

    torch.cuda.set_device(0)
    cases = [("benchmark", build_flow(args.n, args.order), DT)]
    spec = {"nx": 128, "ny": 128, "nz": 128, "Lx": 2 * math.pi, "Ly": math.pi, "Lz": LZ,
            "gamma": 1.9, "Re": 3500.0, "seed": 4321, "cfl": 3.0, "urms": 0.1}
    f, dt = make_flow(spec, order=args.order)
    f.step_sl_bdf2(dt)
    cases.append(("trajectory CFL 3, 128^3 (ensemble recipe)", f, dt))
    for name, flow, dt in cases:
        g, st = flow.sl.native, N.stream_of(flow.u)
        cur, prev = (flow.u, flow.v, flow.w), (flow.u_nm1, flow.v_nm1, flow.w_nm1)
        outs = {k: [torch.zeros_like(t) for t in cur] for k in ("l1", "staged")}
        ncl = torch.zeros((), dtype=torch.int64, device=flow.device)
        stats = (ctypes.c_int64 * 4)()
        N.check(N.lib().slc_gather_stats(g.handle, stats, 1), g.handle)
        res = {"case": name, "grid": [flow.nx, flow.ny, flow.nz], "dt": dt, "order": args.order}
        for key, entry in (("l1", "slc_trace_gather_bdf2"), ("staged", "slc_trace_gather_bdf2_staged")):
            def call():
                g.call(entry, *[N.ptr(t) for t in cur], *[N.ptr(t) for t in prev], float(dt),
                       *[N.ptr(t) for t in outs[key]], N.ptr(ncl), st)
            for _ in range(max(args.warmup, 1)):
                call()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(args.steps):
                call()
            b.record()
            torch.cuda.synchronize()
            res[f"{key}_ms_per_call"] = a.elapsed_time(b) / args.steps
            # the same calls once more with the library's phase events: the
            # U* (and padded-copy) pass apart from the trace+gather launches
            g.timing(True)
            for _ in range(args.steps):
                call()
            ph = g.timing_read()
            g.timing(False)
            res[f"{key}_phases_ms"] = {p: round(ph[p][0] / args.steps, 4) for p in ("mid", "sl")}
        N.check(N.lib().slc_gather_stats(g.handle, stats, 0), g.handle)
        res["staged_stats"] = {"timeouts": stats[0], "blocks": stats[1], "near_boxes_staged": stats[2],
                               "far_boxes_staged": stats[3]}
        res["max_abs_diff"] = max(float((x - y).abs().max()) for x, y in zip(outs["l1"], outs["staged"]))
        print(json.dumps(res), flush=True)
    return 0


def run_b200(args):
    import torch

    from slchannel_b200 import _native as N

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = dist_init(world, "nccl")
    n, order, K, W = args.n, args.order, args.steps, max(args.warmup, 3)
    flow = build_flow(n, order)
    dev = torch.cuda.current_device()
    for _ in range(W):
        flow.step_sl_bdf2(DT)
    torch.cuda.synchronize()

    flow._grid.timing(True)
    gstats = (ctypes.c_int64 * 4)()
    N.check(N.lib().slc_gather_stats(flow._grid.handle, gstats, 1), flow._grid.handle)
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(gpu_smi_id(dev))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = N.kernel_launches()
    sampler.start()
    ev0.record(stream)
    for _ in range(K):
        flow.step_sl_bdf2(DT)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = N.kernel_launches() - launches0
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    phases = flow._grid.timing_read()
    flow._grid.timing(False)
    N.check(N.lib().slc_gather_stats(flow._grid.handle, gstats, 1), flow._grid.handle)
    staged_gather = {"blocks": gstats[1], "near_boxes_staged": gstats[2], "far_boxes_staged": gstats[3],
                     "timeouts": gstats[0]}
    ms_max = ms
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = world * K / (ms_max / 1000.0)

    # correctness riders for the timed state
    from slchannel_b200.utils import compute_divergence

    div = compute_divergence(flow.u, flow.v, flow.w, n, n, n, flow.dx, flow.dy, flow.dz_f)
    max_div = float(div.abs().max())

    # roofline of the dominant kernel (fused trace + gather + BDF2 epilogue)
    sl_ms, sl_cnt = phases["sl"]
    t_sl = sl_ms / 1000.0 / max(sl_cnt, 1)
    bytes_alg, flops_alg, pts = sl_algorithmic(n, order)
    peak, peak_kind = measured_peaks()
    achieved = bytes_alg / t_sl / 1e9
    staged = staged_gather["blocks"] > 0
    tpp = profiled_traffic_per_point("k_sl_tma_staged_gather_o6_fp64_128cubed.txt" if staged
                                     else "k_sl_bdf2_o6_fp64.txt")
    roofline = {
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": achieved / peak, "traffic": (tpp * pts) if tpp else None,
        "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
        "kernel": (f"k_sl_tma_seq<C,{order}> (gather from TMA-staged boxes, one foot after the other)"
                   if staged else f"k_sl<C,{order},BDF2>")
                  + " x3 launches per step (one per velocity component)",
        "staged_gather": staged_gather,
        "algorithmic_bytes_per_step": bytes_alg,
        "kernel_ms_per_step": t_sl * 1000.0,
        "fp64_gflops": flops_alg / t_sl / 1e9,
        "note": "the FP64 gather is bound by L1/LSU load throughput and the FP64 pipe, not HBM",
    }
    # the same kernel's algorithmic FLOP rate against this GPU's FP64 FMA pipe,
    # measured here by the library's FMA-chain kernel (MEASURED_PEAKS.json has
    # no FP64 figure)
    from slchannel_b200 import _native as N

    fp64_peak = N.fma_peak_gflops(True)
    roofline["fp64_pipe"] = {
        "achieved": flops_alg / t_sl / 1e9, "peak": fp64_peak, "unit": "GFLOP/s",
        "frac": flops_alg / t_sl / 1e9 / fp64_peak,
        "flops_per_arrival_point": flops_alg / pts,
        "peak_source": "measured on this GPU: slc_fma_peak (FP64 FMA chains on every SM, best of 3)",
    }
    phase_ms = {p: (v[0] / max(v[1], 1)) for p, v in phases.items() if v[1]}

    # e2e: the host-state API (HostStateStepper -> slc_step_bdf2_host) with the
    # state in pinned HOST memory: every step uploads V^n and V^{n-1} and
    # downloads V^{n+1}, p and (u_bulk, forcing); the library overlaps the
    # chunked copies with each other and with compute.  For comparison, the
    # same protocol serialised on one stream around SLChannelFlow.step_sl_bdf2.
    from slchannel_b200.host import HostStateStepper, pinned_like

    Ke = max(1, args.e2e_steps)  # a sustained loop: fill and drain amortised over Ke steps
    H = [tuple(pinned_like(t) for t in (flow.u, flow.v, flow.w)) for _ in range(3)]
    hp = pinned_like(flow.p)
    hb = torch.zeros(2, dtype=torch.float64).pin_memory()
    for h, d in zip(H[0], (flow.u_nm1, flow.v_nm1, flow.w_nm1)):
        h.copy_(d)
    for h, d in zip(H[1], (flow.u, flow.v, flow.w)):
        h.copy_(d)
    torch.cuda.synchronize()
    h2d = sum(t.numel() * 8 for t in H[0] + H[1])
    d2h = sum(t.numel() * 8 for t in H[2]) + hp.numel() * 8 + 16
    hs = HostStateStepper(flow)
    prev, cur, nxt = H
    hs.step(cur, prev, nxt, hp, hb, DT)  # warm-up: allocates the double-buffered device state
    prev, cur, nxt = cur, nxt, prev
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(Ke):
        hs.step(cur, prev, nxt, hp, hb, DT)
        prev, cur, nxt = cur, nxt, prev
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    # the serialised protocol on one stream (reference point, not the headline)
    host_in = [torch.empty_like(t, device="cpu").pin_memory() for t in
               (flow.u, flow.v, flow.w, flow.u_nm1, flow.v_nm1, flow.w_nm1)]
    host_out = [torch.empty_like(t, device="cpu").pin_memory() for t in (flow.u, flow.v, flow.w, flow.p)]
    host_ub = torch.empty((), dtype=torch.float64).pin_memory()
    for h, d in zip(host_in, (flow.u, flow.v, flow.w, flow.u_nm1, flow.v_nm1, flow.w_nm1)):
        h.copy_(d)
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(Ke):
        for h, name in zip(host_in, ("u", "v", "w", "u_nm1", "v_nm1", "w_nm1")):
            getattr(flow, name).copy_(h, non_blocking=True)
        ub, _f = flow.step_sl_bdf2(DT)
        for h, name in zip(host_out, ("u", "v", "w", "p")):
            h.copy_(getattr(flow, name), non_blocking=True)
        host_ub.copy_(ub, non_blocking=True)
        host_in, host_out = host_out[0:3] + host_in[0:3], host_in[3:6] + host_out[3:4]
    s1.record(stream)
    torch.cuda.synchronize()
    serial_ms = s0.elapsed_time(s1)
    e2e_max = e2e_ms
    if dist:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_max = float(t.item())
    e2e = {"value": world * Ke / (e2e_max / 1000.0), "unit": UNIT, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "steps": Ke, "ms_per_step": e2e_max / Ke,
           "path": "HostStateStepper.step (slc_step_bdf2_host): state in pinned host memory, "
                   "copies in pieces overlapped with compute, the step streamed by x slab",
           "host_step": hs.stats(),
           "serialised_ms_per_step": serial_ms / Ke}

    mixed = None
    if not args.no_mixed:
        mixed = measure_mixed(flow, n, order, K, W, dist)

    # the mixed form's headline figures, compact: early in the line and again
    # as its last key (a reader of only the line's head or tail sees them)
    mixed_summary = None
    if mixed is not None:
        mixed_summary = {"steps_per_s": mixed["value"], "ms_per_step": mixed["ms_per_step"],
                         "vs_fp64_steps_per_s": mixed["value"] / value,
                         "rel_linf_err_vs_fp64": mixed["rel_linf_err_vs_fp64"],
                         "rel_l2_err_vs_fp64": mixed["rel_l2_err_vs_fp64"],
                         "after_steps": mixed["vs_fp64_after_steps"], "max_div": mixed["max_div"]}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(n, order, world),
        "mixed_summary": mixed_summary,
        "mpoint_updates_per_s": value * 3 * n**3 / 1e6,
        "phase_ms": phase_ms, "max_div": max_div,
        "gpu_launches": int(launches), "roofline": roofline, "clocks": clocks, "e2e": e2e,
        "mixed": mixed,
    }
    if world == 1 and not args.no_other_order:
        line["other_order"] = measure_other_order(n, order, K, W)
    if not args.no_ensemble:  # every rank takes part (the instances shard over the ranks)
        line["ensemble"] = measure_ensemble(args.ensemble_n, K, "fp64", world, rank)
        line["ensemble_mixed"] = measure_ensemble(args.ensemble_n, K, "mixed", world, rank)
    if world == 1 and not args.no_adjoint:
        line["adjoint"] = measure_adjoint(args.adjoint_fd_dirs)
    if world == 1 and not args.no_schemes:
        line["scheme_comparison"] = measure_schemes()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t_cpu, desc, threads = cpu_step_sample(n, order, args.cpu_budget_s)
        line["cpu_baseline"] = {"value": 1.0 / t_cpu, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": desc}
    if mixed_summary is not None:
        line["mixed_form"] = mixed_summary  # repeated as the line's last key
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    global MIXED_ERROR_STEPS
    args = parse_args()
    MIXED_ERROR_STEPS = args.mixed_error_steps
    if args.impl == "reference":
        return run_reference(args)
    if args.mixed_report:
        return run_mixed_report(args)
    if args.gather_compare:
        return run_gather_compare(args)
    if args.gather_probe:
        import torch

        from slchannel_b200 import _native as N

        torch.cuda.set_device(0)
        res = N.gather_probe(args.n, max(args.steps, 1))
        res.update(n=args.n, points=args.n**3, reps=max(args.steps, 1),
                   tensor_over_scalar_time=res["tensor_ms"] / res["scalar_ms"])
        print(json.dumps(res), flush=True)
        return 0
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
