"""Ensembles of independent channels advanced together on one GPU.

The reference advances one channel per process (``SLChannelFlow.step_sl_bdf2``,
solver.py:813-1018).  ``ChannelEnsemble`` advances many channels of uneven
grids, Reynolds numbers and time steps with one launch per substep through
the C ABI's ``slc_ensemble_*`` entry points:

* the fused trace+gather is a persistent kernel over an (instance,
  component, tile) work queue;
* the Poisson FFTs are one cuFFT call per group of instances sharing
  (nx, ny);
* the step is captured once per time-level phase into a CUDA graph and
  replayed;
* the SL tile shape of every grid shape is chosen by a timing autotuner.

Per instance the arithmetic is that of the single-channel step, so an
instance in the ensemble follows the same trajectory as the same channel
stepped alone by ``SLChannelFlow`` (the loop this form replaces).

Several GPUs: ``partition_instances`` assigns instances to ranks (greedy
longest-processing-time on the point count); each rank runs its own
ensemble, with no collective on the step path.  ``gather_diagnostics``
collects per-instance scalars at a report cadence.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _native as N
from .fields import synthetic_channel_field
from .solver import SLChannelFlow
from .utils import compute_bulk_velocity

SIZES = (32, 48, 64, 96, 128)


def ensemble_specs(n=48, seed=4, sizes=SIZES, gamma=(1.6, 2.2), Re=(2000.0, 5000.0), cfl=3.0,
                   Lx=2 * math.pi, Ly=math.pi, Lz=2.0, urms=0.1):
    """Seeded instance descriptions: per-axis sizes drawn from `sizes`, tanh
    gamma and bulk Reynolds number uniform in their ranges, a field seed,
    and the trajectory CFL number that fixes each instance's dt."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx, ny, nz = (int(rng.choice(sizes)) for _ in range(3))
        out.append({
            "nx": nx, "ny": ny, "nz": nz, "Lx": Lx, "Ly": Ly, "Lz": Lz,
            "gamma": float(rng.uniform(*gamma)), "Re": float(rng.uniform(*Re)),
            "seed": int(seed * 1000 + i), "cfl": cfl, "urms": urms,
        })
    return out


def _config(spec, order, precision):
    return {
        "grid": {"nx": spec["nx"], "ny": spec["ny"], "nz": spec["nz"]},
        "domain": {"Lx": spec["Lx"], "Ly": spec["Ly"], "Lz": spec["Lz"],
                   "stretching_type": "symmetric"},
        "flow": {"Re": spec["Re"], "Re_tau": 180.0, "U_bulk": 1.0, "gamma": spec["gamma"]},
        "boundary_conditions": {"top_wall": {"type": "dirichlet"}},
        "initialization": {"type": "parabolic"},
        "time": {"dt": 0.01, "dt_update_interval": 0},
        "compute": {"device": "cuda"},
        "sl": {"interp_order": order, "n_traj_iters": 2, "interp_dtype": precision,
               "traj_interp_order": spec.get("traj_order", 2)},
    }


def trajectory_cfl_dt(flow, cfl):
    """dt at which the fastest horizontal velocity crosses `cfl` cells per
    step: dt = cfl / max(max|u| / dx, max|v| / dy) over the interiors."""
    n = (flow.nx, flow.ny, flow.nz)
    u = flow.u[1:n[0] + 1, 1:n[1] + 1, 1:n[2] + 1].abs().max().item()
    v = flow.v[1:n[0] + 1, 1:n[1] + 1, 1:n[2] + 1].abs().max().item()
    return cfl / max(u / flow.dx, v / flow.dy)


def make_flow(spec, order=6, precision="fp64"):
    """One instance as a single-channel solver: the seeded synthetic field
    (Poiseuille + curl of a random potential), bulk velocity 1, projected.
    Returns (flow, dt); the flow has not stepped yet."""
    flow = SLChannelFlow(config=_config(spec, order, precision))
    u, v, w = synthetic_channel_field(
        spec["nx"], spec["ny"], spec["nz"], spec["Lx"], spec["Ly"], spec["Lz"],
        flow.z_f.cpu().numpy(), flow.z_c.cpu().numpy(), urms=spec["urms"], seed=spec["seed"])
    flow.set_state(*(torch.from_numpy(a) for a in (u, v, w)))
    ub = float(compute_bulk_velocity(flow.u, flow.cell_vol_ratio, flow.total_volume))
    flow.u *= flow.U_bulk / ub
    flow._save_and_project_initial()
    return flow, trajectory_cfl_dt(flow, spec["cfl"])


def _desc(flow, order, keep):
    zf = flow.z_f.detach().double().cpu().contiguous()
    zc = flow.z_c.detach().double().cpu().contiguous()
    keep += [zf, zc]
    d = N.GridDesc()
    d.nx, d.ny, d.nz = flow.nx, flow.ny, flow.nz
    d.Lx, d.Ly, d.Lz = float(flow.Lx), float(flow.Ly), float(flow.Lz)
    d.gamma = float(flow.gamma)
    d.stretching = 0 if flow.stretching_type == "symmetric" else 1
    d.order, d.traj_order, d.n_traj_iters = int(order), int(flow.sl_traj_order), int(flow.sl_traj_iters)
    d.top_wall_neumann = 1 if flow.top_wall_bc_type == "neumann" else 0
    d.precision = N.PREC_FP64 if flow.sl_interp_dtype == "fp64" else N.PREC_MIXED
    d.nu = float(flow.nu)
    d.z_f = ctypes.cast(zf.data_ptr(), ctypes.POINTER(ctypes.c_double))
    d.z_c = ctypes.cast(zc.data_ptr(), ctypes.POINTER(ctypes.c_double))
    d.device = flow.device.index if flow.device.index is not None else torch.cuda.current_device()
    d.xy_rhs_lagged = 1 if flow.sl_bdf2_xy_rhs == "lagged" else 0
    return d


def _check(rc, e):
    if rc == N.SLC_OK:
        return
    msg = N.lib().slc_ensemble_last_error(e)
    msg = msg.decode() if msg else f"slc error {rc}"
    raise (ValueError if rc == N.SLC_E_INVALID else RuntimeError)(msg)


class ChannelEnsemble:
    """Many channels stepped together.

    ``flows`` are single-channel solvers that have taken their BDF1
    bootstrap step (``flow.step_sl_bdf2(dt)`` once), ``dts`` their fixed time
    steps.  Their V^{n-1}, V^n and p are copied into the ensemble's own
    buffers; the flows are not modified afterwards.
    """

    def __init__(self, flows, dts, *, use_graph=True, autotune=True, autotune_reps=3):
        if len(flows) != len(dts) or not flows:
            raise ValueError("need one dt per flow and at least one flow")
        order = flows[0].sl_order
        if any(f.sl_order != order for f in flows):
            raise ValueError("all instances of an ensemble share one interp_order")
        if any((f.sl_interp_dtype == "fp64") != (flows[0].sl_interp_dtype == "fp64") for f in flows):
            raise ValueError("all instances of an ensemble share one precision form")
        if any(f.u_nm1 is None for f in flows):
            raise ValueError("every flow must have taken its BDF1 bootstrap step")
        if any(f.sl_bdf2_pressure != "noninc" for f in flows):
            raise ValueError("the ensemble steps the non-incremental pressure form "
                             "(sl.bdf2_pressure: noninc)")
        L = N.lib()
        self.n = len(flows)
        self.device = flows[0].device
        self.use_graph = bool(use_graph)
        self.dts = [float(d) for d in dts]
        self.shapes = [(f.nx, f.ny, f.nz) for f in flows]
        keep = []
        descs = (N.GridDesc * self.n)(*[_desc(f, order, keep) for f in flows])
        h = ctypes.c_void_p()
        rc = L.slc_ensemble_create(descs, self.n, ctypes.byref(h))
        _check(rc, None)
        self._h = h
        # three time levels: level 0 = V^{n-1}, level 1 = V^n, level 2 = spare
        self.lev = []
        for f in flows:
            prev = tuple(t.clone() for t in (f.u_nm1, f.v_nm1, f.w_nm1))
            cur = tuple(t.clone() for t in (f.u, f.v, f.w))
            spare = tuple(torch.zeros_like(t) for t in cur)
            self.lev.append((prev, cur, spare))
        self.p = [f.p.clone() for f in flows]
        self.nclamp = torch.zeros(self.n, dtype=torch.int64, device=self.device)
        self.bulk_out = torch.zeros(2 * self.n, dtype=torch.float64, device=self.device)
        levp = (ctypes.c_void_p * (9 * self.n))(
            *[t.data_ptr() for lv in self.lev for level in lv for t in level])
        pp = (ctypes.c_void_p * self.n)(*[t.data_ptr() for t in self.p])
        dt_arr = (ctypes.c_double * self.n)(*self.dts)
        ub_arr = (ctypes.c_double * self.n)(*[float(f.U_bulk) for f in flows])
        rc = L.slc_ensemble_bind(self._h, levp, pp, dt_arr, ub_arr, N.ptr(self.nclamp),
                                 N.ptr(self.bulk_out))
        _check(rc, self._h)
        self.phase = 0
        self.tune_ms = None
        if autotune:
            self.autotune(autotune_reps)

    # ------------------------------------------------------------------
    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and N._lib is not None:
            N._lib.slc_ensemble_destroy(h)
        self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    @property
    def tiles(self):
        """Per-instance SL tile z-extent (points)."""
        arr = (ctypes.c_int * self.n)()
        _check(N.lib().slc_ensemble_get_tiles(self._h, arr), self._h)
        return [1 << a for a in arr]

    def set_tiles(self, tk):
        arr = (ctypes.c_int * self.n)(*[int(math.log2(t)) for t in tk])
        _check(N.lib().slc_ensemble_set_tiles(self._h, arr), self._h)

    def autotune(self, reps=3):
        """Time tile z-extents 32 / 64 / 128 per grid shape and keep the
        fastest; returns {shape: (chosen extent, [ms per candidate])}."""
        choice = (ctypes.c_int * self.n)()
        ms = (ctypes.c_double * (3 * self.n))()
        rc = N.lib().slc_ensemble_autotune(self._h, self.phase, int(reps), choice, ms,
                                           self._stream())
        _check(rc, self._h)
        self.tune_ms = {}
        for i, s in enumerate(self.shapes):
            self.tune_ms[s] = (1 << choice[i], [ms[3 * i + c] for c in range(3)])
        return self.tune_ms

    def step(self):
        """One SL-BDF2 step of every instance (bulk shift included)."""
        rc = N.lib().slc_ensemble_step_bdf2(self._h, self.phase, 1 if self.use_graph else 0,
                                            self._stream())
        _check(rc, self._h)
        self.phase = (self.phase + 1) % 3

    def run(self, n):
        for _ in range(n):
            self.step()

    def velocity(self, i):
        """Current (u, v, w) of instance i (ghost-shaped views, updated in place by step)."""
        return self.lev[i][(self.phase + 1) % 3]

    def history(self, i):
        """(u, v, w) of the previous time level of instance i."""
        return self.lev[i][self.phase % 3]

    def bulk(self, i):
        """(u_bulk, forcing) of instance i after the last step, 0-D device tensors."""
        return self.bulk_out[2 * i], self.bulk_out[2 * i + 1]

    def points(self):
        return sum(nx * ny * nz for nx, ny, nz in self.shapes)


def loop_step(flows, dts):
    """The plain alternative: step each channel with its own solver."""
    for f, dt in zip(flows, dts):
        f.step_sl_bdf2(dt)


# ----------------------------------------------------------------------
# Several GPUs: instances shard across ranks, no collective on the step path.
# ----------------------------------------------------------------------
def partition_instances(specs, world):
    """Greedy longest-processing-time assignment of instances to `world`
    ranks by point count; returns a list of index lists (ascending inside
    each rank).  Deterministic: ties go to the lower rank."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    cost = [s["nx"] * s["ny"] * s["nz"] for s in specs]
    order = sorted(range(len(specs)), key=lambda i: (-cost[i], i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += cost[i]
    return [sorted(p) for p in parts]


def gather_diagnostics(local, rank_instances, world, group=None):
    """Collect per-instance diagnostics {instance index: value} from every
    rank at a report cadence (host-side; one all_gather_object)."""
    import torch.distributed as dist

    payload = {int(i): local[k] for k, i in enumerate(rank_instances)}
    if world == 1:
        return payload
    out = [None] * world
    dist.all_gather_object(out, payload, group=group)
    merged = {}
    for part in out:
        merged.update(part)
    return dict(sorted(merged.items()))


def reduce_max(value, device=None):
    """The maximum of a float over all ranks of the default group (the value
    itself without torch.distributed).  `device`: where the reduction tensor
    lives -- a CUDA device for NCCL, the CPU for gloo."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def drive_sharded(specs, rank, world, steps, report_every, make_ensemble, timer, *,
                  warmup=3, device=None, group=None):
    """Run rank `rank`'s share of a partitioned ensemble.

    The instances are split by ``partition_instances(specs, world)``;
    ``make_ensemble(indices)`` builds this rank's ensemble (an object with
    ``step()`` and ``diagnostics()``, the latter a list of per-instance
    values in the order of `indices`).  After `warmup` untimed steps the rank
    takes `steps` steps with no collective on the step path; every
    `report_every` steps, and after the last one, the per-instance
    diagnostics of all ranks are gathered (``gather_diagnostics``, outside
    the timed segments).  ``timer()`` returns a fresh stopwatch with
    ``start()`` and ``stop() -> seconds`` (CUDA events on the GPU).

    Returns ``(indices, reports, seconds)``: this rank's instances, the list
    of gathered reports ({step: {instance: diagnostics}}), and the stepping
    time as the maximum over ranks."""
    mine = partition_instances(specs, world)[rank]
    ens = make_ensemble(mine)
    for _ in range(warmup):
        ens.step()
    reports = {}
    total = 0.0
    done = 0
    every = max(1, int(report_every))
    while done < steps:
        seg = min(every - done % every, steps - done)
        sw = timer()
        sw.start()
        for _ in range(seg):
            ens.step()
        total += sw.stop()
        done += seg
        if done % every == 0 or done == steps:
            reports[done] = gather_diagnostics(ens.diagnostics(), mine, world, group=group)
    return mine, reports, reduce_max(total, device)


class EnsembleShard:
    """One rank's ensemble for ``drive_sharded``: the seeded instances
    `indices` of `specs` built as single-channel solvers, bootstrapped, and
    handed to a ChannelEnsemble.  ``diagnostics()`` gives, per instance,
    (u_bulk, forcing, kinetic energy of the interior velocity) after the last
    step (one host synchronisation)."""

    def __init__(self, specs, indices, order=6, precision="fp64", use_graph=True, autotune=True):
        flows, dts = [], []
        for i in indices:
            f, dt = make_flow(specs[i], order=order, precision=precision)
            f.step_sl_bdf2(dt)
            flows.append(f)
            dts.append(dt)
        self.ens = ChannelEnsemble(flows, dts, use_graph=use_graph, autotune=autotune) if flows else None
        self.points = self.ens.points() if self.ens else 0
        self.flows, self.dts = flows, dts  # the single-channel solvers (not stepped by the ensemble)

    def step(self):
        if self.ens is not None:
            self.ens.step()

    def diagnostics(self):
        if self.ens is None:
            return []
        ke = []
        for i, (nx, ny, nz) in enumerate(self.ens.shapes):
            u, v, w = self.ens.velocity(i)
            ke.append(0.5 * (u[1:nx + 1, 1:ny + 1, 1:nz + 1].square().sum()
                             + v[1:nx + 1, 1:ny + 1, 1:nz + 1].square().sum()
                             + w[1:nx + 1, 1:ny + 1, 1:nz].square().sum()))
        ke = torch.stack(ke).cpu().tolist()
        b = self.ens.bulk_out.view(-1, 2).cpu().tolist()
        return [(float(ub), float(fo), float(k)) for (ub, fo), k in zip(b, ke)]

    def close(self):
        if self.ens is not None:
            self.ens.close()
            self.ens = None
        self.flows = []


class CudaStopwatch:
    """start()/stop() -> seconds between CUDA events on the current stream."""

    def start(self):
        self.a = torch.cuda.Event(enable_timing=True)
        self.b = torch.cuda.Event(enable_timing=True)
        self.a.record()

    def stop(self):
        self.b.record()
        self.b.synchronize()
        return self.a.elapsed_time(self.b) / 1000.0
