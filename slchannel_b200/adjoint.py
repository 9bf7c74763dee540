"""Gradients through SL-BDF2 rollouts: the hand-written adjoint of the step
(``slc_adjoint_step`` in the C ABI) behind a ``torch.autograd.Function``,
with step checkpointing for long rollouts.

The reference obtains gradients by torch autograd through its eager FP64
path (the survey of slChannel v1.0.1 checked this against finite
differences).  Here the rollout runs on the GPU step, and the backward pass
runs each step's adjoint:
* the transposed ghost refresh, bulk shift, projection and z-solve;
* the transposed gather as a deterministic segmented scatter-add;
* the gradient through the foot positions.

A rollout of n steps starts from V^0 with the BDF1 bootstrap, followed by
BDF2 steps at a fixed dt; each step includes the exact bulk shift, as
``SLChannelFlow.step_sl_bdf2``.  During the forward pass only every
``checkpoint_every``-th state pair (V^{c-1}, V^c) is kept; the backward pass
recomputes each segment from its checkpoint and runs the segment's adjoint
steps in reverse.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from . import _native as N


def _ptrs(ts):
    return N.ptr_array(ts)


class _Stepper:
    """Forward steps on caller-held ghost-shaped tensors through one handle."""

    def __init__(self, flow):
        if flow.sl_interp_dtype != "fp64":
            raise ValueError("the adjoint is implemented for the FP64 form")
        if flow.sl_bdf2_pressure != "noninc" or flow.sl_traj_order != 2:
            raise ValueError("the adjoint is implemented for the non-incremental pressure form "
                             "with trilinear trajectories (sl.bdf2_pressure: noninc, "
                             "sl.traj_interp_order: 2)")
        self.flow = flow
        self.g = flow._grid
        self.p = torch.zeros_like(flow.p)
        self.ncl = torch.zeros((), dtype=torch.int64, device=flow.device)
        self.out2 = torch.zeros(2, dtype=torch.float64, device=flow.device)
        self.U_bulk = float(flow.U_bulk)

    def stream(self):
        return N.stream_of(self.p)

    def step(self, prev, cur, dt):
        """V^{n+1} from (V^{n-1}, V^n); prev None = BDF1 bootstrap from cur."""
        # zeros: the step writes interiors and refreshes ghosts, and reads the
        # w wall faces of V^{n+1} (impermeable, 0) before the refresh
        nxt = tuple(torch.zeros_like(t) for t in cur)
        pc, kc = _ptrs(cur)
        pn, kn = _ptrs(nxt)
        s = self.stream()
        if prev is None:
            self.g.call("slc_step_bdf1", pc, pn, N.ptr(self.p), float(dt), N.ptr(self.ncl), s)
        else:
            pp, kp = _ptrs(prev)
            self.g.call("slc_step_bdf2", pc, pp, pn, N.ptr(self.p), float(dt), N.ptr(self.ncl), s)
        self.g.call("slc_bulk_shift", N.ptr(nxt[0]), N.ptr(nxt[1]), N.ptr(nxt[2]), self.U_bulk,
                    float(dt), N.ptr(self.out2), s)
        return nxt

    def adjoint(self, n, prev, cur, lam_next, lam_cur, lam_prev, dt):
        """Reverse of step n (n = 0 the bootstrap)."""
        pc, kc = _ptrs(cur)
        pln, k1 = _ptrs(lam_next)
        plc, k2 = _ptrs(lam_cur)
        if n == 0:
            self.g.call("slc_adjoint_step", 1, pc, None, pln, plc, None, float(dt), self.stream())
        else:
            pp, kp = _ptrs(prev)
            plp, k3 = _ptrs(lam_prev)
            self.g.call("slc_adjoint_step", 2, pc, pp, pln, plc, plp, float(dt), self.stream())

    def fold(self, lam):
        self.g.call("slc_adjoint_bc", N.ptr(lam[0]), N.ptr(lam[1]), N.ptr(lam[2]), self.stream())


def rollout(flow, V0, dt, n_steps, checkpoint_every=0):
    """Forward rollout of n_steps from V0 = (u, v, w) (ghost-shaped; ghosts
    are refreshed from the interiors).  Returns (V^N, checkpoints), with
    checkpoints {c: (V^{c-1} or None, V^c)} every checkpoint_every steps
    (0: none)."""
    st = _Stepper(flow)
    cur = tuple(t.detach().clone() for t in V0)
    prev = None
    cps = {}
    for n in range(n_steps):
        if checkpoint_every and n % checkpoint_every == 0:
            cps[n] = (prev, cur)
        nxt = st.step(prev, cur, dt)
        prev, cur = cur, nxt
    return cur, cps


class SLRollout(torch.autograd.Function):
    """(u0, v0, w0) -> (uN, vN, wN) after n_steps SL-BDF2 steps (BDF1
    bootstrap first), differentiable through the hand-written adjoint."""

    @staticmethod
    def forward(ctx, u0, v0, w0, flow, dt, n_steps, checkpoint_every):
        K = int(checkpoint_every) if checkpoint_every else int(n_steps)
        VN, cps = rollout(flow, (u0, v0, w0), dt, n_steps, K)
        ctx.flow, ctx.dt, ctx.n, ctx.K, ctx.cps = flow, float(dt), int(n_steps), K, cps
        return tuple(t.clone() for t in VN)

    @staticmethod
    def backward(ctx, gu, gv, gw):
        grads = adjoint_rollout(ctx.flow, ctx.cps, ctx.dt, ctx.n, ctx.K, (gu, gv, gw))
        ctx.cps = None
        return grads[0], grads[1], grads[2], None, None, None, None


def adjoint_rollout(flow, cps, dt, n_steps, K, lamN):
    """dJ/dV^0 from dJ/dV^N, recomputing each checkpoint segment."""
    st = _Stepper(flow)

    def zeros():
        return tuple(torch.zeros_like(t) for t in lamN)

    lam_next = tuple((t if t is not None else torch.zeros_like(z)).detach().clone().contiguous()
                     for t, z in zip(lamN, cps[0][1]))
    lam_cur, lam_prev = zeros(), zeros()
    starts = sorted(cps)
    for s in reversed(starts):
        e = min(s + K, n_steps)
        prev, cur = cps[s]
        states = {s: cur}
        if prev is not None:
            states[s - 1] = prev
        for n in range(s, e - 1):  # V^{s+1} .. V^{e-1}; V^e is not needed
            states[n + 1] = st.step(states.get(n - 1), states[n], dt)
        for n in range(e - 1, s - 1, -1):
            st.adjoint(n, states.get(n - 1), states[n], lam_next, lam_cur, lam_prev, dt)
            freed = lam_next
            lam_next, lam_cur = lam_cur, lam_prev
            for t in freed:
                t.zero_()
            lam_prev = freed
            states.pop(n + 1, None)
    # lam_next now holds dJ/dV^0
    st.fold(lam_next)
    return lam_next


# ----------------------------------------------------------------------
# Loss, masks and seeded directions
# ----------------------------------------------------------------------
def _positions(flow, comp):
    nx, ny, nz = flow.nx, flow.ny, flow.nz
    x = (np.arange(nx) + (1.0 if comp == 0 else 0.5)) * flow.dx
    y = (np.arange(ny) + (1.0 if comp == 1 else 0.5)) * flow.dy
    zc = flow.z_c.cpu().numpy()
    zf = flow.z_f.cpu().numpy()
    z = zf[1:nz] if comp == 2 else zc[1:nz + 1]
    return np.meshgrid(x, y, z, indexing="ij")


def _smooth(flow, comp, rng, nmodes=6):
    X, Y, Z = _positions(flow, comp)
    s = np.zeros_like(X)
    for _ in range(nmodes):
        m, n, l = rng.integers(0, 3, size=3)
        a, ph1, ph2 = rng.normal(), rng.uniform(0, 2 * math.pi), rng.uniform(0, 2 * math.pi)
        s += a * np.cos(2 * math.pi * m * X / flow.Lx + ph1) * np.cos(2 * math.pi * n * Y / flow.Ly + ph2) \
            * np.cos(math.pi * l * Z / flow.Lz)
    return s


def _interior(t, comp, flow):
    nx, ny, nz = flow.nx, flow.ny, flow.nz
    kz = nz - 1 if comp == 2 else nz
    return t[1:nx + 1, 1:ny + 1, 1:kz + 1]


def smooth_mask(flow, seed):
    """Seeded smooth random weights in (0, 1) at each component's interior
    positions (a logistic of a few low Fourier modes)."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(3):
        s = _smooth(flow, c, rng)
        out.append(torch.from_numpy(1.0 / (1.0 + np.exp(-s))).to(flow.device))
    return out


def kinetic_energy_loss(V, mask, flow):
    """J = 1/2 sum over interior points of mask_c * V_c^2."""
    J = 0.0
    for c in range(3):
        J = J + 0.5 * (mask[c] * _interior(V[c], c, flow) ** 2).sum()
    return J


def random_direction(flow, seed):
    """A seeded smooth perturbation of the interiors (ghosts zero), unit norm."""
    rng = np.random.default_rng(seed)
    d = [torch.zeros_like(t) for t in (flow.u, flow.v, flow.w)]
    for c in range(3):
        _interior(d[c], c, flow).copy_(torch.from_numpy(_smooth(flow, c, rng, nmodes=8)))
    norm = math.sqrt(sum(float((t * t).sum()) for t in d))
    return [t / norm for t in d]


def loss_of(flow, V0, dt, n_steps, mask):
    VN, _ = rollout(flow, V0, dt, n_steps, 0)
    return float(kinetic_energy_loss(VN, mask, flow))


def gradient(flow, V0, dt, n_steps, mask, checkpoint_every=10):
    """(J, dJ/dV^0) through SLRollout and autograd."""
    u0, v0, w0 = (t.detach().clone().requires_grad_(True) for t in V0)
    VN = SLRollout.apply(u0, v0, w0, flow, dt, n_steps, checkpoint_every)
    J = kinetic_energy_loss(VN, mask, flow)
    J.backward()
    return float(J.detach()), (u0.grad, v0.grad, w0.grad)


def central_fd(flow, V0, d, h, dt, n_steps, mask):
    """(J(V0 + h d) - J(V0 - h d)) / (2 h)."""
    plus = tuple(a + h * b for a, b in zip(V0, d))
    minus = tuple(a - h * b for a, b in zip(V0, d))
    return (loss_of(flow, plus, dt, n_steps, mask) - loss_of(flow, minus, dt, n_steps, mask)) / (2 * h)


def dot(a, b):
    return sum(float((x * y).sum()) for x, y in zip(a, b))
