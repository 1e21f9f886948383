"""Gradients of the time-averaged rotor power by the discrete adjoint of the step.

The objective over a window of M steps starting from a state S0 is

    J = (1/M) sum_{n=1..M} P_n,   P_n = sum over turbines of torque x tip rate

(the power of src/alm/alm.h:133, evaluated by the ALM at the start of step n).
`mean_power_gradient` runs the window forward keeping a checkpoint of the
state every `checkpoint` steps, then sweeps back: each segment is recomputed
from its checkpoint (its states held on the device) and falm_step_adjoint
maps the adjoint state back one step at a time, accumulating dJ/d(collective
pitch, per-AP chord, per-AP twist).  Memory: one checkpoint per segment plus
the states of one segment.  By default (checkpoint=None) every state of the
window is kept when that takes at most a quarter of the free device memory,
and nothing is recomputed; otherwise segments of 20 steps.  States live in
one preallocated device buffer that later calls reuse.

`MeanPower` wraps the same computation as a torch.autograd.Function; it is
used only to check the gradients (torch.autograd.gradcheck-style comparisons),
not as a training path.
"""
import numpy as np

FIELDS = ("u", "uu", "p", "nut")


def _power(sim, stats):
    tip = np.asarray(sim.case.alm.tip_rate, dtype=np.float64)
    return float(sum(tq * tr for tq, tr in zip(stats["torque"], tip)))


def _clone(sim):
    return {k: getattr(sim, k).clone() for k in FIELDS}


def _restore(sim, st):
    for k in FIELDS:
        getattr(sim, k).copy_(st[k].reshape(getattr(sim, k).shape))


class _StatePool:
    """device storage for k saved states (FIELDS of a simulation), one allocation
    kept on the simulation and reused while it is large enough"""

    def __init__(self, sim, k):
        torch = sim.ctx.torch
        self.sizes = [getattr(sim, f).numel() for f in FIELDS]
        per = sum(self.sizes)
        buf = getattr(sim, "_adjoint_pool", None)
        if buf is None or buf.numel() < k * per or buf.dtype != sim.u.dtype:
            buf = torch.empty(k * per, dtype=sim.u.dtype, device=sim.u.device)
            sim._adjoint_pool = buf
        self.buf, self.per, self.n = buf, per, 0

    def save(self, sim):
        """copy the simulation's state into the next free slot; returns a dict of views"""
        base = self.n * self.per
        self.n += 1
        st, o = {}, base
        for f, size in zip(FIELDS, self.sizes):
            v = self.buf[o:o + size]
            v.copy_(getattr(sim, f).reshape(-1))
            st[f] = v
            o += size
        return st


def state_bytes(sim):
    return sum(getattr(sim, f).numel() for f in FIELDS) * sim.u.element_size()


def auto_checkpoint(sim, steps, share=0.25):
    """steps (keep every state) when the window's states fit in `share` of the free
    device memory, else 20"""
    torch = sim.ctx.torch
    free, _ = torch.cuda.mem_get_info(sim.u.device)
    return steps if (steps + 2) * state_bytes(sim) <= share * free else 20


def objective(sim, steps):
    """J over the next `steps` steps of sim (advances sim)"""
    J = 0.0
    for _ in range(steps):
        J += _power(sim, sim.step()) / steps
    return J


def mean_power_gradient(sim, steps, checkpoint=None):
    """J over the next `steps` steps of sim and its gradient (pitch, chord[apcount],
    twist[apcount]) by the discrete adjoint; sim ends after the window.  The states
    of the last segment are kept from the forward pass; the other segments are
    recomputed from their checkpoints (checkpoint >= steps keeps every state and
    recomputes nothing; None chooses, see auto_checkpoint)."""
    ctx = sim.ctx
    torch = ctx.torch
    if ctx.precision != "fp64":
        raise ValueError("the discrete adjoint runs in FP64 contexts")
    if checkpoint is None:
        checkpoint = auto_checkpoint(sim, steps)
    checkpoint = max(1, min(checkpoint, steps))
    apc = sim.case.alm.apcount
    ckpts, J = [], 0.0
    it0 = sim.it
    last = ((steps - 1) // checkpoint) * checkpoint   # first step of the last segment
    nseg = (steps + checkpoint - 1) // checkpoint
    # checkpoints (except the last segment's, whose states are all kept), the last
    # segment's states, and one recomputed segment
    pool = _StatePool(sim, (nseg - 1) + (steps - last) + (checkpoint if nseg > 1 else 0) + 2)
    kept = []
    for q in range(steps):
        if q >= last:
            st = pool.save(sim)
            kept.append(st)
            if q == last:
                ckpts.append((sim.it, st))
        elif q % checkpoint == 0:
            ckpts.append((sim.it, pool.save(sim)))
        J += _power(sim, sim.step()) / steps
    kept.append({"u": sim.u.clone()})
    seg_base = pool.n
    end_state, end_it = _clone(sim), sim.it
    n = sim.case.grid.n
    dev, dt = ctx.device, sim.case.dt
    au = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    auu = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    anut = torch.zeros(n, dtype=torch.float64, device=dev)
    grad = torch.zeros(1 + 2 * apc, dtype=torch.float64, device=dev)
    for s in reversed(range(len(ckpts))):
        it_s, st_s = ckpts[s]
        seg = min(checkpoint, it0 + steps - it_s)
        if s == len(ckpts) - 1:
            states = kept   # kept from the forward pass
        else:
            # recompute the segment, keeping the state at the start of each step
            _restore(sim, st_s)
            sim.it = it_s
            states = []
            pool.n = seg_base
            for q in range(seg):
                states.append(pool.save(sim))
                sim.step()
            states.append({"u": sim.u.clone()})   # the velocity after the segment's last step
        for q in reversed(range(seg)):
            S = states[q]
            ctx.step_adjoint(S["u"], S["uu"], S["p"], S["nut"], dt, (it_s + q + 1) * dt, 1.0 / steps, au, auu, anut, grad,
                             u_after=states[q + 1]["u"])
    _restore(sim, end_state)
    sim.it = end_it
    g = grad.cpu().numpy()
    return J, float(g[0]), g[1:1 + apc].copy(), g[1 + apc:].copy()


def _set_params(sim, params):
    """apply (pitch, chord[apcount], twist[apcount]) to the simulation's ALM"""
    alm = sim.case.alm
    apc = alm.apcount
    p = np.asarray(params, dtype=np.float64)
    alm.pitch = float(p[0])
    alm.aps["chord"] = p[1:1 + apc].copy()
    alm.aps["twist"] = p[1 + apc:1 + 2 * apc].copy()
    sim.ctx.alm_init(alm)


def parameters(sim):
    alm = sim.case.alm
    return np.concatenate([[alm.pitch], np.asarray(alm.aps["chord"], dtype=np.float64),
                           np.asarray(alm.aps["twist"], dtype=np.float64)])


def make_mean_power(torch):
    """the torch.autograd.Function (built lazily so that importing this module needs no torch)"""

    class MeanPower(torch.autograd.Function):
        @staticmethod
        def forward(fctx, params, sim, start, steps, checkpoint):
            _set_params(sim, params.detach().cpu().numpy())
            _restore(sim, start[1])
            sim.it = start[0]
            J, gp, gc, gt = mean_power_gradient(sim, steps, checkpoint)
            fctx.save_for_backward(torch.as_tensor(np.concatenate([[gp], gc, gt]), dtype=params.dtype))
            return params.new_tensor(J)

        @staticmethod
        def backward(fctx, gJ):
            (g,) = fctx.saved_tensors
            return gJ * g, None, None, None, None

    return MeanPower
