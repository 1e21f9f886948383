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

`mean_power_gradient_binomial` reverses the window with binomial
checkpointing instead: the states stored at any time are bounded by a number
of slots (or a memory budget), and forward steps are recomputed along the
optimal schedule of the binomial recursion (binomial_table).

Precision: the adjoint fields and gradients are FP64 in every context.  In a
mixed-precision context the forward steps run in mixed precision, the stored
states and checkpoints are FP32 (half the memory of an FP64 context), and the
adjoint of each step is evaluated at those FP32 states.

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

    def slot(self, i):
        """views of the fields of slot i"""
        st, o = {}, i * self.per
        for f, size in zip(FIELDS, self.sizes):
            st[f] = self.buf[o:o + size]
            o += size
        return st

    def put(self, i, sim):
        """copy the simulation's state into slot i"""
        for f, v in self.slot(i).items():
            v.copy_(getattr(sim, f).reshape(-1))

    def save(self, sim):
        """copy the simulation's state into the next free slot; returns a dict of views"""
        self.put(self.n, sim)
        self.n += 1
        return self.slot(self.n - 1)


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


# ---------------------------------------------------------------- binomial checkpointing
_BINOMIAL = {}


def binomial_table(steps, snaps):
    """Optimal reversal schedule of `steps` steps with `snaps` free state slots
    (besides the one holding the start of the window), by dynamic programming
    over the recursion of binomial (revolve-type) checkpointing: to reverse
    t >= 2 steps with s free slots, advance m steps from the start, store that
    state, reverse the last t - m steps with s - 1 slots, then the first m with
    s.  G[t][s] is the least number of forward steps those advances take (each
    reversed step also recomputes its own forward step once); split[t][s] is an
    m that attains it.  With s = 0 every reversal restarts from the start:
    G[t][0] = t (t - 1) / 2."""
    key = (steps, snaps)
    if key in _BINOMIAL:
        return _BINOMIAL[key]
    T, S = steps, snaps
    G = np.zeros((T + 1, S + 1), dtype=np.int64)
    split = np.zeros((T + 1, S + 1), dtype=np.int64)
    t = np.arange(T + 1, dtype=np.int64)
    G[:, 0] = t * (t - 1) // 2
    G[0, :] = 0
    for s in range(1, S + 1):
        for tt in range(2, T + 1):
            m = np.arange(1, tt)
            cost = m + G[tt - m, s - 1] + G[m, s]
            k = int(np.argmin(cost))
            G[tt, s] = cost[k]
            split[tt, s] = m[k]
    _BINOMIAL[key] = (G, split)
    return G, split


def binomial_forward_steps(steps, snaps):
    """forward steps of a binomial reversal (the advances plus the one forward
    step each reversed step recomputes), the initial pass included"""
    G, _ = binomial_table(steps, snaps)
    return int(G[steps, snaps]) + steps


def snaps_for_budget(sim, budget_bytes):
    """free state slots that `budget_bytes` of device memory holds (the slot of the
    window's start not counted)"""
    return max(0, int(budget_bytes // state_bytes(sim)) - 1)


def mean_power_gradient_binomial(sim, steps, snaps=None, budget_bytes=None):
    """J and its gradient (pitch, chord[apcount], twist[apcount]) like
    mean_power_gradient, with binomial checkpointing: besides the window's
    start, its end and one scratch state, at most `snaps` states (or as many as
    `budget_bytes` of device memory holds, by default a quarter of the free
    memory) are stored at any time, and the reversal recomputes forward steps
    from them along the optimal schedule of binomial_table.  Each step's power
    is taken from the first forward evaluation of that step (the step is
    deterministic: every evaluation gives the same value).  sim ends after the
    window."""
    ctx = sim.ctx
    torch = ctx.torch
    if snaps is None:
        if budget_bytes is None:
            budget_bytes = 0.25 * torch.cuda.mem_get_info(sim.u.device)[0]
        snaps = snaps_for_budget(sim, budget_bytes) - 2
    snaps = max(0, min(int(snaps), steps - 1))
    _, split = binomial_table(steps, snaps)
    apc = sim.case.alm.apcount
    it0 = sim.it
    n = sim.case.grid.n
    dev, dt = ctx.device, sim.case.dt
    pool = _StatePool(sim, snaps + 3)
    START, SCRATCH, END = 0, snaps + 1, snaps + 2
    free_slots = list(range(snaps, 0, -1))
    au = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    auu = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    anut = torch.zeros(n, dtype=torch.float64, device=dev)
    grad = torch.zeros(1 + 2 * apc, dtype=torch.float64, device=dev)
    power = {}

    def goto(a, slot):
        _restore(sim, pool.slot(slot))
        sim.it = it0 + a

    def advance(a, m):
        for q in range(m):
            power.setdefault(a + q, _power(sim, sim.step()))

    def reverse_one(a, slot):
        # slot holds the state of step a, which sim is at: its forward step (the
        # power, the velocity after it), then its adjoint
        S = pool.slot(slot)
        power.setdefault(a, _power(sim, sim.step()))
        if a == steps - 1:
            pool.put(END, sim)
        ctx.step_adjoint(S["u"], S["uu"], S["p"], S["nut"], dt, (it0 + a + 1) * dt, 1.0 / steps, au, auu, anut, grad,
                         u_after=sim.u)

    def reverse(a, b, slot, free):
        t = b - a
        if t == 1:
            goto(a, slot)
            reverse_one(a, slot)
        elif free == 0:
            for i in reversed(range(t)):
                goto(a, slot)
                advance(a, i)
                pool.put(SCRATCH, sim)
                reverse_one(a + i, SCRATCH)
        else:
            m = int(split[t, free])
            goto(a, slot)
            advance(a, m)
            s2 = free_slots.pop()
            pool.put(s2, sim)
            reverse(a + m, b, s2, free - 1)
            free_slots.append(s2)
            reverse(a, a + m, slot, free)

    pool.put(START, sim)
    reverse(0, steps, START, snaps)
    J = sum(power[q] for q in range(steps)) / steps
    _restore(sim, pool.slot(END))
    sim.it = it0 + steps
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
