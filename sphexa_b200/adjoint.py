"""Gradients through K steps of the VE hydro propagator with the hand-written adjoint kernels (sphb_sim_step_vjp).

The forward runs K steps at a fixed time step and keeps a checkpoint of the full particle state every
`checkpoint_every` steps. The backward pass walks the checkpoints in reverse: it restores one and replays that
segment's steps once, recording each step's forces (the post-sync state, neighbour lists, derived fields and the
adjoint tape) in a device slot; then it applies the step adjoints in reverse order from those records. Each replayed
step makes the same sort, neighbour lists and branch choices as the forward (they are deterministic functions of the
restored state), so neighbour lists are frozen per step by construction. With recorded=False each step adjoint
recomputes its step's forces instead of reading a record (one more force computation per step, less memory).

Objective: the total kinetic energy sum_i m_i |v_i|^2 / 2 after K steps. Parameters: the initial internal energy per
particle u0 = cv * temp0 (in the order of the initial conditions) and the artificial-viscosity alphamax
(sph/include/sph/hydro_ve/av_switches_kern.hpp).
"""
from __future__ import annotations

import numpy as np

from .ic import CONSERVED_FIELDS
from .simulation import Simulation

FIELD_INDEX = {f: k for k, f in enumerate(CONSERVED_FIELDS)}


def ideal_gas_cv(mui: float, gamma: float) -> float:
    """cv of the reference's ideal gas (sph/include/sph/eos.hpp:19-24)."""
    return 8.317e7 / mui / (gamma - 1.0)


class AdjointRun:
    def __init__(self, ic: dict, precision: str = "fp64", dt: float = 1e-5, steps: int = 20,
                 checkpoint_every: int = 5, recorded: bool = True):
        """recorded: replay each checkpoint segment once and record every step's forces for its adjoint
        (sphb_sim_step_record); otherwise every step adjoint recomputes its forces (sphb_sim_step_vjp)."""
        import torch
        self.torch = torch
        self.ic = ic
        self.precision = precision
        self.dt = float(dt)
        self.steps = int(steps)
        self.every = int(checkpoint_every)
        self.recorded = bool(recorded)
        self.n = int(ic["x"].size)
        self.cv = ideal_gas_cv(ic["params"]["mui"], ic["params"]["gamma"])
        self.sim = None
        self.initial = None
        self.checkpoints = {}
        self.forward_steps = 0

    # state buffers on the device ------------------------------------------------------------------------------
    def _state_buffers(self):
        t = self.torch
        fields = [t.empty(self.n, dtype=t.float64, device="cuda") for _ in CONSERVED_FIELDS]
        ids = t.empty(self.n, dtype=t.int64, device="cuda")
        return fields, ids

    def _store(self):
        fields, ids = self._state_buffers()
        self.sim.store_state(fields, ids)
        return fields, ids

    def _make_sim(self, u0: np.ndarray, alphamax: float) -> Simulation:
        ic = dict(self.ic)
        ic["temp"] = np.asarray(u0, dtype=np.float64) / self.cv
        ic["params"] = dict(self.ic["params"], alphamax=float(alphamax))
        sim = Simulation(ic, self.precision)
        sim.set_fixed_dt(self.dt)
        return sim

    def kinetic_energy(self) -> float:
        t = self.torch
        m = t.empty(self.n, dtype=t.float64, device="cuda")
        self.sim.get_device("m", m)
        e = t.zeros((), dtype=t.float64, device="cuda")
        for f in ("vx", "vy", "vz"):
            v = t.empty(self.n, dtype=t.float64, device="cuda")
            self.sim.get_device(f, v)
            e += 0.5 * (m * v * v).sum()
        return float(e.item())

    # forward and backward -------------------------------------------------------------------------------------
    def forward(self, u0: np.ndarray, alphamax: float, checkpoints: bool = True) -> float:
        """Run the K steps from u0 (initial-condition order) and alphamax; returns the final kinetic energy.
        The first call builds the simulation; later calls restore its initial state with the new u0 and alphamax
        (the physics does not depend on the domain bookkeeping a fresh simulation would rebuild)."""
        if self.sim is None:
            self.sim = self._make_sim(u0, alphamax)
            self.initial = self._store()
        else:
            fields, ids = self.initial
            fields = [f.clone() for f in fields]
            order = ids.cpu().numpy()
            temp = np.asarray(u0, dtype=np.float64)[order] / self.cv
            fields[FIELD_INDEX["temp"]] = self.torch.from_numpy(temp).cuda()
            self.sim.load_state(fields, ids)
            self.sim.set_params(alphamax=float(alphamax))
        self.checkpoints = {}
        for s in range(self.steps):
            if checkpoints and s % self.every == 0:
                self.checkpoints[s] = self._store()
            self.sim.step()
        self.forward_steps = self.steps
        return self.kinetic_energy()

    def backward(self):
        """Returns (dL/du0 in initial-condition order, dL/dalphamax)."""
        t = self.torch
        if not self.checkpoints:
            raise RuntimeError("backward needs a forward run with checkpoints")
        n = self.n
        adj = [t.zeros(n, dtype=t.float64, device="cuda") for _ in CONSERVED_FIELDS]
        m = t.empty(n, dtype=t.float64, device="cuda")
        self.sim.get_device("m", m)
        for f in ("vx", "vy", "vz"):
            v = t.empty(n, dtype=t.float64, device="cuda")
            self.sim.get_device(f, v)
            adj[FIELD_INDEX[f]] = m * v
        nxt = [t.empty(n, dtype=t.float64, device="cuda") for _ in CONSERVED_FIELDS]
        alphamax_bar = 0.0
        if self.recorded:
            self.sim.tape_reserve(self.every)
        for start in sorted(self.checkpoints, reverse=True):
            end = min(start + self.every, self.steps)
            self.sim.load_state(*self.checkpoints[start])
            if self.recorded:
                # replay the segment once, recording every step's forces, then apply the adjoints from the records
                for s in range(start, end):
                    self.sim.step_record(s - start)
                for s in reversed(range(start, end)):
                    alphamax_bar += self.sim.step_vjp_recorded(s - start, adj, nxt)
                    adj, nxt = nxt, adj
            else:
                # replay the segment for its starting states; each step adjoint recomputes its forces
                states = [self.checkpoints[start]]
                for _ in range(start, end - 1):
                    self.sim.step()
                    states.append(self._store())
                for s in reversed(range(start, end)):
                    self.sim.load_state(*states[s - start])
                    alphamax_bar += self.sim.step_vjp(adj, nxt)
                    adj, nxt = nxt, adj
        ids = self.checkpoints[0][1].cpu().numpy()
        gtemp = adj[FIELD_INDEX["temp"]].cpu().numpy()
        grad_u0 = np.empty(n)
        grad_u0[ids] = gtemp / self.cv
        return grad_u0, alphamax_bar

    def close(self):
        if self.sim is not None:
            self.sim.close()
            self.sim = None
            self.initial = None


def kinetic_energy_function():
    """torch.autograd.Function computing the final kinetic energy of an AdjointRun from (u0, alphamax)."""
    import torch

    class KineticEnergy(torch.autograd.Function):
        @staticmethod
        def forward(ctx, u0, alphamax, run):
            value = run.forward(u0.detach().cpu().numpy(), float(alphamax))
            ctx.run = run
            return torch.tensor(value, dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad_out):
            gu, ga = ctx.run.backward()
            g = float(grad_out)
            return torch.from_numpy(gu * g), torch.tensor(ga * g, dtype=torch.float64), None

    return KineticEnergy
