"""GPU tests of the hand-written step adjoint (sphb_sim_step_vjp) through the checkpointed driver and the
torch.autograd.Function wrapper: gradients of the final kinetic energy with respect to the initial internal energy
per particle and alphamax, against central finite differences of the FP64 forward, and the FP32 adjoint against
the FP64 adjoint."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(cuda_device):
    from sphexa_b200 import ic as icm
    from sphexa_b200.adjoint import AdjointRun, ideal_gas_cv
    ic = icm.sedov(16)
    cv = ideal_gas_cv(ic["params"]["mui"], ic["params"]["gamma"])
    u0 = ic["temp"] * cv
    return ic, u0, AdjointRun, cv


def test_step_vjp_matches_central_differences_per_field(cuda_device):
    """One step adjoint against central differences of the FP64 step, for a random linear functional of the state
    after the step and perturbations of one input field at a time (relative perturbations for fields that vanish in
    the quiescent gas, so that no branch of the viscosity switches flips). h after the step carries no weight: it
    depends on the neighbour count, which a perturbation may change by one."""
    import torch
    from sphexa_b200 import ic as icm
    from sphexa_b200.ic import CONSERVED_FIELDS
    from sphexa_b200.simulation import Simulation
    ic = icm.sedov(16)
    n = ic["x"].size
    sim = Simulation(ic, "fp64")
    sim.set_fixed_dt(1e-5)
    for _ in range(12):
        sim.step()

    def buf():
        return ([torch.empty(n, dtype=torch.float64, device="cuda") for _ in CONSERVED_FIELDS],
                torch.empty(n, dtype=torch.int64, device="cuda"))

    s0, i0 = buf()
    sim.store_state(s0, i0)
    rng = np.random.default_rng(1)
    w = [torch.from_numpy(rng.uniform(-1, 1, n)).cuda() for _ in CONSERVED_FIELDS]
    w[CONSERVED_FIELDS.index("m")].zero_()
    w[CONSERVED_FIELDS.index("h")].zero_()

    def run(state):
        sim.load_state(state, i0)
        sim.compute_forces()
        nc = sim.get("nc")
        sim.integrate()
        out, ids = buf()
        sim.store_state(out, ids)
        return out, ids, nc

    base, bids, bnc = run(s0)
    sim.load_state(s0, i0)
    pre = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in CONSERVED_FIELDS]
    am_bar = sim.step_vjp(w, pre)
    for k, f in enumerate(CONSERVED_FIELDS):
        if f == "m":
            continue
        xi = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
        d = xi * 1e-2 if f in ("x", "y", "z") else xi * s0[k]
        if f == "du_m1":
            d = xi * s0[k].abs().max()
        eps = 1e-8 if f == "h" else 1e-7
        sp = [s.clone() for s in s0]
        sp[k] += eps * d
        sm = [s.clone() for s in s0]
        sm[k] -= eps * d
        op, pid, pnc = run(sp)
        om, mid, mnc = run(sm)
        assert torch.equal(pid, bids) and torch.equal(mid, bids), f
        assert np.array_equal(pnc, bnc) and np.array_equal(mnc, bnc), f
        fd = sum(((op[q] - om[q]) * w[q]).sum().item() for q in range(len(CONSERVED_FIELDS))) / (2 * eps)
        ad = (pre[k] * d).sum().item()
        assert abs(fd - ad) <= 1e-4 * abs(fd), (f, fd, ad)
    am0 = sim.params["alphamax"]
    eps = 1e-6
    sim.set_params(alphamax=am0 * (1 + eps))
    op, _, _ = run(s0)
    sim.set_params(alphamax=am0 * (1 - eps))
    om, _, _ = run(s0)
    fd = sum(((op[q] - om[q]) * w[q]).sum().item() for q in range(len(CONSERVED_FIELDS))) / (2 * eps * am0)
    assert am_bar != 0.0 and abs(fd - am_bar) <= 1e-4 * abs(fd), (fd, am_bar)
    sim.close()


def test_gradient_matches_central_differences(setup):
    ic, u0, AdjointRun, _ = setup
    am0 = ic["params"]["alphamax"]
    run = AdjointRun(ic, "fp64", dt=1e-5, steps=10, checkpoint_every=4)
    L0 = run.forward(u0, am0)
    nc0 = run.sim.get("nc")
    gu, ga = run.backward()
    assert np.all(np.isfinite(gu)) and np.isfinite(ga)
    rng = np.random.default_rng(11)
    eps = 1e-6
    assert ga != 0.0  # the alphamax path is exercised
    fd_run = AdjointRun(ic, "fp64", dt=1e-5, steps=10, checkpoint_every=4)
    for _ in range(4):
        xi = rng.uniform(-1.0, 1.0, u0.size)
        zeta = rng.uniform(-1.0, 1.0)
        du, da = xi * u0, zeta * am0
        lp = fd_run.forward(u0 + eps * du, am0 + eps * da, checkpoints=False)
        assert np.array_equal(fd_run.sim.get("nc"), nc0)  # the same neighbour structure
        lm = fd_run.forward(u0 - eps * du, am0 - eps * da, checkpoints=False)
        assert np.array_equal(fd_run.sim.get("nc"), nc0)
        fd = (lp - lm) / (2 * eps)
        ad = float(np.dot(gu, du) + ga * da)
        assert abs(fd - ad) <= 1e-4 * abs(fd), (fd, ad, L0)
    run.close()
    fd_run.close()


def test_autograd_function_and_fp32_adjoint(setup):
    import torch
    from sphexa_b200.adjoint import kinetic_energy_function
    ic, u0, AdjointRun, _ = setup
    KE = kinetic_energy_function()
    grads = {}
    for prec in ("fp64", "mixed"):
        run = AdjointRun(ic, prec, dt=1e-5, steps=4, checkpoint_every=2)
        u = torch.tensor(u0, dtype=torch.float64, requires_grad=True)
        am = torch.tensor(float(ic["params"]["alphamax"]), dtype=torch.float64, requires_grad=True)
        loss = KE.apply(u, am, run)
        loss.backward()
        grads[prec] = (u.grad.numpy().copy(), float(am.grad))
        run.close()
    g64, a64 = grads["fp64"]
    g32, a32 = grads["mixed"]
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    assert rel < 1e-3, rel
    assert abs(a32 - a64) <= 1e-2 * abs(a64) + 1e-30, (a32, a64)


def test_recorded_and_recomputed_adjoints_agree(setup):
    """The backward pass from recorded steps equals the one that recomputes every step's forces (up to the order of
    the atomic scatters)."""
    ic, u0, AdjointRun, _ = setup
    am0 = ic["params"]["alphamax"]
    grads = []
    for recorded in (True, False):
        run = AdjointRun(ic, "fp64", dt=1e-5, steps=7, checkpoint_every=3, recorded=recorded)
        run.forward(u0, am0)
        grads.append(run.backward())
        run.close()
    (g1, a1), (g2, a2) = grads
    assert np.linalg.norm(g1 - g2) <= 1e-10 * np.linalg.norm(g2)
    assert abs(a1 - a2) <= 1e-10 * abs(a2)
