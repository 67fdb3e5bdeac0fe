"""GPU checks of the differentiation of a fixed accepted-step sequence (marked gpu).

The forward is the replay of the steps an adaptive run accepted (d4_replay):
its positions must equal the run's bit for bit.  The adjoint (d4_adjoint) and
the tangent-linear (d4_tangent) are exact derivatives of that discrete map, so:
central finite differences (h = 1e-6) agree with the adjoint to 1e-5 relative
(the bound the engine is held to) on coordinates whose difference quotient is
converged at that h; the adjoint's gradient dotted with a direction equals the
tangent-linear derivative along it to 1e-10 relative (both are exact
derivatives of the same map; they differ by rounding only); the checkpoint
spacing changes nothing; and the torch.autograd.Function returns the adjoint's
gradients.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, STEPS, TAU = 256, 20, 0.08


@pytest.fixture(scope="module")
def setup(pkg):
    x, y, _ = pkg.dconf.generate_internal(N, 1003)
    sd = pkg.SimulationData()
    sd.set_positions(x, y)
    sd.external_stress = pkg.FixedRateProtocol(TAU, 0.0)
    sd.calculate_strain_during_simulation = True
    e = pkg.Engine(sd)
    e.record_steps(True)
    r = e.advance(STEPS)
    xe, _ = e.positions()
    t0s, hs = e.recorded_steps()
    s, g, gt = e.adjoint(x, t0s, hs, checkpoint_every=7)
    return dict(e=e, x=x, y=y, xe=xe, run=r, t0s=t0s, hs=hs, strain=s, g=g, gt=gt)


def test_replay_reproduces_the_run(setup):
    e, t0s, hs = setup["e"], setup["t0s"], setup["hs"]
    assert len(t0s) == STEPS and (hs > 0).all()
    s, x_end = e.replay(setup["x"], t0s, hs)
    assert np.array_equal(x_end, setup["xe"])
    assert abs(s - setup["run"].strain) <= 1e-12 * abs(setup["run"].strain)
    assert s == setup["strain"]


def test_adjoint_vs_central_differences(setup):
    e, x, t0s, hs, g = setup["e"], setup["x"], setup["t0s"], setup["hs"], setup["g"]
    rng = np.random.default_rng(4000)
    h = 1e-6
    for i in rng.choice(N, 8, replace=False):
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        fd = (e.replay(xp, t0s, hs)[0] - e.replay(xm, t0s, hs)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * abs(g[i]), (i, fd, g[i])
    fdt = (e.replay(x, t0s, hs, tau0=TAU + h)[0] - e.replay(x, t0s, hs, tau0=TAU - h)[0]) / (2 * h)
    assert abs(fdt - setup["gt"]) <= 1e-5 * abs(setup["gt"])


def test_adjoint_vs_tangent_linear(setup):
    e, x, t0s, hs = setup["e"], setup["x"], setup["t0s"], setup["hs"]
    rng = np.random.default_rng(7)
    for dtau in (0.0, 0.3):
        d = rng.standard_normal(N)
        s, ds = e.tangent(x, t0s, hs, d, dtau)
        assert s == setup["strain"]
        adj = setup["g"] @ d + setup["gt"] * dtau
        scale = np.abs(setup["g"]).dot(np.abs(d)) + abs(setup["gt"] * dtau)
        assert abs(ds - adj) <= 1e-10 * abs(ds) and abs(ds - adj) <= 1e-12 * scale


def test_checkpoint_spacing_is_invisible(setup):
    e, x, t0s, hs = setup["e"], setup["x"], setup["t0s"], setup["hs"]
    for k in (1, 100):
        s, g, gt = e.adjoint(x, t0s, hs, checkpoint_every=k)
        assert s == setup["strain"] and gt == setup["gt"]
        assert np.array_equal(g, setup["g"])


def test_torch_autograd_function(pkg, setup):
    import importlib
    import torch
    adj = importlib.import_module("2d4_b200.adjoint")
    x0 = torch.tensor(setup["x"], dtype=torch.float64, requires_grad=True)
    tau = torch.tensor(TAU, dtype=torch.float64, requires_grad=True)
    out = adj.strain(x0, tau, setup["e"], setup["t0s"], setup["hs"], 7)
    assert float(out.detach()) == setup["strain"]
    (2.0 * out).backward()
    assert np.array_equal(x0.grad.numpy(), 2.0 * setup["g"])
    assert float(tau.grad) == 2.0 * setup["gt"]


def test_unsupported_forms_rejected(pkg, setup):
    x, y = setup["x"], setup["y"]
    for kw in (dict(precision_mode=pkg._lib.D4_PREC_MIXED),
               dict(cutoff_multiplier=1.0, heaviside_cutoff=True)):
        sd = pkg.SimulationData()
        sd.set_positions(x, y)
        for k, v in kw.items():
            setattr(sd, k, v)
        e = pkg.Engine(sd)
        with pytest.raises(pkg._lib.D4Error):
            e.replay(x, setup["t0s"][:1], setup["hs"][:1])
        e.close()


def test_adjoint_c5_size_vs_central_differences(pkg):
    """The adjoint configuration's own size: N=2048 (seed 1003), tau = 0.08, a
    20-step recorded sequence, checkpoints every 20 steps; central differences
    (h = 1e-6) on 16 coordinates drawn with seed 4000 agree with the adjoint to
    1e-5 relative where the one-sided quotients agree (converged at that h);
    a coordinate whose quotient has not converged at 1e-6 must meet the bound
    at h = 1e-7 or 1e-8, widened by the two quotients' difference (the finite
    differences' own error at those steps)."""
    n = 2048
    x, y, _ = pkg.dconf.generate_internal(n, 1003)
    sd = pkg.SimulationData()
    sd.set_positions(x, y)
    sd.external_stress = pkg.FixedRateProtocol(TAU, 0.0)
    e = pkg.Engine(sd)
    e.record_steps(True)
    e.advance(20)
    t0s, hs = e.recorded_steps()
    s0, _ = e.replay(x, t0s, hs)
    _, g, _ = e.adjoint(x, t0s, hs, checkpoint_every=20)

    def central(i, h):
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        sp, sm = e.replay(xp, t0s, hs)[0], e.replay(xm, t0s, hs)[0]
        return (sp - sm) / (2 * h), (sp - s0) / h, (s0 - sm) / h

    rng = np.random.default_rng(4000)
    for i in rng.choice(n, 16, replace=False):
        q, qp, qm = central(i, 1e-6)
        if abs(qp - qm) <= 1e-4 * abs(q):
            assert abs(q - g[i]) <= 1e-5 * abs(g[i]), (i, q, g[i])
        else:
            # not converged at 1e-6: the quotients at 1e-7 and 1e-8, whose
            # difference bounds their own error, must meet the adjoint within
            # 1e-5 relative plus that bound
            q7, q8 = central(i, 1e-7)[0], central(i, 1e-8)[0]
            best = min(abs(q7 - g[i]), abs(q8 - g[i]))
            assert best <= 1e-5 * abs(g[i]) + abs(q7 - q8), (i, best, abs(q7 - q8), g[i])
    e.close()
