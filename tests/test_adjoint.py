"""Adjoint of the NVE trajectory: gradients of time-averaged observables with
respect to the Kob-Andersen pair parameters.

Bars: the library's observables agree with the float64 torch restatement of
the same forward; the hand-written adjoint's gradient of the matching loss
agrees with torch.autograd through that float64 forward and with its central
finite differences (h = 1e-4, Richardson-extrapolated with h/2 to remove
the O(h^2) truncation) within 1e-4 relative; checkpoint spacing does
not change the result; runs are reproducible.
"""
import numpy as np
import pytest

import gamdpy_b200 as gp
from gamdpy_b200 import adjoint, workloads

RDF = {"bins": 24, "r_lo": 0.7, "r_hi": 2.3, "width": 0.06, "every": 5}
GRAD_TOL = 1e-4


def ka_theta(eps_ab=1.5, sig_ab=0.8):
    sig = workloads.KA_SIGMA.astype(np.float64).copy()
    eps = workloads.KA_EPSILON.astype(np.float64).copy()
    sig[0, 1] = sig[1, 0] = sig_ab
    eps[0, 1] = eps[1, 0] = eps_ab
    return adjoint.theta_from_tables(sig, eps)


def test_theta_tables_round_trip():
    th = ka_theta(1.45, 0.82)
    sig, eps = adjoint.tables_from_theta(th, 2)
    assert np.allclose(sig, sig.T) and np.allclose(eps, eps.T)
    assert eps[0, 1] == 1.45 and sig[0, 1] == 0.82 and sig[1, 1] == np.float64(np.float32(0.88))
    assert np.array_equal(adjoint.theta_from_tables(sig, eps), th)


def test_reference_autograd_matches_finite_differences():
    """The float64 restatement's own autograd against its central differences
    (a dilute KA system: small and fast on the CPU)."""
    import torch

    from oracle import adjoint_torch as R
    conf = workloads.ka_configuration(40, rho=0.25, temperature=0.8, seed=3, jitter=0.3)
    args = (conf["r"], conf["v"], conf.ptype, conf["m"], conf.simbox.lengths, workloads.KA_CUT.astype(np.float64),
            0.004, 12)
    rdf = {"bins": 10, "r_lo": 0.8, "r_hi": 2.2, "width": 0.1, "every": 3}
    th0 = ka_theta()
    target = R.observables(torch.tensor(ka_theta(1.45, 0.82)), *args, rdf=rdf).detach()
    vol = float(np.prod(conf.simbox.lengths))
    dr = (rdf["r_hi"] - rdf["r_lo"]) / rdf["bins"]

    def loss_t(th):
        return adjoint.matching_loss(R.observables(th, *args, rdf=rdf), target, 40, vol, dr)

    th = torch.tensor(th0, requires_grad=True)
    loss_t(th).backward()
    g = th.grad.numpy()
    fd = R.central_differences(lambda x: float(loss_t(torch.tensor(x))), th0, h=1e-4, richardson=True)
    assert np.linalg.norm(g - fd) <= 1e-6 * np.linalg.norm(fd)
    # plain central differences at h = 1e-4 carry their O(h^2) truncation
    fd1 = R.central_differences(lambda x: float(loss_t(torch.tensor(x))), th0, h=1e-4)
    assert np.linalg.norm(g - fd1) <= 1e-3 * np.linalg.norm(fd1)


def small_ka(n=256, temperature=0.6, seed=5):
    return workloads.ka_configuration(n, rho=1.2, temperature=temperature, seed=seed)


@pytest.mark.gpu
def test_forward_observables_match_float64_restatement():
    import torch

    from oracle import adjoint_torch as R
    conf = small_ka()
    eng = adjoint.AdjointNVE(conf, workloads.KA_CUT, dt=0.005, steps=40, checkpoint_every=10, rdf=RDF)
    th = ka_theta()
    got = eng.forward(th)
    ref = R.observables(torch.tensor(th), conf["r"], conf["v"], conf.ptype, conf["m"], conf.simbox.lengths,
                        workloads.KA_CUT.astype(np.float64), 0.005, 40, rdf=RDF).numpy()
    np.testing.assert_allclose(got[:3], ref[:3], rtol=2e-5)
    np.testing.assert_allclose(got[3:], ref[3:], rtol=1e-4, atol=1e-4 * np.max(ref[3:]))


@pytest.mark.gpu
def test_forward_trajectory_matches_plain_path():
    """Same NVE trajectory as the plain simulation path (N^2 list)."""
    conf = small_ka(seed=8)
    eng = adjoint.AdjointNVE(conf, workloads.KA_CUT, dt=0.005, steps=30, checkpoint_every=10)
    eng.forward(ka_theta())
    r_adj, v_adj = eng.final_state()
    c2 = small_ka(seed=8)
    pp = workloads.ka_pair_potential()
    sim = gp.Simulation(c2, pp, gp.integrators.NVE(dt=0.005), [], num_timeblocks=1, steps_per_timeblock=30,
                        compute_plan={"pb": 64, "tp": 1, "skin": 0.5, "UtilizeNIII": False, "gridsync": False,
                                      "nblist": "N squared"}, storage="memory", steps_in_kernel_test=0)
    for _ in sim.run_timeblocks():
        pass
    assert np.max(np.abs(r_adj - c2["r"])) < 1e-4
    assert np.max(np.abs(v_adj - c2["v"])) < 1e-4


def _gradients(n_steps=40, ckpt=10, seed=5):
    import torch

    from oracle import adjoint_torch as R
    conf = small_ka(seed=seed)
    cut = workloads.KA_CUT.astype(np.float64)
    vol = float(np.prod(conf.simbox.lengths))
    dr = (RDF["r_hi"] - RDF["r_lo"]) / RDF["bins"]
    args = (conf["r"], conf["v"], conf.ptype, conf["m"], conf.simbox.lengths, cut, 0.005, n_steps)
    target = R.observables(torch.tensor(ka_theta(1.45, 0.82)), *args, rdf=RDF).detach()
    eng = adjoint.AdjointNVE(conf, cut, dt=0.005, steps=n_steps, checkpoint_every=ckpt, rdf=RDF)
    th = torch.tensor(ka_theta(), requires_grad=True)
    loss = adjoint.matching_loss(eng.observables(th), target, conf.N, vol, dr)
    loss.backward()
    g_adj = th.grad.numpy().copy()
    th_ref = torch.tensor(ka_theta(), requires_grad=True)
    adjoint.matching_loss(R.observables(th_ref, *args, rdf=RDF), target, conf.N, vol, dr).backward()
    return g_adj, th_ref.grad.numpy(), (R, args, target, vol, dr, conf.N)


@pytest.mark.gpu
def test_adjoint_gradient_matches_autograd_and_finite_differences():
    import torch
    g_adj, g_ref, (R, args, target, vol, dr, n) = _gradients()
    assert np.linalg.norm(g_adj - g_ref) <= GRAD_TOL * np.linalg.norm(g_ref), (g_adj, g_ref)
    fd = R.central_differences(
        lambda x: float(adjoint.matching_loss(R.observables(torch.tensor(x), *args, rdf=RDF), target, n, vol, dr)),
        ka_theta(), h=1e-4, richardson=True)
    assert np.linalg.norm(g_adj - fd) <= GRAD_TOL * np.linalg.norm(fd), (g_adj, fd)
    # every component, relative to the gradient's scale
    assert np.all(np.abs(g_adj - fd) <= GRAD_TOL * np.max(np.abs(fd)))


@pytest.mark.gpu
def test_checkpoint_spacing_and_reruns_do_not_change_gradients():
    g1, _, _ = _gradients(n_steps=40, ckpt=10)
    g2, _, _ = _gradients(n_steps=40, ckpt=40)
    g3, _, _ = _gradients(n_steps=40, ckpt=7)
    assert np.array_equal(g1, g2) and np.array_equal(g1, g3)


@pytest.mark.gpu
@pytest.mark.parametrize("window,ckpt", [(10, 10), (8, 10), (15, 7)])
def test_truncated_adjoint_matches_detached_autograd(window, ckpt):
    """Window W: the state at multiples of W is a constant; torch.autograd
    through the float64 forward with the same detaches is the reference."""
    import torch

    from oracle import adjoint_torch as R
    conf = small_ka(seed=12)
    cut = workloads.KA_CUT.astype(np.float64)
    vol = float(np.prod(conf.simbox.lengths))
    dr = (RDF["r_hi"] - RDF["r_lo"]) / RDF["bins"]
    args = (conf["r"], conf["v"], conf.ptype, conf["m"], conf.simbox.lengths, cut, 0.005, 40)
    target = R.observables(torch.tensor(ka_theta(1.45, 0.82)), *args, rdf=RDF).detach()
    eng = adjoint.AdjointNVE(conf, cut, dt=0.005, steps=40, checkpoint_every=ckpt, rdf=RDF, window=window)
    th = torch.tensor(ka_theta(), requires_grad=True)
    adjoint.matching_loss(eng.observables(th), target, conf.N, vol, dr).backward()
    th_ref = torch.tensor(ka_theta(), requires_grad=True)
    adjoint.matching_loss(R.observables(th_ref, *args, rdf=RDF, window=window), target, conf.N, vol,
                          dr).backward()
    g, g_ref = th.grad.numpy(), th_ref.grad.numpy()
    assert np.linalg.norm(g - g_ref) <= GRAD_TOL * np.linalg.norm(g_ref), (g, g_ref)


@pytest.mark.gpu
def test_backward_after_another_forward_reruns_the_forward():
    import torch
    conf = small_ka(seed=9)
    eng = adjoint.AdjointNVE(conf, workloads.KA_CUT, dt=0.005, steps=20, checkpoint_every=5, rdf=RDF)
    th = torch.tensor(ka_theta(), requires_grad=True)
    obs = eng.observables(th)
    (obs[0] + obs[1]).backward()
    g1 = th.grad.clone()
    th.grad = None
    obs = eng.observables(th)
    eng.forward(ka_theta(1.4, 0.85))  # replaces the checkpoints
    (obs[0] + obs[1]).backward()
    assert torch.equal(g1, th.grad)


@pytest.mark.gpu
def test_bad_arguments_raise():
    from gamdpy_b200._lib import GDB_ERR_ARG, GdbError
    with pytest.raises(GdbError) as e:
        adjoint.AdjointNVE(small_ka(), workloads.KA_CUT, dt=-1.0, steps=10)
    assert e.value.args[0] == GDB_ERR_ARG or "bad arguments" in str(e.value)
