"""Gradient of the final annealing energy w.r.t. the schedule values.

* The differentiable forward against the oracle emulator driven with the same
  gates (second-order steps of H(s) = -(1-s) sum X + s sum J ZZ, BP run to a
  tight tolerance): final <Z_v> within 1e-7.
* Each stage's reverse pass (coupling layer of simple updates, regauge with the
  implicit BP adjoint, mixing layer) against central finite differences of the
  same stage followed by the energy, along random state directions:
  1e-5 relative.
* Checkpointed reverse pass of the whole run against central finite
  differences (h = 1e-4) along random schedule directions: 1e-5 relative,
  for checkpoint intervals of 1, 2 and 3 steps (same gradient each time).
"""

import numpy as np
import pytest
import torch

from dequantizer_b200 import workloads as W
from dequantizer_b200.anneal_grad import AnnealingGradient
from oracle.emulator import BPQuantumEmulator as OracleEmulator

pytestmark = pytest.mark.gpu

DT = 0.3


def _instance():
    return W.random_regular_energy(8, 3, seed=21, field_std=0.4)


def test_forward_matches_oracle_emulator():
    energy = _instance()
    s = np.linspace(0.0, 1.0, 5)
    ag = AnnealingGradient(energy, max_chi=4, dt=DT, bp_tol=1e-14)
    gam, lam = ag.final_state(s)
    z = ag.one_site_z(gam, lam).cpu().numpy()
    g = W.tensor_graph_of(energy)
    em = OracleEmulator(g, 3, 4, energy.edges_number, 1e-13, 5000)
    n = energy.fields.shape[0]
    deg = {nid: g.get_node(nid).degree for nid in g.nodes}
    for nid in range(n):
        em.apply_q1(W.HADAMARD, nid)
    for st in s:
        tm, tc = -DT * (1 - st), DT * st
        for nid in range(n):
            em.apply_q1(W.q1_gate(tm / 2), nid)
        for (a, b), J in zip(energy.coupled_spin_pairs, energy.coupling_amplitudes):
            a, b = int(a), int(b)
            em.apply_q2(W.q2_gate(J, energy.fields[a] / deg[a], energy.fields[b] / deg[b], tc), a, b)
        for nid in range(n):
            em.apply_q1(W.q1_gate(tm / 2), nid)
    z_ref = np.array([float((em.dens_q1(nd.id)[0, 0] - em.dens_q1(nd.id)[1, 1]).real) for nd in ag.nodes])
    assert np.abs(z - z_ref).max() < 1e-7


def _state_fd(ag, fn, gam, lam, seed, h=1e-6):
    g = [x.clone().requires_grad_(True) for x in gam]
    l = [x.clone().requires_grad_(True) for x in lam]
    grads = torch.autograd.grad(fn(g, l), g + l, allow_unused=True)
    gen = torch.Generator(device=gam[0].device).manual_seed(seed)
    dg = [torch.randn(x.shape, dtype=x.dtype, device=x.device, generator=gen) for x in gam]
    dl = [torch.randn(x.shape, dtype=x.dtype, device=x.device, generator=gen) for x in lam]
    ad = sum(float((a.conj() * d).real.sum()) for a, d in zip(grads, dg + dl) if a is not None)
    with torch.no_grad():
        ep = float(fn([x + h * d for x, d in zip(gam, dg)], [x + h * d for x, d in zip(lam, dl)]))
        em = float(fn([x - h * d for x, d in zip(gam, dg)], [x - h * d for x, d in zip(lam, dl)]))
    return ad, (ep - em) / (2 * h)


def test_stage_adjoints_match_finite_differences():
    energy = _instance()
    ag = AnnealingGradient(energy, max_chi=4, dt=DT, bp_tol=1e-14)
    dev = ag.device
    gam, lam = ag.initial_state()
    with torch.no_grad():
        for t, st in enumerate([0.3, 0.45, 0.6]):
            gam, lam = ag.step(gam, lam, torch.tensor(st, dtype=torch.float64, device=dev), first=(t == 0))
    tau = torch.tensor(0.21, dtype=torch.float64, device=dev)
    mix = ag.mixing_gate(torch.tensor(-0.1, dtype=torch.float64, device=dev))
    stages = {
        "energy": lambda g, l: ag.energy_of(g, l),
        "regauge": lambda g, l: ag.energy_of(*ag.regauge(g, l)),
        "coupling": lambda g, l: ag.energy_of(*ag.coupling_layer(g, l, tau)),
        "mixing": lambda g, l: ag.energy_of(ag.apply1_all(g, mix), l),
    }
    for i, (name, fn) in enumerate(stages.items()):
        ad, fd = _state_fd(ag, fn, gam, lam, seed=i)
        assert abs(ad - fd) <= 1e-5 * max(abs(fd), 1e-3), (name, ad, fd)


@pytest.mark.parametrize("k", [1, 2, 3])
def test_gradient_matches_finite_differences(k):
    energy = _instance()
    rng = np.random.default_rng(0)
    s = np.clip(np.linspace(0.0, 1.0, 6) + 0.05 * rng.standard_normal(6), 0, 1)
    ag = AnnealingGradient(energy, max_chi=4, dt=DT, checkpoint_every=k, bp_tol=1e-14)
    E, grad = ag.value_and_grad(s)
    assert np.isfinite(grad).all()
    if k == 1:
        test_gradient_matches_finite_differences.ref = grad
    else:
        ref = test_gradient_matches_finite_differences.ref
        assert np.abs(grad - ref).max() < 1e-10 * max(1.0, np.abs(grad).max())
    h = 1e-4
    for trial in range(2 if k == 1 else 1):
        d = rng.standard_normal(6)
        fd = (ag.energy_value(s + h * d) - ag.energy_value(s - h * d)) / (2 * h)
        ad = float(grad @ d)
        assert abs(ad - fd) <= 1e-5 * max(abs(fd), 1e-3), (ad, fd)


def test_stacked_form_equals_per_node_lists():
    """Once every bond is at max_chi the state is carried as one stacked
    tensor per kind (batched stages); with that form switched off the same
    run through per-node lists gives the same energy (1e-12) and gradient
    (1e-9 relative)."""
    energy = _instance()
    s = np.linspace(0.1, 0.9, 6)
    a = AnnealingGradient(energy, max_chi=4, dt=DT, checkpoint_every=2, bp_tol=1e-14)
    b = AnnealingGradient(energy, max_chi=4, dt=DT, checkpoint_every=2, bp_tol=1e-14)
    b.use_stacked = False
    Ea, ga = a.value_and_grad(s)
    Eb, gb = b.value_and_grad(s)
    assert a._stk is not None and b._stk is None, "the stacked form must have run in one and not the other"
    assert abs(Ea - Eb) < 1e-12
    assert np.abs(ga - gb).max() < 1e-9 * max(1.0, np.abs(gb).max())


@pytest.mark.parametrize("batch,m,k", [(3, 512, 32), (600, 40, 8), (5, 6, 9), (2, 7, 7)])
def test_batched_qr_kernel(batch, m, k):
    """dqz_qr_batched: Q R = A, Q^H Q = I, R upper trapezoidal, |diag R| equal to
    LAPACK's (torch.linalg.qr), 1e-12 relative; more matrices than CTAs."""
    from dequantizer_b200.linalg_ad import qr

    gen = torch.Generator(device="cuda").manual_seed(batch + m + k)
    A = torch.randn(batch, m, k, dtype=torch.complex128, device="cuda", generator=gen)
    Q, R = qr(A)
    kk = min(m, k)
    assert Q.shape == (batch, m, kk) and R.shape == (batch, kk, k)
    assert float((Q @ R - A).abs().max() / A.abs().max()) < 1e-12
    eye = torch.eye(kk, dtype=A.dtype, device=A.device)
    assert float((Q.mH @ Q - eye).abs().max()) < 1e-12
    assert float(torch.tril(R, diagonal=-1).abs().max()) == 0.0
    Rt = torch.linalg.qr(A, mode="reduced")[1]
    d1, d2 = torch.diagonal(R, dim1=-2, dim2=-1).abs(), torch.diagonal(Rt, dim1=-2, dim2=-1).abs()
    assert float((d1 - d2).abs().max() / d2.abs().max()) < 1e-12


def test_zero_coupling_step_is_the_documented_nondifferentiable_point():
    """s_0 = 0 makes the first coupling layer the identity: the reverse pass
    returns 0 for that component (the Schmidt values there grow like |tau|),
    while every other component still matches finite differences; just inside
    the interval (s_0 = 0.01) all components match."""
    energy = W.random_regular_energy(8, 3, seed=21, field_std=0.0)
    h = 1e-4
    for s0 in (0.0, 0.01):
        s = np.linspace(0.0, 1.0, 6)
        s[0] = s0
        ag = AnnealingGradient(energy, max_chi=4, dt=DT, checkpoint_every=2, bp_tol=1e-14)
        _, g = ag.value_and_grad(s)
        for j in range(3):
            d = np.zeros(6)
            d[j] = 1.0
            fd = (ag.energy_value(s + h * d) - ag.energy_value(s - h * d)) / (2 * h)
            if s0 == 0.0 and j == 0:
                assert abs(g[0]) < 1e-12 and abs(fd) > 1e-2
            else:
                assert abs(g[j] - fd) <= 1e-5 * max(abs(fd), 1e-3), (s0, j, g[j], fd)
