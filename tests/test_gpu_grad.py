"""Adjoint sweep (gsb_grad_run) behind torch.autograd: d log2 Pr(b) / d theta for the rotation layer.

Checks, on the differentiation workload's construction (matching circuit, trainable U3 layer):
  * Z(b) from the sweep gives the same log2 Pr as the executor's 'prob' (complex128) with the same matrices;
  * on n = 20 the gradient of -mean log2 Pr equals a complex128 statevector-autograd gradient (torch, CPU);
  * on n = 48 (width about 22) selected gradient entries equal central finite differences (h = 1e-3, FP64).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _instance(n, seed, iters=20000):
    import workloads
    return workloads.rotation_instance(n, n, seed=seed, order_seed=12, iters=iters)


def _targets(w, count, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, 2, size=(count, len(w["steps"])), dtype=np.int8)


def _loss(theta, w, bits, sweep):
    import adjoint
    return -adjoint.log2_prob(theta, w["M0"], w["step_vertices"], bits, sweep).mean()


def test_sweep_log2p_matches_executor():
    import adjoint
    import gsb
    w = _instance(20, 3)
    bits = _targets(w, 16, 1)
    M = adjoint.step_matrices(torch.tensor(w["theta0"]), w["M0"], w["step_vertices"]).numpy()
    sweep = gsb.GradSweep(w["plan"])
    z, dz = sweep.run(M, bits)
    lp = np.log2(np.abs(z) ** 2) - w["n"]
    with gsb.Engine.from_text(w["plan"], precision=gsb.GSB_C128) as eng:
        eng.set_matrices(M)
        want = eng.prob(bits)
    assert np.max(np.abs(lp - want)) < 1e-9
    assert dz.shape == (16, len(w["steps"]), 2)


def _statevector_loss(theta, w, bits):
    """-mean log2 |<b|psi(theta)>|^2 with psi = U3 layer after the Clifford body (complex128, torch autograd)."""
    from oracle.statevector import dense_state_torch
    import adjoint
    n = w["n"]
    psi = dense_state_torch(n, w["body"], device="cpu").reshape([2] * n)
    G = adjoint.u3(theta)
    for q in range(n):
        psi = torch.movedim(torch.tensordot(G[q], psi, dims=([1], [q])), 0, q)
    psi = psi.reshape(-1)
    # string bit k belongs to qubit step_vertices[k]; qubit 0 is the most significant index bit
    sv = w["step_vertices"]
    idx = np.zeros(len(bits), np.int64)
    for k, q in enumerate(sv):
        idx |= bits[:, k].astype(np.int64) << (n - 1 - q)
    amp = psi[torch.from_numpy(idx)]
    return -(torch.log2(amp.abs() ** 2)).mean()


def test_gradient_matches_statevector_autograd_n20():
    import gsb
    w = _instance(20, 5)
    bits = _targets(w, 64, 2)
    sweep = gsb.GradSweep(w["plan"], every=4)
    th = torch.tensor(w["theta0"], requires_grad=True)
    loss = _loss(th, w, bits, sweep)
    loss.backward()
    g_sweep = th.grad.clone()
    th2 = torch.tensor(w["theta0"], requires_grad=True)
    loss2 = _statevector_loss(th2, w, bits)
    loss2.backward()
    assert abs(loss.item() - loss2.item()) < 1e-9
    assert torch.max(torch.abs(g_sweep - th2.grad)) < 1e-8 * max(1.0, float(torch.max(torch.abs(th2.grad))))


def test_gradient_matches_finite_differences_n48():
    import gsb
    w = _instance(48, 7, iters=20000)
    assert w["width"] <= 24
    bits = _targets(w, 8, 3)
    sweep = gsb.GradSweep(w["plan"], every=4)
    th = torch.tensor(w["theta0"], requires_grad=True)
    _loss(th, w, bits, sweep).backward()
    h = 1e-3
    rng = np.random.default_rng(11)
    for q, a in zip(rng.integers(0, 48, 6), rng.integers(0, 3, 6)):
        tp, tm = torch.tensor(w["theta0"]), torch.tensor(w["theta0"])
        tp[q, a] += h
        tm[q, a] -= h
        fd = (float(_loss(tp, w, bits, sweep)) - float(_loss(tm, w, bits, sweep))) / (2 * h)
        # central differences: error O(h^2) times the third derivative
        assert abs(fd - float(th.grad[q, a])) < 1e-4 * max(1.0, abs(fd)), (q, a, fd, float(th.grad[q, a]))


def test_checkpoint_interval_and_partial_batches_do_not_change_gradients():
    """every = 1 (a checkpoint before every step), 3 and 64 (one segment: the whole sweep recomputed once) give the
    same Z and dZ; 37 strings (not a multiple of the strings swept per launch) give the same rows as 5 of them."""
    import adjoint
    import gsb
    w = _instance(20, 5)
    bits = _targets(w, 37, 4)
    M = adjoint.step_matrices(torch.tensor(w["theta0"]), w["M0"], w["step_vertices"]).numpy()
    ref_z, ref_dz = gsb.GradSweep(w["plan"], every=4).run(M, bits)
    for every in (1, 3, 64):
        z, dz = gsb.GradSweep(w["plan"], every=every).run(M, bits)
        assert np.max(np.abs(z - ref_z)) <= 1e-12 * np.max(np.abs(ref_z))
        assert np.max(np.abs(dz - ref_dz)) <= 1e-12 * np.max(np.abs(ref_dz))
    z5, dz5 = gsb.GradSweep(w["plan"], every=4).run(M, bits[:5])
    assert np.array_equal(z5, ref_z[:5]) and np.array_equal(dz5, ref_dz[:5])
