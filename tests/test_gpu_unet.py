"""GPU parity of the learned preconditioner's tcgen05 kernels with the CPU
oracle (forward activations, output, loss, every layer's weight gradient),
on-GPU training, and the learned solver with its automatic fallback."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

# BF16 activations and weights, FP32 accumulation on both sides; the oracle
# rounds at the same points in double arithmetic, so the gap is summation
# order plus the occasional differently rounded bf16 value.
FWD_TOL = 2e-2
GRAD_TOL = 3e-2


def _torch():
    import torch
    return torch


def _weights(seed, n_params):
    rng = np.random.default_rng(seed)
    w = np.zeros(n_params, dtype=np.float32)
    for name, (sl, (_, cout, cin)) in O.unet_layer_slices().items():
        w[sl] = rng.normal(0.0, 1.0 / np.sqrt(27 * cin), sl.stop - sl.start)
    return w


@pytest.fixture(scope="module")
def ctx():
    import dare_b200 as D
    return D.Context(0)


@pytest.mark.parametrize("n", [(16, 24, 32), (8, 8, 8), (32, 16, 8)])
def test_forward_matches_oracle(ctx, n):
    import dare_b200 as D
    torch = _torch()
    net = D.LearnedPreconditioner(ctx, n, seed=3)
    w = _weights(11, net.num_params)
    net.set_weights(w)
    N = int(np.prod(n))
    g = torch.Generator().manual_seed(5)
    u = torch.randn(N, generator=g, dtype=torch.float32).cuda()
    z = torch.empty_like(u)
    net.apply(u.data_ptr(), z.data_ptr())
    torch.cuda.synchronize()
    zo, acts = O.unet_forward(n, w, u.cpu().double().numpy(), bf16=True, with_acts=True)
    errs = {}
    for i, (name, _, _) in enumerate(O.UNET_ACTS):
        errs[name] = rel_l2(net.activation(i), acts[name])
    uu = u.cpu().double().numpy()
    errs["U(u)"] = rel_l2(z.cpu().double().numpy() - uu, zo - uu)
    print(n, errs)
    assert all(e < FWD_TOL for e in errs.values()), errs


def test_input_off_the_16_byte_grid(ctx):
    """enc0 reads its FP32 input through a TMA map, which needs a 16-byte
    base: a vector that starts 4 bytes off goes through a pitched staging
    copy first and must give the same output, bit for bit."""
    import dare_b200 as D
    torch = _torch()
    n = (16, 24, 32)
    net = D.LearnedPreconditioner(ctx, n, seed=3)
    net.set_weights(_weights(12, net.num_params))
    N = int(np.prod(n))
    g = torch.Generator().manual_seed(6)
    buf = torch.randn(N + 4, generator=g, dtype=torch.float32).cuda()
    shifted = buf[1:N + 1]
    assert shifted.data_ptr() % 16 == 4
    aligned = shifted.clone()
    assert aligned.data_ptr() % 16 == 0
    z0, z1 = torch.empty(N, device="cuda"), torch.empty(N, device="cuda")
    net.apply(aligned.data_ptr(), z0.data_ptr())
    net.apply(shifted.data_ptr(), z1.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(z0, z1)


def test_identity_at_initialisation(ctx):
    # dec0 starts at zero: N = I exactly before any training
    import dare_b200 as D
    torch = _torch()
    n = (16, 16, 16)
    net = D.LearnedPreconditioner(ctx, n, seed=0)
    u = torch.randn(int(np.prod(n)), dtype=torch.float32).cuda()
    z = torch.empty_like(u)
    net.apply(u.data_ptr(), z.data_ptr())
    assert torch.equal(z, u)


def test_gradients_match_oracle(ctx):
    import dare_b200 as D
    torch = _torch()
    n = (16, 24, 32)
    net = D.LearnedPreconditioner(ctx, n, seed=3)
    w = _weights(12, net.num_params)
    net.set_weights(w)
    N = int(np.prod(n))
    g = torch.Generator().manual_seed(9)
    r = torch.randn(2, N, generator=g, dtype=torch.float32).cuda()
    e = torch.randn(2, N, generator=g, dtype=torch.float32).cuda()
    loss, grad = net.loss_grad(r.data_ptr(), e.data_ptr(), 2)
    lo, go = O.unet_loss_grad(n, w, r.cpu().double().numpy(), e.cpu().double().numpy(), bf16=True)
    errs = {"loss": abs(loss - lo) / lo}
    for name, (sl, _) in O.unet_layer_slices().items():
        errs[name] = rel_l2(grad[sl], go[sl])
    print(errs)
    assert all(v < GRAD_TOL for v in errs.values()), errs
    # and the BF16 gradient is close to the exact (FP64, unrounded) one
    _, gx = O.unet_loss_grad(n, w, r.cpu().double().numpy(), e.cpu().double().numpy(), bf16=False)
    assert rel_l2(grad, gx) < 5e-2


def test_train_step_reduces_loss(ctx):
    import dare_b200 as D
    torch = _torch()
    n = (16, 16, 16)
    net = D.LearnedPreconditioner(ctx, n, seed=4)
    N = int(np.prod(n))
    # target: a fixed smoothing of the input (a linear map the net can represent)
    g = torch.Generator().manual_seed(2)
    r = torch.randn(4, N, generator=g, dtype=torch.float32).cuda()
    x = r.view(4, *n)
    e = (x + 0.25 * (torch.roll(x, 1, 1) + torch.roll(x, -1, 1) + torch.roll(x, 1, 3) + torch.roll(x, -1, 3)))
    e = e.reshape(4, N).contiguous()
    p = net.train_params(lr=3e-3)
    losses = [net.train_step(r.data_ptr(), e.data_ptr(), 4, p) for _ in range(60)]
    print(losses[0], losses[-1])
    assert losses[-1] < 0.5 * losses[0]
    assert net.stats()["steps"] == 60


def _operator(ctx, n, seed):
    from dare_b200 import training
    return training.Operator(ctx, training.sample_case(n, seed, "cuda:0"))


def test_learned_solver_fallback_and_fp64_residual(ctx):
    import dare_b200 as D
    n = 32
    net = D.LearnedPreconditioner(ctx, (n, n, n), seed=5)
    op = _operator(ctx, n, 101)
    solver = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 500, "tol_relative": 1})
    op.assemble()
    plain = solver.solve(op.system)
    x_plain = op.system.solution()
    # a budget of one inner iteration cannot reach 1e-10: the plain solve takes over
    op.assemble()
    rep = net.solve(op.system, solver, net.learned_params(iteration_budget=1))
    assert rep["fallback_used"] == 1 and rep["converged"] == 1
    assert rep["true_res_abs"] <= rep["tol_abs"] * 1.0000001
    # a normal budget: converged by the learned phase, checked by the FP64 residual
    op.assemble()
    rep = net.solve(op.system, solver)
    print(plain, rep)
    assert rep["converged"] == 1 and rep["fallback_used"] == 0
    assert rep["true_res_abs"] <= rep["tol_abs"]
    assert rel_l2(op.system.solution(), x_plain) < 1e-8


def test_trained_network_gains_over_identity(ctx):
    """Training on the plain solver's pairs lowers the iterations the learned
    solver needs, against the same solver with N = I (the untrained net)."""
    import dare_b200 as D
    from dare_b200 import training
    n = 32
    ident = D.LearnedPreconditioner(ctx, (n, n, n), seed=6)
    net = D.LearnedPreconditioner(ctx, (n, n, n), seed=6)
    p = net.train_params(steps=24, batch=4, lr=2e-4)
    reps = training.train(net, ctx, n, operators=6, steps_per_operator=3, params=p, seed=1000)
    first, last = reps[0]["loss_first"], np.mean([r["loss_last"] for r in reps[-3:]])
    solver = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 500, "tol_relative": 1})
    # a deep inner reduction per refinement, so the inner solves are long
    # enough for the preconditioner to show (each takes at least 2 iterations)
    lp = net.learned_params(inner_rel_tol=1e-5)
    its = {"identity": [], "trained": []}
    for seed in (5001, 5002):
        op = _operator(ctx, n, seed)
        for name, m in (("identity", ident), ("trained", net)):
            op.reset()
            op.assemble()
            r = m.solve(op.system, solver, lp)
            assert r["converged"] == 1 and r["true_res_abs"] <= r["tol_abs"]
            its[name].append(r["inner_iters"])
    print({"loss_first": first, "loss_last": last, "iters": its})
    assert last < first
    assert sum(its["trained"]) < sum(its["identity"])


# ---- the coarse-correction form N(u) = u + P U(R u) -------------------------------
def _restrict(u, n):
    """Mean of the 8 children of every coarse cell (cell layout)."""
    a = u.reshape(n[0] // 2, 2, n[1] // 2, 2, n[2] // 2, 2)
    return a.mean(axis=(1, 3, 5)).reshape(-1)


def _prolong(c, nc):
    a = c.reshape(nc)
    return np.repeat(np.repeat(np.repeat(a, 2, 0), 2, 1), 2, 2).reshape(-1)


@pytest.mark.parametrize("n", [(32, 16, 48), (16, 16, 16)])
def test_coarse_forward_matches_oracle(ctx, n):
    """z = u + P (N_c(R u) - R u) with the oracle's network N_c on the
    restricted grid and exact restriction / prolongation."""
    import dare_b200 as D
    torch = _torch()
    net = D.LearnedPreconditioner(ctx, n, seed=3, coarse=True)
    assert net.net_shape == tuple(x // 2 for x in n)
    w = _weights(13, net.num_params)
    net.set_weights(w)
    N = int(np.prod(n))
    g = torch.Generator().manual_seed(7)
    u = torch.randn(N, generator=g, dtype=torch.float32).cuda()
    z = torch.empty_like(u)
    net.apply(u.data_ptr(), z.data_ptr())
    torch.cuda.synchronize()
    uh = u.cpu().double().numpy()
    uc = _restrict(uh, n)
    zc = O.unet_forward(net.net_shape, w, uc, bf16=True)
    zo = uh + _prolong(zc - uc, net.net_shape)
    err = rel_l2(z.cpu().double().numpy() - uh, zo - uh)
    print(n, err)
    assert err < FWD_TOL
    # the restriction the network saw: its first activation is enc0 of R u
    acts = O.unet_forward(net.net_shape, w, uc, bf16=True, with_acts=True)[1]
    assert rel_l2(net.activation(0), acts["S0"]) < FWD_TOL


def test_coarse_input_off_the_16_byte_grid(ctx):
    """The level transfers use 16-byte accesses: vectors 4 bytes off that
    grid are copied first and give the same output, bit for bit."""
    import dare_b200 as D
    torch = _torch()
    n = (32, 16, 48)
    net = D.LearnedPreconditioner(ctx, n, seed=3, coarse=True)
    net.set_weights(_weights(14, net.num_params))
    N = int(np.prod(n))
    g = torch.Generator().manual_seed(8)
    buf = torch.randn(N + 4, generator=g, dtype=torch.float32).cuda()
    shifted = buf[1:N + 1]
    aligned = shifted.clone()
    out = torch.empty(N + 4, device="cuda")
    z0 = torch.empty(N, device="cuda")
    net.apply(aligned.data_ptr(), z0.data_ptr())
    net.apply(shifted.data_ptr(), out[1:N + 1].data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(z0, out[1:N + 1])


def test_coarse_identity_at_initialisation(ctx):
    import dare_b200 as D
    torch = _torch()
    n = (32, 32, 32)
    net = D.LearnedPreconditioner(ctx, n, seed=0, coarse=True)
    u = torch.randn(int(np.prod(n)), dtype=torch.float32).cuda()
    z = torch.empty_like(u)
    net.apply(u.data_ptr(), z.data_ptr())
    assert torch.equal(z, u)


def test_coarse_training_pairs_are_restrictions(ctx):
    """The ring of a coarse-form network holds (R r, R e) of the plain
    solver's pairs: the loss of its first step equals the loss of those
    restricted pairs recomputed through the public loss on the coarse grid."""
    import dare_b200 as D
    n = 32
    net = D.LearnedPreconditioner(ctx, (n, n, n), seed=8, coarse=True)
    op = _operator(ctx, n, 303)
    op.assemble()
    rep = net.train_on_system(op.system, 1e-10, net.train_params(steps=4, batch=2))
    assert rep["pairs_added"] >= 1 and rep["steps"] == 4 and np.isfinite(rep["loss_last"])


def test_coarse_learned_solver(ctx):
    """The learned solve with a coarse-form network converges to the FP64
    residual and the plain solution; after training on the plain solver's
    pairs it needs no more inner iterations than with N = I."""
    import dare_b200 as D
    from dare_b200 import training
    n = 32
    ident = D.LearnedPreconditioner(ctx, (n, n, n), seed=6, coarse=True)
    net = D.LearnedPreconditioner(ctx, (n, n, n), seed=6, coarse=True)
    p = net.train_params(steps=24, batch=4, lr=5e-4)
    reps = training.train(net, ctx, n, operators=6, steps_per_operator=3, params=p, seed=1000)
    first, last = reps[0]["loss_first"], np.mean([r["loss_last"] for r in reps[-3:]])
    solver = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 500, "tol_relative": 1})
    lp = net.learned_params(inner_rel_tol=1e-5)
    its = {"identity": [], "trained": []}
    for seed in (5001, 5002):
        op = _operator(ctx, n, seed)
        op.assemble()
        solver.solve(op.system)
        x_plain = op.system.solution()
        for name, m in (("identity", ident), ("trained", net)):
            op.reset()
            op.assemble()
            r = m.solve(op.system, solver, lp)
            assert r["converged"] == 1 and r["true_res_abs"] <= r["tol_abs"]
            assert rel_l2(op.system.solution(), x_plain) < 1e-8
            its[name].append(r["inner_iters"])
    print({"loss_first": first, "loss_last": last, "iters": its})
    assert last < first
    assert sum(its["trained"]) <= sum(its["identity"])


def test_bounded_wait_times_out_and_the_network_recovers(ctx):
    """Failure detection without a GPU fault.  A one-shot test hook leaves one
    input plane of one CTA of the next forward convolution unstaged, so that
    CTA's MMA issuer waits for a phase that never completes.  With a short
    run-time limit (1000 polls) the wait runs out: the CTA raises its abort
    flag, its roles leave their loops, it waits for its own work in flight,
    frees its tensor memory and returns.  The call reports DARE_ERR_TIMEOUT
    with the message on the context, and the next call on the same network
    and context gives the correct output bit for bit (its CTAs allocate
    tensor memory again, so none was left held)."""
    import dare_b200 as D
    torch = _torch()
    n = (16, 24, 32)
    net = D.LearnedPreconditioner(ctx, n, seed=3)
    net.set_weights(_weights(15, net.num_params))
    N = int(np.prod(n))
    u = torch.randn(N, generator=torch.Generator().manual_seed(4), dtype=torch.float32).cuda()
    z0, z1, z2 = (torch.empty_like(u) for _ in range(3))
    net.apply(u.data_ptr(), z0.data_ptr())
    net.set_wait_limit(1000)
    net.debug_skip_plane()
    with pytest.raises(D.DareError) as err:
        net.apply(u.data_ptr(), z1.data_ptr())
    assert "timed out" in str(err.value) and "status -6" in str(err.value)
    assert "timed out" in D.lib().dare_ctx_last_error(ctx.h).decode()
    net.set_wait_limit(0)
    net.apply(u.data_ptr(), z2.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(z2, z0)
