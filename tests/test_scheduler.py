"""The learned scheduler: FP64 oracle of its MLP (CPU), GPU training-kernel
gradients against it, GPU inference against it, and what training gains
over the fixed rule on held-out traces."""
import numpy as np
import pytest

from oracle import mlp_oracle as M


def random_problem(seed, n=200):
    rng = np.random.default_rng(seed)
    P = rng.normal(0, 0.3, M.NUM_PARAMS)
    X = rng.uniform(0, 1, (n, 6))
    T = rng.uniform(0.01, 1.0, (n, 8))
    T[rng.uniform(size=T.shape) < 0.1] = -1  # some schedules not measured
    return P, X, T


def test_oracle_gradient_matches_finite_differences():
    P, X, T = random_problem(1, n=30)
    loss, g = M.loss_and_grad(P, X, T)
    rng = np.random.default_rng(2)
    for i in rng.choice(M.NUM_PARAMS, 40, replace=False):
        e = np.zeros_like(P)
        e[i] = 1e-6
        num = (M.loss_and_grad(P + e, X, T)[0] - M.loss_and_grad(P - e, X, T)[0]) / 2e-6
        assert abs(num - g[i]) <= 1e-6 + 1e-4 * abs(num), (i, num, g[i])


def test_targets_prefer_fast_schedules():
    q = M.targets(np.array([[1.0, 2.0, -1, 1.0, 4.0, 1.1, 9.0, 1.0]]))
    assert q[0, 2] == 0 and np.isclose(q.sum(), 1)
    assert q[0, 0] == q[0, 3] > q[0, 5] > q[0, 1] > q[0, 4]


@pytest.mark.gpu
def test_gpu_gradient_matches_fp64_oracle(gpu_ctx):
    for seed in (3, 4):
        P, X, T = random_problem(seed, n=777)
        g_gpu, l_gpu = gpu_ctx.scheduler_grad(P.astype(np.float32), X.astype(np.float32),
                                              T.astype(np.float32))
        l_ref, g_ref = M.loss_and_grad(P.astype(np.float32).astype(np.float64),
                                       X.astype(np.float32), T.astype(np.float32))
        assert abs(l_gpu - l_ref) <= 1e-4 * max(1.0, abs(l_ref))
        scale = np.abs(g_ref).max()
        np.testing.assert_allclose(g_gpu, g_ref, atol=2e-4 * scale, rtol=1e-3)


@pytest.mark.gpu
def test_gpu_pick_matches_oracle(gpu_ctx):
    P, X, _ = random_problem(5, n=500)
    P = P.astype(np.float32)
    gpu_ctx.scheduler_set_weights(P)
    got = gpu_ctx.scheduler_pick(X.astype(np.float32))
    o = M.forward(P.astype(np.float64), X.astype(np.float32))[4]
    top2 = np.sort(o, axis=1)[:, -2:]
    clear = (top2[:, 1] - top2[:, 0]) > 1e-4  # skip near-ties (FP32 vs FP64)
    assert (got[clear] == o.argmax(axis=1)[clear]).all()


def scheduler_families(seed):
    from medusa_b200 import api
    return [api.rmat_params(14, 1 << 18, 0.45, 0.15, 0.15, seed=seed, wmin=1, wmax=1000),
            api.uniform_params(1 << 14, 1 << 18, seed=seed, wmin=1, wmax=1000),
            api.grid_params(40, 40, 0.1, 0.005, seed=seed)]


def collect(ctx, seeds):
    X, T, S = [], [], []
    for seed in seeds:
        for p in scheduler_families(seed):
            g = ctx.generate(p)
            for app in (0, 1):
                x, t, s = ctx.scheduler_collect(g, app, 0)
                X.append(x); T.append(t); S.append(s)
            g.close()
    return np.concatenate(X), np.concatenate(T), np.concatenate(S)


@pytest.fixture(scope="module")
def trained(gpu_ctx):
    """Scheduler trained on traces of two seeds of three generator families
    (R-MAT, uniform, grid; BFS and SSSP), plus held-out traces of a third seed."""
    train = collect(gpu_ctx, (11, 12))
    test = collect(gpu_ctx, (99,))
    loss = gpu_ctx.scheduler_train(train[0], train[1], epochs=1500, lr=3e-3, seed=7)
    yield gpu_ctx, loss, train, test
    gpu_ctx.set_policy(0)


@pytest.mark.gpu
def test_traces_are_well_formed(trained):
    _, _, (X, T, S), _ = trained
    assert len(X) > 50
    assert ((X >= 0) & (X <= 1.0001)).all()
    assert ((S >= 0) & (S < 8)).all()
    measured = T[np.arange(len(T)), S]
    assert (measured > 0).all()  # the fixed rule's own choice was timed


@pytest.mark.gpu
def test_learned_beats_or_matches_fixed_rule_on_held_out_traces(trained):
    ctx, loss, _, (X, T, S) = trained
    assert np.isfinite(loss)
    pick = ctx.scheduler_pick(X)
    t_learned = T[np.arange(len(T)), pick]
    t_fixed = T[np.arange(len(T)), S]
    assert (t_learned > 0).all()
    # per-superstep times summed: the learned choices must not lose to the
    # fixed rule by more than timer noise on graphs it never saw
    assert t_learned.sum() <= 1.05 * t_fixed.sum(), (t_learned.sum(), t_fixed.sum())


@pytest.mark.gpu
def test_learned_policy_results_identical(trained, gpu_ctx):
    """Whatever the MLP picks, BFS levels and SSSP distances are the fixed
    rule's, bit for bit."""
    ctx = trained[0]
    for p in scheduler_families(99):
        g = ctx.generate(p)
        ctx.set_policy(0)
        lv0, _ = g.bfs([3, 17])
        d0, _ = g.sssp([3, 17])
        ctx.set_policy(1)
        lv1, _ = g.bfs([3, 17])
        d1, _ = g.sssp([3, 17])
        ctx.set_policy(0)
        g.close()
        assert np.array_equal(lv0, lv1)
        assert np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
