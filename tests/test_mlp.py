"""The learned warm start's network: tensor-core inference against a float64
reference of the same weights, training-kernel gradients against autograd,
and training on a smooth synthetic target."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from pippin_b200 import warm

# weight array offsets (include/pippin_b200_mlp.h)
IN_MEAN, IN_SCALE, OUT_SCALE = 0, 24, 48
W1, B1 = 51, 51 + 128 * 24
W2, B2 = B1 + 128, B1 + 128 + 128 * 128
W3, B3 = B2 + 128, B2 + 128 + 128 * 128
W4, B4 = B3 + 128, B3 + 128 + 3 * 128


def random_weights(rng):
    w = np.zeros(warm.WEIGHTS, np.float32)
    w[IN_MEAN:IN_MEAN + 24] = rng.normal(0, 0.5, 24)
    w[IN_SCALE:IN_SCALE + 24] = rng.uniform(0.5, 2.0, 24)
    w[OUT_SCALE:OUT_SCALE + 3] = rng.uniform(0.5, 3.0, 3)
    for off, rows, cols in ((W1, 128, 24), (W2, 128, 128), (W3, 128, 128), (W4, 3, 128)):
        w[off:off + rows * cols] = rng.uniform(-1, 1, rows * cols) * np.sqrt(6.0 / cols)
    for off, n in ((B1, 128), (B2, 128), (B3, 128), (B4, 3)):
        w[off:off + n] = rng.normal(0, 0.1, n)
    return w


def reference(w, X, Y=None):
    """The network in float64 torch; with Y, the normalised MSE."""
    t = lambda a: torch.tensor(np.asarray(a, np.float64))
    p = t(w[W1:]).requires_grad_(Y is not None)
    off = lambda o: o - W1
    Wt = lambda o, r, c: p[off(o):off(o) + r * c].reshape(r, c)
    bt = lambda o, n: p[off(o):off(o) + n]
    x = (t(X) - t(w[IN_MEAN:IN_MEAN + 24])) * t(w[IN_SCALE:IN_SCALE + 24])
    h = torch.relu(x @ Wt(W1, 128, 24).T + bt(B1, 128))
    h = torch.relu(h @ Wt(W2, 128, 128).T + bt(B2, 128))
    h = torch.relu(h @ Wt(W3, 128, 128).T + bt(B3, 128))
    o = h @ Wt(W4, 3, 128).T + bt(B4, 3)
    if Y is None:
        return (o * t(w[OUT_SCALE:OUT_SCALE + 3])).detach().numpy()
    loss = ((o - t(Y) / t(w[OUT_SCALE:OUT_SCALE + 3])) ** 2).mean()
    loss.backward()
    return loss.item(), p.grad.numpy()


def test_forward_matches_reference():
    """BF16 operands, FP32 accumulation: within 2% of the output scale."""
    rng = np.random.default_rng(0)
    w = random_weights(rng)
    X = rng.normal(0, 1.5, (1000, 24)).astype(np.float32)
    got = warm.forward(w, X)
    ref = reference(w, X)
    scale = np.abs(ref).max(axis=0)
    assert np.all(np.abs(got - ref).max(axis=0) < 0.02 * scale), (np.abs(got - ref).max(axis=0), scale)
    assert np.abs(warm.forward(w, X[:7]) - got[:7]).max() == 0.0  # batch-independent


def test_gradients_match_autograd():
    rng = np.random.default_rng(1)
    w = random_weights(rng)
    X = rng.normal(0, 1.5, (300, 24)).astype(np.float32)
    Y = rng.normal(0, 2.0, (300, 3)).astype(np.float32)
    loss, g = warm.loss_grad(w, X, Y)
    rloss, rg = reference(w, X, Y)
    assert abs(loss - rloss) < 1e-5 * max(abs(rloss), 1.0)
    assert np.abs(g - rg).max() < 1e-4 * np.abs(rg).max(), np.abs(g - rg).max()


def test_training_fits_a_smooth_target():
    rng = np.random.default_rng(2)
    X = rng.normal(0, 1.0, (20000, 24)).astype(np.float32)
    Y = np.stack([np.sin(X[:, 0]) + X[:, 1] * X[:, 2], np.maximum(X[:, 3], 0) * 3.0, X[:, 4] - X[:, 5] ** 2],
                 axis=1).astype(np.float32)
    w, losses = warm.train(X, Y, epochs=30, batch=1000, lr=2e-3, seed=3)
    assert losses[-1] < 0.1 * losses[0], losses
    pred = warm.forward(w, X[:2000])
    assert np.mean((pred - Y[:2000]) ** 2) < 0.2 * np.mean(Y[:2000] ** 2)


def _ant(n, seed):
    from pippin_b200 import CudaPhysics, Field, mjcf, scenes
    m = mjcf.load_string(scenes.ant_xml(tolerance=1e-10, iterations=30))
    p = CudaPhysics(mjcf.to_blob(m), n)
    rng = np.random.default_rng(seed)
    p.set(Field.QPOS, range(n), np.tile(np.array(m.qpos0), (n, 1)) + rng.uniform(-0.1, 0.1, (n, m.nq)))
    p.set(Field.QVEL, range(n), rng.normal(0, 0.1, (n, m.nv)))
    return m, p, rng


def test_learned_warm_start_on_ant():
    """Train on converged Ant contact forces, then start Newton from the
    learned candidate (the minimiser of the cost on the active set the
    predicted forces give): the solution is the same as from a cold start
    (both stop at the 1e-10 gradient tolerance), and the iterations, counted
    as the reference counts them from the start the cost gate keeps, do not
    exceed the cold start's by more than 3% (forming the candidate costs one
    factorisation outside that count)."""
    from pippin_b200 import Field, WarmStart
    m, p, rng = _ant(2048, 0)
    X, F = warm.collect(p, 120, controls=lambda t: rng.uniform(-1, 1, (2048, m.nu)), skip=20)
    assert len(X) > 20000, len(X)
    assert np.all(np.isfinite(F)) and np.mean(F[:, 0] >= -1e-6) > 0.99  # normal forces push
    w, losses = warm.train(X, F, epochs=15, batch=2048, lr=1e-3, seed=1)
    assert losses[-1] < 0.5 * losses[0], losses
    # held-out states: cold vs learned on identical inputs, step by step
    m, g, rng = _ant(1024, 5)
    g.set_warm_mlp(w)
    n = 1024
    for t in range(40):
        g.set(Field.CTRL, range(n), rng.uniform(-1, 1, (n, m.nu)))
        g.step(range(n), 1)
    iters = {"cold": [], "learned": []}
    worst = 0.0
    for t in range(40):
        g.set(Field.CTRL, range(n), rng.uniform(-1, 1, (n, m.nu)))
        st = {f: g.get(f, range(n)) for f in (Field.QPOS, Field.QVEL, Field.QACC)}
        out = {}
        for mode, wm in (("cold", WarmStart.COLD), ("learned", WarmStart.LEARNED)):
            for f in st:
                g.set(f, range(n), st[f])
            g.set_solver(warm=int(wm))
            g.step(range(n), 1)
            s = g.stats()
            rows = s["nrows"] > 0
            iters[mode].append(s["iters"][rows])
            out[mode] = g.get(Field.QACC, range(n))
        scale = np.maximum(np.abs(out["cold"]).max(axis=1), 1.0)
        worst = max(worst, float((np.abs(out["learned"] - out["cold"]).max(axis=1) / scale).max()))
    cold, learned = np.concatenate(iters["cold"]), np.concatenate(iters["learned"])
    assert worst < 1e-8, worst
    assert learned.mean() < 1.03 * cold.mean(), (learned.mean(), cold.mean())


def test_learned_warm_start_on_tabletop():
    """The learned start on a model with many dof trees (the tile Newton with
    islands): training pairs come from converged island solves, and starting
    from the prediction gives the cold start's solution (both stop at the
    1e-10 gradient tolerance, behind the same per-island cost gate)."""
    from pippin_b200 import CudaPhysics, Field, Param, WarmStart, mjcf, scenes
    n = 512
    plan = scenes.tabletop(n, seed=3)
    m = mjcf.load_string(plan.xml)
    p = CudaPhysics(mjcf.to_blob(m), n)
    p.set_solver(tolerance=1e-10)
    plan.apply(lambda pid, elem, vals: p.set_param(Param(pid), elem, range(n), vals), lambda: p.reset(range(n)))
    X, F = warm.collect(p, 160, skip=60)
    assert len(X) > 20000, len(X)
    assert np.all(np.isfinite(F)) and np.mean(F[:, 0] >= -1e-6) > 0.99  # normal forces push
    w, losses = warm.train(X, F, epochs=10, batch=2048, lr=1e-3, seed=1)
    assert losses[-1] < 0.5 * losses[0], losses
    # held-out envs, still landing: cold vs learned on identical inputs
    plan = scenes.tabletop(n, seed=4)
    g = CudaPhysics(mjcf.to_blob(mjcf.load_string(plan.xml)), n)
    g.set_solver(tolerance=1e-10)
    plan.apply(lambda pid, elem, vals: g.set_param(Param(pid), elem, range(n), vals), lambda: g.reset(range(n)))
    g.set_warm_mlp(w)
    g.step(range(n), 60)
    worst, used = 0.0, 0
    iters = {"cold": [], "learned": []}
    for t in range(30):
        st = {f: g.get(f, range(n)) for f in (Field.QPOS, Field.QVEL, Field.QACC)}
        out = {}
        for mode, wm in (("cold", WarmStart.COLD), ("learned", WarmStart.LEARNED)):
            for f in st:
                g.set(f, range(n), st[f])
            g.set_solver(warm=int(wm))
            g.step(range(n), 1)
            s = g.stats()
            assert not s["status"].any()
            used += int((s["nrows"] > 0).sum())
            iters[mode].append(s["iters"][s["nrows"] > 0])
            out[mode] = g.get(Field.QACC, range(n))
        scale = np.maximum(np.abs(out["cold"]).max(axis=1), 1.0)
        worst = max(worst, float((np.abs(out["learned"] - out["cold"]).max(axis=1) / scale).max()))
    assert used > n * 10
    assert worst < 1e-8, worst
    # the candidate (the minimiser on the predicted active set) counts as an
    # iteration and still takes fewer than the cold start on resting contacts
    cold, learned = np.concatenate(iters["cold"]), np.concatenate(iters["learned"])
    assert learned.mean() <= cold.mean(), (learned.mean(), cold.mean())
