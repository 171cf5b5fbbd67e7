"""The batched engine (vcl_batch_*) and the serving loop (vcl_server_*):
jobs of different sizes give the same results alone and in the mix.

The fused step accumulates texel and vertex gradients with float atomics,
so two runs of the same job differ in summation order only; parameters are
compared with the Adam-step tolerance used for the fit tests (bulk to FP32
rounding, a few sign-flipped near-zero-gradient entries within the step
budget) and losses to 1e-4 relative."""
import numpy as np
import pytest

from vcl_b200 import scenes

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from vcl_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()


def assert_adam_close(got, want, lr, steps, name=""):
    """Over several Adam steps a sign flip at one step moves an entry by up to
    2*lr and perturbs its neighbours through the next forward pass, so: every
    entry within the step budget, 99% of them within FP32 rounding."""
    d = np.abs(np.asarray(got, np.float64) - np.asarray(want, np.float64)).reshape(-1)
    scale = max(1.0, float(np.abs(want).max()))
    assert d.max() <= 2.0 * lr * steps, (name, d.max())
    assert np.quantile(d, 0.99) <= 1e-5 * scale * steps, (name, np.quantile(d, 0.99))
    assert np.mean(d > 1e-5 * scale * steps) <= 0.01, (name, np.mean(d > 1e-5 * scale * steps))


def _mix():
    return [
        scenes.small(seed=31, W=96, H=64, views=2, subdiv=3, tex=64, K=6),
        scenes.small(seed=32, W=40, H=40, views=1, subdiv=1, tex=32, K=8),
        scenes.small(seed=33, W=128, H=96, views=3, subdiv=4, tex=128, K=12),
        scenes.small(seed=34, W=64, H=48, views=4, subdiv=2, tex=256, K=3),
    ]


def _target(S):
    return np.random.default_rng(S.seed + 3).random((S.W * S.H * S.views, S.C)).astype(np.float32)


def _alone(ctx, S, steps):
    from vcl_b200 import capi
    fit = capi.Fit(ctx, S, strategy=capi.FIT_FUSED)
    fit.set_target(_target(S))
    st = torch.cuda.Stream()
    for _ in range(steps):
        fit.step(st.cuda_stream)
    loss = fit.read_loss(st.cuda_stream)
    pos, tex, lobes = fit.read_params(st.cuda_stream)
    fit.close()
    return loss, pos, tex, lobes


def _compare(S, got, want, steps):
    (gl, gp, gt, (ga, gs, gm)), (wl, wp, wt, (wa, ws, wm)) = got, want
    assert abs(gl - wl) <= 1e-4 * abs(wl), (S.name, gl, wl)
    for name, g, w in (("pos", gp, wp), ("tex", gt, wt), ("axis", ga, wa), ("sharp", gs, ws), ("amp", gm, wm)):
        assert_adam_close(g, w, S.lr, steps, f"{S.name}:{name}")


def test_batch_step_equals_jobs_stepped_alone(ctx):
    from vcl_b200 import capi
    steps = 3
    mix = _mix()
    alone = [_alone(ctx, S, steps) for S in mix]
    batch = capi.Batch(ctx)
    fits = []
    for S in mix:
        f = capi.Fit(ctx, S)
        f.set_target(_target(S))
        batch.add(f)
        fits.append(f)
    assert len(batch) == len(mix)
    assert batch.launches_per_step() == sum(f.launches_per_step() for f in fits)
    st = torch.cuda.Stream()
    for _ in range(steps):
        batch.step(st.cuda_stream)
    for S, f, want in zip(mix, fits, alone):
        got = (f.read_loss(st.cuda_stream),) + f.read_params(st.cuda_stream)
        _compare(S, got, want, steps)
    for f in fits:
        batch.remove(f)
        f.close()
    batch.close()


def test_batch_membership_changes_between_steps(ctx):
    """A job that joins late and one that leaves early each see exactly their
    own number of iterations."""
    from vcl_b200 import capi
    mix = _mix()[:3]
    want = [_alone(ctx, S, n) for S, n in zip(mix, (4, 2, 3))]
    batch = capi.Batch(ctx)
    st = torch.cuda.Stream()
    f = [capi.Fit(ctx, S) for S in mix]
    for x, S in zip(f, mix):
        x.set_target(_target(S))
    batch.add(f[0]); batch.add(f[1])
    batch.step(st.cuda_stream)              # f0: 1, f1: 1
    batch.add(f[2])
    batch.step(st.cuda_stream)              # f0: 2, f1: 2, f2: 1
    batch.remove(f[1])
    batch.step(st.cuda_stream)              # f0: 3, f2: 2
    batch.step(st.cuda_stream)              # f0: 4, f2: 3
    for S, x, w, n in zip(mix, f, want, (4, 2, 3)):
        got = (x.read_loss(st.cuda_stream),) + x.read_params(st.cuda_stream)
        _compare(S, got, w, n)
    batch.close()
    for x in f:
        x.close()


def test_batch_repeat_runs_several_iterations_per_step(ctx):
    """A member set to three iterations per batch step advances three
    iterations each step (chained in the batch graph), the others one."""
    from vcl_b200 import capi
    mix = _mix()[:2]
    want = [_alone(ctx, mix[0], 6), _alone(ctx, mix[1], 2)]
    batch = capi.Batch(ctx)
    st = torch.cuda.Stream()
    f = [capi.Fit(ctx, S) for S in mix]
    for x, S in zip(f, mix):
        x.set_target(_target(S))
        batch.add(x)
    batch.set_repeat(f[0], 3)
    assert batch.launches_per_step() == 3 * f[0].launches_per_step() + f[1].launches_per_step()
    batch.step(st.cuda_stream)
    batch.step(st.cuda_stream)
    for S, x, w, n in zip(mix, f, want, (6, 2)):
        got = (x.read_loss(st.cuda_stream),) + x.read_params(st.cuda_stream)
        _compare(S, got, w, n)
    batch.close()
    for x in f:
        x.close()


def test_server_results_same_alone_and_in_mix(ctx):
    """Jobs submitted together, admitted under a budget that holds only part
    of them at once, interleaved in batched ticks: each job's final
    parameters and loss equal the job run alone."""
    from vcl_b200 import capi
    mix = _mix()
    iters = [5, 2, 4, 3]
    want = [_alone(ctx, S, n) for S, n in zip(mix, iters)]
    fp = [capi.footprint(S) for S in mix]
    budget = int(sorted(fp)[-1] + sorted(fp)[-2])   # the two largest fit, not all four
    srv = capi.Server(ctx, budget, max_live=3)
    st = torch.cuda.Stream()
    ids = [srv.submit(S, _target(S), n, keep_result=True) for S, n in zip(mix, iters)]
    peak = 0
    for _ in range(1000):
        live, _ = srv.tick(st.cuda_stream)
        peak = max(peak, srv.stats()["resident_bytes"])
        assert live <= 3
        if srv.pending() == 0:
            break
    assert srv.pending() == 0
    assert peak <= budget
    stats = srv.stats()
    assert stats["completed"] == len(mix)
    assert stats["iterations"] == sum(iters)
    assert 0 < stats["p50_ms"] <= stats["p99_ms"]
    for S, jid, w, n in zip(mix, ids, want, iters):
        s = srv.status(jid)
        assert s["state"] == capi.JOB_DONE and s["iters"] == n
        assert s["submit_ms"] <= s["admit_ms"] <= s["done_ms"]
        pos, tex, lobes, loss = srv.result(jid)
        _compare(S, (loss, pos, tex, lobes), w, n)
    srv.close()


def test_server_rejects_job_larger_than_budget(ctx):
    from vcl_b200 import capi
    S = _mix()[2]
    srv = capi.Server(ctx, capi.footprint(S) - 1, max_live=4)
    jid = srv.submit(S, _target(S), 2)
    assert srv.status(jid)["state"] == capi.JOB_FAILED
    srv.drain(None)
    assert srv.stats()["completed"] == 0
    srv.close()
