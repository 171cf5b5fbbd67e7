"""Fit jobs on the GPU (vcl_fit_*): the plain and fused strategies against
full fit iterations of the CPU oracle, and against each other."""
import numpy as np
import pytest

import chain
from oracle import oracle as O
from vcl_b200 import scenes

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max(initial=0.0) / max(np.abs(b).max(initial=0.0), 1e-30)


@pytest.fixture(scope="module")
def ctx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from vcl_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()


def assert_adam_close(got, want, lr, steps, name=""):
    """Parameters after Adam steps: an Adam step is ~lr * m/sqrt(v), which
    flips with the sign of a near-zero gradient, so a few entries may differ
    by up to the step budget; the bulk must agree to FP32 rounding."""
    d = np.abs(np.asarray(got, np.float64) - np.asarray(want, np.float64)).reshape(-1)
    scale = max(1.0, float(np.abs(want).max()))
    assert d.max() <= 2.0 * lr * steps, (name, d.max())
    assert np.quantile(d, 0.99) <= 1e-5 * scale, (name, np.quantile(d, 0.99))
    assert np.mean(d > 1e-5 * scale) <= 0.01, (name, np.mean(d > 1e-5 * scale))


def _scene():
    return scenes.small(seed=21, W=96, H=64, views=2, subdiv=3, tex=64, K=6)


def _target(S):
    return np.random.default_rng(S.seed + 3).random((S.W * S.H * S.views, S.C)).astype(np.float32)


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("strategy", [0, 1])
@pytest.mark.parametrize("K", [6, 40, 70])
def test_fit_steps_match_oracle(ctx, mode, strategy, K):
    # K = 40 and 70 put two and three lobes on each lane of the fused
    # lobe-gradient kernel
    from vcl_b200 import capi
    S = _scene() if K == 6 else scenes.small(seed=21, W=96, H=64, views=2, subdiv=3, tex=64, K=K)
    tgt = _target(S)
    steps = 3
    ref = chain.oracle_fit(S, mode, steps, tgt)
    ctx.set_mode(mode)
    fit = capi.Fit(ctx, S, strategy=strategy)
    fit.set_target(tgt)
    stream = torch.cuda.Stream()
    losses = []
    for _ in range(steps):
        fit.step(stream.cuda_stream)
        losses.append(fit.read_loss(stream.cuda_stream))
    pos, tex, (ax, sh, am) = fit.read_params(stream.cuda_stream)
    fit.close()
    ctx.set_mode(0)
    assert np.allclose(losses, ref["losses"], rtol=1e-5), (losses, ref["losses"])
    # three Adam steps of size ~lr: parameters agree to far better than lr
    for name, got, want in (("tex", tex, ref["tex"]), ("pos", pos, ref["pos"]), ("axis", ax, ref["axis"]),
                            ("sharp", sh, ref["sharp"]), ("amp", am, ref["amp"])):
        assert_adam_close(got, want, S.lr, steps, name)


@pytest.mark.parametrize("mode", [0, 1])
def test_fused_odd_sizes_match_oracle(ctx, mode):
    """Image sizes that are not multiples of the kernels' tiles and warps
    (130 x 97: partial antialias tiles, warps spanning two pixel rows in the
    per-pixel backward's run aggregation, partial record chunks), three
    views and 16 lobes (two lobe groups per warp)."""
    from vcl_b200 import capi
    S = scenes.small(seed=5, W=130, H=97, views=3, subdiv=3, tex=128, K=16)
    tgt = _target(S)
    steps = 2
    ref = chain.oracle_fit(S, mode, steps, tgt)
    ctx.set_mode(mode)
    fit = capi.Fit(ctx, S, strategy=capi.FIT_FUSED)
    fit.set_target(tgt)
    stream = torch.cuda.Stream()
    losses = []
    for _ in range(steps):
        fit.step(stream.cuda_stream)
        losses.append(fit.read_loss(stream.cuda_stream))
    pos, tex, (ax, sh, am) = fit.read_params(stream.cuda_stream)
    fit.close()
    ctx.set_mode(0)
    assert np.allclose(losses, ref["losses"], rtol=1e-5), (losses, ref["losses"])
    for name, got, want in (("tex", tex, ref["tex"]), ("pos", pos, ref["pos"]), ("axis", ax, ref["axis"]),
                            ("sharp", sh, ref["sharp"]), ("amp", am, ref["amp"])):
        assert_adam_close(got, want, S.lr, steps, name)


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("strategy", [0, 1])
def test_fit_with_non_finite_target_pixels_matches_oracle(ctx, mode, strategy):
    """NaN and +-inf target pixels (a hole in a mask, a broken image) make the
    loss NaN and every gradient that flows from those pixels non-finite.  The
    reference drops such terms where it adds through its guarded add
    (common.h:181: the SG lobe sums, material.cu:428-436; the mip gradient
    push-down, buffer.cu:615-648; the Adam update, optimize.cu:106) and lets
    them through where it does not (antialias, texture and raster
    backward), so the parameters whose update was dropped keep their values
    and all parameters stay finite.  Both strategies must leave every
    parameter as the oracle's fit does."""
    from vcl_b200 import capi
    S = _scene()
    tgt = _target(S)
    N = S.W * S.H * S.views
    pick = np.random.default_rng(5).choice(N, 12, replace=False)
    tgt[pick[:4], 1] = np.nan
    tgt[pick[4:8]] = np.inf
    tgt[pick[8:], 2] = -np.inf
    steps = 3
    with np.errstate(invalid="ignore"):
        ref = chain.oracle_fit(S, mode, steps, tgt)
    ctx.set_mode(mode)
    fit = capi.Fit(ctx, S, strategy=strategy)
    fit.set_target(tgt)
    stream = torch.cuda.Stream()
    losses = []
    for _ in range(steps):
        fit.step(stream.cuda_stream)
        losses.append(fit.read_loss(stream.cuda_stream))
    pos, tex, (ax, sh, am) = fit.read_params(stream.cuda_stream)
    fit.close()
    ctx.set_mode(0)
    assert not np.isfinite(ref["losses"]).any() and not np.isfinite(losses).any(), (losses, ref["losses"])
    for name, got, want in (("tex", tex, ref["tex"]), ("pos", pos, ref["pos"]), ("axis", ax, ref["axis"]),
                            ("sharp", sh, ref["sharp"]), ("amp", am, ref["amp"])):
        assert np.isfinite(want).all() and np.isfinite(got).all(), name
        assert_adam_close(got, want, S.lr, steps, name)


@pytest.mark.parametrize("strategy", [0, 1])
def test_state_save_load_resumes(ctx, strategy):
    """A job saved after 3 steps and loaded into a fresh job of the same
    shapes continues as the original does (losses and parameters of the next
    2 steps); a state of other shapes, or not a state at all, is refused."""
    from vcl_b200 import capi
    S = _scene()
    tgt = _target(S)
    st = torch.cuda.Stream()
    a = capi.Fit(ctx, S, strategy=strategy)
    a.set_target(tgt)
    for _ in range(3):
        a.step(st.cuda_stream)
    state = a.save_state(st.cuda_stream)
    la = []
    for _ in range(2):
        a.step(st.cuda_stream)
        la.append(a.read_loss(st.cuda_stream))
    pa = a.read_params(st.cuda_stream)
    a.close()
    b = capi.Fit(ctx, S, strategy=strategy)
    b.set_target(tgt)
    b.load_state(state, st.cuda_stream)
    lb = []
    for _ in range(2):
        b.step(st.cuda_stream)
        lb.append(b.read_loss(st.cuda_stream))
    pb = b.read_params(st.cuda_stream)
    b.close()
    assert np.allclose(la, lb, rtol=1e-5), (la, lb)
    assert_adam_close(pb[0], pa[0], S.lr, 2, "pos")
    assert_adam_close(pb[1], pa[1], S.lr, 2, "tex")
    for x, y in zip(pb[2], pa[2]):
        assert_adam_close(x, y, S.lr, 2, "lobes")
    other = capi.Fit(ctx, scenes.small(seed=3, W=32, H=24, views=1, subdiv=1, tex=32, K=4), strategy=strategy)
    with pytest.raises(capi.VclError, match="another job shape"):
        other.load_state(state, st.cuda_stream)
    with pytest.raises(capi.VclError, match="bad magic"):
        other.load_state(b"x" * len(state), st.cuda_stream)
    other.close()


def test_fused_equals_plain(ctx):
    """One step from the same state agrees to rounding; over ten steps the
    two trajectories stay together (losses within 1e-3, parameters within
    the Adam step budget) -- they differ only in summation order."""
    from vcl_b200 import capi
    S = _scene()
    tgt = _target(S)
    stream = torch.cuda.Stream()
    for steps in (1, 10):
        res = []
        for strategy in (capi.FIT_PLAIN, capi.FIT_FUSED):
            fit = capi.Fit(ctx, S, strategy=strategy)
            fit.set_target(tgt)
            ls = []
            for _ in range(steps):
                fit.step(stream.cuda_stream)
                ls.append(fit.read_loss(stream.cuda_stream))
            res.append((ls, fit.read_params(stream.cuda_stream)))
            fit.close()
        (l0, (p0, t0, lb0)), (l1, (p1, t1, lb1)) = res
        if steps == 1:
            assert np.allclose(l0, l1, rtol=1e-5)
            assert_adam_close(t1, t0, S.lr, 1, "tex")
            assert_adam_close(p1, p0, S.lr, 1, "pos")
            for a, b in zip(lb0, lb1):
                assert_adam_close(b, a, S.lr, 1, "lobes")
        else:
            assert np.allclose(l0, l1, rtol=1e-3)
            for a, b in ((t0, t1), (p0, p1)) + tuple(zip(lb0, lb1)):
                assert np.abs(a - b).max() <= 2 * S.lr * steps
            assert l1[-1] < l1[0]       # the fit makes progress


def test_fused_graph_and_direct_launch_agree(ctx):
    from vcl_b200 import capi
    S = _scene()
    tgt = _target(S)
    out = []
    for use_stream in (False, True):
        fit = capi.Fit(ctx, S, strategy=capi.FIT_FUSED)
        fit.set_target(tgt)
        st = torch.cuda.Stream() if use_stream else None
        h = st.cuda_stream if st else None
        for _ in range(4):
            fit.step(h)
        torch.cuda.synchronize()
        out.append(fit.read_params(h))
        fit.close()
    for a, b in zip(out[0][:2], out[1][:2]):
        assert_adam_close(a, b, S.lr, 4)


def test_render_is_deterministic_and_switching_strategy_keeps_step_count(ctx):
    from vcl_b200 import capi
    S = _scene()
    fit = capi.Fit(ctx, S)
    img = [torch.zeros(S.W * S.H * S.views * S.C, device="cuda") for _ in range(2)]
    fit.render(img[0]); fit.render(img[1])
    torch.cuda.synchronize()
    assert torch.equal(img[0], img[1])      # forward is atomic-free: bit-identical reruns
    tgt = _target(S)
    fit.set_target(tgt)
    stream = torch.cuda.Stream()
    lm = []
    for strategy in (capi.FIT_PLAIN, capi.FIT_FUSED, capi.FIT_PLAIN):
        fit.set_strategy(strategy)
        fit.step(stream.cuda_stream)
        lm.append(fit.read_loss(stream.cuda_stream))
    p_mixed = fit.read_params(stream.cuda_stream)
    fit.close()
    ref = capi.Fit(ctx, S)
    ref.set_target(tgt)
    lp = []
    for _ in range(3):
        ref.step(stream.cuda_stream)
        lp.append(ref.read_loss(stream.cuda_stream))
    p_plain = ref.read_params(stream.cuda_stream)
    ref.close()
    # a stale gradient or a wrong step index would show up here at the size
    # of a whole Adam step; what remains is summation-order noise
    assert np.allclose(lm, lp, rtol=1e-4), (lm, lp)
    for a, b in zip(p_mixed, p_plain):
        if isinstance(a, tuple):
            for x, y in zip(a, b):
                assert np.abs(x - y).max() <= 2 * S.lr * 3
        else:
            assert np.abs(a - b).max() <= 2 * S.lr * 3


def test_staged_target_upload_equals_set_target(ctx):
    """vcl_fit_stage_target (upload on a copy stream, consumed by the next
    step) gives the same iterations as vcl_fit_set_target before each step."""
    from vcl_b200 import capi
    S = _scene()
    rng = np.random.default_rng(7)
    targets = [rng.random((S.W * S.H * S.views, S.C)).astype(np.float32) for _ in range(3)]
    stream, copy = torch.cuda.Stream(), torch.cuda.Stream()
    res = []
    for staged in (False, True):
        fit = capi.Fit(ctx, S, strategy=capi.FIT_FUSED)
        pinned = [torch.from_numpy(t.reshape(-1)).pin_memory() for t in targets]
        losses = []
        if staged:
            fit.stage_target(pinned[0], copy.cuda_stream)
        for i in range(3):
            if not staged:
                fit.set_target(targets[i], stream.cuda_stream)
            fit.step(stream.cuda_stream)
            if staged and i + 1 < 3:
                fit.stage_target(pinned[i + 1], copy.cuda_stream)
            losses.append(fit.read_loss(stream.cuda_stream))
        res.append((losses, fit.read_params(stream.cuda_stream)))
        if staged:
            with pytest.raises(capi.VclError):
                fit.stage_target(pinned[0], copy.cuda_stream)
                fit.stage_target(pinned[0], copy.cuda_stream)   # the first one was not consumed
        copy.synchronize()
        fit.close()
    (l0, p0), (l1, p1) = res
    assert np.allclose(l0, l1, rtol=1e-5)
    for a, b in zip(p0[:2], p1[:2]):
        assert_adam_close(b, a, S.lr, 3)
