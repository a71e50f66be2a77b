"""Neural path guiding: the CPU oracle against finite differences and Monte
Carlo, the CUDA network against the oracle, training, and the guided render
(unbiased, and better than plain cosine sampling at equal samples)."""
import os
import sys

import numpy as np
import pytest

import azimuth_b200 as az

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import guide_oracle as go  # noqa: E402


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _rows(rng, n, lo, hi):
    pos = lo + (hi - lo) * rng.random((n, 3))
    nrm = _unit(rng, n)
    wo = _unit(rng, n)
    wi = _unit(rng, n)
    wi = np.where(((wi * nrm).sum(1) < 0)[:, None] & (rng.random((n, 1)) < 0.7), -wi, wi)
    w = rng.uniform(0.1, 2.0, n)
    rows = np.zeros((n, 16), np.float32)
    rows[:, 0:3] = pos
    rows[:, 3] = w
    rows[:, 4:7] = nrm
    rows[:, 8:11] = wo
    rows[:, 12:15] = wi
    return rows


def _small_params(rng, scale=0.25):
    return {"mlp": rng.normal(scale=scale, size=(4, 64, 64)), "bias": rng.normal(scale=0.5, size=64)}


# ---------------------------------------------------------------- CPU: oracle
def test_oracle_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    n = 6
    o = rng.normal(size=(n, 64))
    nrm = _unit(rng, n)
    wi = _unit(rng, n)
    w = rng.uniform(0.5, 1.5, n)
    _, do = go.loss_and_grad(o, nrm, wi, w)
    eps = 1e-6
    for j in list(range(41)):
        op, om = o.copy(), o.copy()
        op[:, j] += eps
        om[:, j] -= eps
        fd = (go.loss_and_grad(op, nrm, wi, w)[0] - go.loss_and_grad(om, nrm, wi, w)[0]) / (2 * eps)
        assert abs(fd - do[:, j].sum()) <= 1e-5 * max(1.0, abs(fd)), j


def test_oracle_network_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    n = 5
    p = _small_params(rng)
    x = np.zeros((n, 64))
    x[:, :39] = rng.normal(size=(n, 39))
    nrm, wi, w = _unit(rng, n), _unit(rng, n), rng.uniform(0.5, 1.5, n)

    def loss(params, xx):
        o, _ = go.forward(params, xx, bf=False)
        return go.loss_and_grad(o, nrm, wi, w)[0]

    o, inputs = go.forward(p, x, bf=False)
    _, do = go.loss_and_grad(o, nrm, wi, w)
    dmlp, dbias, enc = go.backward(p, inputs, do, bf=False)
    eps = 1e-6
    for (l, i, j) in [(0, 3, 5), (1, 10, 20), (2, 63, 0), (3, 7, 40), (3, 12, 4)]:
        q = {"mlp": p["mlp"].copy(), "bias": p["bias"]}
        q["mlp"][l, i, j] += eps
        up = loss(q, x)
        q["mlp"][l, i, j] -= 2 * eps
        fd = (up - loss(q, x)) / (2 * eps)
        assert abs(fd - dmlp[l, i, j]) <= 1e-5 * max(1.0, abs(fd)), (l, i, j)
    for j in [0, 17, 31]:
        xp, xm = x.copy(), x.copy()
        xp[2, j] += eps
        xm[2, j] -= eps
        fd = (loss(p, xp) - loss(p, xm)) / (2 * eps)
        assert abs(fd - enc[2, j]) <= 1e-5 * max(1.0, abs(fd)), j


def test_vmf_mixture_density_integrates_to_one_and_sampler_follows_it():
    rng = np.random.default_rng(2)
    o = rng.normal(size=(1, 64))
    o[0, 3:40:5] = np.log([0.5, 2.0, 5.0, 20.0, 1.0, 8.0, 3.0, 50.0])
    nrm = np.array([[0.0, 0.0, 1.0]])
    m = 400000
    w = _unit(rng, m)
    q = go.mixture_pdf(np.repeat(o, m, 0), np.repeat(nrm, m, 0), w)
    assert abs(q.mean() * 4 * np.pi - 1.0) < 0.02
    # the lobe sampler: mean cosine to the lobe axis matches coth(kappa) - 1/kappa
    mu = np.repeat(np.array([[0.0, 0.6, 0.8]]), m, 0)
    for kap in (0.3, 4.0, 60.0):
        d = go.sample_vmf(mu, kap, rng.random(m), rng.random(m))
        assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-9)
        mean_cos = (d * mu).sum(1).mean()
        assert abs(mean_cos - (1.0 / np.tanh(kap) - 1.0 / kap)) < 5e-3


# ---------------------------------------------------------------- GPU
def _guide(gpu_scene, seed=0, **kw):
    return az.Guide(gpu_scene, seed=seed, **kw)


def _bounds(info):
    lo = info["lo"].astype(np.float64)
    return lo, lo + 1.0 / info["inv_ext"].astype(np.float64)


KERNELS = pytest.mark.parametrize("kernels", [az.GUIDE_TCGEN05, az.GUIDE_MMA_SYNC], ids=["tcgen05", "mma_sync"])


@pytest.mark.gpu
@KERNELS
def test_guide_forward_and_gradients_match_oracle(gpu, kernels):
    """Outputs, loss and every gradient of both network kernel sets (tcgen05:
    128-row tiles; mma.sync: 16-row warp tiles) against the FP64 oracle, on a
    row count that leaves a partial tile."""
    rng = np.random.default_rng(3)
    scene = az.generate_scene(az.SCENE_CORNELL, width=8, height=8, spp=1)
    with az.GpuScene(scene) as g, _guide(g, kernels=kernels) as guide:
        info = guide.info()
        assert list(info["res"]) == list(go.level_res())
        mlp = rng.normal(scale=0.2, size=(4, 64, 64)).astype(np.float32)
        bias = rng.normal(scale=0.5, size=64).astype(np.float32)
        grid = rng.uniform(-1.0, 1.0, size=(16, 1 << 19, 2)).astype(np.float32)
        guide.set_params(mlp, bias, grid)
        lo, hi = _bounds(info)
        rows = _rows(rng, 500, lo, hi)
        got = guide.eval(rows)
        ref = go.evaluate({"mlp": mlp.astype(np.float64), "bias": bias.astype(np.float64)},
                          grid.astype(np.float16).astype(np.float64), rows, info["lo"], info["inv_ext"])
    o_gpu, o_ref = got["outputs"][:, :41], ref["outputs"][:, :41]
    scale = np.abs(o_ref).max()
    assert np.abs(o_gpu - o_ref).max() <= 1e-2 * scale, np.abs(o_gpu - o_ref).max()
    assert abs(got["loss"] - ref["loss"]) <= 2e-3 * abs(ref["loss"])

    def rel(a, b):
        return np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b)
    assert rel(got["bias_grad"], ref["bias_grad"]) < 2e-2
    assert rel(got["mlp_grad"], ref["mlp_grad"]) < 3e-2
    assert rel(got["enc_grad"], ref["enc_grad"]) < 3e-2


@pytest.mark.gpu
def test_guide_training_fits_a_direction_field(gpu):
    """Maximum-likelihood fit (unit weights) of directions scattered around an
    axis that depends on the position (16 surface points, 512 directions each):
    the loss drops and the learned density peaks on the axis."""
    rng = np.random.default_rng(4)
    scene = az.generate_scene(az.SCENE_CORNELL, width=8, height=8, spp=1)
    with az.GpuScene(scene) as g, _guide(g, seed=1) as guide:
        lo, hi = _bounds(guide.info())
        n = 8192
        rows = _rows(rng, n, lo, hi)
        points = lo + (hi - lo) * rng.random((16, 3))
        rows[:, 0:3] = points[np.arange(n) % 16]
        axis = np.where((rows[:, 0:1] < (lo[0] + hi[0]) / 2), [[0.0, 1.0, 0.0]], [[0.0, 0.0, 1.0]])
        rows[:, 12:15] = go.sample_vmf(axis, 30.0, rng.random(n), rng.random(n))
        rows[:, 4:7] = axis          # normal along the axis: the cosine part can help too
        rows[:, 3] = 1.0
        losses = guide.train(rows, 300)
        after = guide.eval(rows)
    per_row = losses / n
    assert per_row[-1] < per_row[0] - 1.0, (per_row[0], per_row[-1])
    q = go.mixture_pdf(after["outputs"].astype(np.float64), rows[:, 4:7].astype(np.float64), axis)
    assert np.median(q) > 2.0     # cosine alone gives 1/pi at the axis


def _relmse(img, ref):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def _film_image(film):
    f = film.cpu().numpy().astype(np.float64)
    return f[..., :3] / f[..., 3:4]


@pytest.mark.gpu
def test_guided_render_is_unbiased(gpu):
    """Cornell box (light noise, so the image mean is measurable to a fraction of
    a percent): after training, many guided renders average to the converged
    plain render."""
    import torch
    scene = az.generate_scene(az.SCENE_CORNELL, seed=0, width=64, height=64, spp=16)
    w, h = scene.resolution()
    with az.GpuScene(scene) as g:
        film = torch.zeros((h, w, 4), device="cuda")
        ref = np.zeros((h, w, 3))
        for k in range(64):
            film.zero_()
            g.render_device(film.data_ptr(), seed=1000 + k)
            ref += _film_image(film)
        ref /= 64
        with _guide(g, seed=5) as guide:
            for k in range(12):
                film.zero_()
                guide.render(film.data_ptr(), train=True, seed=2000 + k)
            gm = np.zeros_like(ref)
            for k in range(64):
                film.zero_()
                guide.render(film.data_ptr(), train=False, seed=3000 + k)
                gm += _film_image(film)
            gm /= 64
    print("cornell 64x64: image mean reference %.6g, guided %.6g" % (ref.mean(), gm.mean()))
    assert np.isfinite(gm).all()
    assert abs(gm.mean() - ref.mean()) <= 0.01 * ref.mean()
    # per channel as well
    assert np.allclose(gm.mean(axis=(0, 1)), ref.mean(axis=(0, 1)), rtol=0.015)


@pytest.mark.gpu
def test_guided_render_beats_cosine_sampling(gpu):
    """Interior (light in room 1, camera in room 3): against an FP64-accumulated
    converged plain render, trained guides' images at equal samples have a
    lower relMSE than plain cosine sampling (medians over five renders each: one
    16-spp image's error is dominated by a few rare paths)."""
    import torch
    scene = az.generate_scene(az.SCENE_INTERIOR, seed=0, width=64, height=36, spp=16, detail=4)
    w, h = scene.resolution()
    with az.GpuScene(scene) as g:
        film = torch.zeros((h, w, 4), device="cuda")
        ref = np.zeros((h, w, 3))
        passes = 48
        for k in range(passes):                     # converged reference: 48 x 16 spp, FP64 sums
            film.zero_()
            g.render_device(film.data_ptr(), seed=1000 + k)
            ref += _film_image(film)
        ref /= passes
        e_plain = []
        for s in range(5):
            film.zero_()
            g.render_device(film.data_ptr(), seed=7 + s)
            e_plain.append(_relmse(_film_image(film), ref))
        e_guided = []
        # training sums gradients with float atomics, so a trained network varies
        # from run to run: three guides, 64 training renders each, and the median
        # over all their renders
        for gseed in (2, 3, 4):
            with _guide(g, seed=gseed) as guide:
                for k in range(64):
                    film.zero_()
                    guide.render(film.data_ptr(), train=True, seed=2000 + 100 * gseed + k)
                assert guide.info()["steps"] >= 64
                for s in range(5):
                    film.zero_()
                    guide.render(film.data_ptr(), train=False, seed=7 + s)
                    guided = _film_image(film)
                    assert np.isfinite(guided).all()
                    e_guided.append(_relmse(guided, ref))
    e_plain, e_guided = float(np.median(e_plain)), float(np.median(e_guided))
    print("interior 64x36, 16 spp: median relMSE plain %.4g, guided %.4g" % (e_plain, e_guided))
    assert e_guided < e_plain


@pytest.mark.gpu
@KERNELS
def test_adam_step_matches_the_oracle_and_training_is_deterministic(gpu, kernels):
    """One Adam step (learning rate 1e-2, betas 0.9 / 0.99, eps 1e-8) on the
    gradients az_guide_eval reports: the first step moves every parameter by
    lr * g / (|g| + eps) (both moments bias-corrected), the MLP and bias from
    the reported gradients, the hash grid from the encoding gradients scattered
    to the corners of each row's cells.  Two guides with the same seed trained
    on the same rows end with bit-identical parameters: the gradient sums do
    not depend on the order in which the GPU's threads add them."""
    rng = np.random.default_rng(6)
    scene = az.generate_scene(az.SCENE_CORNELL, width=8, height=8, spp=1)
    lr, eps = 1e-2, 1e-8
    with az.GpuScene(scene) as g:
        with _guide(g, seed=2, kernels=kernels) as guide:
            info = guide.info()
            lo, hi = _bounds(info)
            rows = _rows(rng, 4096, lo, hi)
            mlp0, bias0, grid0 = guide.params()
            grads = guide.eval(rows)
            guide.train(rows, 1)
            mlp1, bias1, grid1 = guide.params()
        finals = []
        for _ in range(2):
            with _guide(g, seed=9, kernels=kernels) as gd:
                gd.train(rows, 3)
                finals.append(gd.params())
    for p0, p1, gr in ((mlp0, mlp1, grads["mlp_grad"]), (bias0, bias1, grads["bias_grad"])):
        gr = gr.astype(np.float64)
        want = p0.astype(np.float64) - lr * gr / (np.abs(gr) + eps)
        assert np.abs(p1 - want).max() <= 2e-7 + 1e-6 * lr, np.abs(p1 - want).max()
    # the grid: encoding gradients of every row scattered to its cells' corners
    p01 = go.normalise_positions(rows[:, 0:3].astype(np.float64), info["lo"], info["inv_ext"])
    res = go.level_res()
    gg = np.zeros((16, 1 << 19, 2))
    enc = grads["enc_grad"].astype(np.float64)
    for lv in range(16):
        idx, wts = go.corners(p01, lv, res)
        for k in range(8):
            np.add.at(gg[lv], idx[:, k], wts[:, k:k + 1] * enc[:, 2 * lv:2 * lv + 2])
    touched = np.abs(gg) > 1e-5
    step = grid1.astype(np.float64) - grid0.astype(np.float64)
    assert touched.sum() > 1000
    want = -lr * gg[touched] / (np.abs(gg[touched]) + eps)
    assert np.abs(step[touched] - want).max() <= 2e-4 * lr + 1e-7
    assert np.abs(step[np.abs(gg) == 0.0]).max() == 0.0
    for a, b in zip(finals[0], finals[1]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.gpu
def test_tensor_core_inference_matches_oracle_and_the_mma_sync_path(gpu):
    """The tcgen05 proposal kernel (128 rows per CTA, BF16 operands in shared
    memory, FP32 accumulators in tensor memory) gives the network outputs of the
    numpy oracle within the BF16 tolerance of the forward test, and guided
    renders with either inference kernel give the same image."""
    import torch
    rng = np.random.default_rng(8)
    scene = az.generate_scene(az.SCENE_CORNELL, width=48, height=32, spp=4)
    with az.GpuScene(scene) as g, _guide(g, seed=5) as guide:
        info = guide.info()
        mlp = rng.normal(scale=0.2, size=(4, 64, 64)).astype(np.float32)
        bias = rng.normal(scale=0.5, size=64).astype(np.float32)
        grid = rng.uniform(-1.0, 1.0, size=(16, 1 << 19, 2)).astype(np.float32)
        guide.set_params(mlp, bias, grid)
        lo, hi = _bounds(info)
        rows = _rows(rng, 1000, lo, hi)     # not a multiple of the 128-row tile
        got = guide.infer(rows)
        ref = go.evaluate({"mlp": mlp.astype(np.float64), "bias": bias.astype(np.float64)},
                          grid.astype(np.float16).astype(np.float64), rows, info["lo"], info["inv_ext"])
        films = []
        for kind in (az.GUIDE_TCGEN05, az.GUIDE_MMA_SYNC):
            with _guide(g, seed=5, kernels=kind) as gd:
                gd.set_params(mlp, bias, grid)
                w, h = scene.resolution()
                f = torch.zeros((h, w, 4), device="cuda")
                gd.render(f.data_ptr(), train=False, seed=3)
                torch.cuda.synchronize()
                films.append(f.cpu().numpy())
    o_gpu, o_ref = got[:, :41], ref["outputs"][:, :41]
    assert np.abs(o_gpu - o_ref).max() <= 1e-2 * np.abs(o_ref).max(), np.abs(o_gpu - o_ref).max()
    a, b = films
    floor = 1e-3 * float(np.abs(b[..., :3]).mean())
    err = (np.abs(a - b)[..., :3] / np.maximum(np.abs(b[..., :3]), floor)).max(axis=-1)
    assert (err <= 1e-3).mean() >= 0.97, float((err <= 1e-3).mean())
