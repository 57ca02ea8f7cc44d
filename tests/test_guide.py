"""Learned path guiding: the tensor-core network kernels against the float64
restatement (oracle/guide_mlp.py), the vMF mixture sampler against its pdf,
unbiasedness of guided rendering, and the gain of the trained network.

Tolerances: forward outputs |gpu - cpu| <= 2e-3 + 1e-2 |cpu| (bf16 hidden
activations may round differently after FP32 vs FP64 accumulation); the
gradient (bf16 deltas on the device) within cosine 0.999 and 3 % in norm.
"""
import numpy as np
import pytest

import guide_mlp as G
from raymond_b200 import api, scenes
from raymond_b200._abi import SAMPLING_BSDF, SceneDesc
from raymond_b200.metrics import relmse


def _records(rng, n):
    """Random training records: features in [0, 1], unit directions, BSDF pdfs and targets."""
    f = rng.uniform(0, 1, (n, 7))
    w = rng.normal(size=(n, 3))
    w /= np.linalg.norm(w, axis=1, keepdims=True)
    pb = rng.uniform(0.05, 2.0, n)
    y = rng.exponential(1.0, n) * (rng.uniform(0, 1, n) < 0.7)
    return np.concatenate([f, w, pb[:, None], y[:, None]], axis=1).astype(np.float32)


def _sphere(m):
    """Fibonacci-sphere quadrature points."""
    k = np.arange(m) + 0.5
    z = 1 - 2 * k / m
    phi = np.pi * (1 + 5 ** 0.5) * k
    r = np.sqrt(1 - z * z)
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)


# ------------------------------------------------------------------ CPU
def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    params = G.init_params(5).astype(np.float64)
    params[-G.OUTPUTS:] += rng.normal(0, 0.3, G.OUTPUTS)  # move the output biases off their start
    rec = _records(rng, 64)
    loss, grad = G.loss_and_grad(params, rec, emulate_bf16=False)
    assert np.isfinite(loss) and grad.shape == (G.PARAMS,)
    # the descent direction is the gradient of -y log q plus the selection term with q held fixed
    q0 = G.mixture_pdf_at_records(params, rec)
    idx = np.concatenate([rng.choice(G.PARAMS, 40, replace=False), np.arange(G.PARAMS - G.OUTPUTS, G.PARAMS - 15)])
    for i in idx:
        h = 1e-6 * max(1.0, abs(params[i]))
        p1, p0 = params.copy(), params.copy()
        p1[i] += h
        p0[i] -= h
        fd = (G.surrogate(p1, rec, q0) - G.surrogate(p0, rec, q0)) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, grad[i])


def test_oracle_mixture_is_normalised():
    rng = np.random.default_rng(1)
    dirs = _sphere(200000)
    for o in rng.normal(0, 1.5, (3, G.OUTPUTS)):
        integral = G.mixture_pdf(G.decode(o[None]), dirs).mean() * 4 * np.pi
        assert abs(integral - 1) < 2e-3, integral


def test_guide_param_count(built):
    assert api.guide_param_count() == G.PARAMS == 21744


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
def test_guide_forward_matches_oracle(gpu_ctx):
    rng = np.random.default_rng(7)
    params = G.init_params(11)
    params[-G.OUTPUTS:] += rng.normal(0, 0.5, G.OUTPUTS).astype(np.float32)
    feats = rng.uniform(0, 1, (1003, 7)).astype(np.float32)  # ragged: not a multiple of 16
    feats[:5] = [0, 1, 0.5, 0, 1, 0.999, 0.001]             # bin edges
    gpu = api.guide_forward(params, feats)
    cpu, _ = G.forward(params, feats)
    err = np.abs(gpu - cpu)
    assert np.all(err <= 2e-3 + 1e-2 * np.abs(cpu)), float(err.max())


@pytest.mark.gpu
def test_guide_gradient_matches_oracle(gpu_ctx):
    rng = np.random.default_rng(9)
    params = G.init_params(2)
    params[-G.OUTPUTS:] += rng.normal(0, 0.5, G.OUTPUTS).astype(np.float32)
    rec = _records(rng, 4099)
    grad, loss = api.guide_gradient(params, rec)
    loss_c, grad_c = G.loss_and_grad(params, rec)
    cos = grad @ grad_c / (np.linalg.norm(grad) * np.linalg.norm(grad_c))
    assert cos > 0.999, cos
    assert np.linalg.norm(grad - grad_c) <= 0.03 * np.linalg.norm(grad_c)
    assert abs(loss - loss_c) <= 1e-3 * abs(loss_c) + 1e-4, (loss, loss_c)
    # per layer as well (the input layer sees the sparse one-blob inputs)
    off = 0
    for i, o in G.LAYERS:
        sl = slice(off, off + i * o + o)
        g, c = grad[sl], grad_c[sl]
        assert g @ c / (np.linalg.norm(g) * np.linalg.norm(c)) > 0.998
        off += i * o + o


@pytest.mark.gpu
def test_guide_adam_matches_oracle(gpu_ctx):
    """The device Adam step (k_guide_adam) against the float64 Adam of the
    oracle (with the device's FP32 coefficients), for a first step and a
    later one with non-zero moments: new parameters within 1e-6 relative
    (+1e-9), moments within 1e-5 relative (+1e-9 for the first moment, whose
    two terms can cancel), and the BF16 weight copy equal to the new FP32
    weights rounded."""
    rng = np.random.default_rng(21)
    n = api.guide_param_count()
    params = G.init_params(4)
    grad = (rng.normal(0, 1e-2, n) * rng.uniform(0, 1, n) ** 4).astype(np.float32)
    grad[rng.uniform(0, 1, n) < 0.1] = 0.0  # parameters without gradient (inputs never active)
    for step, m, v in [(1, np.zeros(n), np.zeros(n)),
                       (37, rng.normal(0, 1e-3, n), rng.uniform(0, 1e-4, n))]:
        m32, v32 = m.astype(np.float32), v.astype(np.float32)
        p_g, m_g, v_g, bits = api.guide_adam(params, grad, m32, v32, step, 1e-3)
        p_c, m_c, v_c = G.adam_step(params, grad, m32, v32, step, 1e-3)
        np.testing.assert_allclose(m_g, m_c, rtol=1e-5, atol=1e-9)
        np.testing.assert_allclose(v_g, v_c, rtol=1e-5, atol=1e-15)
        np.testing.assert_allclose(p_g, p_c, rtol=1e-6, atol=1e-9)
        wmask = G.weight_mask()
        want = (G.bf16(p_g[wmask]).astype(np.float32).view(np.uint32) >> 16).astype(np.uint16)
        np.testing.assert_array_equal(bits[:wmask.sum()], want)


@pytest.mark.gpu
def test_guide_mixture_sampling_matches_pdf(gpu_ctx):
    rng = np.random.default_rng(4)
    out = rng.normal(0, 1.0, G.OUTPUTS).astype(np.float32)
    out[2:32:4] = rng.uniform(0, 4, 8)  # concentrated lobes
    n = 1 << 20
    u = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    m = 1 << 18
    q = _sphere(m).astype(np.float32)
    samples, pdf_q = api.guide_mixture(out, u, q)
    # pdf normalised and close to the unpacked float64 mixture (bf16 packing)
    assert abs(pdf_q.mean() * 4 * np.pi - 1) < 5e-3
    ref = G.mixture_pdf(G.decode(out[None]), q)[0]
    assert np.all(np.abs(pdf_q - ref) <= 0.03 * ref + 1e-4)
    d = samples[:, :3]
    assert np.allclose(np.linalg.norm(d, axis=1), 1, atol=1e-5)
    # each sample's pdf is the mixture's pdf at it
    _, pdf_s = api.guide_mixture(out, u[:4096], d[:4096])
    assert np.allclose(samples[:4096, 3], pdf_s, rtol=1e-6)

    # histogram of the samples over equal-area bins against the pdf's mass
    def bins(v):
        cz = np.clip(((v[:, 2] + 1) / 2 * 32).astype(int), 0, 31)
        ph = np.clip(((np.arctan2(v[:, 1], v[:, 0]) + np.pi) / (2 * np.pi) * 64).astype(int), 0, 63)
        return cz * 64 + ph
    hist = np.bincount(bins(d), minlength=2048) / n
    mass = np.bincount(bins(q), weights=pdf_q.astype(np.float64), minlength=2048) * (4 * np.pi / m)
    tol = 4 * np.sqrt(mass / n) + 2e-4
    assert np.all(np.abs(hist - mass) <= tol), float(np.abs(hist - mass).max())


def _scene(gpu_ctx, desc_dict):
    desc = SceneDesc(desc_dict)
    return desc, api.Scene(gpu_ctx, desc)


@pytest.mark.gpu
def test_guided_render_is_unbiased(gpu_ctx):
    """Guided rendering with online training converges to the plain tracer's image."""
    _, scene = _scene(gpu_ctx, scenes.cornell(seed=1, envmap_exponent=6))
    W = H = 64
    spp = 4096
    plain = api.Renderer(scene, W, H)
    plain.render(spp=spp, max_depth=8, film_fp64=True, seed=1)
    a = plain.film64() / spp
    guided = api.Renderer(scene, W, H)
    guided.set_guide(sampling=True, training=True, batch_size=1 << 14, steps_per_batch=4, seed=3)
    guided.render(spp=spp, max_depth=8, film_fp64=True, seed=2)
    b = guided.film64() / spp
    st = guided.guide_stats()
    assert st["steps"] > 10 and np.isfinite(st["last_loss"])
    assert guided.stats()["ms_guide"] > 0
    assert abs(b.mean() / a.mean() - 1) < 0.01, (a.mean(), b.mean())
    ba = a.reshape(8, 8, 8, 8, 3).mean(axis=(1, 3))
    bb = b.reshape(8, 8, 8, 8, 3).mean(axis=(1, 3))
    assert np.all(np.abs(bb - ba) <= 0.05 * ba + 1e-3)


@pytest.mark.gpu
def test_trained_guide_lowers_error(gpu_ctx):
    """What the trained network gains: in the Cornell box traced with BSDF
    sampling alone (no light sampling), the guide learns where the small
    ceiling light is, and at equal sample count its relMSE against a
    converged reference is well below the unguided tracer's and below that of
    the same guide untrained."""
    _, scene = _scene(gpu_ctx, scenes.cornell(seed=1, envmap_exponent=6))
    W = H = 128
    depth = 8
    ref = api.Renderer(scene, W, H)
    ref.render(spp=16384, max_depth=depth, film_fp64=True, seed=9)
    reference = ref.film64() / 16384

    def relmse_of(r, seeds):
        out = []
        for s in seeds:
            r.reset()
            r.render(spp=16, max_depth=depth, seed=s, sampling_mode=SAMPLING_BSDF)
            out.append(relmse(r.film(normalize=True), reference))
        return float(np.mean(out))

    plain = api.Renderer(scene, W, H)
    e_plain = relmse_of(plain, range(100, 104))
    opts = dict(batch_size=1 << 16, step_records=1 << 14, steps_per_batch=8, seed=1)
    guided = api.Renderer(scene, W, H)
    guided.set_guide(sampling=True, training=True, **opts)
    guided.render(spp=192, max_depth=depth, seed=2, sampling_mode=SAMPLING_BSDF)  # online training
    st = guided.guide_stats()
    guided.set_guide(sampling=True, training=False, **opts)
    e_guided = relmse_of(guided, range(100, 104))
    untrained = api.Renderer(scene, W, H)
    untrained.set_guide(sampling=True, training=False, **opts)
    e_untrained = relmse_of(untrained, range(100, 104))
    print(f"relMSE plain {e_plain:.4f} untrained {e_untrained:.4f} trained {e_guided:.4f} ({st['steps']} steps)")
    assert st["steps"] > 100
    assert e_guided < 0.5 * e_plain, (e_plain, e_guided)
    assert e_guided < 0.5 * e_untrained, (e_untrained, e_guided)


@pytest.mark.gpu
def test_guide_switch_selects_the_shading_kernel(gpu_ctx):
    """A renderer compiles its shading kernel without the guide's code until
    guiding is switched on, then takes the kernel with it on the next render,
    and the plain one again once guiding is off: the plain image after the
    guided render equals the one before it, bit for bit (two samples per
    pixel, so the film's atomic sums do not depend on their order)."""
    _, scene = _scene(gpu_ctx, scenes.cornell(seed=1, envmap_exponent=6))
    W = H = 64
    r = api.Renderer(scene, W, H)
    r.render(spp=2, max_depth=8, seed=5, first_sample=0)
    before = r.film()
    r.set_guide(sampling=True, training=True, batch_size=1 << 10, steps_per_batch=2, seed=3)
    r.reset()
    r.render(spp=8, max_depth=8, seed=5, first_sample=0)
    guided = r.film()
    assert np.isfinite(guided).all() and guided.mean() > 0
    assert r.guide_stats()["steps"] > 0 and r.stats()["ms_guide"] > 0
    r.set_guide(sampling=False, training=False)
    r.reset()
    r.render(spp=2, max_depth=8, seed=5, first_sample=0)
    assert r.stats()["ms_guide"] == 0
    assert np.array_equal(r.film(), before)
