"""The path-replay adjoint on the GPU (pulse_render_backward).

  * against the FP64 CPU adjoint on the same seeded paths (the GPU's FP32
    forward is the oracle's bit for bit, so both replay identical paths);
  * the emission-homogeneity identity sum_c Le_c dL/dLe_c == sum w.I;
  * against central finite differences (eps 1e-3) of the MSE loss of the
    rendered image, over all 8 x 5 material-group parameters of the Cornell
    box (the differentiable workload at reduced resolution): of the seeded
    estimator (albedo and emission, in which the sampling does not move), and
    of the detached-sampling estimator the adjoint differentiates (every
    parameter, roughness included);
  * roughness, whose seeded differences also move the GGX-sampled directions:
    the adjoint and the seeded differences agree in expectation, tested over
    32 independent seeds.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from pulse_b200 import _ffi, diff, scenes
from pulse_b200.tracer import PulseError, Scene, Target, make_view, render_backward, render_forward, render_params

pytestmark = pytest.mark.gpu

PARAMS = dict(max_depth=6, nee_mode=2, light_pick=1, quirks=0)


@pytest.fixture(scope="module")
def cornell():
    d = scenes.cornell(32, 24)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 16, 4)


@pytest.mark.parametrize("no_roulette", [0, 1])
def test_backward_matches_fp64_oracle(ctx, cornell, no_roulette):
    desc, sb = cornell
    W, H, n = desc.width, desc.height, 8
    params = dict(PARAMS, no_roulette=no_roulette)
    w = np.random.default_rng(5).normal(size=(H, W, 4)).astype(np.float32)
    ref = oracle.backward(sb, desc.view, W, H, n, w, **params)[:, :7]
    sc = Scene(ctx)
    sc.set_buffers(sb)
    got = render_backward(sc, desc.view, W, H, n, w, **params)
    sc.close()
    scale = np.abs(ref).max()
    assert scale > 0
    err = np.abs(got - ref).max() / scale
    assert err < 2e-4, err


def test_emission_homogeneity_gpu(ctx, cornell):
    desc, sb = cornell
    W, H, n = desc.width, desc.height, 4
    w = np.random.default_rng(6).normal(size=(H, W, 4)).astype(np.float32)
    sc = Scene(ctx)
    sc.set_buffers(sb)
    tg = Target(ctx, W, H)
    for acc in range(n):
        render_forward(sc, desc.view, tg, acc, **PARAMS)
    img = tg.download()
    g = render_backward(sc, desc.view, W, H, n, w, **PARAMS)
    tg.close()
    sc.close()
    lhs = float(np.sum(w[..., :3].astype(np.float64) * img[..., :3]))
    le = np.array(desc.materials[3].emissive[:3], np.float64)
    assert float(g[3, 3:6] @ le) == pytest.approx(lhs, rel=1e-4)


def test_backward_rejects_unsupported(ctx, cornell):
    desc, sb = cornell
    sc = Scene(ctx)
    sc.set_buffers(sb)
    lib = ctx.lib
    v = make_view(desc.view)
    w = np.zeros((desc.height, desc.width, 4), np.float32)
    out = (_ffi.MaterialGrad * 8)()
    for bad in (dict(PARAMS, nee_mode=0), dict(PARAMS, nee_mode=1)):
        p = render_params(**bad)
        rc = lib.pulse_render_backward(sc.h, C.byref(v), desc.width, desc.height, 1, C.byref(p),
                                       w.ctypes.data_as(C.c_void_p), out)
        assert rc == _ffi.PULSE_ERR_INVALID_ARG
    p = render_params(**PARAMS)
    rc = lib.pulse_render_backward(sc.h, C.byref(v), desc.width, desc.height, 0, C.byref(p),
                                   w.ctypes.data_as(C.c_void_p), out)
    assert rc == _ffi.PULSE_ERR_INVALID_ARG
    sc.close()


def _diff_setup(ctx, W, H):
    desc = scenes.cornell(W, H)
    sc = Scene(ctx)
    ids = [sc.upload_mesh(m, 16, 4) for m in desc.meshes]
    sc.set_materials(desc.materials)
    sc.set_instances(desc.instances, ids)
    return desc, sc


def test_gradient_matches_central_differences(ctx):
    """All 40 group parameters; FD of the same seeded estimator (eps 1e-3)."""
    W, H, spp = 128, 128, 64
    desc, sc = _diff_setup(ctx, W, H)
    tg = Target(ctx, W, H)
    mats = desc.materials
    base_em = diff.base_emission(mats)
    theta = diff.GroupParams.of_materials(mats)
    theta.roughness[:] = 0.6  # inside (0, 1): the central difference stays in range
    rng = np.random.default_rng(1)
    hidden = diff.GroupParams(rng.uniform(0.1, 0.9, (8, 3)).astype(np.float32),
                              rng.uniform(0.1, 0.9, 8).astype(np.float32),
                              rng.uniform(0.1, 0.9, 8).astype(np.float32))
    # Without Russian roulette the seeded estimator is a smooth function of the
    # albedos (no path ends on a draw that moves with them), so its central
    # differences are not dominated by termination flips.
    render = dict(PARAMS, spp=spp, no_roulette=1)
    sc.set_materials(diff.apply(mats, base_em, hidden))
    ref = diff.render_image(sc, desc.view, tg, 1, **render)
    loss, grad, _ = diff.loss_and_grad(sc, desc.view, tg, mats, base_em, theta, ref, 1, **render)
    g = grad.flat()
    eps = 1e-3
    x0 = theta.flat()
    fd = np.zeros_like(x0)
    for k in range(x0.size):
        vals = []
        for s in (1, -1):
            x = x0.copy()
            x[k] += s * eps
            sc.set_materials(diff.apply(mats, base_em, diff.GroupParams.from_flat(x, 8)))
            vals.append(diff.mse(diff.render_image(sc, desc.view, tg, 1, **render), ref))
        fd[k] = (vals[0] - vals[1]) / (2 * eps)
    tg.close()
    sc.close()
    rel = np.linalg.norm(g - fd) / np.linalg.norm(fd)
    # albedo (24) and emission scale (8): the estimator is smooth in them
    sm = np.r_[0:24, 32:40]
    rel_smooth = np.linalg.norm(g[sm] - fd[sm]) / np.linalg.norm(fd[sm])
    print("relative L2 error adjoint vs FD: all", rel, "albedo+emission", rel_smooth)
    assert rel_smooth < 2e-3, (rel_smooth, g[sm], fd[sm])
    # roughness moves the GGX-sampled directions, so the seeded FD carries
    # visibility-change noise; at 1M paths it stays a few percent overall
    assert rel < 6e-2, (rel, g, fd)


def _group_rows(mats, base_em):
    def rows_at(x):
        return np.stack([m.to_words() for m in diff.apply(mats, base_em, diff.GroupParams.from_flat(x, 8))])
    return rows_at


def test_gradient_matches_detached_central_differences(ctx):
    """All 40 group parameters, roughness included, against central
    differences (eps 1e-3) of the estimator the adjoint differentiates: the
    same seeded paths with sampling detached (directions, light picks, MIS
    weights and pdfs at the current parameters), weighted by the BSDF values
    and emissions at the perturbed parameters (oracle.detached_fd, which
    evaluates eval_g itself, not its derivatives).  The loss is the MSE
    against an image rendered from hidden parameters."""
    W, H, spp = 64, 48, 16
    desc, sc = _diff_setup(ctx, W, H)
    tg = Target(ctx, W, H)
    mats = desc.materials
    base_em = diff.base_emission(mats)
    theta = diff.GroupParams.of_materials(mats)
    theta.roughness[:] = 0.6
    rng = np.random.default_rng(1)
    hidden = diff.GroupParams(rng.uniform(0.1, 0.9, (8, 3)).astype(np.float32),
                              rng.uniform(0.1, 0.9, 8).astype(np.float32),
                              rng.uniform(0.1, 0.9, 8).astype(np.float32))
    render = dict(PARAMS, spp=spp, no_roulette=1)
    sc.set_materials(diff.apply(mats, base_em, hidden))
    ref = diff.render_image(sc, desc.view, tg, 1, **render)
    loss, grad, img = diff.loss_and_grad(sc, desc.view, tg, mats, base_em, theta, ref, 1, **render)
    tg.close()
    sc.close()
    g = grad.flat()
    sb = oracle.assemble(desc.meshes, diff.apply(mats, base_em, theta), desc.instances, 16, 4)
    fd = oracle.detached_fd(sb, desc.view, W, H, spp, diff.dmse(img, ref), _group_rows(mats, base_em), theta.flat(),
                            eps=1e-3, **dict(PARAMS, no_roulette=1))
    for name, idx in (("albedo", np.r_[0:24]), ("roughness", np.r_[24:32]), ("emission", np.r_[32:40])):
        rel = np.linalg.norm(g[idx] - fd[idx]) / np.linalg.norm(fd[idx])
        print(f"{name}: relative L2 error {rel:.2e}")
        assert np.linalg.norm(fd[idx]) > 0
        assert rel < 1e-2, (name, rel, g[idx], fd[idx])


def test_roughness_gradient_agrees_with_seeded_fd_over_seeds(ctx):
    """The detached gradient and the seeded central differences (sampling
    moves with roughness: GGX half vectors, mixture pdfs, MIS weights) are two
    estimators of the same derivative of the expected image.  For a fixed
    linear functional sum(w . I) both are averaged over 32 independent seeds;
    their mean difference per roughness parameter must be within 4.5 standard
    errors (8 parameters)."""
    W, H, spp, seeds, eps = 64, 48, 32, 32, 1e-3
    desc, sc = _diff_setup(ctx, W, H)
    tg = Target(ctx, W, H)
    mats = desc.materials
    base_em = diff.base_emission(mats)
    theta = diff.GroupParams.of_materials(mats)
    theta.roughness[:] = 0.6
    w = np.random.default_rng(9).normal(size=(H, W, 4)).astype(np.float32) / (W * H)
    wv = w[..., :3].astype(np.float64)
    render = dict(PARAMS, spp=spp, no_roulette=1)
    x0 = theta.flat()
    d = np.zeros((seeds, 8))
    for s in range(seeds):
        sc.set_materials(diff.apply(mats, base_em, theta))
        gm = render_backward(sc, desc.view, W, H, spp, w, **dict(render, seed=s))
        g = diff.group_grad(gm, base_em).flat()[24:32]
        for j in range(8):
            vals = []
            for sgn in (1, -1):
                x = x0.copy()
                x[24 + j] += sgn * eps
                sc.set_materials(diff.apply(mats, base_em, diff.GroupParams.from_flat(x, 8)))
                vals.append(float(np.sum(wv * diff.render_image(sc, desc.view, tg, 1, **dict(render, seed=s))[..., :3])))
            step = float(np.float32(x0[24 + j] + eps)) - float(np.float32(x0[24 + j] - eps))
            d[s, j] = g[j] - (vals[0] - vals[1]) / step
    tg.close()
    sc.close()
    z = d.mean(axis=0) / (d.std(axis=0, ddof=1) / np.sqrt(seeds))
    print("roughness: mean difference in standard errors", np.round(z, 2))
    assert np.all(np.abs(z) <= 4.5), z


def test_materials_set_relights_prepared_scene(ctx):
    """Doubling the only light's emission doubles every texel exactly (each
    contribution is a product with Le; the one-light CDF stays 1), so a
    material update must reach the renderer and its light data."""
    desc, sc = _diff_setup(ctx, 40, 30)
    tg = Target(ctx, 40, 30)
    a = diff.render_image(sc, desc.view, tg, 2, **PARAMS)
    mats = list(desc.materials)
    light = mats[3]
    mats[3] = type(light)(light.base_color, tuple(2.0 * x for x in light.emissive[:3]) + (1.0,),
                          light.perceptual_roughness, light.reflectance, light.metallic)
    sc.set_materials(mats)
    b = diff.render_image(sc, desc.view, tg, 2, **PARAMS)
    assert np.array_equal(b[..., :3], 2.0 * a[..., :3])
    sc.set_materials(mats[:3])  # the instances use material 7: not ready until they are set again
    with pytest.raises(PulseError) as e:
        diff.render_image(sc, desc.view, tg, 1, **PARAMS)
    assert e.value.code == _ffi.PULSE_ERR_NOT_READY
    tg.close()
    sc.close()
