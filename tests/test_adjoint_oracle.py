"""The FP64 CPU adjoint (oracle.backward) on its own: the BRDF derivative
against central differences, and exact identities of the detached estimator.

  * Homogeneity: with one light the image is linear in that light's emissive
    color (the sampling does not depend on it), so for any dloss/dimage w,
    sum_c Le_c * d(sum w.I)/dLe_c == sum w.I over the image.
  * Linearity: the gradient is linear in dloss/dimage.
"""
import numpy as np
import pytest

import oracle
from pulse_b200 import scenes
from pulse_b200.layout import Material


@pytest.fixture(scope="module")
def cornell():
    d = scenes.cornell(24, 20)
    return d, oracle.assemble(d.meshes, d.materials, d.instances, 16, 4)


PARAMS = dict(max_depth=6, nee_mode=2, light_pick=1, quirks=0)


def _unit(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("metal,rough", [(0.0, 1.0), (0.0, 0.3), (1.0, 0.5), (0.4, 0.12)])
def test_eval_g_grad_matches_central_differences(metal, rough):
    rng = np.random.default_rng(7)
    for _ in range(20):
        n = _unit(rng.normal(size=3))
        wo = _unit(n + 0.8 * rng.normal(size=3))
        wi = _unit(n + 0.8 * rng.normal(size=3))
        if n @ wo <= 0.05 or n @ wi <= 0.05:
            continue
        base = rng.uniform(0.1, 0.9, 3)
        row = Material((*base, 1.0), (0, 0, 0, 1), rough, 0.5, metal).to_words()
        g = oracle.eval_g_grad(n, wo, wi, row)
        h = 1e-3
        for c in range(3):
            rp, rm = row.copy(), row.copy()
            rp[c] += h
            rm[c] -= h
            fd = (oracle.eval_g_grad(n, wo, wi, rp)[0, c] - oracle.eval_g_grad(n, wo, wi, rm)[0, c]) / (2 * h)
            assert g[1, c] == pytest.approx(fd, rel=2e-3, abs=1e-6)
        rp, rm = row.copy(), row.copy()
        rp[8] += h
        rm[8] -= h
        fd = (oracle.eval_g_grad(n, wo, wi, rp)[0] - oracle.eval_g_grad(n, wo, wi, rm)[0]) / (2 * h)
        assert np.allclose(g[2], fd, rtol=5e-3, atol=1e-6)


def test_emission_homogeneity(cornell):
    desc, sb = cornell
    W, H, n = desc.width, desc.height, 4
    rng = np.random.default_rng(3)
    w = rng.normal(size=(H, W, 4)).astype(np.float32)
    g = oracle.backward(sb, desc.view, W, H, n, w, **PARAMS)
    # sum w . I with I the mean over samples 0..n-1 (FP64 accumulation of the FP32 paths)
    img = np.zeros((H, W, 4), np.float32)
    for acc in range(n):
        oracle.render(sb, desc.view, W, H, acc, image=img, **PARAMS)
    lhs = float(np.sum(w[..., :3].astype(np.float64) * img[..., :3]))
    light = 3  # the ceiling light's material
    le = np.array(desc.materials[light].emissive[:3], np.float64)
    rhs = float(g[light, 3:6] @ le)
    assert rhs == pytest.approx(lhs, rel=1e-4)
    # the other materials emit nothing: their emissive gradient is still defined
    assert np.isfinite(g).all()


def test_backward_linear_in_dloss(cornell):
    desc, sb = cornell
    W, H = desc.width, desc.height
    rng = np.random.default_rng(4)
    a = rng.normal(size=(H, W, 4)).astype(np.float32)
    b = rng.normal(size=(H, W, 4)).astype(np.float32)
    ga = oracle.backward(sb, desc.view, W, H, 2, a, **PARAMS)
    gb = oracle.backward(sb, desc.view, W, H, 2, b, **PARAMS)
    gab = oracle.backward(sb, desc.view, W, H, 2, (2 * a + b).astype(np.float32), **PARAMS)
    scale = np.abs(gab).max()
    assert np.allclose(gab, 2 * ga + gb, atol=1e-5 * scale)
    gz = oracle.backward(sb, desc.view, W, H, 2, np.zeros((H, W, 4), np.float32), **PARAMS)
    assert not gz.any()


def test_backward_rejects_other_modes(cornell):
    desc, sb = cornell
    with pytest.raises(ValueError):
        # the wrapper forces nee_mode 2; the C entry point refuses others
        oracle.lib().oracle_backward.argtypes  # noqa: B018 -- bound
        p = oracle.make_params(**dict(PARAMS, nee_mode=0))
        import ctypes as C
        rc = oracle.lib().oracle_backward(None, None, None, 1, 1, 1, C.byref(p), None, 0, None, 1)
        if rc != 0:
            raise ValueError("refused")


def _group_setup(W, H, rough=0.6):
    from pulse_b200 import diff
    desc = scenes.cornell(W, H)
    mats = desc.materials
    base_em = diff.base_emission(mats)
    theta = diff.GroupParams.of_materials(mats)
    theta.roughness[:] = rough
    sb = oracle.assemble(desc.meshes, diff.apply(mats, base_em, theta), desc.instances, 16, 4)

    def rows_at(x):
        return np.stack([m.to_words() for m in diff.apply(mats, base_em, diff.GroupParams.from_flat(x, 8))])
    return desc, sb, theta, base_em, rows_at


def test_adjoint_matches_detached_central_differences():
    """The FP64 adjoint against central differences (eps 1e-3) of the
    detached-sampling estimator (oracle.detached_fd: the same FP32 paths,
    weighted by the perturbed materials), for all 8 x 5 group parameters
    including roughness.  The differences evaluate eval_g itself, not the
    derivative formulas, so this pins the adjoint's roughness derivative
    independently of its derivation."""
    from pulse_b200 import diff
    W, H, n = 20, 16, 8
    desc, sb, theta, base_em, rows_at = _group_setup(W, H)
    params = dict(PARAMS, no_roulette=1)
    w = np.random.default_rng(11).normal(size=(H, W, 4)).astype(np.float32)
    g = oracle.backward(sb, desc.view, W, H, n, w, **params)[:, :7]
    grad = diff.group_grad(g, base_em).flat()
    fd = oracle.detached_fd(sb, desc.view, W, H, n, w, rows_at, theta.flat(), eps=1e-3, **params)
    for name, idx in (("albedo", np.r_[0:24]), ("roughness", np.r_[24:32]), ("emission", np.r_[32:40])):
        rel = np.linalg.norm(grad[idx] - fd[idx]) / np.linalg.norm(fd[idx])
        assert np.linalg.norm(fd[idx]) > 0, name
        assert rel < 1e-3, (name, rel, grad[idx], fd[idx])
