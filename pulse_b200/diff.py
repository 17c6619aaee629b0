"""Differentiable rendering on top of render_forward / render_backward.

Parameters are per material group: RGB albedo (the material's base color),
scalar GGX roughness (perceptual roughness) and an emission scale (the
material's emissive color = scale x the group's base emission).  The loss is
the mean squared error of the image against a target image:

    loss = mean over texels and RGB of (I - target)^2,
    dloss/dI = 2 (I - target) / (3 W H)    (alpha channel ignored)

``loss_and_grad`` renders the image (frames x spp samples per texel, the
running-mean accumulation of the forward), evaluates the loss, and calls the
path-replay adjoint for the gradient of every parameter.
"""
from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np

from .layout import Material
from .tracer import Scene, Target, render_backward, render_forward


@dataclass
class GroupParams:
    """Parameters of n material groups (float32)."""

    albedo: np.ndarray          # (n, 3)
    roughness: np.ndarray       # (n,)
    emission_scale: np.ndarray  # (n,)

    def flat(self) -> np.ndarray:
        return np.concatenate([self.albedo.ravel(), self.roughness, self.emission_scale]).astype(np.float64)

    @staticmethod
    def from_flat(v, n: int) -> "GroupParams":
        v = np.asarray(v, dtype=np.float32)
        return GroupParams(v[:3 * n].reshape(n, 3).copy(), v[3 * n:4 * n].copy(), v[4 * n:5 * n].copy())

    @staticmethod
    def of_materials(materials) -> "GroupParams":
        n = len(materials)
        return GroupParams(np.array([m.base_color[:3] for m in materials], np.float32),
                           np.array([m.perceptual_roughness for m in materials], np.float32),
                           np.ones(n, np.float32))


def apply(materials, base_emission: np.ndarray, params: GroupParams):
    """The materials with the group parameters applied (one group per material)."""
    out = []
    for i, m in enumerate(materials):
        em = base_emission[i] * params.emission_scale[i]
        out.append(replace(m, base_color=(*params.albedo[i], m.base_color[3] if len(m.base_color) > 3 else 1.0),
                           emissive=(*em, 1.0), perceptual_roughness=float(params.roughness[i])))
    return out


def base_emission(materials) -> np.ndarray:
    return np.array([m.emissive[:3] for m in materials], np.float32)


def render_image(scene: Scene, view, target: Target, frames: int, **params) -> np.ndarray:
    """The mean of frames x spp samples per texel (sample indices 0 .. frames*spp - 1)."""
    for acc in range(frames):
        render_forward(scene, view, target, acc, **params)
    return target.download()


def mse(img: np.ndarray, ref: np.ndarray) -> float:
    d = img[..., :3].astype(np.float64) - ref[..., :3]
    return float(np.mean(d * d))


def dmse(img: np.ndarray, ref: np.ndarray) -> np.ndarray:
    h, w = img.shape[:2]
    g = np.zeros_like(img, dtype=np.float32)
    g[..., :3] = (2.0 * (img[..., :3].astype(np.float64) - ref[..., :3]) / (3.0 * h * w)).astype(np.float32)
    return g


def group_grad(mat_grads: np.ndarray, base_em: np.ndarray) -> GroupParams:
    """Material gradients (n, 7: base rgb, emissive rgb, roughness) -> group
    parameter gradients (the emission scale's through emissive = scale x base)."""
    return GroupParams(mat_grads[:, 0:3].astype(np.float32), mat_grads[:, 6].astype(np.float32),
                       np.sum(mat_grads[:, 3:6] * base_em, axis=1).astype(np.float32))


def loss_and_grad(scene: Scene, view, target: Target, materials, base_em, params: GroupParams, ref: np.ndarray,
                  frames: int, **render):
    """(loss, GroupParams gradient, image) of the MSE against ref at params."""
    scene.set_materials(apply(materials, base_em, params))
    h, w = ref.shape[:2]
    spp = int(render.get("spp", 1))
    img = render_image(scene, view, target, frames, **render)
    g = render_backward(scene, view, w, h, frames * spp, dmse(img, ref), **render)
    return mse(img, ref), group_grad(g, base_em), img
