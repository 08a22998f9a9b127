"""The texture unit's linear filter, pinned by golden vectors fetched through the reference's own
texture objects (tests/golden/tex_probe.npz, made on a B200 by tests/golden/make_tex_golden.py
with oracle/_ref/ref_fdk --texprobe: NDArrayTexture, src/cuda/data/nd_array_texture.cuh:33-56,
filled by copyDevToDevTexture).

The reference backprojects through tex1D / tex2D (src/cuda/recon/back_proj.cuh:38,75); what the
unit returns is therefore part of the reference's result. Measured rule: the sample position
snaps to the nearest 1/256 of a texel on each axis, and the bilinear corner weight a b snaps to
the nearest 1/256 as well, the other three weights being a - w11, b - w11 and 1 - a - b + w11.
The FP64 oracle's lerp_bits=8 mode (or_tex_fetch, the interpolation or_fdk uses) reproduces all
8192 probe fetches to within float32 rounding of the unit's result (<= 6e-8 absolute on values
up to 1 and <= 2e-5 on values up to 513); exact weights, position truncation instead of rounding,
and products of snapped weights without the corner rule all miss by 1e-3 or more.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as orc

GOLDEN = Path(__file__).resolve().parent / "golden" / "tex_probe.npz"
PROBES = ("d1_alt", "d1_rand", "d2_alt", "d2_rand")


def _probe(name):
    z = np.load(GOLDEN)
    return z[f"{name}_texels"], z[f"{name}_xy"], z[f"{name}_fetched"].astype(np.float64)


@pytest.mark.parametrize("name", PROBES)
def test_oracle_fetch_reproduces_the_texture_unit(name):
    tex, xy, fetched = _probe(name)
    got = orc.tex_fetch(tex, xy, lerp_bits=8)
    tol = 2.0 ** -24 * max(1.0, float(np.abs(fetched).max())) * 2
    assert np.abs(got - fetched).max() <= tol


@pytest.mark.parametrize("name", ["d1_rand", "d2_rand"])
def test_other_rules_do_not(name):
    tex, xy, fetched = _probe(name)
    assert np.abs(orc.tex_fetch(tex, xy, lerp_bits=0) - fetched).max() > 1e-3
    h, w = tex.shape
    x, y = xy[:, 0].astype(np.float64) - 0.5, xy[:, 1].astype(np.float64) - 0.5

    def emulate(snap, corner):
        xs, ys = snap(x), snap(y)
        i, j = np.floor(xs).astype(int), np.floor(ys).astype(int)
        a, b = xs - i, ys - j

        def T(ii, jj):
            ok = (ii >= 0) & (ii < w) & (jj >= 0) & (jj < h)
            return np.where(ok, tex[np.clip(jj, 0, h - 1), np.clip(ii, 0, w - 1)], 0.0)
        w11 = corner(a, b)
        return (1 - a - b + w11) * T(i, j) + (a - w11) * T(i + 1, j) + (b - w11) * T(i, j + 1) + w11 * T(i + 1, j + 1)
    down = lambda v: np.floor(v * 256) / 256
    near = lambda v: np.floor(v * 256 + 0.5) / 256
    assert np.abs(emulate(down, lambda a, b: near(a * b)) - fetched).max() > 1e-3
    if name == "d2_rand":
        assert np.abs(emulate(near, lambda a, b: a * b) - fetched).max() > 1e-3
    assert np.abs(emulate(near, lambda a, b: near(a * b)) - fetched).max() < 1e-6


def test_probe_covers_steps_borders_and_both_dimensions():
    for name in PROBES:
        tex, xy, fetched = _probe(name)
        h, w = tex.shape
        assert len(xy) == len(fetched) == 2048
        x = xy[:, 0].astype(np.float64) - 0.5
        assert (x < 0).any() and (x > w - 1).any()  # border texels
        assert np.unique(np.floor((x[:1024] - np.floor(x[:1024])) * 256)).size == 256  # every 1/256 step
        if name.startswith("d2"):
            y = xy[:, 1].astype(np.float64) - 0.5
            assert (y < 0).any() and (y > h - 1).any()
