"""Golden vectors of the reference's texture fetch: what the texture unit returns when the
reference's own texture objects (NDArrayTexture, src/cuda/data/nd_array_texture.cuh:33-56: linear
filter, border address mode, unnormalised float coordinates, filled by copyDevToDevTexture) are
sampled at chosen coordinates. They pin the weight rule the FP64 oracle emulates with lerp_bits.

Needs a CUDA device and oracle/_ref/ref_fdk (oracle/build_ref.sh). Usage:
    python tests/golden/make_tex_golden.py [--out tests/golden/tex_probe.npz]

Four probes, each with its texels, the (x, y) coordinates passed to tex1D / tex2D and the fetched
values: 1D and 2D textures of alternating 0 / 1 texels (the fetch returns the interpolation weight
itself, or one minus it) and of seeded random texels (the whole interpolation), at coordinates on
a 1/1024-texel grid across quantisation steps, at random coordinates, and around the borders.
"""
from __future__ import annotations

import argparse
import struct
import subprocess
import tempfile
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
REF_FDK = REPO / "oracle" / "_ref" / "ref_fdk"


def probe_inputs(seed: int = 4321) -> dict:
    rs = np.random.RandomState(seed)
    out = {}
    for dim in (1, 2):
        w, h = (256, 1) if dim == 1 else (64, 48)
        n = 2048
        # texel positions: a fine grid through two texels, random positions, and the borders
        grid = 3.0 + np.arange(1024) / 1024.0 + 1e-4
        rnd = rs.uniform(-1.5, w + 0.5, size=n - 1024 - 64)
        edge = np.concatenate([rs.uniform(-2.0, 0.5, 32), rs.uniform(w - 1.5, w + 1.0, 32)])
        xs = np.concatenate([grid, rnd, edge]).astype(np.float32) + np.float32(0.5)
        if dim == 1:
            ys = np.full(n, 0.5, dtype=np.float32)
        else:
            ys = (np.concatenate([rs.uniform(1.0, h - 2.0, 1024), rs.uniform(-1.5, h + 0.5, n - 1024)]) + 0.5)
            ys = ys.astype(np.float32)
        xy = np.stack([xs, ys], 1).astype(np.float32)
        alt = np.zeros((h, w), np.float32)
        if dim == 1:
            alt[0, 1::2] = 1.0
        else:
            alt[1::2, :] = 1.0  # rows alternate: the fetch returns the row weight
            alt[:, 1::2] += 512.0  # columns alternate with weight 512: both weights readable from one value
        out[f"d{dim}_alt"] = (alt, xy)
        out[f"d{dim}_rand"] = (rs.uniform(-1.0, 1.0, size=(h, w)).astype(np.float32), xy)
    return out


def fetch(texels: np.ndarray, xy: np.ndarray, dim: int) -> np.ndarray:
    h, w = texels.shape
    with tempfile.TemporaryDirectory() as td:
        inp, outp = Path(td) / "in.bin", Path(td) / "out.bin"
        with open(inp, "wb") as f:
            f.write(struct.pack("<4i", dim, w, h, len(xy)))
            f.write(np.ascontiguousarray(texels, np.float32).tobytes())
            f.write(np.ascontiguousarray(xy, np.float32).tobytes())
        res = subprocess.run([str(REF_FDK), "--texprobe", str(inp), str(outp)], capture_output=True, text=True,
                             timeout=120)
        if res.returncode != 0:
            raise RuntimeError(res.stderr)
        return np.fromfile(outp, dtype=np.float32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent / "tex_probe.npz"))
    args = ap.parse_args()
    arrays = {}
    for name, (tex, xy) in probe_inputs().items():
        dim = 1 if name.startswith("d1") else 2
        arrays[f"{name}_texels"] = tex
        arrays[f"{name}_xy"] = xy
        arrays[f"{name}_fetched"] = fetch(tex, xy, dim)
    np.savez_compressed(args.out, **arrays)
    print(args.out)


if __name__ == "__main__":
    main()
