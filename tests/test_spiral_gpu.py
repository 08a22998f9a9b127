"""Spiral (helical) FDK on the GPU against the FP64 oracle's restatement of the reference's
spiral FDK (src/cuda/recon/fdk_spiral.cuh:33-94: cosine weights and the ramp filter without
Parker weights, each slice backprojecting the rotation of views centred on its nearest view,
slices without a complete rotation left zero).

Tolerances (relative RMS over the reconstructed slices): FP32 quads 1e-4, FP16 quads 1e-3; the
slices outside the helix's complete rotations are exactly zero; host-buffer paths against one
device launch: <= 1e-6 (FP32), 1e-5 (FP16: chunked view scales can flip a half rounding).
"""
import numpy as np
import pytest

import gct_b200 as g
from cases import make_spiral_case, spiral_projections
from conftest import rel_rms
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _plan(case, storage=g.STORAGE_F32, filt=g.FILTER_FFT):
    return g.FdkPlan(case.cg, case.vg, opts=g.FdkOptions(storage=storage, filter=filt, scan=g.SCAN_SPIRAL))


def _execute(plan, case, proj):
    import torch
    vol = torch.full(case.vg.shape, float("nan"), dtype=torch.float32, device="cuda")
    plan.execute(torch.from_numpy(proj).cuda(), vol)
    torch.cuda.synchronize()
    return vol.cpu().numpy()


@pytest.mark.parametrize("storage", [g.STORAGE_F32, g.STORAGE_F16])
@pytest.mark.parametrize("name", ["cone_cyl", "cone_flat"])
def test_spiral_matches_oracle(name, storage):
    case = make_spiral_case(name)
    proj = spiral_projections(case)
    with _plan(case, storage) as p:
        got = _execute(p, case, proj)
    ref = orc.fdk_spiral(case.og, case.ov, proj)
    wins = orc.spiral_windows(case.og, case.ov)
    on = np.array([w is not None for w in wins])
    assert on.any() and not on.all()
    assert np.all(got[~on] == 0.0)
    tol = 1e-4 if storage == g.STORAGE_F32 else 1e-3
    assert rel_rms(got[on], ref[on]) <= tol


def test_spiral_host_paths_agree():
    case = make_spiral_case("cone_cyl")
    proj = spiral_projections(case)
    with _plan(case) as p:
        dev = _execute(p, case, proj)
        host = np.empty(case.vg.shape, np.float32)
        p.execute_host(proj, host)
        assert rel_rms(host, dev) <= 1e-6
        pix = case.cg.num_rows * case.cg.num_cols
        per_view = 2 * pix * 4 + (case.cg.num_rows + 4) * (case.cg.num_cols + 4) * 16
        p.execute_host_budget(proj, host, 25 * per_view + 4096)
        assert rel_rms(host, dev) <= 1e-6
    img = g.ReconImg(case.vg)
    g.reconstruct(case.cg, g.ProjectionStack(case.cg.num_cols, case.cg.num_views, case.cg.num_rows, proj), img)
    assert np.array_equal(img.elements, dev)


def test_spiral_toeplitz_filter():
    case = make_spiral_case("cone_flat")
    proj = spiral_projections(case)
    with _plan(case, g.STORAGE_F16, g.FILTER_TOEPLITZ_BF16X4) as p:
        got = _execute(p, case, proj)
        p.check()
    ref = orc.fdk_spiral(case.og, case.ov, proj)
    on = np.array([w is not None for w in orc.spiral_windows(case.og, case.ov)])
    assert rel_rms(got[on], ref[on]) <= 1e-3


def test_spiral_plans_are_not_batched():
    import torch
    case = make_spiral_case("cone_cyl")
    with _plan(case) as p:
        d = torch.zeros((case.cg.num_views, case.cg.num_rows, case.cg.num_cols), device="cuda")
        v = torch.zeros(case.vg.shape, device="cuda")
        with pytest.raises(g.GctError, match="spiral"):
            g.FdkBatch([(p, d, v)])


def test_spiral_matches_the_reference(tmp_path):
    """Against the reference's own spiral FDK (oracle/_ref/ref_fdk --spiral: its stage functions in
    the order of src/cuda/recon/fdk_spiral.cuh:33-94 on a cylindrical detector). The reference
    samples through the texture unit (1/256-texel positions) and the engine exactly: the whole gap
    must be the reference's own distance from the FP64 oracle (the texture's quantisation), within
    the bound measured on the axial cases (1.5e-4)."""
    import test_reference_gpu as tr
    if not tr.REF_FDK.exists():
        pytest.skip("oracle/_ref/ref_fdk not built")
    case = make_spiral_case("cone_cyl")
    proj = spiral_projections(case)
    with _plan(case) as p:
        got = _execute(p, case, proj)
    ref = tr.run_reference(case, proj, tmp_path, "--spiral")
    on = np.array([w is not None for w in orc.spiral_windows(case.og, case.ov)])
    # the same slices are reconstructed and the same ones left zero
    assert np.array_equal(np.any(ref != 0, axis=(1, 2)), on)
    exact = orc.fdk_spiral(case.og, case.ov, proj)
    e_ref, e_ref_oracle = rel_rms(got[on], ref[on]), rel_rms(ref[on], exact[on])
    print(f"spiral: engine-ref {e_ref:.2e}  ref-oracle {e_ref_oracle:.2e}  "
          f"engine-oracle {rel_rms(got[on], exact[on]):.2e}")
    assert e_ref <= 1.5e-4
    assert abs(e_ref - e_ref_oracle) <= 0.05 * e_ref_oracle + 2e-6
