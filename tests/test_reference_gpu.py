"""Parity against satidev/gct's own CUDA FDK on identical inputs (all seven geometries).

oracle/_ref/ref_fdk is the reference's GCT::Recon::CUDA::reconstruct compiled from its sources
for sm_100a by oracle/build_ref.sh; it reads the same geometry (cast to FP32, as the reference
stores it) and the same float32 projections. The reference samples its filtered projections
through the texture unit, whose bilinear weights carry 8 fractional bits; the engine interpolates
exactly. That part of the difference is quantified separately with the FP64 oracle run both ways
(exact and 8-bit lerp weights).

Measured on B200 (geometry of the reference's own integration tests, 7 kinds): engine vs exact FP64
oracle 1.1e-6 .. 2.5e-6 relative RMS; reference vs exact oracle 1.1e-4 .. 1.4e-4; engine vs
reference equal to the latter to three digits. The whole engine/reference gap is therefore the
reference's own texture interpolation error. Asserted: engine vs exact oracle <= 1e-5; engine vs
reference <= 1.5e-4 and within 2% of the reference's distance to the exact oracle.
"""
import math
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

import gct_b200 as g
from cases import KINDS, make_case, oracle_projections
from conftest import rel_rms
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
REF_FDK = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "ref_fdk"


def run_reference(case, proj, tmp_path):
    cg, vg = case.cg, case.vg
    det = cg.det_geom()
    du = det[0].sampling_width
    dv = det[1].sampling_width if len(det) > 1 else 1.0
    nz = vg.z.num_samples if vg.z is not None else 1
    dz = vg.z.sampling_width if vg.z is not None else 1.0
    mid = tuple(vg.mid_point) + (0.0,) * (3 - len(vg.mid_point))
    inp = tmp_path / "in.bin"
    out = tmp_path / "out.bin"
    recs = np.zeros((cg.num_views, 17), dtype=np.float32)
    v = cg.views
    recs[:, 0], recs[:, 1], recs[:, 2] = v["rot_ang"], v["det_row_center"], v["det_col_center"]
    recs[:, 3], recs[:, 4] = v["src_det_dist"], v["src_iso_dist"]
    recs[:, 5:8], recs[:, 8:11], recs[:, 11:14], recs[:, 14:17] = v["src_pos"], v["det_row_dir"], v["det_col_dir"], \
        v["iso_ray_dir"]
    with open(inp, "wb") as f:
        f.write(struct.pack("<7i", int(cg.kind), cg.num_cols, cg.num_rows, cg.num_views, vg.x.num_samples,
                            vg.y.num_samples, nz))
        f.write(struct.pack("<8f", du, dv, vg.x.sampling_width, vg.y.sampling_width, dz, *mid))
        f.write(recs.tobytes())
        f.write(np.ascontiguousarray(proj, dtype=np.float32).tobytes())
    res = subprocess.run([str(REF_FDK), str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    return np.fromfile(out, dtype=np.float32).reshape(vg.shape)


def run_engine(case, proj):
    import torch
    dproj = torch.from_numpy(proj).cuda()
    vol = torch.empty(case.vg.shape, dtype=torch.float32, device="cuda")
    with g.FdkPlan(case.cg, case.vg) as plan:
        plan.execute(dproj, vol)
    torch.cuda.synchronize()
    return vol.cpu().numpy()


@pytest.fixture(scope="module")
def ref_fdk():
    if not REF_FDK.exists():
        pytest.skip("oracle/_ref/ref_fdk not built (run oracle/build_ref.sh where the reference tree exists)")
    return REF_FDK


def reference_sized_case(kind):
    """Geometry of the reference's own FDK integration tests (test/cuda/recon/fdk_axial_tests.cu:
    15-537): 360 views at 1 degree, 256 x 256 (x 5) voxels at 1 mm, SID/SDD 500/1000 (arc, flat,
    cylindrical) or 1000/1536 (line, cone-parallel), detector widths 0.8961 mm (parallel),
    0.0017922 rad (arc), 2.0 mm (line, flat) and 1.14 mm (rows); 512 columns, 32 rows."""
    return make_case(kind, nv=360, nc=512, nr=32, n=256, nz=5, vox=1.0, reference_sizes=True)


def _errors(case, proj, tmp_path):
    ref = run_reference(case, proj, tmp_path)
    got = run_engine(case, proj)
    exact = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
    return got, ref, exact


@pytest.mark.parametrize("kind", KINDS)
def test_engine_matches_reference_fdk(kind, ref_fdk, tmp_path, record_property):
    case = reference_sized_case(kind)
    proj = oracle_projections(case, scale=3.0)
    got, ref, exact = _errors(case, proj, tmp_path)
    e_ref, e_ref_exact, e_eng_exact = rel_rms(got, ref), rel_rms(ref, exact), rel_rms(got, exact)
    record_property("engine_vs_reference", e_ref)
    record_property("reference_vs_oracle_exact", e_ref_exact)
    record_property("engine_vs_oracle_exact", e_eng_exact)
    print(f"{kind}: engine-ref {e_ref:.2e}  ref-oracle(exact) {e_ref_exact:.2e}  engine-oracle(exact) {e_eng_exact:.2e}")
    assert e_eng_exact <= 1e-5
    assert e_ref <= 1.5e-4, f"{kind}: engine vs reference relRMS {e_ref:.3e}"
    assert abs(e_ref - e_ref_exact) <= 0.02 * e_ref_exact + 2e-6


@pytest.mark.parametrize("kind", KINDS)
def test_difference_is_the_reference_texture_lerp(kind, ref_fdk, tmp_path):
    # Coarse sampling magnifies the reference's 8-bit texture interpolation error. The engine's
    # own error (vs the exact FP64 oracle) stays tiny, and its distance to the reference equals
    # the reference's distance to the exact oracle; the oracle's 8-bit lerp emulation moves
    # towards the reference.
    case = make_case(kind)
    proj = oracle_projections(case)
    got, ref, exact = _errors(case, proj, tmp_path)
    tex8 = orc.fdk(case.og, case.ov, proj, lerp_bits=8).reshape(got.shape)
    e_ref, e_ref_exact, e_eng_exact = rel_rms(got, ref), rel_rms(ref, exact), rel_rms(got, exact)
    print(f"{kind}: engine-ref {e_ref:.2e}  ref-oracle(exact) {e_ref_exact:.2e}  "
          f"ref-oracle(8-bit lerp) {rel_rms(ref, tex8):.2e}  engine-oracle(exact) {e_eng_exact:.2e}")
    assert e_eng_exact <= 1e-5
    assert abs(e_ref - e_ref_exact) <= 0.02 * e_ref_exact + 2e-6
    assert rel_rms(ref, tex8) < e_ref_exact


@pytest.mark.parametrize("kind", ["cone_flat", "fan_arc"])
def test_reference_short_scan_ccw(kind, ref_fdk, tmp_path):
    case = make_case(kind, nv=100, range_rad=math.pi + 0.5, rot_dir=g.RotDir.CCW, init_ang=math.pi / 2)
    proj = oracle_projections(case)
    got, ref, exact = _errors(case, proj, tmp_path)
    assert rel_rms(got, exact) <= 1e-5
    assert abs(rel_rms(got, ref) - rel_rms(ref, exact)) <= 0.02 * rel_rms(ref, exact) + 2e-6
