"""The Toeplitz-GEMM ramp filter (split BF16 or FP16 pieces on tcgen05, FP32 accumulation) against
the FP64 oracle and against the FFT filter.

Tolerances (relative RMS): filtered rows vs the FP64 oracle <= 3e-4 (the dropped lo x lo term and
BF16 rounding of the split give ~1e-4 on small detectors, where the alternating ramp taps cancel
most of the products); full FDK with FP32 quads <= 1e-4, with FP16 quads <= 1e-3. The four-term
BF16 form (three pieces of the rows and of the central taps) and the FP16 form (rows in two FP16
pieces under a per-row scale, far taps as their hi piece with the column sums kept exact) are held
to the same bounds and must be at least as accurate as the three-term form on noisy rows; the FP16
form is also checked on rows scaled by 1e-20 and 1e20 and on all-zero views (per-row scales).
"""
import numpy as np
import pytest

import gct_b200 as g
from cases import KINDS, make_case, oracle_projections
from conftest import rel_rms
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

TOEPLITZ = g.FILTER_TOEPLITZ_BF16X3
BOTH = [g.FILTER_TOEPLITZ_BF16X3, g.FILTER_TOEPLITZ_BF16X4, g.FILTER_TOEPLITZ_F16X2]


def _filter(case, proj, filt=TOEPLITZ, params=None):
    import torch
    dproj = torch.from_numpy(proj).cuda()
    out = torch.empty_like(dproj)
    with g.FdkPlan(case.cg, case.vg, filt=params, opts=g.FdkOptions(filter=filt)) as plan:
        plan.filter(dproj, out)
        plan.check()
    return out.cpu().numpy()


def _fdk(case, proj, storage, filt=TOEPLITZ):
    import torch
    dproj = torch.from_numpy(proj).cuda()
    vol = torch.empty(case.vg.shape, dtype=torch.float32, device="cuda")
    with g.FdkPlan(case.cg, case.vg, opts=g.FdkOptions(filter=filt, storage=storage)) as plan:
        plan.execute(dproj, vol)
        plan.check()
    return vol.cpu().numpy()


@pytest.mark.parametrize("filt", BOTH)
@pytest.mark.parametrize("kind", ["cone_flat", "fan_arc"])
def test_toeplitz_filter_matches_oracle(kind, filt):
    case = make_case(kind)
    proj = oracle_projections(case)
    got = _filter(case, proj, filt)
    ref = orc.filter_stack(case.og, proj).reshape(got.shape)
    assert rel_rms(got, ref) <= 3e-4


@pytest.mark.parametrize("filt", BOTH)
@pytest.mark.parametrize("kind", ["cone_flat", "fan_arc"])
def test_toeplitz_windowed_taps(kind, filt):
    # cut-off 0.8 with a Hann window: other taps, other far-field sums (the FP16 form folds them)
    case = make_case(kind)
    proj = oracle_projections(case)
    got = _filter(case, proj, filt, g.FiltParams(0.8, g.ApodFunc.HANN))
    ref = orc.filter_stack(case.og, proj, cut_off=0.8, apod=1).reshape(got.shape)
    assert rel_rms(got, ref) <= 3e-4


@pytest.mark.parametrize("filt", BOTH)
@pytest.mark.parametrize("nc,nr,nv", [(75, 13, 37), (300, 40, 20), (1024, 8, 6), (1240, 5, 4), (2100, 4, 3)])
def test_toeplitz_odd_sizes(nc, nr, nv, filt):
    # K and N not multiples of the 64 / 256 tiles, M not a multiple of 128; K up to 1024, 2048
    # and beyond (the FP16 split keeps a row in registers up to K = 2048, two passes above)
    case = make_case("cone_flat", nv=nv, nc=nc, nr=nr)
    proj = oracle_projections(case)
    got = _filter(case, proj, filt)
    ref = orc.filter_stack(case.og, proj).reshape(got.shape)
    assert rel_rms(got, ref) <= 3e-4


@pytest.mark.parametrize("filt", BOTH)
@pytest.mark.parametrize("kind", KINDS)
def test_toeplitz_fdk_matches_oracle(kind, filt):
    case = make_case(kind)
    proj = oracle_projections(case)
    ref = orc.fdk(case.og, case.ov, proj).reshape(case.vg.shape)
    assert rel_rms(_fdk(case, proj, g.STORAGE_F32, filt), ref) <= 1e-4
    assert rel_rms(_fdk(case, proj, g.STORAGE_F16, filt), ref) <= 1e-3


def test_four_terms_at_least_as_accurate_on_noisy_rows():
    # Poisson-noisy line integrals of a large object: two BF16 pieces of the rows and of the taps
    # leave residuals of the smooth part that the ramp filter does not cancel
    case = make_case("cone_flat", nc=512, nr=16, nv=24)
    rng = np.random.default_rng(5)
    proj = oracle_projections(case, scale=3.0) * np.float32(4.0)
    counts = rng.poisson(1e5 * np.exp(-proj.astype(np.float64)))
    proj = (-np.log(np.maximum(counts, 1) / 1e5)).astype(np.float32)
    ref = orc.filter_stack(case.og, proj).reshape(proj.shape)
    e3 = rel_rms(_filter(case, proj, g.FILTER_TOEPLITZ_BF16X3), ref)
    e4 = rel_rms(_filter(case, proj, g.FILTER_TOEPLITZ_BF16X4), ref)
    e16 = rel_rms(_filter(case, proj, g.FILTER_TOEPLITZ_F16X2), ref)
    assert e4 <= e3 and e16 <= e3
    assert e4 <= 2e-4 and e16 <= 2e-4


@pytest.mark.parametrize("factor", [1e-20, 1e20])
def test_f16_form_row_scales(factor):
    # each row gets its own power-of-two scale: tiny and huge rows, and all-zero views, filter like
    # unit rows (the oracle's filter is linear)
    case = make_case("cone_flat", nc=300, nr=12, nv=10)
    proj = oracle_projections(case)
    proj[3] = 0.0
    ref = orc.filter_stack(case.og, proj).reshape(proj.shape)
    got = _filter(case, (proj.astype(np.float64) * factor).astype(np.float32), g.FILTER_TOEPLITZ_F16X2)
    assert np.all(got[3] == 0.0)
    assert rel_rms(got / factor, ref) <= 3e-4


def test_toeplitz_and_fft_agree():
    case = make_case("cone_cyl")
    proj = oracle_projections(case)
    a = _fdk(case, proj, g.STORAGE_F32, TOEPLITZ)
    b = _fdk(case, proj, g.STORAGE_F32, g.FILTER_FFT)
    assert rel_rms(a, b) <= 1e-4
