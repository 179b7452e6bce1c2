"""The FP64 reference of the merge and gather (gi_rc_merge_gather_f64) against the oracle's FP64 restatement, and the
atlas precision study (f32/f16/bf16 irradiance against it, colonnade with moving boxes)."""
import numpy as np
import pytest

import gi_cases
from oracle import bind
from rtgi import _lib, configs, gpu, precision

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = gpu.Context(0)
    yield c
    c.destroy()


def test_f64_reference_matches_oracle(ctx):
    case = gi_cases.room_lit("f32")
    sg = gpu.SceneGpu(ctx, case.scene)
    vw = gpu.VoxWorld(sg, case.vox)
    rc = gpu.Rc(ctx, case.rc, case.width, case.height)
    try:
        rc.set_frame(case.frame)
        rc.render_gbuffer(sg)
        vw.update(case.scene.camera.eye)
        with pytest.raises(_lib.GiError):
            rc.merge_gather_f64()          # traced intervals not kept yet
        rc.set_debug_hits(True)
        rc.solve(vw)
        rc.merge_gather_f64()
        irr64 = rc.read_irradiance_f64()
        irr32 = rc.read_irradiance()
        depth = rc.read_buffer(_lib.GI_RC_DEPTH).view(np.float32).reshape(case.height, case.width)
        normal = rc.read_buffer(_lib.GI_RC_NORMAL).view(np.float16).reshape(case.height, case.width, 4)
        probes = rc.read_buffer(_lib.GI_RC_PROBES).view(bind.PROBE_DTYPE)
        traced = rc.read_atlas(_lib.GI_RC_RAD_TRACED)
        rounded = {}
        for mask in (0b00001, 0b10110, 0b11111):
            rc.merge_gather_f64(f16_cascades=mask)
            rounded[mask] = rc.read_irradiance_f64()
    finally:
        for h in (rc, vw, sg):
            h.destroy()
    lay = dict(configs.cascade_layout(case.rc, case.width, case.height))
    ref = bind.merge_gather_f64(lay, case.frame, depth, normal.astype(np.float32), probes, traced)
    assert np.array_equal(irr64[..., 3], ref[..., 3])
    scale = np.abs(ref[..., :3]).max()
    assert scale > 0.0, "the lit room must carry irradiance"
    # same double operations in the same order; only exp() may differ in the last bit
    np.testing.assert_allclose(irr64, ref, rtol=1e-12, atol=1e-12 * scale)
    # the storage of some cascades rounded to f16 (round to nearest even, in the traced intervals and the merged
    # radiances above cascade 0), every stage still in double.  Rounding a merged radiance to f16 is discontinuous: where
    # exp()'s last bit moves it across a rounding boundary, GPU and oracle store neighbouring f16 values, so those
    # masks agree to 1e-12 except at a few pixels, which stay within a fraction of one f16 step.
    for mask, got in rounded.items():
        want = bind.merge_gather_f64(lay, case.frame, depth, normal.astype(np.float32), probes, traced, f16_cascades=mask)
        assert np.array_equal(got[..., 3], want[..., 3])
        assert not np.array_equal(got, irr64)
        if mask == 0b00001:   # cascade 0: only the traced intervals (identical inputs) are rounded
            np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * scale, err_msg=f"f16 cascades {mask:05b}")
            continue
        off = np.abs(got - want) > 1e-12 * scale + 1e-12 * np.abs(want)
        assert off.mean() < 0.01, f"f16 cascades {mask:05b}: {off.mean():.4f} of the values differ"
        np.testing.assert_allclose(got, want, rtol=2.0 ** -14, atol=2.0 ** -14 * scale, err_msg=f"f16 cascades {mask:05b}")
    # the f32 path's irradiance against its own FP64 merge + gather
    valid = ref[..., 3] > 0
    d = irr32[..., :3][valid].astype(np.float64) - ref[..., :3][valid]
    assert np.sqrt((d * d).sum() / (ref[..., :3][valid] ** 2).sum()) < 1e-5


def test_f64_reference_needs_f32_atlas(ctx):
    case = gi_cases.config0("f16")
    rc = gpu.Rc(ctx, case.rc, case.width, case.height)
    try:
        rc.set_debug_hits(True)
        with pytest.raises(_lib.GiError):
            rc.merge_gather_f64()
    finally:
        rc.destroy()


def test_precision_study_small(ctx):
    """Three frames of the study at 480x270: every mode valid where the reference is, errors ordered by precision."""
    r = precision.run(ctx, frames=3, width=480, height=270)
    a = r["atlases"]
    for m in ("f32", "f16", "bf16", "f16-f32out", "bf16-f32out"):
        assert a[m]["alpha_mismatch"] == 0
        assert a[m]["values"] > 0
    assert a["f32"]["rel_l2"] < 1e-5
    assert a["f32"]["rel_l2"] < a["f16"]["rel_l2"] < a["bf16"]["rel_l2"]
    assert a["f16"]["rel_l2"] < 2e-3
    assert a["bf16"]["rel_l2"] < 2e-2
    # SH and irradiance in f32: only the atlas and the merge round to 16 bits
    assert a["f16-f32out"]["rel_l2"] < a["f16"]["rel_l2"] and a["bf16-f32out"]["rel_l2"] < a["bf16"]["rel_l2"]
    # storage rounding with every stage in double: more cascades rounded, fewer atlas bytes and a larger error
    m = r["storage_rounding"]["modes"]
    assert m["c0-c4"]["atlas_bytes"] * 2 == r["storage_rounding"]["atlas_bytes_f32"]
    assert m["c4"]["atlas_bytes"] > m["c3-c4"]["atlas_bytes"] > m["c2-c4"]["atlas_bytes"] > m["c1-c4"]["atlas_bytes"]
    assert 0.0 < m["c4"]["rel_l2"] <= m["c1-c4"]["rel_l2"] <= m["c0-c4"]["rel_l2"] < 2.0 ** -10
    assert all(x["alpha_mismatch"] == 0 for x in m.values())
