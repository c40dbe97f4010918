"""Light-tree NEE of the CUDA path tracer in a closed lamp-lit room: per-pixel parity with the
oracle with NEE on and off, then NEE with MIS against the plain path tracer at many samples (the
reference's unbiasedness test, tests/trace_test.cpp:3100-3173: mean ratio in [0.97, 1.03], 16 x
16-block PSNR above 30 dB over the pixels that do not see a lamp directly)."""
import numpy as np
import pytest

import oracle_lib
from test_light_nee_oracle import compare_light, lamp_box
from test_trace_gpu import assert_radiance_close, assert_scene_equal

pytestmark = pytest.mark.gpu


def device_render(r, vs, width, height, spp, seed, nee):
    import torch

    out = torch.zeros(height * width * 3, dtype=torch.float32, device="cuda")
    r.set_light_nee(nee)
    r.render(out, width, height, vs.camera, bounces=4, seed=seed, spp=spp)
    return out.cpu().numpy().reshape(height, width, 3)


def test_lamp_room_parity_and_unbiased_nee(cuda_device, oracle):
    import caelix_b200

    vs = lamp_box()
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    osc = oracle_lib.OracleScene(oracle, vs)
    assert_scene_equal(scene, osc, vs)
    r = caelix_b200.Renderer(cuda_device, scene)
    for nee in (True, False):
        gpu = device_render(r, vs, 48, 48, 2, 7, nee)
        ref, rays = osc.render(48, 48, spp=2, bounces=4, seed=7, light_nee=nee, threads=8)
        st = r.stats()
        assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == tuple(int(x) for x in rays)
        assert_radiance_close(gpu, ref)
    pt = device_render(r, vs, 64, 64, 8192, 100000, False)
    nee_img = device_render(r, vs, 64, 64, 2048, 200000, True)
    ref_mean, test_mean, psnr = compare_light(pt, nee_img, direct=8.0, block=16)
    assert ref_mean > 0.01
    assert 0.97 < test_mean / ref_mean < 1.03, (ref_mean, test_mean)
    assert psnr > 30.0, psnr
    r.close()
    scene.close()
