"""The adjoint (caelix_renderer_backward) on the differentiation workload: the solid-brick world of
the plain light-tree build (4096 brick records in a 32^3 brick grid), 256 x 256, 8 spp, 3 bounces,
L2 loss against a target rendered with albedo and power perturbed by up to 10 %.
* the backward call's forward image is bit-identical to caelix_renderer_render;
* its gradients match the double-precision reference (oracle oc_adjoint: the same estimator with
  the sampling quantities held fixed, reverse accumulation in double) within 1e-3 relative;
* they match central finite differences (eps = 1e-3) of the frozen estimator, evaluated in
  double, within 1e-3 relative, on the largest albedo and power gradients."""
import numpy as np
import pytest

import oracle_lib
from caelix_b200 import workloads

pytestmark = pytest.mark.gpu

W = H = 256
SPP = 8
BOUNCES = 3
EPS = 1e-3
REL = 1e-3


@pytest.fixture(scope="module")
def workload(cuda_device, oracle):
    import torch

    import caelix_b200

    vs = workloads.solid_brick_scene()
    target_vs = workloads.perturbed(vs)
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    tscene = caelix_b200.Scene.from_voxel_scene(cuda_device, target_vs)
    r = caelix_b200.Renderer(cuda_device, scene)
    tr = caelix_b200.Renderer(cuda_device, tscene)
    img = torch.zeros(H * W * 3, device="cuda")
    tgt = torch.zeros(H * W * 3, device="cuda")
    r.render(img, W, H, vs.camera, bounces=BOUNCES, seed=1, spp=SPP)
    tr.render(tgt, W, H, vs.camera, bounces=BOUNCES, seed=1, spp=SPP)
    d_rad = 2.0 * (img - tgt)
    d_alb = torch.zeros(65536 * 3, device="cuda")
    d_pow = torch.zeros(vs.brick_count, device="cuda")
    fwd = torch.zeros_like(img)
    r.backward(d_rad, W, H, vs.camera, d_alb, d_pow, bounces=BOUNCES, seed=1, spp=SPP, image=fwd)
    torch.cuda.synchronize()
    osc = oracle_lib.OracleScene(oracle, vs)
    _, rA, rP = osc.adjoint(W, H, spp=SPP, bounces=BOUNCES, seed=1, d_radiance=d_rad.cpu().numpy(), threads=8)
    out = dict(vs=vs, img=img.cpu().numpy(), tgt=tgt.cpu().numpy().astype(np.float64), fwd=fwd.cpu().numpy(),
               gA=d_alb.cpu().numpy().reshape(65536, 3).astype(np.float64), gP=d_pow.cpu().numpy().astype(np.float64),
               rA=rA, rP=rP, osc=osc)
    yield out
    osc.close()
    r.close()
    tr.close()
    scene.close()
    tscene.close()


def test_backward_forward_image_is_the_render(workload):
    assert workload["fwd"].view(np.uint32).tobytes() == workload["img"].view(np.uint32).tobytes()


def close(gpu, ref, floor):
    """Per-entry relative error within REL for entries at least `floor` of the largest."""
    scale = np.abs(ref).max()
    big = np.abs(ref) >= floor * scale
    rel = np.abs(gpu[big] - ref[big]) / np.abs(ref[big])
    assert big.sum() > 0
    return float(rel.max()), int(big.sum()), float(np.abs(gpu - ref).max() / scale)


def test_gradients_match_the_double_reference(workload):
    codes = 0x8000 + np.arange(1, 65)  # the workload's material codes
    rel_a, n_a, abs_a = close(workload["gA"][codes], workload["rA"][codes], 1e-3)
    rel_p, n_p, abs_p = close(workload["gP"], workload["rP"], 1e-3)
    assert rel_a <= REL and abs_a <= REL, (rel_a, abs_a)
    assert rel_p <= REL and abs_p <= REL, (rel_p, abs_p)
    assert n_a >= 100 and n_p >= 50


def test_gradients_match_central_differences(workload):
    vs, osc = workload["vs"], workload["osc"]
    A0 = osc.albedo_table.astype(np.float64)  # the material table's albedo, by code
    P0 = vs.power.astype(np.float64)

    def loss(A=None, P=None):
        image, _, _ = osc.adjoint(W, H, spp=SPP, bounces=BOUNCES, seed=1, A=A, P=P, threads=8)
        return float(((image.reshape(-1) - workload["tgt"]) ** 2).sum())

    gA, gP = workload["gA"], workload["gP"]
    rows = sorted([tuple(x) for x in np.argwhere(np.abs(gA) > 0)], key=lambda rc: -abs(gA[rc]))[:4]
    for rc in rows:
        Ap, Am = A0.copy(), A0.copy()
        Ap[rc] += EPS
        Am[rc] -= EPS
        fd = (loss(A=Ap) - loss(A=Am)) / (2 * EPS)
        assert abs(gA[rc] - fd) <= REL * abs(fd), (rc, gA[rc], fd)
    for b in np.argsort(-np.abs(gP))[:4]:
        Pp, Pm = P0.copy(), P0.copy()
        Pp[b] += EPS
        Pm[b] -= EPS
        fd = (loss(P=Pp) - loss(P=Pm)) / (2 * EPS)
        assert abs(gP[b] - fd) <= REL * abs(fd), (b, gP[b], fd)
