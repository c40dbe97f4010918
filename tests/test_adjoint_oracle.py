"""The double-precision adjoint reference (oracle oc_adjoint) on the CPU: its gradients against
central finite differences (eps = 1e-3) of the same frozen estimator in double, its image against
the fp32 oracle render, on a small solid-brick world."""
import numpy as np
import pytest

import oracle_lib
from caelix_b200 import workloads

EPS = 1e-3


@pytest.fixture(scope="module")
def small(oracle):
    vs = workloads.solid_brick_scene(n=160, grid_bricks=16, seed=3)
    osc = oracle_lib.OracleScene(oracle, vs)
    target = workloads.perturbed(vs, seed=5)
    tsc = oracle_lib.OracleScene(oracle, target)
    w = h = 24
    img, _ = osc.render(w, h, spp=2, bounces=3, seed=1, threads=8)
    tgt, _ = tsc.render(w, h, spp=2, bounces=3, seed=1, threads=8)
    grad = (2.0 * (img.astype(np.float64) - tgt)).astype(np.float32)
    yield dict(vs=vs, osc=osc, tgt=tgt.astype(np.float64), img=img, grad=grad, w=w, h=h)
    osc.close()
    tsc.close()


def loss(small, A=None, P=None):
    image, _, _ = small["osc"].adjoint(small["w"], small["h"], spp=2, bounces=3, seed=1, A=A, P=P)
    return float(((image - small["tgt"]) ** 2).sum())


def test_frozen_image_matches_fp32_render(small):
    image, _, _ = small["osc"].adjoint(small["w"], small["h"], spp=2, bounces=3, seed=1)
    ref = small["img"].astype(np.float64)
    assert np.allclose(image, ref, rtol=1e-5, atol=1e-6)


def test_gradients_match_central_differences(small):
    vs = small["vs"]
    _, dA, dP = small["osc"].adjoint(small["w"], small["h"], spp=2, bounces=3, seed=1, d_radiance=small["grad"])
    A0 = small["osc"].albedo_table.astype(np.float64)  # the material table's albedo, by code
    P0 = vs.power.astype(np.float64)
    # The albedo entries and bricks with the largest gradients, and a few others.
    rows = [tuple(x) for x in np.argwhere(np.abs(dA) > 0)]
    rows = sorted(rows, key=lambda rc: -abs(dA[rc]))[:6]
    bricks = list(np.argsort(-np.abs(dP))[:6])
    assert rows and bricks
    for rc in rows:
        Ap, Am = A0.copy(), A0.copy()
        Ap[rc] += EPS
        Am[rc] -= EPS
        fd = (loss(small, A=Ap) - loss(small, A=Am)) / (2 * EPS)
        assert abs(fd - dA[rc]) <= 1e-6 * max(abs(fd), 1e-12) + 1e-9, (rc, fd, dA[rc])
    for b in bricks:
        Pp, Pm = P0.copy(), P0.copy()
        Pp[b] += EPS
        Pm[b] -= EPS
        fd = (loss(small, P=Pp) - loss(small, P=Pm)) / (2 * EPS)
        assert abs(fd - dP[b]) <= 1e-6 * max(abs(fd), 1e-12) + 1e-9, (b, fd, dP[b])
