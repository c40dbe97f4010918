"""Failure detection without a GPU fault: a bounded device wait that runs out.

The look-back of the radix sort waits for the status words of earlier tiles. Here one tile of the
first pass never publishes its words (caelix_radix_sort_pairs_wait_test), and every wait is limited
to a few hundred polls: the tile after it must give up, set the look-back timeout bit, and finish.
The host reads the failure as CAELIX_ERROR_DEVICE_STATUS from caelix_device_check; the device stays
usable (a normal sort afterwards is correct and reports nothing). Nothing traps or hangs."""
import ctypes as C

import numpy as np
import pytest

import caelix_b200

pytestmark = pytest.mark.gpu

STATUS_LOOKBACK_TIMEOUT = 1 << 0


def test_lookback_wait_gives_up_and_reports(cuda_device):
    import torch

    lib = cuda_device.L.lib
    f = lib.caelix_radix_sort_pairs_wait_test
    f.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64]
    f.restype = C.c_int
    n = 3 * 4096 + 17  # four tiles of 4096 pairs
    rng = np.random.default_rng(5)
    keys = torch.from_numpy(rng.integers(0, 1 << 31, size=n).astype(np.int32)).cuda()
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    assert cuda_device.check_status() == 0
    # Arguments outside the hook's range are refused before anything runs.
    assert f(cuda_device.handle, keys.data_ptr(), vals.data_ptr(), n, 0, 256, 0) == caelix_b200.CAELIX_ERROR_INVALID_ARGUMENT
    assert f(cuda_device.handle, keys.data_ptr(), vals.data_ptr(), n, 4, 256, 0) == caelix_b200.CAELIX_ERROR_INVALID_ARGUMENT
    assert f(cuda_device.handle, keys.data_ptr(), vals.data_ptr(), 4096, 1, 256, 0) == caelix_b200.CAELIX_ERROR_INVALID_ARGUMENT
    assert f(cuda_device.handle, keys.data_ptr(), vals.data_ptr(), n, 1, 0, 0) == caelix_b200.CAELIX_ERROR_INVALID_ARGUMENT
    # Tile 1 never publishes: tile 2's waits run out after 256 polls.
    assert f(cuda_device.handle, keys.data_ptr(), vals.data_ptr(), n, 1, 256, 0) == caelix_b200.CAELIX_OK
    status = C.c_uint32(0)
    code = lib.caelix_device_check(cuda_device.handle, C.byref(status))
    assert code == caelix_b200.CAELIX_ERROR_DEVICE_STATUS
    assert status.value & STATUS_LOOKBACK_TIMEOUT
    # The device still works: a normal sort is correct and reports nothing.
    k = rng.integers(0, 1 << 31, size=n).astype(np.int32)
    dk = torch.from_numpy(k).cuda()
    dv = torch.zeros(n, dtype=torch.int32, device="cuda")
    cuda_device.radix_sort_pairs(dk, dv, n, identity_values=True)
    assert cuda_device.check_status() == 0
    order = np.argsort(k, kind="stable")
    assert np.array_equal(dk.cpu().numpy(), k[order])
    assert np.array_equal(dv.cpu().numpy(), order.astype(np.int32))
