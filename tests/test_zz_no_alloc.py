"""caelix_radix_sort_pairs_static, the sort for callers that cannot allocate device memory while
they record GPU work (an engine render thread that must not stall a frame on an allocation, a host
with a fixed memory budget): it uses a scratch array compiled into the library instead of cudaMalloc.

Checked through the C ABI against caelix_radix_sort_pairs (the allocating entry point) on two calls
in a row with different data (the second call must not see the first call's leftovers in the
shared array); integer sort results must be identical. This file is collected last so that a run
stopping at the first failure has already run every other test; it also passes alone."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1 << 18


def sort_both(dev, lib, keys_np, vals_np, identity):
    import torch

    n = len(keys_np)
    k1 = torch.from_numpy(keys_np.view(np.int32)).cuda()
    v1 = torch.from_numpy(vals_np.view(np.int32)).cuda()
    k2 = k1.clone()
    v2 = v1.clone()
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    dev.radix_sort_pairs(k1, v1, n, identity_values=identity)
    code = lib.caelix_radix_sort_pairs_static(C.c_uint64(k2.data_ptr()), C.c_uint64(v2.data_ptr()), n,
                                              1 if identity else 0, C.c_uint64(status.data_ptr()), C.c_uint64(0))
    assert code == 0
    torch.cuda.synchronize()
    assert int(status[0].item()) == 0
    assert dev.check_status() == 0
    return k1.cpu().numpy(), v1.cpu().numpy(), k2.cpu().numpy(), v2.cpu().numpy()


def bind(lib):
    f = lib.caelix_radix_sort_pairs_static
    f.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64]
    f.restype = C.c_int
    return lib


def test_static_sort_matches_allocating_sort_twice(cuda_device):
    lib = bind(cuda_device.L.lib)
    rng = np.random.default_rng(11)
    for call, (n, identity) in enumerate([(MAX_PAIRS, False), (100003, True)]):
        keys = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
        keys[:: 5 + call] = keys[0]
        vals = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
        k1, v1, k2, v2 = sort_both(cuda_device, lib, keys, vals, identity)
        assert np.array_equal(k1, k2), f"call {call}: keys differ"
        assert np.array_equal(v1, v2), f"call {call}: values differ"
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(k2.view(np.uint32), keys[order])


def test_static_sort_small_sizes_match_allocating_sort(cuda_device):
    # 1 and 4096 pairs take the one-CTA path (the whole sort in shared memory, no scratch words);
    # 4097 is the smallest count of the multi-tile path. Two rounds, so that the second round runs
    # on what the first left in the shared array.
    lib = bind(cuda_device.L.lib)
    rng = np.random.default_rng(12)
    for round_ in range(2):
        for n in (1, 4096, 4097):
            for identity in (False, True):
                keys = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
                keys[:: 3] = keys[0]
                vals = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
                k1, v1, k2, v2 = sort_both(cuda_device, lib, keys, vals, identity)
                assert np.array_equal(k1, k2), f"round {round_}, n {n}: keys differ"
                assert np.array_equal(v1, v2), f"round {round_}, n {n}: values differ"
                order = np.argsort(keys, kind="stable")
                assert np.array_equal(k2.view(np.uint32), keys[order])


def test_static_sort_rejects_sizes_above_its_scratch(cuda_device):
    import torch

    lib = bind(cuda_device.L.lib)
    k = torch.zeros(MAX_PAIRS + 1, dtype=torch.int32, device="cuda")
    v = torch.zeros(MAX_PAIRS + 1, dtype=torch.int32, device="cuda")
    code = lib.caelix_radix_sort_pairs_static(C.c_uint64(k.data_ptr()), C.c_uint64(v.data_ptr()), MAX_PAIRS + 1, 0,
                                              C.c_uint64(0), C.c_uint64(0))
    assert code == 1  # CAELIX_ERROR_INVALID_ARGUMENT
