"""Python host binding of libcaelix_b200 (include/caelix_b200.h) over ctypes.

The binding mirrors the reference's C ABI (include/caelix/caelix.h of betairylia/Caelix-Renderer):
the same entry point names, CaelixResult codes raised as CaelixError, borrowed arrays. Device
buffers are passed as CUDA device pointers; torch tensors are accepted for convenience (their
data_ptr() is used) but the library itself never sees a torch type.

There is no CPU fallback: importing this module loads the CUDA library and fails loudly when it is
missing (build it with `make -C caelix-renderer_b200`).
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libcaelix_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(os.path.dirname(_HERE)), "include", "caelix_b200.h")

CAELIX_OK = 0
CAELIX_ERROR_INVALID_ARGUMENT = 1
CAELIX_ERROR_UNSUPPORTED = 2
CAELIX_ERROR_CUDA = 3
CAELIX_ERROR_OUT_OF_MEMORY = 4
CAELIX_ERROR_DEVICE_STATUS = 5
RESULT_NAMES = {
    0: "CAELIX_OK",
    1: "CAELIX_ERROR_INVALID_ARGUMENT",
    2: "CAELIX_ERROR_UNSUPPORTED",
    3: "CAELIX_ERROR_CUDA",
    4: "CAELIX_ERROR_OUT_OF_MEMORY",
    5: "CAELIX_ERROR_DEVICE_STATUS",
}


class CaelixError(RuntimeError):
    def __init__(self, code: int, what: str, log: list[str]):
        self.code = code
        self.what = what
        self.log = list(log)
        super().__init__(f"{what}: {RESULT_NAMES.get(code, code)}" + (f" ({log[-1]})" if log else ""))


# ---------------------------------------------------------------------------------------------
# Structs (byte layouts of include/caelix_b200.h)


class CaelixVersion(C.Structure):
    _fields_ = [("major", C.c_uint32), ("minor", C.c_uint32), ("patch", C.c_uint32), ("abi", C.c_uint32)]


class CaelixDeviceDesc(C.Structure):
    _fields_ = [("cuda_device", C.c_int32), ("reserved", C.c_uint32)]


class CaelixLightBvhInput(C.Structure):
    _fields_ = [
        ("records", C.c_uint64),
        ("count", C.c_uint32),
        ("group_count", C.c_uint32),
        ("record_group", C.c_uint64),
        ("record_entry", C.c_uint64),
        ("group_frames", C.c_uint64),
    ]


class CaelixLightBvhView(C.Structure):
    _fields_ = [
        (name, C.c_uint64)
        for name in (
            "leaves", "nodes", "header", "keys", "values", "left", "right", "parent",
            "leaf_parent", "depth", "wide", "aggregates",
        )
    ] + [("leaf_capacity", C.c_uint32), ("node_capacity", C.c_uint32)]


class CaelixLightBvhStats(C.Structure):
    _fields_ = [
        ("leaves", C.c_uint32),
        ("nodes", C.c_uint32),
        ("root", C.c_uint32),
        ("builds", C.c_uint32),
        ("leaves_found", C.c_uint32),
        ("leaves_dropped", C.c_uint32),
        ("node_overflow", C.c_uint32),
        ("status", C.c_uint32),
        ("bounds", C.c_float * 6),
        ("gpu_ms", C.c_float),
        ("kernel_launches", C.c_uint32),
        ("stage_ms", C.c_float * 7),
        ("pad", C.c_uint32),
    ]


LOG_CALLBACK = C.CFUNCTYPE(None, C.c_int, C.c_char_p, C.c_void_p)

# ---------------------------------------------------------------------------------------------
# Library


def _ptr(x) -> int:
    """A device pointer from an int, None (0) or an object with data_ptr() (torch tensor)."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    return int(x.data_ptr())


class Library:
    """The loaded libcaelix_b200.so with its prototypes and a log sink."""

    def __init__(self, path: str = LIB_PATH):
        if not os.path.exists(path):
            raise OSError(f"libcaelix_b200.so not built: {path} (run make -C caelix-renderer_b200)")
        self.path = path
        self.lib = C.CDLL(path)
        self.log: list[str] = []
        self._callback = LOG_CALLBACK(self._on_log)
        L = self.lib
        vp = C.c_void_p
        L.caelix_get_version.argtypes = [C.POINTER(CaelixVersion)]
        L.caelix_get_version.restype = None
        L.caelix_version_string.argtypes = []
        L.caelix_version_string.restype = C.c_char_p
        L.caelix_set_log_callback.argtypes = [LOG_CALLBACK, vp]
        L.caelix_set_log_callback.restype = None
        L.caelix_device_create.argtypes = [C.POINTER(CaelixDeviceDesc), C.POINTER(vp)]
        L.caelix_device_destroy.argtypes = [vp]
        L.caelix_device_destroy.restype = None
        L.caelix_device_check.argtypes = [vp, C.POINTER(C.c_uint32)]
        L.caelix_light_bvh_create.argtypes = [vp, C.c_uint32, C.POINTER(vp)]
        L.caelix_light_bvh_destroy.argtypes = [vp]
        L.caelix_light_bvh_destroy.restype = None
        L.caelix_light_bvh_build.argtypes = [vp, C.POINTER(CaelixLightBvhInput), C.c_uint64]
        L.caelix_light_bvh_get_view.argtypes = [vp, C.POINTER(CaelixLightBvhView)]
        L.caelix_light_bvh_get_stats.argtypes = [vp, C.POINTER(CaelixLightBvhStats)]
        L.caelix_light_bvh_set_profiling.argtypes = [vp, C.c_uint32]
        L.caelix_radix_sort_pairs.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64]
        for name in (
            "caelix_device_create", "caelix_device_check", "caelix_light_bvh_create",
            "caelix_light_bvh_build", "caelix_light_bvh_get_view", "caelix_light_bvh_get_stats",
            "caelix_radix_sort_pairs", "caelix_light_bvh_set_profiling",
        ):
            getattr(L, name).restype = C.c_int
        L.caelix_set_log_callback(self._callback, None)

    def _on_log(self, level, message, user):
        self.log.append(message.decode("utf-8", "replace"))

    def check(self, code: int, what: str):
        if code != CAELIX_OK:
            raise CaelixError(code, what, self.log)

    def version(self) -> CaelixVersion:
        v = CaelixVersion()
        self.lib.caelix_get_version(C.byref(v))
        return v


_LIB: Library | None = None


def library() -> Library:
    global _LIB
    if _LIB is None:
        _LIB = Library()
    return _LIB


class Device:
    """caelix_device_create / caelix_device_destroy."""

    def __init__(self, cuda_device: int = 0):
        self.L = library()
        handle = C.c_void_p()
        desc = CaelixDeviceDesc(cuda_device, 0)
        self.L.check(self.L.lib.caelix_device_create(C.byref(desc), C.byref(handle)), "caelix_device_create")
        self.handle = handle

    def close(self):
        if self.handle:
            self.L.lib.caelix_device_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check_status(self) -> int:
        status = C.c_uint32(0)
        code = self.L.lib.caelix_device_check(self.handle, C.byref(status))
        self.L.check(code, "caelix_device_check")
        return status.value

    def radix_sort_pairs(self, keys, values, count: int, identity_values: bool = False, stream: int = 0):
        code = self.L.lib.caelix_radix_sort_pairs(
            self.handle, _ptr(keys), _ptr(values), count, 1 if identity_values else 0, stream
        )
        self.L.check(code, "caelix_radix_sort_pairs")


class LightBvh:
    """caelix_light_bvh_*: one light tree's device buffers and its build."""

    def __init__(self, device: Device, leaf_capacity: int):
        self.device = device
        self.L = device.L
        handle = C.c_void_p()
        self.L.check(
            self.L.lib.caelix_light_bvh_create(device.handle, leaf_capacity, C.byref(handle)),
            "caelix_light_bvh_create",
        )
        self.handle = handle

    def close(self):
        if self.handle:
            self.L.lib.caelix_light_bvh_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build(self, records, count: int, record_group=None, record_entry=None, group_frames=None, group_count=None,
              stream: int = 0):
        if group_frames is not None and group_count is None:
            raise ValueError("group_count is required with group_frames")
        inp = CaelixLightBvhInput(_ptr(records), count, group_count or 0, _ptr(record_group), _ptr(record_entry),
                                  _ptr(group_frames))
        self.L.check(self.L.lib.caelix_light_bvh_build(self.handle, C.byref(inp), stream), "caelix_light_bvh_build")

    def set_profiling(self, enabled: bool):
        self.L.check(self.L.lib.caelix_light_bvh_set_profiling(self.handle, 1 if enabled else 0),
                     "caelix_light_bvh_set_profiling")

    def view(self) -> CaelixLightBvhView:
        v = CaelixLightBvhView()
        self.L.check(self.L.lib.caelix_light_bvh_get_view(self.handle, C.byref(v)), "caelix_light_bvh_get_view")
        return v

    def stats(self, check: bool = True) -> CaelixLightBvhStats:
        s = CaelixLightBvhStats()
        code = self.L.lib.caelix_light_bvh_get_stats(self.handle, C.byref(s))
        if check:
            self.L.check(code, "caelix_light_bvh_get_stats")
        return s
