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


class CaelixWorldInfo(C.Structure):
    _fields_ = [("version", C.c_uint16), ("has_player_pose", C.c_uint16), ("entity_count", C.c_uint32),
                ("sector_count", C.c_uint64), ("player_position", C.c_float * 3), ("player_rotation", C.c_float * 4)]


class CaelixWorldEntity(C.Structure):
    _fields_ = [("guid", C.c_uint8 * 16), ("position", C.c_float * 3), ("rotation", C.c_float * 4),
                ("velocity", C.c_float * 6), ("require_update_flags", C.c_uint16), ("flags", C.c_uint8),
                ("is_protected", C.c_uint8), ("sector_count", C.c_uint32)]


class CaelixWorldSector(C.Structure):
    _fields_ = [("entity", C.c_uint32), ("coord", C.c_int32 * 3), ("region_offset", C.c_uint64),
                ("region_size", C.c_uint32), ("pad", C.c_uint32)]

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

    def __init__(self, path: str | None = None):
        path = path or os.environ.get("CAELIX_B200_LIB", LIB_PATH)
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
        L.caelix_world_open.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.caelix_world_close.argtypes = [vp]
        L.caelix_world_close.restype = None
        L.caelix_world_get_info.argtypes = [vp, C.POINTER(CaelixWorldInfo)]
        L.caelix_world_get_entity.argtypes = [vp, C.c_uint32, C.POINTER(CaelixWorldEntity)]
        L.caelix_world_get_sector.argtypes = [vp, C.c_uint64, C.POINTER(CaelixWorldSector)]
        L.caelix_world_decode_sector.argtypes = [vp, C.c_uint64, C.c_uint32, vp, vp, vp, C.POINTER(C.c_uint32),
                                                 C.POINTER(C.c_uint64)]
        L.caelix_world_upload_entity.argtypes = [vp, C.c_uint32, vp, C.c_uint32, C.POINTER(C.c_int32),
                                                 C.POINTER(C.c_uint64)]
        L.caelix_world_load.argtypes = [vp, vp, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
        for name in (
            "caelix_world_open", "caelix_world_get_info", "caelix_world_get_entity", "caelix_world_get_sector",
            "caelix_world_decode_sector", "caelix_world_upload_entity", "caelix_world_load",
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


# ---------------------------------------------------------------------------------------------
# Scene and renderer


class CaelixEntityDesc(C.Structure):
    _fields_ = [("guid", C.c_uint8 * 16), ("position", C.c_float * 3), ("rotation", C.c_float * 4)]


class CaelixSceneDesc(C.Structure):
    _fields_ = [("staging_bytes", C.c_uint64), ("records_per_page", C.c_uint32), ("group_shift", C.c_uint32),
                ("block_bytes", C.c_uint32), ("encoding", C.c_uint32), ("scratch_bytes", C.c_uint64)]


assert C.sizeof(CaelixSceneDesc) == 32

ENCODING_PACKED = 0
ENCODING_BLOCK_ID = 1


class CaelixBrickKey(C.Structure):
    _fields_ = [("x", C.c_int32), ("y", C.c_int32), ("z", C.c_int32)]


class CaelixMaterial(C.Structure):
    _fields_ = [
        ("albedo", C.c_float * 3), ("smoothness", C.c_float), ("emission", C.c_float * 3), ("metallic", C.c_float),
        ("ior", C.c_float), ("extinction", C.c_float), ("sss_model", C.c_uint32), ("sss_probability", C.c_float),
        ("sss_albedo", C.c_float * 3), ("sss_anisotropy", C.c_float), ("sss_steps", C.c_uint32),
        ("sss_params", C.c_float * 8), ("texture_set", C.c_uint32), ("connect_group", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


assert C.sizeof(CaelixMaterial) == 112


class CaelixMaterialEntry(C.Structure):
    _fields_ = [("code", C.c_uint32), ("material", CaelixMaterial)]


assert C.sizeof(CaelixMaterialEntry) == 116


class CaelixLightOptions(C.Structure):
    _fields_ = [("enabled", C.c_uint32), ("min_emission", C.c_float), ("heap_bytes", C.c_uint64)]


class CaelixFrameDesc(C.Structure):
    _fields_ = [("command_buffer", C.c_uint64), ("frame_number", C.c_uint64), ("safe_frame_number", C.c_uint64)]


class CaelixLightStats(C.Structure):
    _fields_ = [
        ("enabled", C.c_uint32), ("light_groups", C.c_uint32), ("light_bricks", C.c_uint64),
        ("light_faces", C.c_uint64), ("bricks_dropped", C.c_uint64), ("heap_bytes_used", C.c_uint64),
        ("heap_bytes_capacity", C.c_uint64), ("passes", C.c_uint32), ("failed_passes", C.c_uint32),
        ("records_recomputed", C.c_uint32), ("records_copied", C.c_uint32), ("gpu_ms", C.c_float),
        ("pad", C.c_uint32), ("tree_leaves", C.c_uint32 * 2), ("tree_nodes", C.c_uint32 * 2),
        ("tree_builds", C.c_uint32 * 2), ("tree_leaves_dropped", C.c_uint32 * 2),
    ]


assert C.sizeof(CaelixLightStats) == 104


class CaelixSceneView(C.Structure):
    _fields_ = [("grid", C.c_uint32 * 3), ("group_shift", C.c_uint32), ("groups", C.c_uint32 * 3),
                ("brick_count", C.c_uint32), ("hash_capacity", C.c_uint32), ("hash_slot_count", C.c_uint32),
                ("hash_max_probe", C.c_uint32), ("light_count", C.c_uint32), ("heap_words", C.c_uint32),
                ("group_count", C.c_uint32)] + [(n, C.c_uint64) for n in (
                    "keys", "records", "hash_slots", "bitmap", "heap", "group_rows", "light_headers", "light_group",
                    "light_entry", "light_brick", "tree_header", "tree_nodes", "tree_leaves")] + [
                ("origin", C.c_int32 * 3), ("encoding", C.c_uint32)]


class CaelixCamera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("pad0", C.c_float), ("right", C.c_float * 3), ("pad1", C.c_float),
                ("up", C.c_float * 3), ("pad2", C.c_float), ("forward", C.c_float * 3), ("pad3", C.c_float),
                ("tan_half_fov_y", C.c_float), ("aspect", C.c_float), ("near_z", C.c_float), ("far_z", C.c_float),
                ("projection", C.c_float * 16), ("jitter", C.c_float * 2)]


class CaelixRenderTargets(C.Structure):
    _fields_ = [("radiance", C.c_uint64), ("width", C.c_uint32), ("height", C.c_uint32), ("voxel_id", C.c_uint64)]


class CaelixRenderOptions(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("bounce_count", C.c_uint32), ("frame_seed", C.c_uint32), ("spp", C.c_uint32),
                ("voxel_id_tmax", C.c_float), ("reserved", C.c_uint32 * 3)]


def render_options(bounces: int, seed: int, spp: int, voxel_id_tmax: float = 0.0) -> CaelixRenderOptions:
    return CaelixRenderOptions(1, bounces, seed, spp, float(voxel_id_tmax), (C.c_uint32 * 3)(0, 0, 0))


class CaelixLightNeeOptions(C.Structure):
    _fields_ = [("enabled", C.c_uint32), ("flags", C.c_uint32), ("hint_patch", C.c_uint32), ("reserved", C.c_uint32)]


class CaelixGpuTimings(C.Structure):
    _fields_ = [("trace_ms", C.c_float), ("flush_ms", C.c_float), ("frame_number", C.c_uint64),
                ("composite_ms", C.c_float), ("denoise_ms", C.c_float), ("upscale_ms", C.c_float),
                ("pad", C.c_float)]


class CaelixRenderStats(C.Structure):
    _fields_ = [("primary_rays", C.c_uint64), ("bounce_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("kernel_launches", C.c_uint32), ("pad", C.c_uint32)]


def _bind_scene(L):
    vp = C.c_void_p
    proto = {
        "caelix_scene_create": [vp, C.POINTER(CaelixSceneDesc), C.POINTER(vp)],
        "caelix_scene_upload_bricks": [vp, C.c_uint32, C.c_uint32, vp, vp, C.POINTER(C.c_uint32)],
        "caelix_scene_set_brick_power": [vp, C.c_uint32, C.c_uint32, vp, vp],
        "caelix_scene_remove_bricks": [vp, C.c_uint32, C.c_uint32, vp],
        "caelix_scene_add_entity": [vp, C.POINTER(CaelixEntityDesc), C.POINTER(C.c_uint32)],
        "caelix_scene_remove_entity": [vp, C.c_uint32],
        "caelix_scene_set_entity_transform": [vp, C.c_uint32, vp, vp],
        "caelix_scene_set_entity_motion": [vp, C.c_uint32, C.c_uint32],
        "caelix_scene_set_materials": [vp, vp, C.c_uint32],
        "caelix_scene_set_material_entries": [vp, vp, C.c_uint32],
        "caelix_scene_get_material": [vp, C.c_uint32, C.POINTER(CaelixMaterial)],
        "caelix_scene_set_light_options": [vp, C.POINTER(CaelixLightOptions)],
        "caelix_scene_flush": [vp, C.POINTER(CaelixFrameDesc)],
        "caelix_scene_get_view": [vp, C.POINTER(CaelixSceneView)],
        "caelix_renderer_create": [vp, vp, C.POINTER(vp)],
        "caelix_renderer_render": [vp, C.POINTER(CaelixFrameDesc), C.POINTER(CaelixRenderTargets),
                                   C.POINTER(CaelixCamera), C.POINTER(CaelixRenderOptions)],
        "caelix_renderer_set_light_nee_options": [vp, C.POINTER(CaelixLightNeeOptions)],
        "caelix_renderer_get_stats": [vp, C.POINTER(CaelixRenderStats)],
        "caelix_renderer_set_trace_mode": [vp, C.c_uint32, C.c_uint32],
        "caelix_renderer_backward": [vp, C.POINTER(CaelixFrameDesc), C.POINTER(CaelixRenderTargets),
                                     C.POINTER(CaelixCamera), C.POINTER(CaelixRenderOptions), C.c_uint64, C.c_uint64,
                                     C.c_uint64],
    }
    for name, args in proto.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.caelix_scene_destroy.argtypes = [vp]
    L.caelix_scene_destroy.restype = None
    L.caelix_renderer_destroy.argtypes = [vp]
    L.caelix_renderer_destroy.restype = None
    L.caelix_scene_get_light_stats.argtypes = [vp, C.POINTER(CaelixLightStats)]
    L.caelix_scene_get_light_stats.restype = None
    L.caelix_scene_get_light_tree.argtypes = [vp]
    L.caelix_scene_get_light_tree.restype = C.c_uint64
    L.caelix_renderer_get_gpu_timings.argtypes = [vp, C.POINTER(CaelixGpuTimings)]
    L.caelix_renderer_get_gpu_timings.restype = None


class Scene:
    """caelix_scene_*: bricks, brick power, materials, flush."""

    def __init__(self, device: Device, group_shift: int = 4, encoding: int = ENCODING_PACKED):
        self.device = device
        self.L = device.L
        _bind_scene(self.L.lib)
        handle = C.c_void_p()
        desc = CaelixSceneDesc(0, 0, group_shift, 0, encoding, 0)
        self.L.check(self.L.lib.caelix_scene_create(device.handle, C.byref(desc), C.byref(handle)), "caelix_scene_create")
        self.handle = handle
        self.frame = 0

    def close(self):
        if self.handle:
            self.L.lib.caelix_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload_bricks(self, keys, voxels, entity: int = 0):
        import numpy as np

        keys = np.ascontiguousarray(keys, np.int32)
        voxels = np.ascontiguousarray(voxels, np.uint16)
        consumed = C.c_uint32(0)
        self.L.check(self.L.lib.caelix_scene_upload_bricks(self.handle, entity, len(keys), keys.ctypes.data,
                                                           voxels.ctypes.data, C.byref(consumed)),
                     "caelix_scene_upload_bricks")
        return consumed.value

    def add_entity(self, position, rotation=(0.0, 0.0, 0.0, 1.0), guid=b""):
        """caelix_scene_add_entity: an entity with no bricks at `position` with the unit quaternion
        `rotation` (x, y, z, w); returns its id (1, 2, ...)."""
        d = CaelixEntityDesc()
        g = bytes(guid)[:16]
        d.guid[: len(g)] = list(g)
        d.position[:] = [float(v) for v in position]
        d.rotation[:] = [float(v) for v in rotation]
        out = C.c_uint32(0)
        self.L.check(self.L.lib.caelix_scene_add_entity(self.handle, C.byref(d), C.byref(out)), "caelix_scene_add_entity")
        return out.value

    def remove_entity(self, entity: int):
        self.L.check(self.L.lib.caelix_scene_remove_entity(self.handle, entity), "caelix_scene_remove_entity")

    def set_entity_transform(self, entity: int, position, rotation):
        p = (C.c_float * 3)(*[float(v) for v in position])
        q = (C.c_float * 4)(*[float(v) for v in rotation])
        self.L.check(self.L.lib.caelix_scene_set_entity_transform(self.handle, entity, p, q),
                     "caelix_scene_set_entity_transform")

    def set_entity_motion(self, entity: int, motion: int):
        self.L.check(self.L.lib.caelix_scene_set_entity_motion(self.handle, entity, motion),
                     "caelix_scene_set_entity_motion")

    def remove_bricks(self, keys, entity: int = 0):
        """caelix_scene_remove_bricks: keys the scene does not have are ignored; the next flush
        rebuilds the tables from the remaining bricks."""
        import numpy as np

        keys = np.ascontiguousarray(keys, np.int32).reshape(-1, 3)
        self.L.check(self.L.lib.caelix_scene_remove_bricks(self.handle, entity, len(keys), keys.ctypes.data),
                     "caelix_scene_remove_bricks")

    def set_brick_power(self, keys, power, entity: int = 0):
        import numpy as np

        keys = np.ascontiguousarray(keys, np.int32)
        power = np.ascontiguousarray(power, np.float32)
        self.L.check(self.L.lib.caelix_scene_set_brick_power(self.handle, entity, len(keys), keys.ctypes.data,
                                                             power.ctypes.data), "caelix_scene_set_brick_power")

    def set_materials(self, materials):
        """caelix_scene_set_materials: entries [0, len) from (albedo, emission) pairs, the rest built-in."""
        entries = (CaelixMaterial * max(len(materials), 1))()
        for i, (a, e) in enumerate(materials):
            entries[i].albedo[:] = [float(v) for v in a]
            entries[i].emission[:] = [float(v) for v in e]
            entries[i].ior = 1.5
        self.L.check(self.L.lib.caelix_scene_set_materials(self.handle, entries, len(materials)),
                     "caelix_scene_set_materials")

    def set_material_entries(self, entries):
        """caelix_scene_set_material_entries: [(code, albedo rgb, emission rgb)] over the current table."""
        arr = (CaelixMaterialEntry * max(len(entries), 1))()
        for i, (code, a, e) in enumerate(entries):
            arr[i].code = int(code)
            arr[i].material.albedo[:] = [float(v) for v in a]
            arr[i].material.emission[:] = [float(v) for v in e]
            arr[i].material.ior = 1.5
        self.L.check(self.L.lib.caelix_scene_set_material_entries(self.handle, arr, len(entries)),
                     "caelix_scene_set_material_entries")

    def material(self, code: int) -> CaelixMaterial:
        m = CaelixMaterial()
        self.L.check(self.L.lib.caelix_scene_get_material(self.handle, code, C.byref(m)), "caelix_scene_get_material")
        return m

    def set_albedo(self, albedo):
        """The block-ID materials of the benchmark worlds: code 0x8000 | i gets albedo[i] and an emission
        of 1 on every channel (the brick's power is its voxels' radiance)."""
        self.set_material_entries([(0x8000 | i, a, (1.0, 1.0, 1.0)) for i, a in enumerate(albedo)])

    def flush(self, stream: int = 0):
        self.frame += 1
        fd = CaelixFrameDesc(stream, self.frame, self.frame - 1)
        self.L.check(self.L.lib.caelix_scene_flush(self.handle, C.byref(fd)), "caelix_scene_flush")

    def set_light_options(self, enabled: bool = True, min_emission: float = 0.5, heap_bytes: int = 16 << 20):
        """caelix_scene_set_light_options (the library's default min_emission is 20; the benchmark
        worlds' emission is 1, so 0.5 here); with the tree already on and the light codes unchanged,
        the next flush rebuilds only the light tree."""
        o = CaelixLightOptions(1 if enabled else 0, float(min_emission), int(heap_bytes))
        self.L.check(self.L.lib.caelix_scene_set_light_options(self.handle, C.byref(o)),
                     "caelix_scene_set_light_options")

    def view(self) -> CaelixSceneView:
        v = CaelixSceneView()
        self.L.check(self.L.lib.caelix_scene_get_view(self.handle, C.byref(v)), "caelix_scene_get_view")
        return v

    def light_stats(self) -> CaelixLightStats:
        s = CaelixLightStats()
        self.L.lib.caelix_scene_get_light_stats(self.handle, C.byref(s))
        return s

    @classmethod
    def for_voxel_scene(cls, device: Device, vs):
        """An empty device scene with a workloads.VoxelScene's encoding, materials and light options."""
        s = cls(device, vs.group_shift, vs.encoding)
        entries = vs.material_entries()
        if entries:
            s.set_material_entries(entries)
        s.set_light_options(vs.lights, vs.min_emission)
        return s

    @classmethod
    def from_voxel_scene(cls, device: Device, vs):
        """A device scene holding a workloads.VoxelScene (bricks, every brick's power, materials,
        light options), flushed."""
        s = cls.for_voxel_scene(device, vs)
        s.upload_bricks(vs.keys, vs.voxels)
        if vs.brick_count:
            s.set_brick_power(vs.keys, vs.power)
        s.flush()
        return s


class WorldFile:
    """caelix_world_*: a .cxw world file (format version 8 and older) read on the host."""

    def __init__(self, path: str):
        self.L = library()
        handle = C.c_void_p()
        self.L.check(self.L.lib.caelix_world_open(os.fsencode(path), C.byref(handle)), "caelix_world_open")
        self.handle = handle

    def close(self):
        if self.handle:
            self.L.lib.caelix_world_close(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> CaelixWorldInfo:
        out = CaelixWorldInfo()
        self.L.check(self.L.lib.caelix_world_get_info(self.handle, C.byref(out)), "caelix_world_get_info")
        return out

    def entities(self) -> list:
        out = []
        for i in range(self.info().entity_count):
            e = CaelixWorldEntity()
            self.L.check(self.L.lib.caelix_world_get_entity(self.handle, i, C.byref(e)), "caelix_world_get_entity")
            out.append(e)
        return out

    def sectors(self) -> list:
        out = []
        for i in range(self.info().sector_count):
            s = CaelixWorldSector()
            self.L.check(self.L.lib.caelix_world_get_sector(self.handle, i, C.byref(s)), "caelix_world_get_sector")
            out.append(s)
        return out

    def decode(self, index: int):
        """(keys int32 [n, 3], blocks uint16 [n, 512], summaries uint32 [n], non-zero value count)."""
        import numpy as np

        n = C.c_uint32(0)
        voxels = C.c_uint64(0)
        self.L.check(self.L.lib.caelix_world_decode_sector(self.handle, index, 0, None, None, None, C.byref(n),
                                                           C.byref(voxels)), "caelix_world_decode_sector")
        keys = np.zeros((n.value, 3), np.int32)
        blocks = np.zeros((n.value, 512), np.uint16)
        summaries = np.zeros(n.value, np.uint32)
        self.L.check(self.L.lib.caelix_world_decode_sector(
            self.handle, index, n.value, keys.ctypes.data, blocks.ctypes.data, summaries.ctypes.data, C.byref(n),
            C.byref(voxels)), "caelix_world_decode_sector")
        return keys, blocks, summaries, voxels.value

    def upload_entity(self, entity: int, scene: "Scene", threads: int = 0):
        """Decodes an entity's sectors and uploads its bricks to the scene; returns (origin, bricks)."""
        origin = (C.c_int32 * 3)()
        bricks = C.c_uint64(0)
        self.L.check(self.L.lib.caelix_world_upload_entity(self.handle, entity, scene.handle, threads, origin,
                                                           C.byref(bricks)), "caelix_world_upload_entity")
        return tuple(origin), bricks.value

    def load(self, scene: "Scene", threads: int = 0):
        """caelix_world_load: file entity 0 into the scene's world, every other entity as a scene
        entity; returns (scene entity id of every file entity, bricks uploaded)."""
        n = self.info().entity_count
        ids = (C.c_uint32 * max(n, 1))()
        bricks = C.c_uint64(0)
        self.L.check(self.L.lib.caelix_world_load(self.handle, scene.handle, threads, ids, C.byref(bricks)),
                     "caelix_world_load")
        return list(ids)[:n], bricks.value


def camera_struct(cam) -> CaelixCamera:
    c = CaelixCamera()
    c.position[:] = [float(v) for v in cam["position"]]
    c.right[:] = [float(v) for v in cam["right"]]
    c.up[:] = [float(v) for v in cam["up"]]
    c.forward[:] = [float(v) for v in cam["forward"]]
    c.tan_half_fov_y = float(cam["tan_half_fov_y"])
    c.aspect = float(cam["aspect"])
    return c


class Renderer:
    """caelix_renderer_*: the trace of a scene into a device radiance buffer."""

    def __init__(self, device: Device, scene: Scene):
        self.device = device
        self.scene = scene
        self.L = device.L
        handle = C.c_void_p()
        self.L.check(self.L.lib.caelix_renderer_create(device.handle, scene.handle, C.byref(handle)),
                     "caelix_renderer_create")
        self.handle = handle
        self.frame = 0

    def close(self):
        if self.handle:
            self.L.lib.caelix_renderer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    TRACE_WAVEFRONT = 0
    TRACE_MEGAKERNEL = 1

    def set_trace_mode(self, mode: int, wave_capacity: int = 0):
        """caelix_renderer_set_trace_mode: TRACE_WAVEFRONT (default; wave_capacity bounds the paths in
        flight, 0 = one per pixel) or TRACE_MEGAKERNEL."""
        self.L.check(self.L.lib.caelix_renderer_set_trace_mode(self.handle, mode, wave_capacity),
                     "caelix_renderer_set_trace_mode")

    def set_light_nee(self, enabled: bool):
        o = CaelixLightNeeOptions(1 if enabled else 0, 0, 0, 0)
        self.L.check(self.L.lib.caelix_renderer_set_light_nee_options(self.handle, C.byref(o)),
                     "caelix_renderer_set_light_nee_options")

    def render(self, radiance, width: int, height: int, camera, bounces: int = 4, seed: int = 1, spp: int = 1,
               stream: int = 0, voxel_id=None, voxel_id_tmax: float = 0.0):
        """caelix_renderer_render; voxel_id (device, height x width x 2 uint32, optional) receives the
        voxel id target."""
        self.frame += 1
        fd = CaelixFrameDesc(stream, self.frame, self.frame - 1)
        t = CaelixRenderTargets(_ptr(radiance), width, height, _ptr(voxel_id) if voxel_id is not None else 0)
        cam = camera if isinstance(camera, CaelixCamera) else camera_struct(camera)
        o = render_options(bounces, seed, spp, voxel_id_tmax)
        self.L.check(self.L.lib.caelix_renderer_render(self.handle, C.byref(fd), C.byref(t), C.byref(cam), C.byref(o)),
                     "caelix_renderer_render")

    def backward(self, d_radiance, width: int, height: int, camera, d_albedo, d_power, bounces: int = 4,
                 seed: int = 1, spp: int = 1, image=None, stream: int = 0):
        """caelix_renderer_backward: d_radiance = dL/d(radiance) (device, height x width x 3); writes
        dL/dalbedo into d_albedo (device, 65536 x 3, by material code) and dL/dpower into d_power (device, one per brick
        in the scene's order); image (device, optional) receives the forward radiance."""
        self.frame += 1
        fd = CaelixFrameDesc(stream, self.frame, self.frame - 1)
        t = CaelixRenderTargets(_ptr(image) if image is not None else 0, width, height, 0)
        cam = camera if isinstance(camera, CaelixCamera) else camera_struct(camera)
        o = render_options(bounces, seed, spp)
        self.L.check(self.L.lib.caelix_renderer_backward(self.handle, C.byref(fd), C.byref(t), C.byref(cam),
                                                         C.byref(o), _ptr(d_radiance), _ptr(d_albedo),
                                                         _ptr(d_power)), "caelix_renderer_backward")

    def stats(self) -> CaelixRenderStats:
        s = CaelixRenderStats()
        self.L.check(self.L.lib.caelix_renderer_get_stats(self.handle, C.byref(s)), "caelix_renderer_get_stats")
        return s

    def timings(self) -> CaelixGpuTimings:
        t = CaelixGpuTimings()
        self.L.lib.caelix_renderer_get_gpu_timings(self.handle, C.byref(t))
        return t


class CaelixBatchView(C.Structure):
    _fields_ = [("renderer", C.c_void_p), ("camera", CaelixCamera), ("target", CaelixRenderTargets),
                ("options", CaelixRenderOptions)]


class CaelixBatchDesc(C.Structure):
    _fields_ = [("view_count", C.c_uint32), ("rebuild_light_trees", C.c_uint32),
                ("views", C.POINTER(CaelixBatchView)), ("reserved", C.c_uint32 * 4)]


class CaelixBatchTuning(C.Structure):
    _fields_ = [("min_blocks", C.c_uint32), ("wavefront", C.c_uint32), ("block_width", C.c_uint32),
                ("refill_min", C.c_uint32), ("sort_keys_per_thread", C.c_uint32), ("order", C.c_uint32),
                ("kernel", C.c_uint32), ("reserved", C.c_uint32)]

    def as_dict(self) -> dict:
        return {n: int(getattr(self, n)) for n, _ in self._fields_ if n != "reserved"}


class CaelixBatchStats(C.Structure):
    _fields_ = [("primary_rays", C.c_uint64), ("bounce_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("gpu_ms", C.c_float), ("kernel_launches", C.c_uint32), ("light_tree_builds", C.c_uint32),
                ("wavefront", C.c_uint32), ("graph_captures", C.c_uint32), ("pad", C.c_uint32)]


def _bind_batch(L):
    vp = C.c_void_p
    proto = {
        "caelix_batch_create": [vp, C.POINTER(CaelixBatchDesc), C.POINTER(vp)],
        "caelix_batch_run": [vp, C.POINTER(CaelixFrameDesc)],
        "caelix_batch_set_tuning": [vp, C.POINTER(CaelixBatchTuning)],
        "caelix_batch_get_tuning": [vp, C.POINTER(CaelixBatchTuning)],
        "caelix_batch_autotune": [vp, C.POINTER(CaelixFrameDesc), C.c_char_p, C.c_uint32,
                                  C.POINTER(CaelixBatchTuning)],
        "caelix_batch_get_stats": [vp, C.POINTER(CaelixBatchStats)],
        "caelix_batch_get_view_stats": [vp, C.c_uint32, C.POINTER(CaelixRenderStats)],
    }
    for name, args in proto.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.caelix_batch_destroy.argtypes = [vp]
    L.caelix_batch_destroy.restype = None


class Batch:
    """caelix_batch_*: many views (renderer, target, camera, options) in one CUDA graph launch per run.
    `views`: (renderer, radiance buffer, width, height, camera, bounces, seed, spp) tuples."""

    def __init__(self, device: Device, views, rebuild_light_trees: bool = True):
        self.device = device
        self.L = device.L
        _bind_scene(self.L.lib)
        _bind_batch(self.L.lib)
        self.renderers = [v[0] for v in views]  # kept alive with the batch
        arr = (CaelixBatchView * len(views))()
        for i, (renderer, radiance, width, height, camera, bounces, seed, spp) in enumerate(views):
            arr[i].renderer = renderer.handle
            arr[i].camera = camera if isinstance(camera, CaelixCamera) else camera_struct(camera)
            arr[i].target = CaelixRenderTargets(_ptr(radiance), width, height, 0)
            arr[i].options = render_options(bounces, seed, spp)
        desc = CaelixBatchDesc(len(views), 1 if rebuild_light_trees else 0, arr, (C.c_uint32 * 4)(0, 0, 0, 0))
        handle = C.c_void_p()
        self.L.check(self.L.lib.caelix_batch_create(device.handle, C.byref(desc), C.byref(handle)),
                     "caelix_batch_create")
        self.handle = handle
        self.frame = 0

    def close(self):
        if self.handle:
            self.L.lib.caelix_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, stream: int = 0):
        self.frame += 1
        fd = CaelixFrameDesc(stream, self.frame, self.frame - 1)
        self.L.check(self.L.lib.caelix_batch_run(self.handle, C.byref(fd)), "caelix_batch_run")

    def tuning(self) -> CaelixBatchTuning:
        t = CaelixBatchTuning()
        self.L.check(self.L.lib.caelix_batch_get_tuning(self.handle, C.byref(t)), "caelix_batch_get_tuning")
        return t

    def set_tuning(self, **fields):
        t = self.tuning()
        for k, v in fields.items():
            setattr(t, k, int(v))
        self.L.check(self.L.lib.caelix_batch_set_tuning(self.handle, C.byref(t)), "caelix_batch_set_tuning")

    def autotune(self, cache_path: str | None = None, repeats: int = 2, stream: int = 0) -> CaelixBatchTuning:
        fd = CaelixFrameDesc(stream, self.frame + 1, self.frame)
        t = CaelixBatchTuning()
        path = cache_path.encode() if cache_path else None
        self.L.check(self.L.lib.caelix_batch_autotune(self.handle, C.byref(fd), path, repeats, C.byref(t)),
                     "caelix_batch_autotune")
        return t

    def stats(self) -> CaelixBatchStats:
        s = CaelixBatchStats()
        self.L.check(self.L.lib.caelix_batch_get_stats(self.handle, C.byref(s)), "caelix_batch_get_stats")
        return s

    def view_stats(self, index: int) -> CaelixRenderStats:
        s = CaelixRenderStats()
        self.L.check(self.L.lib.caelix_batch_get_view_stats(self.handle, index, C.byref(s)),
                     "caelix_batch_get_view_stats")
        return s
