"""ctypes binding of the CPU oracle (oracle/liboracle.so). Test infrastructure: only the tests,
the smoke check and the benchmark's CPU-baseline leg load it, as the checker."""
import ctypes as C
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")

LEAF_DTYPE = np.dtype([("face", "<f4", (6,)), ("lo", "<f4", (3,)), ("hi", "<f4", (3,)),
                       ("group", "<u4"), ("entry", "<u4"), ("pad", "<u4"), ("parent", "<u4")])
NODE_DTYPE = np.dtype([("child_face", "<f4", (4, 6)), ("child_lo", "<f4", (4, 3)), ("child_hi", "<f4", (4, 3)),
                       ("child", "<u4", (4,)), ("parent", "<u4"), ("parent_slot", "<u4"), ("pad", "<u4", (2,))])
HEADER_DTYPE = np.dtype([("face", "<f4", (6,)), ("lo", "<f4", (3,)), ("hi", "<f4", (3,)),
                         ("root", "<u4"), ("leaf_count", "<u4"), ("node_count", "<u4"), ("pad", "<u4")])
SUMMARY_DTYPE = np.dtype([("face", "<f4", (6,)), ("lo", "<f4", (3,)), ("hi", "<f4", (3,))])
assert LEAF_DTYPE.itemsize == 64 and NODE_DTYPE.itemsize == 224 and HEADER_DTYPE.itemsize == 64


class BuildOut(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "leaves", "nodes", "header", "keys", "values", "left", "right", "parent", "leaf_parent",
        "depth", "wide", "aggregates", "bounds", "node_overflow")]


def build_oracle():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def load():
    if not os.path.exists(ORACLE_SO):
        build_oracle()
    lib = C.CDLL(ORACLE_SO)
    lib.oc_morton.argtypes = [C.c_uint32] * 3
    lib.oc_morton.restype = C.c_uint32
    lib.oc_radix_sort_pairs.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
    lib.oc_radix_sort_pairs.restype = None
    lib.oc_lt_build.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                C.POINTER(BuildOut)]
    lib.oc_lt_build.restype = C.c_int
    return lib


def _p(a):
    return None if a is None else a.ctypes.data


def lt_build(lib, records, record_group=None, record_entry=None, group_frames=None, leaf_capacity=None):
    """Runs the oracle build; returns a dict of numpy arrays (the oracle's full output)."""
    n = len(records)
    cap = max(leaf_capacity or n, 2)
    out = {
        "leaves": np.zeros(cap, LEAF_DTYPE),
        "nodes": np.zeros(cap, NODE_DTYPE),
        "header": np.zeros(1, HEADER_DTYPE),
        "keys": np.zeros(cap, np.uint32),
        "values": np.zeros(cap, np.uint32),
        "left": np.zeros(cap, np.uint32),
        "right": np.zeros(cap, np.uint32),
        "parent": np.zeros(cap, np.uint32),
        "leaf_parent": np.zeros(cap, np.uint32),
        "depth": np.zeros(cap, np.uint32),
        "wide": np.zeros(cap, np.uint32),
        "aggregates": np.zeros(cap, SUMMARY_DTYPE),
        "bounds": np.zeros(6, np.float32),
        "node_overflow": np.zeros(1, np.uint32),
    }
    bo = BuildOut(*[out[k].ctypes.data for k in (
        "leaves", "nodes", "header", "keys", "values", "left", "right", "parent", "leaf_parent",
        "depth", "wide", "aggregates", "bounds", "node_overflow")])
    records = np.ascontiguousarray(records)
    status = lib.oc_lt_build(_p(records), n, _p(record_group), _p(record_entry), _p(group_frames),
                             leaf_capacity or n, cap, C.byref(bo))
    out["status"] = status
    out["n"] = n
    return out


# ---------------------------------------------------------------------------------------------
# Scene and trace


class SceneDesc(C.Structure):
    _fields_ = [("grid", C.c_uint32 * 3), ("group_shift", C.c_uint32), ("brick_count", C.c_uint32),
                ("encoding", C.c_uint32), ("origin", C.c_int32 * 3), ("lights", C.c_uint32),
                ("min_emission", C.c_float), ("pad", C.c_uint32), ("keys", C.c_void_p), ("voxels", C.c_void_p),
                ("power", C.c_void_p), ("emission", C.c_void_p)]


class Scene(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("grid0", "grid1", "grid2", "group_shift")] + [
        ("origin", C.c_int32 * 3), ("encoding", C.c_uint32), ("emission", C.c_void_p), ("light_codes", C.c_void_p),
        ("keys", C.c_void_p)] + [(n, C.c_uint32) for n in (
        "brick_count", "hash_capacity", "hash_slot_count",
        "hash_max_probe", "bitmap_words", "light_count", "heap_words", "group_count", "groups0", "groups1",
        "groups2", "pad")] + [(n, C.c_void_p) for n in (
        "records", "hash_slots", "bitmap", "light_headers", "light_group", "light_entry", "light_brick",
        "heap", "group_rows", "group_frames")] + [("entities", C.c_void_p), ("entity_count", C.c_uint32),
                                                   ("pad2", C.c_uint32), ("dyn", C.c_void_p), ("dyn_tree", C.c_void_p),
                                                   ("dyn_power", C.c_void_p)]


class Entity(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("rot", C.c_float * 9), ("pos", C.c_float * 3), ("group_base", C.c_uint32),
                ("id", C.c_uint32), ("tree", C.c_uint32), ("power", C.c_void_p)]


class Camera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("right", C.c_float * 3), ("up", C.c_float * 3),
                ("forward", C.c_float * 3), ("tan_half_fov_y", C.c_float), ("aspect", C.c_float)]


class RenderDesc(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in (
        "width", "height", "spp", "bounce_count", "frame_seed", "light_nee", "x0", "y0", "x1", "y1")] + [
        ("voxel_id", C.c_void_p), ("voxel_id_tmax", C.c_float), ("pad", C.c_uint32)]


class LightTree(C.Structure):
    _fields_ = [("leaves", C.c_void_p), ("nodes", C.c_void_p), ("header", C.c_void_p)]


class Hit(C.Structure):
    _fields_ = [("hit", C.c_uint32), ("t", C.c_float), ("attrib", C.c_uint32), ("record", C.c_uint32),
                ("group", C.c_uint32), ("normal", C.c_float * 3), ("object_hit", C.c_float * 3)]


def _bind_scene(lib):
    if getattr(lib, "_scene_bound", False):
        return
    lib.oc_scene_build.argtypes = [C.POINTER(SceneDesc), C.POINTER(Scene)]
    lib.oc_scene_build.restype = C.c_int
    lib.oc_scene_free.argtypes = [C.POINTER(Scene)]
    lib.oc_scene_free.restype = None
    lib.oc_hash_lookup.argtypes = [C.POINTER(Scene), C.c_int32, C.c_int32, C.c_int32]
    lib.oc_hash_lookup.restype = C.c_uint32
    lib.oc_trace_ray.argtypes = [C.POINTER(Scene), C.c_void_p, C.c_void_p, C.c_float, C.c_float]
    lib.oc_trace_ray.restype = Hit
    lib.oc_render.argtypes = [C.POINTER(Scene), C.POINTER(LightTree), C.c_void_p, C.c_void_p, C.POINTER(Camera),
                              C.POINTER(RenderDesc), C.c_void_p, C.c_void_p, C.c_int]
    lib.oc_render.restype = None
    lib.oc_adjoint.argtypes = [C.POINTER(Scene), C.POINTER(LightTree), C.c_void_p, C.c_void_p, C.POINTER(Camera),
                               C.POINTER(RenderDesc), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_int]
    lib.oc_adjoint.restype = None
    lib.oc_light_sample.argtypes = [C.POINTER(Scene), C.POINTER(LightTree), C.c_void_p, C.c_void_p, C.c_uint32,
                                    C.c_void_p, C.c_void_p]
    lib.oc_light_sample.restype = C.c_int
    lib.oc_light_point_pdf.argtypes = [C.POINTER(Scene), C.POINTER(LightTree), C.c_void_p, C.c_void_p, C.c_uint32,
                                       C.c_void_p, C.c_uint32, C.c_uint32]
    lib.oc_light_point_pdf.restype = C.c_float
    lib.oc_light_point_pdf_tree.argtypes = [C.POINTER(Scene), C.POINTER(LightTree), C.c_void_p, C.c_void_p,
                                            C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32]
    lib.oc_light_point_pdf_tree.restype = C.c_float
    lib.oc_light_draws.argtypes = [C.POINTER(Scene), C.POINTER(LightTree), C.c_void_p, C.c_void_p, C.c_uint32,
                                   C.c_uint32, C.c_void_p]
    lib.oc_light_draws.restype = None
    lib.oc_mis_weight.argtypes = [C.c_float, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_int]
    lib.oc_mis_weight.restype = C.c_float
    lib.oc_entity_rows.argtypes = [C.c_void_p, C.c_void_p]
    lib.oc_entity_rows.restype = None
    lib.oc_sincos.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    lib.oc_sincos.restype = None
    lib._scene_bound = True


class OracleScene:
    """The oracle's scene (records, hash table, light blocks) and light tree for a VoxelScene."""

    def __init__(self, lib, scene):
        _bind_scene(lib)
        self.lib = lib
        self.src = scene
        self.origin, self.grid = scene.box()
        self.albedo_table, self.emission_table = scene.material_tables()
        self.desc = SceneDesc((C.c_uint32 * 3)(*self.grid), scene.group_shift, scene.brick_count, scene.encoding,
                              (C.c_int32 * 3)(*self.origin), 1 if scene.lights else 0, scene.min_emission, 0,
                              scene.keys.ctypes.data, scene.voxels.ctypes.data, scene.power.ctypes.data,
                              self.emission_table.ctypes.data)
        self.s = Scene()
        lib.oc_scene_build(C.byref(self.desc), C.byref(self.s))
        s = self.s
        n = scene.brick_count
        self.records = np.ctypeslib.as_array(C.cast(s.records, C.POINTER(C.c_uint32)), (max(n, 1) * 274,))[: n * 274].reshape(n, 274).copy()
        self.hash_slots = np.ctypeslib.as_array(C.cast(s.hash_slots, C.POINTER(C.c_uint32)), (s.hash_slot_count * 4,)).reshape(-1, 4).copy()
        m = s.light_count
        self.light_count = m
        if m:
            hdr = np.ctypeslib.as_array(C.cast(s.light_headers, C.POINTER(C.c_uint8)), (m * 48,))
            from caelix_b200 import workloads

            self.light_headers = hdr.view(workloads.RECORD_DTYPE).copy()
            self.light_group = np.ctypeslib.as_array(C.cast(s.light_group, C.POINTER(C.c_uint32)), (m,)).copy()
            self.light_entry = np.ctypeslib.as_array(C.cast(s.light_entry, C.POINTER(C.c_uint32)), (m,)).copy()
            self.light_brick = np.ctypeslib.as_array(C.cast(s.light_brick, C.POINTER(C.c_uint32)), (m,)).copy()
        self.heap = np.ctypeslib.as_array(C.cast(s.heap, C.POINTER(C.c_uint32)), (max(s.heap_words, 1),))[: s.heap_words].copy()
        self.group_rows = np.ctypeslib.as_array(C.cast(s.group_rows, C.POINTER(C.c_uint32)), (s.group_count * 8,)).reshape(-1, 8).copy()
        from caelix_b200 import workloads

        fr = np.ctypeslib.as_array(C.cast(s.group_frames, C.POINTER(C.c_uint8)), (s.group_count * 60,))
        self.group_frames = fr.view(workloads.FRAME_DTYPE).copy()
        # The light tree over the light records (leaf = gather order).
        if m:
            self.tree = lt_build(lib, self.light_headers, record_group=self.light_group, record_entry=self.light_entry,
                                 group_frames=self.group_frames)
        else:
            self.tree = lt_build(lib, np.zeros(0, RECORD_DTYPE_LOCAL()), leaf_capacity=1)
        self.lt = LightTree(self.tree["leaves"].ctypes.data, self.tree["nodes"].ctypes.data,
                            self.tree["header"].ctypes.data)
        self._set_tree0(None)

    def _set_tree0(self, merged):
        """Tree 0 and its light set: the world's own (merged None), or a merged static set (the
        world's light blocks first at their own indices, then the static entities'): the scene's
        heap, group rows and frames point at it, `lt` is its tree and `power0` its power."""
        s = self.s
        if not hasattr(self, "_own0"):
            self._own0 = (s.heap, s.heap_words, s.group_rows, s.group_frames, s.group_count, s.light_count, self.lt,
                          self.tree)
        own = self._own0
        if merged is None:
            s.heap, s.heap_words, s.group_rows, s.group_frames, s.group_count, s.light_count = own[:6]
            self.lt, self.tree = own[6], own[7]
            self.heap0, self.rows0, self.frames0 = self.heap, self.group_rows, self.group_frames
            self.power0 = self.src.power
            self._merged0 = None
            return
        self._merged0 = merged
        s.heap = merged["heap"].ctypes.data
        s.heap_words = len(merged["heap"])
        s.group_rows = merged["rows"].ctypes.data
        s.group_frames = merged["frames"].ctypes.data
        s.group_count = len(merged["rows"])
        s.light_count = merged["lights"]
        self.tree = merged["tree"]
        self.lt = LightTree(self.tree["leaves"].ctypes.data, self.tree["nodes"].ctypes.data,
                            self.tree["header"].ctypes.data)
        self.heap0, self.rows0, self.frames0 = merged["heap"], merged["rows"], merged["frames"]
        self.power0 = merged["power"]

    def _merge(self, parts, leaf_flag, world):
        """A merged light set: with `world` the scene's own light tables first (unchanged), then
        each part (index, OracleScene, rotation rows, position) with its groups, heap units, brick
        indices and leaves after the earlier ones' (the index entries' brick and leaf words moved,
        the leaf word marked with leaf_flag), every group's frame the part's transform. Returns the
        arrays, the light tree over the records and every part's group base."""
        from caelix_b200 import workloads

        heaps, rows, frames, powers, headers, lgroup, lentry, bases = [], [], [], [], [], [], [], []
        group_base = unit_base = record_base = light_base = 0
        if world:
            heaps.append(self.heap)
            rows.append(self.group_rows)
            frames.append(self.group_frames)
            powers.append(self.src.power)
            if self.light_count:
                headers.append(self.light_headers)
                lgroup.append(self.light_group)
                lentry.append(self.light_entry)
            group_base, unit_base, record_base, light_base = (len(self.group_rows), len(self.heap) // 4,
                                                              self.src.brick_count, self.light_count)
        for _, osc, rot, pos in parts:
            heap = osc.heap.copy()
            r = osc.group_rows.copy()
            for g in np.nonzero(r[:, 1])[0]:
                block = int(r[g, 0]) * 4
                for e in range(int(heap[block])):
                    ie = block + 4 + 4 * e
                    heap[ie + 1] += record_base
                    if heap[ie + 3] != 0xFFFFFFFF:
                        heap[ie + 3] = leaf_flag | (light_base + (int(heap[ie + 3]) & 0x7FFFFFFF))
                r[g, 0] += unit_base
            heaps.append(heap)
            rows.append(r)
            fr = osc.group_frames.copy()
            fr["rotation"] = rot
            fr["translation"] = np.asarray(pos, np.float32)
            frames.append(fr)
            powers.append(osc.src.power)
            if osc.light_count:
                headers.append(osc.light_headers)
                lgroup.append(osc.light_group + group_base)
                lentry.append(osc.light_entry)
            bases.append(group_base)
            group_base += len(r)
            unit_base += len(heap) // 4
            record_base += osc.src.brick_count
            light_base += osc.light_count
        if not light_base:
            return None, bases
        out = dict(heap=np.ascontiguousarray(np.concatenate(heaps), np.uint32),
                   rows=np.ascontiguousarray(np.concatenate(rows), np.uint32),
                   frames=np.ascontiguousarray(np.concatenate(frames)),
                   power=np.ascontiguousarray(np.concatenate(powers), np.float32),
                   headers=np.ascontiguousarray(np.concatenate(headers)).view(workloads.RECORD_DTYPE),
                   group=np.ascontiguousarray(np.concatenate(lgroup), np.uint32),
                   entry=np.ascontiguousarray(np.concatenate(lentry), np.uint32), lights=light_base)
        out["tree"] = lt_build(self.lib, out["headers"], record_group=out["group"], record_entry=out["entry"],
                               group_frames=out["frames"])
        return out, bases

    def set_entities(self, entities, ids=None, motions=None):
        """Entities beside the scene's bricks: (OracleScene of the entity's bricks, quaternion x y z w,
        position) each, traversed in order; rotation rows as the library computes them; ids: their
        entity ids (the voxel id's entity word; default 1, 2, ...); motions: 0 (static, the
        library's default) or 1 (dynamic) each. The dynamic entities' light records are merged into
        one light set in entity order with its own light tree (tree 1; leaf words marked
        0x80000000); with lights in static entities, the world's light set and the static
        entities' are merged (the world's first, at its own indices) and tree 0 built over them.
        In a merged set an entity's groups follow the earlier parts' group counts, its heap units,
        brick indices and leaves theirs, and every group's frame is the entity's transform."""
        motions = list(motions) if motions is not None else [0] * len(entities)
        self._set_tree0(None)
        self._entity_scenes = [e[0] for e in entities]
        arr = (Entity * max(len(entities), 1))()
        dyn_parts, stat_parts = [], []
        for i, (osc, q, pos) in enumerate(entities):
            qf = np.ascontiguousarray(q, np.float32)
            rot = np.zeros(9, np.float32)
            self.lib.oc_entity_rows(qf.ctypes.data, rot.ctypes.data)
            arr[i].scene = C.cast(C.pointer(osc.s), C.c_void_p)
            arr[i].rot[:] = [float(v) for v in rot]
            arr[i].pos[:] = [float(v) for v in np.asarray(pos, np.float32)]
            arr[i].group_base = 0
            arr[i].id = int(ids[i]) if ids is not None else i + 1
            arr[i].tree = 0xFFFFFFFF
            arr[i].power = osc.src.power.ctypes.data
            (dyn_parts if motions[i] == 1 else stat_parts).append((i, osc, rot, pos))
        self._entities = arr
        self.s.entities = C.cast(arr, C.c_void_p) if entities else None
        self.s.entity_count = len(entities)
        self.s.dyn = self.s.dyn_tree = self.s.dyn_power = None
        dyn, bases = self._merge(dyn_parts, 0x80000000, world=False)
        if dyn is not None:
            for (i, _, _, _), b in zip(dyn_parts, bases):
                arr[i].group_base = b
                arr[i].tree = 1
            self.dyn_heap, self.dyn_rows, self.dyn_frames = dyn["heap"], dyn["rows"], dyn["frames"]
            self.dyn_power, self.dyn_headers = dyn["power"], dyn["headers"]
            self.dyn_group, self.dyn_entry, self.dyn_tree = dyn["group"], dyn["entry"], dyn["tree"]
            self._dyn_lt = LightTree(self.dyn_tree["leaves"].ctypes.data, self.dyn_tree["nodes"].ctypes.data,
                                     self.dyn_tree["header"].ctypes.data)
            d = Scene()
            d.group_shift = self.s.group_shift
            d.encoding = self.s.encoding
            d.emission = self.s.emission
            d.light_codes = self.s.light_codes
            d.group_count = len(self.dyn_rows)
            d.light_count = dyn["lights"]
            d.heap_words = len(self.dyn_heap)
            d.heap = self.dyn_heap.ctypes.data
            d.group_rows = self.dyn_rows.ctypes.data
            d.group_frames = self.dyn_frames.ctypes.data
            self._dyn = d
            self.s.dyn = C.cast(C.pointer(d), C.c_void_p)
            self.s.dyn_tree = C.cast(C.pointer(self._dyn_lt), C.c_void_p)
            self.s.dyn_power = self.dyn_power.ctypes.data
        if any(osc.light_count for _, osc, _, _ in stat_parts):
            stat, bases = self._merge(stat_parts, 0, world=True)
            for (i, _, _, _), b in zip(stat_parts, bases):
                arr[i].group_base = b
                arr[i].tree = 0
            self._set_tree0(stat)

    def close(self):
        if self.s.records:
            self._set_tree0(None)
            self.s.entities = None
            self.s.entity_count = 0
            self.s.dyn = self.s.dyn_tree = self.s.dyn_power = None
            self.lib.oc_scene_free(C.byref(self.s))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def lookup(self, x, y, z):
        return self.lib.oc_hash_lookup(C.byref(self.s), x, y, z)

    def trace(self, origin, direction, tmin=0.0, tmax=1e30):
        o = np.asarray(origin, np.float32)
        d = np.asarray(direction, np.float32)
        return self.lib.oc_trace_ray(C.byref(self.s), o.ctypes.data, d.ctypes.data, tmin, tmax)

    def render(self, width, height, spp=1, bounces=4, seed=1, light_nee=True, window=None, threads=1, camera=None,
               voxel_ids=False, voxel_id_tmax=0.0):
        """Radiance [height][width][3] and ray counts; with voxel_ids also the voxel id image
        [height][width][2] (the first sample's camera rays; outside the window 0)."""
        cam = self.src.camera if camera is None else camera
        c = Camera((C.c_float * 3)(*cam["position"]), (C.c_float * 3)(*cam["right"]), (C.c_float * 3)(*cam["up"]),
                   (C.c_float * 3)(*cam["forward"]), float(cam["tan_half_fov_y"]), float(cam["aspect"]))
        x0, y0, x1, y1 = window or (0, 0, width, height)
        ids = np.zeros((height, width, 2), np.uint32) if voxel_ids else None
        r = RenderDesc(width, height, spp, bounces, seed, 1 if light_nee else 0, x0, y0, x1, y1,
                       ids.ctypes.data if voxel_ids else None, float(voxel_id_tmax), 0)
        out = np.zeros((height, width, 3), np.float32)
        rays = np.zeros(3, np.uint64)
        self.lib.oc_render(C.byref(self.s), C.byref(self.lt), self.albedo_table.ctypes.data,
                           self.power0.ctypes.data, C.byref(c), C.byref(r), out.ctypes.data, rays.ctypes.data,
                           threads)
        if voxel_ids:
            return out, rays, ids
        return out, rays


    def adjoint(self, width, height, spp=1, bounces=4, seed=1, d_radiance=None, A=None, P=None, threads=8):
        """The double-precision adjoint reference (oc_adjoint): the frozen estimator's image at
        (A, P) (None: the scene's own fp32 parameters) and, with d_radiance = dL/d(pixel), the
        gradients dL/dalbedo [65536][3] (by material code) and dL/dpower [brick_count]. A: the albedo
        table [65536][3] (None: the scene's)."""
        cam = self.src.camera
        c = Camera((C.c_float * 3)(*cam["position"]), (C.c_float * 3)(*cam["right"]), (C.c_float * 3)(*cam["up"]),
                   (C.c_float * 3)(*cam["forward"]), float(cam["tan_half_fov_y"]), float(cam["aspect"]))
        r = RenderDesc(width, height, spp, bounces, seed, 1, 0, 0, width, height, None, 0.0, 0)
        nb = max(self.s.brick_count, 1)
        image = np.zeros((height, width, 3), np.float64)
        dA = np.zeros((65536, 3), np.float64)
        dP = np.zeros(nb, np.float64)
        a_ptr = p_ptr = None
        if A is not None:
            A = np.ascontiguousarray(A, np.float64)
            a_ptr = A.ctypes.data
        if P is not None:
            P = np.ascontiguousarray(P, np.float64)
            p_ptr = P.ctypes.data
        g_ptr = None
        if d_radiance is not None:
            d_radiance = np.ascontiguousarray(d_radiance, np.float32)
            g_ptr = d_radiance.ctypes.data
        self.lib.oc_adjoint(C.byref(self.s), C.byref(self.lt), self.albedo_table.ctypes.data, self.power0.ctypes.data,
                            C.byref(c), C.byref(r), a_ptr, p_ptr, g_ptr, image.ctypes.data, dA.ctypes.data,
                            dP.ctypes.data, threads)
        return image, dA, dP[: self.s.brick_count]


def RECORD_DTYPE_LOCAL():
    from caelix_b200 import workloads

    return workloads.RECORD_DTYPE


def group_frames_of(origin, grid, group_shift):
    """The frames of a scene's groups (identity rotation, the group's voxel origin), in group order."""
    from caelix_b200 import workloads

    groups = [(g + (1 << group_shift) - 1) >> group_shift for g in grid]
    n = groups[0] * groups[1] * groups[2]
    fr = np.zeros(n, workloads.FRAME_DTYPE)
    g = np.arange(n)
    cell = np.stack([g % groups[0], (g // groups[0]) % groups[1], g // (groups[0] * groups[1])], -1)
    fr["origin"] = (8 * (np.asarray(origin, np.int64) + (cell.astype(np.int64) << group_shift))).astype(np.float32)
    fr["rotation"][:, [0, 4, 8]] = 1.0
    return fr, groups


class TablesScene(OracleScene):
    """The oracle's trace over a scene's device-built tables (records, hash table, bitmap, light
    blocks and light records, as CaelixSceneView hands them out), with the light tree built by the
    oracle from those light records: for worlds whose full oracle build would take too long, the
    trace and the light tree are still the oracle's own restatement."""

    def __init__(self, lib, vs, view):
        import gpu_util
        from caelix_b200 import workloads

        _bind_scene(lib)
        lib.oc_light_codes.argtypes = [C.c_void_p, C.c_uint32, C.c_float, C.c_void_p]
        lib.oc_light_codes.restype = None
        self.lib = lib
        self.src = vs
        v = view
        self.origin = tuple(int(x) for x in v.origin)
        self.grid = tuple(int(x) for x in v.grid)
        self.albedo_table, self.emission_table = vs.material_tables()
        n = int(v.brick_count)
        self.records = gpu_util.from_device(v.records, np.uint32, 274 * n)
        self.hash_slots = gpu_util.from_device(v.hash_slots, np.uint32, 4 * int(v.hash_slot_count))
        cells = self.grid[0] * self.grid[1] * self.grid[2]
        self.bitmap = gpu_util.from_device(v.bitmap, np.uint32, (cells + 31) // 32)
        self.keys_dev = gpu_util.from_device(v.keys, np.int32, 3 * n)
        m = int(v.light_count)
        self.light_count = m
        self.light_headers = gpu_util.from_device(v.light_headers, workloads.RECORD_DTYPE, m)
        self.light_group = gpu_util.from_device(v.light_group, np.uint32, m)
        self.light_entry = gpu_util.from_device(v.light_entry, np.uint32, m)
        self.light_brick = gpu_util.from_device(v.light_brick, np.uint32, m)
        self.heap = gpu_util.from_device(v.heap, np.uint32, int(v.heap_words))
        self.group_rows = gpu_util.from_device(v.group_rows, np.uint32, 8 * int(v.group_count)).reshape(-1, 8)
        self.group_frames, groups = group_frames_of(self.origin, self.grid, int(v.group_shift))
        self.light_codes = np.zeros(2048, np.uint32)
        lib.oc_light_codes(self.emission_table.ctypes.data, vs.encoding, vs.min_emission, self.light_codes.ctypes.data)
        s = Scene()
        s.grid0, s.grid1, s.grid2 = self.grid
        s.group_shift = int(v.group_shift)
        s.origin[:] = self.origin
        s.encoding = vs.encoding
        s.emission = self.emission_table.ctypes.data
        s.light_codes = self.light_codes.ctypes.data
        s.keys = self.keys_dev.ctypes.data
        s.brick_count = n
        s.hash_capacity = int(v.hash_capacity)
        s.hash_slot_count = int(v.hash_slot_count)
        s.hash_max_probe = int(v.hash_max_probe)
        s.bitmap_words = len(self.bitmap)
        s.light_count = m
        s.heap_words = int(v.heap_words)
        s.group_count = int(v.group_count)
        s.groups0, s.groups1, s.groups2 = groups
        s.records = self.records.ctypes.data
        s.hash_slots = self.hash_slots.ctypes.data
        s.bitmap = self.bitmap.ctypes.data
        s.light_headers = self.light_headers.ctypes.data
        s.light_group = self.light_group.ctypes.data
        s.light_entry = self.light_entry.ctypes.data
        s.light_brick = self.light_brick.ctypes.data
        s.heap = self.heap.ctypes.data
        s.group_rows = self.group_rows.ctypes.data
        s.group_frames = self.group_frames.ctypes.data
        self.s = s
        self.tree = lt_build(lib, self.light_headers, record_group=self.light_group, record_entry=self.light_entry,
                             group_frames=self.group_frames, leaf_capacity=max(m, 1))
        self.lt = LightTree(self.tree["leaves"].ctypes.data, self.tree["nodes"].ctypes.data,
                            self.tree["header"].ctypes.data)
        self._set_tree0(None)

    def close(self):
        pass  # the arrays are numpy-owned
