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
