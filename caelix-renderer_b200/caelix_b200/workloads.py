"""Seeded synthetic workloads of the benchmark configurations (host-side generators).

Every generator is deterministic and vectorised (numpy): the CUDA path and the CPU oracle consume
the same host arrays.

  PCG32          O'Neill's pcg32 (64-bit LCG state, XSH-RR output), `stream` selects the
                 increment; draws are produced by LCG jump-ahead, so n draws cost O(log n) numpy
                 passes.
  doubles        53-bit uniform doubles from two draws: ((a >> 5) * 2^26 + (b >> 6)) / 2^53.
  log-normal     exp(mu + sigma z), z from Box-Muller over PCG32 doubles, cast to fp32.

Brick light records follow the reference's BrickLightRecordHeader layout
(lib/src/light/light_tree_layout.h:298-323): face sums, packed group-local voxel box, pos,
entry count, family counts.
"""
from __future__ import annotations

import numpy as np

MULT = np.uint64(6364136223846793005)

RECORD_DTYPE = np.dtype(
    [
        ("face", "<f4", (6,)),
        ("box_lo", "<u4"),
        ("box_hi", "<u4"),
        ("pos", "<u4"),
        ("entry_count", "<u4"),
        ("counts_lo", "<u4"),
        ("counts_hi", "<u4"),
    ]
)
assert RECORD_DTYPE.itemsize == 48

FRAME_DTYPE = np.dtype([("origin", "<f4", (3,)), ("rotation", "<f4", (9,)), ("translation", "<f4", (3,))])
assert FRAME_DTYPE.itemsize == 60


class Pcg32:
    """pcg32 with explicit state and stream (the reference implementation's seeding: state = 0,
    step, state += seed, step)."""

    def __init__(self, seed: int, stream: int):
        self.inc = np.uint64(((stream << 1) | 1) & 0xFFFFFFFFFFFFFFFF)
        self.state = np.uint64(0)
        self._advance_one()
        self.state = np.uint64((int(self.state) + seed) & 0xFFFFFFFFFFFFFFFF)
        self._advance_one()

    def _advance_one(self):
        with np.errstate(over="ignore"):
            self.state = self.state * MULT + self.inc

    def next_u32(self, n: int) -> np.ndarray:
        """The next n outputs as uint32."""
        if n <= 0:
            return np.zeros(0, np.uint32)
        with np.errstate(over="ignore"):
            # states[k] = state after k steps (output k uses the state before its step).
            mult = np.ones(1, np.uint64)
            plus = np.zeros(1, np.uint64)
            step_mult = MULT
            step_plus = self.inc
            while mult.size < n:
                # Extend with the transform of `mult.size` steps applied after the existing ones.
                m_ext = mult * step_mult
                p_ext = plus * step_mult + step_plus
                mult = np.concatenate([mult, m_ext])
                plus = np.concatenate([plus, p_ext])
                step_plus = step_plus * step_mult + step_plus
                step_mult = step_mult * step_mult
            mult = mult[:n]
            plus = plus[:n]
            old = self.state * mult + plus
            # Advance the generator by n steps.
            self.state = old[-1] * MULT + self.inc
            xorshifted = (((old >> np.uint64(18)) ^ old) >> np.uint64(27)).astype(np.uint32)
            rot = (old >> np.uint64(59)).astype(np.uint32)
            out = (xorshifted >> rot) | (xorshifted << ((np.uint32(32) - rot) & np.uint32(31)))
        return out.astype(np.uint32)

    def next_doubles(self, n: int) -> np.ndarray:
        u = self.next_u32(2 * n).reshape(n, 2)
        a = (u[:, 0] >> np.uint32(5)).astype(np.float64)
        b = (u[:, 1] >> np.uint32(6)).astype(np.float64)
        return (a * 67108864.0 + b) / 9007199254740992.0

    def lognormal(self, n: int, mu: float = 0.0, sigma: float = 1.0) -> np.ndarray:
        d = self.next_doubles(2 * n).reshape(n, 2)
        u1 = 1.0 - d[:, 0]  # (0, 1]
        z = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * d[:, 1])
        return np.exp(mu + sigma * z).astype(np.float32)


def pack_voxel(x, y, z) -> np.ndarray:
    return (np.asarray(x, np.uint32) | (np.asarray(y, np.uint32) << np.uint32(10)) |
            (np.asarray(z, np.uint32) << np.uint32(20))).astype(np.uint32)


def brick_light_records(n: int, grid_bricks: int = 32, seed: int = 1, stream: int = 1, group_shift: int | None = None):
    """Brick light records of the plain light-tree build: brick coordinates uniform in
    [0, grid_bricks)^3, box = the brick's voxels [8b, 8b + 8), power log-normal(0, 1) split evenly
    over the six faces. Returns (records, record_group, group_frames): with group_shift None every
    record is in group 0 at origin 0 (the box is world-space); else the bricks are put in render
    groups of (1 << group_shift)^3 bricks with an identity frame at the group's voxel origin (what
    the large instances need: a group-local box is 10 bits per axis)."""
    rng = Pcg32(seed, stream)
    bits = int(grid_bricks).bit_length() - 1
    assert 1 << bits == grid_bricks, "grid_bricks must be a power of two"
    coords = rng.next_u32(3 * n).reshape(n, 3) >> np.uint32(32 - bits) if bits > 0 else np.zeros((n, 3), np.uint32)
    power = rng.lognormal(n)
    rec = np.zeros(n, RECORD_DTYPE)
    rec["face"] = (power / np.float32(6.0)).astype(np.float32)[:, None]
    if group_shift is None:
        lo = coords * np.uint32(8)
        rec["box_lo"] = pack_voxel(lo[:, 0], lo[:, 1], lo[:, 2])
        rec["box_hi"] = pack_voxel(lo[:, 0] + 8, lo[:, 1] + 8, lo[:, 2] + 8)
        rec["pos"] = pack_voxel(coords[:, 0], coords[:, 1], coords[:, 2])
        return rec, None, None
    g_bits = bits - group_shift
    assert g_bits >= 0
    local = coords & np.uint32((1 << group_shift) - 1)
    gc = coords >> np.uint32(group_shift)
    groups_per_axis = 1 << g_bits
    group = (gc[:, 0] + groups_per_axis * (gc[:, 1] + groups_per_axis * gc[:, 2])).astype(np.uint32)
    lo = local * np.uint32(8)
    rec["box_lo"] = pack_voxel(lo[:, 0], lo[:, 1], lo[:, 2])
    rec["box_hi"] = pack_voxel(lo[:, 0] + 8, lo[:, 1] + 8, lo[:, 2] + 8)
    rec["pos"] = (local[:, 0] | (local[:, 1] << np.uint32(group_shift)) |
                  (local[:, 2] << np.uint32(2 * group_shift))).astype(np.uint32)
    count = groups_per_axis ** 3
    frames = np.zeros(count, FRAME_DTYPE)
    g = np.arange(count, dtype=np.int64)
    edge = 8 << group_shift
    frames["origin"][:, 0] = (g % groups_per_axis) * edge
    frames["origin"][:, 1] = ((g // groups_per_axis) % groups_per_axis) * edge
    frames["origin"][:, 2] = (g // (groups_per_axis * groups_per_axis)) * edge
    frames["rotation"][:] = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1], np.float32)
    return rec, group, frames
