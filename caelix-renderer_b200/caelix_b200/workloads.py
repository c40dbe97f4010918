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


def pcg_hash(v: np.ndarray) -> np.ndarray:
    """PcgHash of caelix_random.hlsl:18-23 (vectorised, uint32)."""
    v = np.asarray(v, np.uint32)
    with np.errstate(over="ignore"):
        state = v * np.uint32(747796405) + np.uint32(2891336453)
        word = ((state >> ((state >> np.uint32(28)) + np.uint32(4))) ^ state) * np.uint32(277803737)
    return (word >> np.uint32(22)) ^ word


def value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """Seeded 3D value noise in [0, 1): lattice values from a PcgHash chain of the integer lattice
    point and the seed, trilinear interpolation with smoothstep weights (float64)."""
    p = np.asarray(p, np.float64)
    i0 = np.floor(p).astype(np.int64)
    f = p - i0
    w = f * f * (3.0 - 2.0 * f)
    s = pcg_hash(np.uint32(seed))

    def lattice(ix, iy, iz):
        h = pcg_hash(np.asarray(iz, np.int64).astype(np.uint32) ^ s)
        h = pcg_hash(np.asarray(iy, np.int64).astype(np.uint32) ^ h)
        h = pcg_hash(np.asarray(ix, np.int64).astype(np.uint32) ^ h)
        return (h >> np.uint32(8)).astype(np.float64) / 16777216.0

    out = np.zeros(p.shape[:-1])
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                v = lattice(i0[..., 0] + dx, i0[..., 1] + dy, i0[..., 2] + dz)
                wx = w[..., 0] if dx else 1.0 - w[..., 0]
                wy = w[..., 1] if dy else 1.0 - w[..., 1]
                wz = w[..., 2] if dz else 1.0 - w[..., 2]
                out += v * wx * wy * wz
    return out


ENCODING_PACKED = 0
ENCODING_BLOCK_ID = 1
MATERIAL_CODES = 65536


def _hash32(v: np.ndarray) -> np.ndarray:
    v = np.asarray(v, np.uint32).copy()
    v ^= v >> np.uint32(16)
    v *= np.uint32(0x7FEB352D)
    v ^= v >> np.uint32(15)
    v *= np.uint32(0x846CA68B)
    v ^= v >> np.uint32(16)
    return v


def _pastel(h: np.ndarray) -> np.ndarray:
    out = np.empty(h.shape + (3,), np.float32)
    for c in range(3):
        b = ((h >> np.uint32(8 * c)) & np.uint32(0xFF)).astype(np.float32)
        out[..., c] = np.float32(0.35) + np.float32(0.6) * (b / np.float32(255.0))
    return out


def builtin_materials(encoding: int):
    """The library's built-in material table of an encoding (include/caelix_b200.h, CaelixMaterial):
    albedo and emission [65536][3] fp32 by code."""
    code = np.arange(MATERIAL_CODES, dtype=np.uint32)
    albedo = np.ones((MATERIAL_CODES, 3), np.float32)
    emission = np.zeros((MATERIAL_CODES, 3), np.float32)
    if encoding == ENCODING_PACKED:
        rgb5 = (code & np.uint32(0x8000)) != 0
        rgb4 = ((code & np.uint32(0xC000)) == np.uint32(0x4000))
        for c, shift in enumerate((10, 5, 0)):
            v = ((code >> np.uint32(shift)) & np.uint32(31)).astype(np.float32) / np.float32(31.0)
            albedo[rgb5, c] = v[rgb5]
        strength = np.exp2(np.float32(3.0) * (code & np.uint32(3)).astype(np.float32)).astype(np.float32)
        for c, shift in enumerate((10, 6, 2)):
            v = ((code >> np.uint32(shift)) & np.uint32(15)).astype(np.float32) / np.float32(15.0)
            albedo[rgb4, c] = v[rgb4]
            emission[rgb4, c] = (v * strength)[rgb4]
    else:
        opaque = (code & np.uint32(0x8000)) != 0
        albedo[opaque] = _pastel(_hash32(code[opaque] & np.uint32(0x7FFF)))
        ids = code & np.uint32(0x1FF)
        tr = ~opaque & (ids != 0)
        albedo[tr] = _pastel(_hash32(ids[tr] | np.uint32(0x10000)))
    return albedo, emission


def scene_grid(keys: np.ndarray, group_shift: int):
    """The box of a set of brick keys as the library's flush computes it: origin = the smallest key
    per axis rounded down to a multiple of the group edge, grid = the bricks from there to the
    largest key."""
    keys = np.asarray(keys, np.int64).reshape(-1, 3)
    if len(keys) == 0:
        return (0, 0, 0), (1, 1, 1)
    edge = 1 << group_shift
    lo = keys.min(axis=0)
    origin = (lo // edge) * edge  # floor division rounds toward -inf
    grid = keys.max(axis=0) - origin + 1
    return tuple(int(v) for v in origin), tuple(int(v) for v in grid)


class VoxelScene:
    """A voxel world of 8^3-voxel bricks: brick keys (in increasing linear brick index of their
    box), raw block values, per-brick emitter power, a material table and a camera.

    The material table is the encoding's built-in table with, for the block-ID worlds of the
    benchmark generators, the entries of codes 0x8000 | i (i < len(albedo)) set to albedo[i] and an
    emission of 1 on every channel (a brick's power then is its voxels' emitted radiance; bricks
    of power 0 emit nothing), plus `entries` ({code: (albedo rgb, emission rgb)}) over it. Light
    voxels: codes whose emission luminance reaches min_emission, in bricks with power above 0."""

    def __init__(self, grid, keys, voxels, power, albedo, camera, group_shift=4, encoding=ENCODING_BLOCK_ID,
                 entries=None, min_emission=0.5, lights=True):
        self.grid = tuple(int(g) for g in grid)
        self.keys = np.ascontiguousarray(keys, np.int32)
        self.voxels = np.ascontiguousarray(voxels, np.uint16)
        self.power = np.ascontiguousarray(power, np.float32)
        self.albedo = np.ascontiguousarray(albedo if albedo is not None else np.zeros((0, 3)), np.float32)
        self.camera = camera
        self.group_shift = group_shift
        self.encoding = encoding
        self.entries = dict(entries or {})
        self.min_emission = float(min_emission)
        self.lights = bool(lights)

    @property
    def brick_count(self):
        return len(self.keys)

    def material_entries(self):
        """[(code, albedo rgb, emission rgb)]: the entries the host sets over the built-in table."""
        out = []
        if self.encoding == ENCODING_BLOCK_ID:
            for i, a in enumerate(self.albedo):
                out.append((0x8000 | i, tuple(float(v) for v in a), (1.0, 1.0, 1.0)))
        for code, (a, e) in sorted(self.entries.items()):
            out.append((int(code), tuple(float(v) for v in a), tuple(float(v) for v in e)))
        return out

    def material_tables(self):
        """The whole table: albedo and emission [65536][3] fp32 by code."""
        albedo, emission = builtin_materials(self.encoding)
        for code, a, e in self.material_entries():
            albedo[code] = np.asarray(a, np.float32)
            emission[code] = np.asarray(e, np.float32)
        return albedo, emission

    def box(self):
        """(origin, grid) of the keys, as the library's flush computes them."""
        return scene_grid(self.keys, self.group_shift)

    def like(self, **changes):
        """A copy with some fields replaced (keys, voxels, power, albedo, ...)."""
        fields = dict(grid=self.grid, keys=self.keys, voxels=self.voxels, power=self.power, albedo=self.albedo,
                      camera=self.camera, group_shift=self.group_shift, encoding=self.encoding,
                      entries=self.entries, min_emission=self.min_emission, lights=self.lights)
        fields.update(changes)
        return VoxelScene(**fields)


def look_at(position, target, tan_half_fov_y=0.5, aspect=1.0):
    """A camera (Unity convention: +X right, +Y up, +Z forward) at `position` looking at `target`."""
    pos = np.asarray(position, np.float64)
    fwd = np.asarray(target, np.float64) - pos
    fwd /= np.linalg.norm(fwd)
    right = np.cross(np.array([0.0, 1.0, 0.0]), fwd)
    right /= np.linalg.norm(right)
    up = np.cross(fwd, right)
    return {
        "position": pos.astype(np.float32),
        "right": right.astype(np.float32),
        "up": up.astype(np.float32),
        "forward": fwd.astype(np.float32),
        "tan_half_fov_y": np.float32(tan_half_fov_y),
        "aspect": np.float32(aspect),
    }


def noise_world(grid_bricks=(16, 16, 16), brick_occupancy=0.30, voxel_fill=0.5, emissive_fraction=0.01,
                seed=2, brick_scale=0.25, voxel_scale=0.25, camera=None) -> VoxelScene:
    """The plain trace scene: a grid of bricks, the `brick_occupancy` fraction of them occupied
    (the bricks with the highest value noise at brick scale), their voxels solid where the value
    noise at voxel scale exceeds 1 - voxel_fill, materials uniform in [1, 64] (block-ID value
    0x8000 | m), `emissive_fraction` of the occupied bricks emissive with power log-normal(0, 1),
    albedo uniform in [0.1, 0.9] per material and channel. Seeded PCG32 streams of `seed`."""
    gx, gy, gz = grid_bricks
    total = gx * gy * gz
    lin = np.arange(total, dtype=np.int64)
    bx, by, bz = lin % gx, (lin // gx) % gy, lin // (gx * gy)
    centres = np.stack([bx, by, bz], -1).astype(np.float64) + 0.5
    nb = value_noise(centres * brick_scale, seed * 7919 + 1)
    occupied_count = int(round(brick_occupancy * total))
    order = np.lexsort((lin, -nb))  # highest noise first, ties by index
    occupied = np.sort(order[:occupied_count])
    keys = np.stack([bx[occupied], by[occupied], bz[occupied]], -1).astype(np.int32)
    n = len(occupied)
    v = np.arange(512)
    vx, vy, vz = v % 8, (v // 8) % 8, v // 64
    pos = (keys[:, None, :].astype(np.float64) * 8 + np.stack([vx, vy, vz], -1)[None, :, :] + 0.5)
    nv = value_noise(pos * voxel_scale, seed * 7919 + 2)
    solid = nv > (1.0 - voxel_fill)
    mat = Pcg32(seed, 2).next_u32(n * 512).reshape(n, 512)
    material = (np.uint32(1) + (mat >> np.uint32(26))).astype(np.uint16)
    voxels = np.where(solid, np.uint16(0x8000) | material, np.uint16(0)).astype(np.uint16)
    emitters = max(1, int(round(emissive_fraction * n)))
    perm = np.lexsort((np.arange(n), Pcg32(seed, 3).next_u32(n)))
    power = np.zeros(n, np.float32)
    power[np.sort(perm[:emitters])] = Pcg32(seed, 4).lognormal(emitters)
    albedo = np.zeros((128, 3), np.float32)
    albedo[1:65] = (0.1 + 0.8 * Pcg32(seed, 5).next_doubles(64 * 3)).reshape(64, 3).astype(np.float32)
    world = np.array([gx, gy, gz], np.float64) * 8
    if camera is None:
        camera = look_at(np.array([-0.25, 1.2, -0.35]) * world, world * np.array([0.5, 0.35, 0.5]))
    return VoxelScene(grid_bricks, keys, voxels, power, albedo, camera)


def _torch_pcg_hash(v):
    import torch

    v = v & 0xFFFFFFFF
    state = (v * 747796405 + 2891336453) & 0xFFFFFFFF
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & 0xFFFFFFFF
    return ((word >> 22) ^ word) & 0xFFFFFFFF


def _torch_value_noise(p, seed: int):
    """value_noise on a torch int64/float64 device tensor p[..., 3] (the same lattice hash)."""
    import torch

    i0 = torch.floor(p).to(torch.int64)
    f = p - i0.to(torch.float64)
    w = f * f * (3.0 - 2.0 * f)
    s = int(pcg_hash(np.uint32(seed)))
    out = torch.zeros(p.shape[:-1], dtype=torch.float64, device=p.device)
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                h = _torch_pcg_hash((i0[..., 2] + dz) ^ s)
                h = _torch_pcg_hash((i0[..., 1] + dy) ^ h)
                h = _torch_pcg_hash((i0[..., 0] + dx) ^ h)
                v = (h >> 8).to(torch.float64) / 16777216.0
                wx = w[..., 0] if dx else 1.0 - w[..., 0]
                wy = w[..., 1] if dy else 1.0 - w[..., 1]
                wz = w[..., 2] if dz else 1.0 - w[..., 2]
                out += v * wx * wy * wz
    return out


def noise_world_large(grid_bricks=(256, 256, 64), occupied_bricks=2_000_000, voxel_fill=0.25, emissive_bricks=100_000,
                      seed=3, brick_scale=1.0 / 16, voxel_scale=0.125, chunk=1 << 16, camera=None) -> VoxelScene:
    """The large trace scene, generated on the GPU (torch): a grid of bricks, `occupied_bricks` of
    them occupied (highest value noise at brick scale), their voxels solid where the voxel-scale
    value noise exceeds 1 - voxel_fill, materials uniform in [1, 64] (PcgHash of the voxel's global
    index, so no host stream of a billion draws is needed), `emissive_bricks` of the
    occupied bricks emissive with power log-normal(0, 1) (PCG32 streams of `seed`). Returns host
    arrays (the oracle and the C ABI take host memory)."""
    import torch

    gx, gy, gz = grid_bricks
    total = gx * gy * gz
    dev = "cuda"
    lin = torch.arange(total, dtype=torch.int64, device=dev)
    b = torch.stack([lin % gx, (lin // gx) % gy, lin // (gx * gy)], -1)
    nb = _torch_value_noise((b.to(torch.float64) + 0.5) * brick_scale, seed * 7919 + 1)
    # Highest noise first, ties by index: a stable sort of -noise.
    order = torch.sort(-nb, stable=True).indices
    occupied = torch.sort(order[:occupied_bricks]).values
    keys = b[occupied].to(torch.int32)
    n = keys.shape[0]
    v = torch.arange(512, dtype=torch.int64, device=dev)
    local = torch.stack([v % 8, (v // 8) % 8, v // 64], -1).to(torch.float64)
    mat_seed = int(pcg_hash(np.uint32(seed * 7919 + 3)))
    voxels = torch.empty((n, 512), dtype=torch.int32, device=dev)
    # The solid threshold: the (1 - voxel_fill) quantile of the voxel noise over the first bricks,
    # so that voxel_fill of the voxels of occupied bricks are solid.
    probe = min(n, 4096)
    pos = keys[:probe, None, :].to(torch.float64) * 8 + local[None] + 0.5
    sample = _torch_value_noise(pos * voxel_scale, seed * 7919 + 2).reshape(-1)
    threshold = float(torch.kthvalue(sample.cpu(), max(1, int((1.0 - voxel_fill) * sample.numel()))).values)
    for start in range(0, n, chunk):
        end = min(n, start + chunk)
        pos = keys[start:end, None, :].to(torch.float64) * 8 + local[None] + 0.5
        nv = _torch_value_noise(pos * voxel_scale, seed * 7919 + 2)
        index = torch.arange(start * 512, end * 512, dtype=torch.int64, device=dev).view(end - start, 512)
        material = 1 + (_torch_pcg_hash(index ^ mat_seed) >> 26)  # uniform in [1, 64]
        voxels[start:end] = torch.where(nv > threshold, (0x8000 | material).to(torch.int32),
                                        torch.zeros_like(material, dtype=torch.int32))
    keys_h = keys.cpu().numpy()
    vox_h = voxels.cpu().numpy().astype(np.uint16)
    emitters = min(emissive_bricks, n)
    perm = np.lexsort((np.arange(n), Pcg32(seed, 3).next_u32(n)))
    power = np.zeros(n, np.float32)
    power[np.sort(perm[:emitters])] = Pcg32(seed, 4).lognormal(emitters)
    albedo = np.zeros((128, 3), np.float32)
    albedo[1:65] = (0.1 + 0.8 * Pcg32(seed, 5).next_doubles(64 * 3)).reshape(64, 3).astype(np.float32)
    world = np.array([gx, gy, gz], np.float64) * 8
    if camera is None:
        camera = look_at(world * np.array([-0.05, 1.0, -0.05]) + np.array([0.0, 200.0, 0.0]),
                         world * np.array([0.45, 0.3, 0.45]), tan_half_fov_y=0.5, aspect=16.0 / 9.0)
    return VoxelScene(grid_bricks, keys_h, vox_h, power, albedo, camera)


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


BATCH_VIEWPORTS = (256, 512, 1024)


def batch_plan(count: int = 64, min_bricks: int = 1000, max_bricks: int = 500_000, seed: int = 4):
    """The batched workload's scene list: `count` scenes with brick counts log-uniform in
    [min_bricks, max_bricks] and square viewports uniform among BATCH_VIEWPORTS (PCG32 streams of
    `seed`). Returns [(brick_count, side)]."""
    u = Pcg32(seed, 11).next_doubles(count)
    bricks = np.rint(np.exp(np.log(min_bricks) + u * (np.log(max_bricks) - np.log(min_bricks)))).astype(np.int64)
    sides = np.array(BATCH_VIEWPORTS)[Pcg32(seed, 12).next_u32(count) % np.uint32(len(BATCH_VIEWPORTS))]
    return [(int(b), int(s)) for b, s in zip(bricks, sides)]


def batch_scene(bricks: int, seed: int, occupancy: float = 0.30, emissive_fraction: float = 0.01) -> VoxelScene:
    """One scene of the batched workload: the plain scene's generator (value noise, `occupancy` of
    the bricks of a cubic grid occupied, half the voxels of an occupied brick solid, materials
    uniform in [1, 64], `emissive_fraction` of the bricks emissive with log-normal(0, 1) power)
    at `bricks` occupied bricks, on the GPU; the camera of the plain scene, aspect 1."""
    side = int(np.ceil(np.cbrt(bricks / occupancy)))
    world = np.array([side, side, side], np.float64) * 8
    camera = look_at(np.array([-0.25, 1.2, -0.35]) * world, world * np.array([0.5, 0.35, 0.5]))
    return noise_world_large(grid_bricks=(side, side, side), occupied_bricks=bricks, voxel_fill=0.5,
                             emissive_bricks=max(1, int(round(emissive_fraction * bricks))), seed=seed,
                             brick_scale=0.25, voxel_scale=0.25, camera=camera)


def solid_brick_scene(n: int = 4096, grid_bricks: int = 32, seed: int = 1, stream: int = 1) -> VoxelScene:
    """The plain light-tree build's bricks as a voxel world (the differentiation scene): brick
    coordinates and powers from brick_light_records' PCG32 stream (uniform in [0, grid_bricks)^3,
    power log-normal(0, 1); a repeated coordinate keeps its first draw), every brick solid (AABB =
    the brick), voxel materials uniform in [1, 64] (PCG32 stream 2), every brick emissive, albedo
    uniform in [0.1, 0.9] per material and channel (stream 5); bricks in increasing linear index;
    a camera looking into the grid, aspect 1."""
    rng = Pcg32(seed, stream)
    bits = int(grid_bricks).bit_length() - 1
    assert 1 << bits == grid_bricks, "grid_bricks must be a power of two"
    coords = (rng.next_u32(3 * n).reshape(n, 3) >> np.uint32(32 - bits)).astype(np.int64)
    power = rng.lognormal(n)
    lin = coords[:, 0] + grid_bricks * (coords[:, 1] + grid_bricks * coords[:, 2])
    _, first = np.unique(lin, return_index=True)  # sorted by linear index, first occurrence of each
    keys = coords[first].astype(np.int32)
    power = power[first].astype(np.float32)
    m = len(keys)
    mat = Pcg32(seed, 2).next_u32(m * 512).reshape(m, 512)
    voxels = (np.uint16(0x8000) | (np.uint32(1) + (mat >> np.uint32(26))).astype(np.uint16)).astype(np.uint16)
    albedo = np.zeros((128, 3), np.float32)
    albedo[1:65] = (0.1 + 0.8 * Pcg32(seed, 5).next_doubles(64 * 3)).reshape(64, 3).astype(np.float32)
    world = np.array([grid_bricks] * 3, np.float64) * 8
    camera = look_at(np.array([-0.25, 1.2, -0.35]) * world, world * np.array([0.5, 0.35, 0.5]))
    return VoxelScene((grid_bricks,) * 3, keys, voxels, power, albedo, camera)


def perturbed(vs: VoxelScene, seed: int = 7, amount: float = 0.10) -> VoxelScene:
    """The same world with albedo and power each scaled by (1 + amount * u), u uniform in [-1, 1]
    (PCG32 streams 21 and 22 of `seed`): the target of the differentiation workload."""
    ua = 2.0 * Pcg32(seed, 21).next_doubles(vs.albedo.size).reshape(vs.albedo.shape) - 1.0
    up = 2.0 * Pcg32(seed, 22).next_doubles(len(vs.power)) - 1.0
    albedo = (vs.albedo * (1.0 + amount * ua)).astype(np.float32)
    power = (vs.power * (1.0 + amount * up)).astype(np.float32)
    return vs.like(power=power, albedo=albedo)
