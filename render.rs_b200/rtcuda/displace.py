"""Displacement at tessellation time (src/geometry/displace.rs): every
vertex moves along its normal by amplitude x an fBm of classic Perlin
gradient noise, then the normals are rebuilt from the displaced faces
(src/geometry/subdiv.rs:329-358). The noise is the same field the
PxrFractal pattern reads on the device (csrc/pattern.cuh): a 64-bit hashed
integer lattice, the 12 cube-edge gradients, quintic fade."""
import numpy as np

_M1 = np.uint64(0x9E3779B97F4A7C15)
_M2 = np.uint64(0xBF58476D1CE4E5B9)


def _lattice_hash(key):
    """displace.rs:36-43 on uint64 arrays: multiply, xor with the arithmetic
    shift right by 29, multiply, xor with the arithmetic shift by 32."""
    x = key * _M1
    x = x ^ (x.view(np.int64) >> np.int64(29)).view(np.uint64)
    x = x * _M2
    x = x ^ (x.view(np.int64) >> np.int64(32)).view(np.uint64)
    return (x & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def perlin(p):
    """displace.rs:45-80 for points p (n, 3), f64."""
    p = np.asarray(p, dtype=np.float64).reshape(-1, 3)
    cell = np.floor(p)
    f = p - cell
    ic = cell.astype(np.int64)
    corner = np.empty((len(p), 8))
    with np.errstate(over="ignore"):
        for k in range(8):
            d = np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1], dtype=np.int64)
            c = (ic + d).view(np.uint64)
            key = c[:, 0] * np.uint64(73856093) ^ c[:, 1] * np.uint64(19349663) ^ c[:, 2] * np.uint64(83492791)
            h = _lattice_hash(key) % np.uint32(12)
            # h 0-3: (+-1, +-1, 0); 4-7: (+-1, 0, +-1); 8-11: (0, +-1, +-1).
            g0 = np.where(h < 8, np.where(h & 1, -1.0, 1.0), 0.0)
            g1 = np.where(h < 4, np.where(h & 2, -1.0, 1.0), np.where(h < 8, 0.0, np.where(h & 1, -1.0, 1.0)))
            g2 = np.where(h < 4, 0.0, np.where(h & 2, -1.0, 1.0))
            fd = f - d
            corner[:, k] = g0 * fd[:, 0] + g1 * fd[:, 1] + g2 * fd[:, 2]

    def fade(t):
        return t * t * t * (t * (t * 6.0 - 15.0) + 10.0)

    def lerp(a, b, t):
        return a + (b - a) * t

    u, v, w = fade(f[:, 0]), fade(f[:, 1]), fade(f[:, 2])
    y0 = lerp(lerp(corner[:, 0], corner[:, 1], u), lerp(corner[:, 2], corner[:, 3], u), v)
    y1 = lerp(lerp(corner[:, 4], corner[:, 5], u), lerp(corner[:, 6], corner[:, 7], u), v)
    return lerp(y0, y1, w)


def fbm(p, frequency=1.0, octaves=4, gain=0.5, lacunarity=2.0, offset=(0.0, 0.0, 0.0)):
    """displace.rs:82-97."""
    p = np.asarray(p, dtype=np.float64).reshape(-1, 3)
    off = np.asarray(offset, dtype=np.float64)
    total, amp, freq = np.zeros(len(p)), 1.0, frequency
    for _ in range(max(int(octaves), 1)):
        total += amp * perlin(p * freq + off)
        amp *= gain
        freq *= lacunarity
    return total


def smooth_normals(positions, indices):
    """Area-weighted vertex normals (subdiv.rs:329-358): unnormalised face
    normals summed in f64, normalised, stored as f32."""
    P = np.asarray(positions, dtype=np.float32).astype(np.float64)
    I = np.asarray(indices, dtype=np.int64).reshape(-1, 3)
    n = np.cross(P[I[:, 1]] - P[I[:, 0]], P[I[:, 2]] - P[I[:, 0]])
    acc = np.zeros_like(P)
    for k in range(3):
        np.add.at(acc, I[:, k], n)
    ln = np.maximum(np.linalg.norm(acc, axis=1, keepdims=True), 1e-12)
    return (acc / ln).astype(np.float32)


def displace_mesh(positions, indices, normals, amplitude=0.1, frequency=1.0, octaves=4, gain=0.5, lacunarity=2.0,
                  offset=(0.0, 0.0, 0.0)):
    """displace_mesh (displace.rs:99-123): (positions, normals) after
    moving every vertex along its normal (given, else smooth) by
    fbm * amplitude."""
    P = np.asarray(positions, dtype=np.float32).reshape(-1, 3)
    N = smooth_normals(P, indices) if normals is None else np.asarray(normals, dtype=np.float32).reshape(-1, 3)
    d = fbm(P.astype(np.float64), frequency, octaves, gain, lacunarity, offset) * amplitude
    Q = (P.astype(np.float64) + N.astype(np.float64) * d[:, None]).astype(np.float32)
    return Q, smooth_normals(Q, indices)
