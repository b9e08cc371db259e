"""Seeded synthetic scenes for the delta projection.

Every scene is plain numpy data in the reference's layouts (code/water-core/src/delta3d.rs:24-28):
cells and columns x-fastest, faces u/v/w per axis, SDF nodes (nx+1)(ny+1)(nz+1) x-fastest.
Scalar f32 arithmetic that the reference performs in f32 is done here in f32 too, and
transcendental functions go through the C library's `sinf`/`expf` (what Rust's f32 methods call
on Linux), so that the oracle and the GPU see bit-identical inputs.

Scenes:
  * `s385_case`       the multigrid bench of code/water-core/examples/delta3d_multigrille.rs:26-94
  * `noise`           the xorshift U[-1,1) generator of code/water-core/src/tests_delta3d.rs:66-75
  * `sphere_lake`     64^3 closed box, 8 random spheres, lower half liquid, U[-1,1] faces
  * `box_basin`       128^3, 16 random boxes, sinusoidal surface, curl background + N(0,0.5)
Random draws use the project's SplitMix64 (`SplitMix64`), never numpy's global generator.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

_libm = C.CDLL("libm.so.6")
_libm.sinf.argtypes = [C.c_float]
_libm.sinf.restype = C.c_float
_libm.expf.argtypes = [C.c_float]
_libm.expf.restype = C.c_float

f32 = np.float32
TAU32 = f32(2.0 * math.pi)  # core::f32::consts::TAU


def sinf(x) -> np.float32:
    return f32(_libm.sinf(float(f32(x))))


def expf(x) -> np.float32:
    return f32(_libm.expf(float(f32(x))))


class SplitMix64:
    """SplitMix64 (Steele, Lea, Flood 2014): the project's seeded generator."""

    M = (1 << 64) - 1

    def __init__(self, seed: int):
        self.s = seed & self.M

    def next_u64(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & self.M
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.M
        return z ^ (z >> 31)

    def uniform(self, lo=0.0, hi=1.0) -> float:
        return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / (1 << 53)))

    def normal_array(self, n: int, sigma: float) -> np.ndarray:
        """n draws of N(0, sigma) by Box-Muller on SplitMix64 uniforms (vectorised)."""
        m = (n + 1) // 2
        raw = np.empty(2 * m, dtype=np.uint64)
        for q in range(2 * m):
            raw[q] = self.next_u64()
        u = ((raw >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / (1 << 53))
        r = np.sqrt(-2.0 * np.log(u[:m]))
        t = 2.0 * np.pi * u[m:]
        z = np.concatenate([r * np.cos(t), r * np.sin(t)])[:n]
        return (sigma * z).astype(np.float32)

    def uniform_array(self, n: int, lo: float, hi: float) -> np.ndarray:
        """n draws of U[lo, hi) as f32, from a fast counter-based SplitMix64 stream seeded here."""
        base = np.uint64(self.next_u64())
        idx = np.arange(n, dtype=np.uint64)
        with np.errstate(over="ignore"):
            z = base + (idx + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            z = z ^ (z >> np.uint64(31))
        x = (z >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))
        return (lo + (hi - lo) * x).astype(np.float32)


def noise(n: int, seed: int) -> np.ndarray:
    """Deterministic U[-1,1) f32 (tests_delta3d.rs:66-75): xorshift on a u64 state."""
    M = (1 << 64) - 1
    s = ((seed * 0x9E3779B97F4A7C15) & M) | 1
    out = np.empty(n, dtype=np.float32)
    for q in range(n):
        s ^= (s << 13) & M
        s ^= s >> 7
        s ^= (s << 17) & M
        out[q] = f32(f32(f32(s >> 40) / f32(1 << 24)) * f32(2.0)) - f32(1.0)
    return out


# ----------------------------------------------------------------------------------------------
# The reference's multigrid bench (examples/delta3d_multigrille.rs): 8 x 4 x 6 m, surface at rest
# 4 m, a 1 cm sine along x, dt = 2 ms; flat bottom or the off-centre bump of S324.
S385_LX, S385_LZ, S385_A = f32(8.0), f32(4.0), f32(0.01)
S385_RHO, S385_G, S385_DT_US = 1025.0, 9.81, 2000


def s385_bump(x: np.float32, y: np.float32) -> np.float32:
    a = f32(f32(x - f32(3.0)) / f32(1.2))
    b = f32(f32(y - f32(1.3)) / f32(0.9))
    return f32(0.4) + f32(0.6) * expf(-(f32(a * a) + f32(b * b)))


def s385_case(nx: int, bump: bool = False) -> dict:
    """Domain, bottom (None for flat) and free surface of the S385 bench at resolution nx."""
    ny, nz = nx // 2, 3 * nx // 4
    dx = f32(S385_LX / f32(nx))
    row = np.array([S385_LZ + S385_A * sinf(f32(f32(TAU32 * f32(f32(i) + f32(0.5))) * dx) / S385_LX)
                    for i in range(nx)], dtype=np.float32)
    eta = np.tile(row, ny)
    bottom = None
    if bump:
        bottom = np.array([s385_bump(f32(f32(f32(i) + f32(0.5)) * dx), f32(f32(f32(j) + f32(0.5)) * dx))
                           for j in range(ny) for i in range(nx)], dtype=np.float32)
    return dict(nx=nx, ny=ny, nz=nz, dx=float(dx), rho=S385_RHO, g=S385_G, bottom=bottom, eta=eta,
                rest=float(S385_LZ), dt_us=S385_DT_US)
