"""Seeded synthetic multi-view scenes for the motion-stereo path.

Stands in for the ICL-NUIM / TUM sequences the reference was run on (evaluate.cc:30-40):
six random 3D planes (normals within 40 degrees of the optical axis, depth 1-8 m at a random
pixel), textured with 4-octave value noise, ray-cast to uint8 grayscale with N(0, sigma^2)
pixel noise.  Source frames sit at baselines of 5-15 cm in a random direction with rotations
of at most 2 degrees about a random axis.  Poses are camera-to-world (R, T), the convention of
StereoMapper::update (stereo_mapper.cpp:79-80).  Everything is FP64 and seeded.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def rodrigues(axis: np.ndarray, angle: float) -> np.ndarray:
    axis = np.asarray(axis, np.float64)
    axis = axis / np.linalg.norm(axis)
    k = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + np.sin(angle) * k + (1 - np.cos(angle)) * (k @ k)


def _unit(rng) -> np.ndarray:
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


@dataclass
class Camera:
    W: int
    H: int
    f: float

    @property
    def cx(self) -> float:
        return self.W / 2.0

    @property
    def cy(self) -> float:
        return self.H / 2.0

    @property
    def K(self) -> np.ndarray:
        return np.array([[self.f, 0.0, self.cx], [0.0, self.f, self.cy], [0.0, 0.0, 1.0]])


class Scene:
    """Six textured planes, stored in world coordinates."""

    OCTAVES = 4
    LATTICE = 256

    def __init__(self, cam: Camera, seed: int, R0: np.ndarray, T0: np.ndarray, n_planes: int = 6):
        rng = np.random.default_rng(seed)
        self.cam = cam
        Kinv = np.linalg.inv(cam.K)
        self.n, self.c, self.e1, self.e2 = [], [], [], []
        self.tables = []
        for _ in range(n_planes):
            # normal within 40 degrees of -z (facing the reference camera)
            theta = np.deg2rad(40.0) * np.sqrt(rng.uniform())
            phi = rng.uniform(0, 2 * np.pi)
            n_cam = np.array([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), -np.cos(theta)])
            px = np.array([rng.uniform(0, cam.W), rng.uniform(0, cam.H), 1.0])
            z = rng.uniform(1.0, 8.0)
            X_cam = z * (Kinv @ px)
            n_w = R0 @ n_cam
            X_w = R0 @ X_cam + T0
            a = np.cross(n_w, [1.0, 0.0, 0.0])
            if np.linalg.norm(a) < 1e-3:
                a = np.cross(n_w, [0.0, 1.0, 0.0])
            e1 = a / np.linalg.norm(a)
            e2 = np.cross(n_w, e1)
            self.n.append(n_w)
            self.c.append(X_w)
            self.e1.append(e1)
            self.e2.append(e2)
            self.tables.append(rng.uniform(0.0, 1.0, size=(self.OCTAVES, self.LATTICE, self.LATTICE)))
        self.base_cell = 0.30   # metres per lattice cell at the coarsest octave

    def _noise(self, k: int, s: np.ndarray, t: np.ndarray) -> np.ndarray:
        out = np.zeros_like(s)
        amp, tot = 1.0, 0.0
        L = self.LATTICE
        for o in range(self.OCTAVES):
            cell = self.base_cell / (2 ** o)
            fs, ft = s / cell, t / cell
            i0, j0 = np.floor(fs), np.floor(ft)
            a, b = fs - i0, ft - j0
            a = a * a * (3 - 2 * a)
            b = b * b * (3 - 2 * b)
            i0 = i0.astype(np.int64) % L
            j0 = j0.astype(np.int64) % L
            i1, j1 = (i0 + 1) % L, (j0 + 1) % L
            tab = self.tables[k][o]
            v = ((1 - a) * (1 - b) * tab[j0, i0] + a * (1 - b) * tab[j0, i1]
                 + (1 - a) * b * tab[j1, i0] + a * b * tab[j1, i1])
            out += amp * v
            tot += amp
            amp *= 0.5
        return out / tot

    def render(self, R: np.ndarray, T: np.ndarray, rng, noise_sigma: float = 2.0):
        """Ray-cast a camera with camera-to-world pose (R, T).  Returns (uint8 image, depth)."""
        cam = self.cam
        u, v = np.meshgrid(np.arange(cam.W, dtype=np.float64), np.arange(cam.H, dtype=np.float64))
        rays_c = np.stack([(u - cam.cx) / cam.f, (v - cam.cy) / cam.f, np.ones_like(u)], -1)
        rays_w = rays_c @ R.T
        best_t = np.full(u.shape, np.inf)
        best_k = np.full(u.shape, -1, np.int64)
        for k, (n, c) in enumerate(zip(self.n, self.c)):
            den = rays_w @ n
            with np.errstate(divide="ignore", invalid="ignore"):
                t = (n @ (c - T)) / den
            ok = (t > 1e-6) & (t < best_t)
            best_t = np.where(ok, t, best_t)
            best_k = np.where(ok, k, best_k)
        img = np.zeros(u.shape)
        for k in range(len(self.n)):
            m = best_k == k
            if not m.any():
                continue
            X = T + rays_w[m] * best_t[m][:, None]
            d = X - self.c[k]
            s = d @ self.e1[k]
            t = d @ self.e2[k]
            img[m] = self._noise(k, s, t)
        img = 255.0 * np.clip(0.5 + 1.6 * (img - 0.5), 0.0, 1.0)
        img = img + rng.normal(0.0, noise_sigma, size=img.shape)
        img8 = np.clip(np.rint(img), 0, 255).astype(np.uint8)
        depth = np.where(np.isfinite(best_t), best_t, 0.0)   # rays_c has unit z: t is depth
        return img8, depth


@dataclass
class FrameSet:
    """One reference frame with its source frames (one depth map of work)."""
    ref: np.ndarray          # (H, W) uint8
    srcs: np.ndarray         # (S, H, W) uint8
    K: np.ndarray
    R_ref: np.ndarray
    T_ref: np.ndarray
    R_srcs: np.ndarray       # (S, 3, 3)
    T_srcs: np.ndarray       # (S, 3)
    gt_depth: np.ndarray     # (H, W) float64, depth along the optical axis


def random_source_pose(rng, R_ref, T_ref, bmin=0.05, bmax=0.15, max_rot_deg=2.0):
    b = rng.uniform(bmin, bmax)
    T = T_ref + R_ref @ (b * _unit(rng))
    R = R_ref @ rodrigues(_unit(rng), np.deg2rad(max_rot_deg) * rng.uniform())
    return R, T


def make_sequence(W: int, H: int, f: float, S: int, n_keyframes: int, seed: int,
                  noise_sigma: float = 2.0, step: float = 0.04) -> list[FrameSet]:
    """Keyframes along a smooth sideways path through one scene, each with S sources."""
    cam = Camera(W, H, f)
    rng = np.random.default_rng(seed)
    R0 = rodrigues(_unit(rng), np.deg2rad(5.0) * rng.uniform())
    T0 = rng.normal(0.0, 0.5, size=3)
    scene = Scene(cam, int(rng.integers(1 << 31)), R0, T0)
    heading = R0 @ np.array([1.0, 0.0, 0.0])
    out = []
    for k in range(n_keyframes):
        R_ref = R0 @ rodrigues(np.array([0.0, 1.0, 0.0]), np.deg2rad(0.5) * k)
        T_ref = T0 + heading * step * k
        ref, depth = scene.render(R_ref, T_ref, rng, noise_sigma)
        Rs, Ts, imgs = [], [], []
        for _ in range(S):
            R, T = random_source_pose(rng, R_ref, T_ref)
            img, _ = scene.render(R, T, rng, noise_sigma)
            Rs.append(R)
            Ts.append(T)
            imgs.append(img)
        out.append(FrameSet(ref, np.stack(imgs), cam.K, R_ref, T_ref, np.stack(Rs), np.stack(Ts), depth))
    return out


def make_stream(W: int, H: int, f: float, n_frames: int, seed: int, noise_sigma: float = 2.0,
                step: float = 0.01, yaw_deg: float = 0.15):
    """A continuous camera stream through one scene (for the sequence driver): frame k sits
    step * k metres along a sideways heading and is turned yaw_deg * k about the camera's y axis.
    Returns (images (n, H, W) uint8, R (n, 3, 3), T (n, 3), K)."""
    cam = Camera(W, H, f)
    rng = np.random.default_rng(seed)
    R0 = rodrigues(_unit(rng), np.deg2rad(5.0) * rng.uniform())
    T0 = rng.normal(0.0, 0.5, size=3)
    scene = Scene(cam, int(rng.integers(1 << 31)), R0, T0)
    heading = R0 @ np.array([1.0, 0.0, 0.0])
    imgs, Rs, Ts = [], [], []
    for k in range(n_frames):
        R = R0 @ rodrigues(np.array([0.0, 1.0, 0.0]), np.deg2rad(yaw_deg) * k)
        T = T0 + heading * step * k
        img, _ = scene.render(R, T, rng, noise_sigma)
        imgs.append(img)
        Rs.append(R)
        Ts.append(T)
    return np.stack(imgs), np.stack(Rs), np.stack(Ts), cam.K


def make_frameset(W: int, H: int, f: float, S: int, seed: int, noise_sigma: float = 2.0) -> FrameSet:
    return make_sequence(W, H, f, S, 1, seed, noise_sigma)[0]


def plane_range(D: int, rho_min: float = 0.1, rho_max: float = 2.0):
    """(rho0, drho) for D planes uniform in [rho_min, rho_max] m^-1."""
    return rho_min, (rho_max - rho_min) / (D - 1)
