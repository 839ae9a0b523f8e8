"""Seeded synthetic stereo workloads: speckle-projected scenes rendered by ray casting.

Stands in for the reference's test-data generator (libs/synth, which needs Eigen/TBB) with the scene
parameters the benchmarks name. Nothing here is on the hot path: it makes the input bytes that both
the CUDA path and the CPU reference then consume.

Model
- Cameras: pinhole + Brown-Conrady distortion (k1, k2, p1, p2, k3), as
  libs/core/include/einstar/core/camera.hpp:23-30 defines `distort_normalized`.
- Rig: left camera at the origin looking down +z; the right camera's centre at (+baseline, 0, 0)
  in the left frame, optionally rotated about y (a converging rig).
- Projector: between the cameras, casting a random binary pattern of ~3 px cells at 50% fill; the
  pattern is sampled bilinearly (soft-edged dots) and shaded by the incidence angle.
- Noise: Gaussian, sigma in DN, then clipped to [0, 255] and rounded to uint8.
- Rectification (raw configurations): the Bouguet split of libs/calib/src/rectify.cpp:11-98 with one
  shared principal point (cx_offset = 0), and float32 remap tables built as in
  libs/calib/src/rectify.cpp:117-131. The tables are shared inputs of the CPU and GPU paths.

Geometry is computed in float64 with torch (CPU or CUDA device); outputs are numpy arrays.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

# --------------------------------------------------------------------------------------------------
# cameras and rig


@dataclass
class Camera:
    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float
    dist: tuple = (0.0, 0.0, 0.0, 0.0, 0.0)  # k1 k2 p1 p2 k3

    def distort(self, x, y):
        """Normalised (undistorted) -> distorted pixel coordinates (camera.hpp:23-30)."""
        k1, k2, p1, p2, k3 = self.dist
        r2 = x * x + y * y
        radial = 1 + k1 * r2 + k2 * r2 * r2 + k3 * r2 * r2 * r2
        xd = x * radial + 2 * p1 * x * y + p2 * (r2 + 2 * x * x)
        yd = y * radial + p1 * (r2 + 2 * y * y) + 2 * p2 * x * y
        return self.fx * xd + self.cx, self.fy * yd + self.cy

    def undistort(self, u, v, iterations=12):
        """Distorted pixel -> normalised coordinates, by fixed-point/Newton iteration."""
        x = (u - self.cx) / self.fx
        y = (v - self.cy) / self.fy
        if not any(self.dist):
            return x, y
        h = 1e-6
        for _ in range(iterations):
            ex = u - self.distort(x, y)[0]
            ey = v - self.distort(x, y)[1]
            jxx = (self.distort(x + h, y)[0] - self.distort(x - h, y)[0]) / (2 * h)
            jxy = (self.distort(x, y + h)[0] - self.distort(x, y - h)[0]) / (2 * h)
            jyx = (self.distort(x + h, y)[1] - self.distort(x - h, y)[1]) / (2 * h)
            jyy = (self.distort(x, y + h)[1] - self.distort(x, y - h)[1]) / (2 * h)
            det = jxx * jyy - jxy * jyx
            x = x + (jyy * ex - jxy * ey) / det
            y = y + (-jyx * ex + jxx * ey) / det
        return x, y


def rot_axis(axis, angle) -> np.ndarray:
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + math.sin(angle) * K + (1 - math.cos(angle)) * (K @ K)


@dataclass
class Rig:
    left: Camera
    right: Camera
    R: np.ndarray  # right-camera coords = R @ left coords + t
    t: np.ndarray

    @property
    def baseline(self) -> float:
        return float(np.linalg.norm(self.t))


def make_rig(width, height, f, baseline, *, k1=0.0, k2=0.0, yaw_deg=0.0) -> Rig:
    """Right camera centre at (+baseline, 0, 0) in the left frame, rotated by yaw_deg about y."""
    cam = Camera(width, height, f, f, (width - 1) / 2.0, (height - 1) / 2.0, (k1, k2, 0.0, 0.0, 0.0))
    R = rot_axis((0, 1, 0), math.radians(yaw_deg))
    centre = np.array([baseline, 0.0, 0.0])
    t = -R @ centre
    return Rig(cam, Camera(**{**cam.__dict__}), R, t)


# --------------------------------------------------------------------------------------------------
# rectification (Bouguet split, shared principal point)


@dataclass
class Rectification:
    R_left: np.ndarray
    R_right: np.ndarray
    f: float
    cx: float
    cy: float
    width: int
    height: int
    baseline: float
    cx_offset: float = 0.0


def compute_rectification(rig: Rig) -> Rectification:
    """Each camera turns by half the relative rotation, then both align x with the baseline
    (libs/calib/src/rectify.cpp:11-98, shared-principal-point branch :84-93)."""
    R, t = rig.R, rig.t
    angle = math.acos(max(-1.0, min(1.0, (np.trace(R) - 1) / 2)))
    if angle < 1e-12:
        r_half = np.eye(3)
    else:
        axis = np.array([R[2, 1] - R[1, 2], R[0, 2] - R[2, 0], R[1, 0] - R[0, 1]]) / (2 * math.sin(angle))
        r_half = rot_axis(axis, -0.5 * angle)
    l_half = r_half.T
    tr = r_half @ t
    e1 = -tr / np.linalg.norm(tr)
    e2 = np.cross([0.0, 0.0, 1.0], e1)
    if np.linalg.norm(e2) < 1e-9:
        e2 = np.array([0.0, 1.0, 0.0])
    e2 = e2 / np.linalg.norm(e2)
    e3 = np.cross(e1, e2)
    r_align = np.stack([e1, e2, e3])
    R_left, R_right = r_align @ l_half, r_align @ r_half
    f = min(rig.left.fx, rig.left.fy, rig.right.fx, rig.right.fy)
    w, h = rig.left.width, rig.left.height

    def centre_ray(cam, Rr):
        x, y = cam.undistort(np.float64(cam.width * 0.5), np.float64(cam.height * 0.5))
        ray = Rr @ np.array([x, y, 1.0])
        return ray[:2] / ray[2]

    c = 0.5 * (centre_ray(rig.left, R_left) + centre_ray(rig.right, R_right))
    return Rectification(R_left, R_right, f, w * 0.5 - f * c[0], h * 0.5 - f * c[1], w, h, rig.baseline)


def build_remap(cam: Camera, R_rect: np.ndarray, rect: Rectification, device="cpu"):
    """For each rectified pixel, the source pixel in the distorted image (rectify.cpp:117-131)."""
    dev = torch.device(device)
    ys, xs = torch.meshgrid(torch.arange(rect.height, dtype=torch.float64, device=dev),
                            torch.arange(rect.width, dtype=torch.float64, device=dev), indexing="ij")
    rx, ry = (xs - rect.cx) / rect.f, (ys - rect.cy) / rect.f
    Ri = torch.tensor(R_rect.T, dtype=torch.float64, device=dev)
    X = Ri[0, 0] * rx + Ri[0, 1] * ry + Ri[0, 2]
    Y = Ri[1, 0] * rx + Ri[1, 1] * ry + Ri[1, 2]
    Z = Ri[2, 0] * rx + Ri[2, 1] * ry + Ri[2, 2]
    u, v = cam.distort(X / Z, Y / Z)
    return u.float().cpu().numpy(), v.float().cpu().numpy()


# --------------------------------------------------------------------------------------------------
# scene primitives (world = left camera frame, mm)


@dataclass
class Plane:
    point: tuple
    normal: tuple


@dataclass
class Sphere:
    centre: tuple
    radius: float


@dataclass
class Box:
    centre: tuple
    R: np.ndarray  # box axes in world (columns)
    half: tuple


@dataclass
class Cylinder:
    centre: tuple
    axis: tuple
    radius: float
    half_height: float


@dataclass
class Projector:
    position: tuple
    f: float = 900.0
    width: int = 1280
    height: int = 800
    cell: float = 3.0
    seed: int = 7
    fill: float = 0.5
    R: np.ndarray | None = None  # world -> projector rotation (None: axes of the world)


@dataclass
class Scene:
    primitives: list = field(default_factory=list)
    projector: Projector = field(default_factory=lambda: Projector((30.0, 15.0, 0.0)))


def _hit_plane(o, d, p: Plane):
    n = torch.tensor(p.normal, dtype=torch.float64, device=o.device)
    n = n / n.norm()
    q = torch.tensor(p.point, dtype=torch.float64, device=o.device)
    den = (d * n).sum(-1)
    t = ((q - o) * n).sum(-1) / torch.where(den.abs() < 1e-12, torch.full_like(den, 1e-12), den)
    nrm = n.expand_as(d)
    return torch.where(t > 1e-6, t, torch.full_like(t, math.inf)), nrm


def _hit_sphere(o, d, s: Sphere):
    c = torch.tensor(s.centre, dtype=torch.float64, device=o.device)
    oc = o - c
    b = (oc * d).sum(-1)
    cc = (oc * oc).sum(-1) - s.radius ** 2
    disc = b * b - cc
    sq = torch.sqrt(torch.clamp(disc, min=0))
    t0, t1 = -b - sq, -b + sq
    t = torch.where(t0 > 1e-6, t0, t1)
    t = torch.where((disc >= 0) & (t > 1e-6), t, torch.full_like(t, math.inf))
    p = o + d * t.unsqueeze(-1).clamp(max=1e9)
    return t, (p - c) / s.radius


def _hit_box(o, d, b: Box):
    R = torch.tensor(np.asarray(b.R), dtype=torch.float64, device=o.device)
    c = torch.tensor(b.centre, dtype=torch.float64, device=o.device)
    half = torch.tensor(b.half, dtype=torch.float64, device=o.device)
    ol = (o - c) @ R
    dl = d @ R
    inv = 1.0 / torch.where(dl.abs() < 1e-12, torch.full_like(dl, 1e-12), dl)
    ta, tb = (-half - ol) * inv, (half - ol) * inv
    tmin, tmax = torch.minimum(ta, tb), torch.maximum(ta, tb)
    tn, axis = tmin.max(-1)
    tf = tmax.min(-1).values
    hit = (tn <= tf) & (tf > 1e-6)
    t = torch.where(tn > 1e-6, tn, tf)
    t = torch.where(hit, t, torch.full_like(t, math.inf))
    nl = torch.zeros_like(dl)
    nl.scatter_(-1, axis.unsqueeze(-1), 1.0)
    nl = nl * -torch.sign(dl)
    return t, nl @ R.T


def _hit_cylinder(o, d, cy: Cylinder):
    a = torch.tensor(cy.axis, dtype=torch.float64, device=o.device)
    a = a / a.norm()
    c = torch.tensor(cy.centre, dtype=torch.float64, device=o.device)
    oc = o - c
    da, oa = (d * a).sum(-1), (oc * a).sum(-1)
    dp, op = d - da.unsqueeze(-1) * a, oc - oa.unsqueeze(-1) * a
    A = (dp * dp).sum(-1)
    B = 2 * (dp * op).sum(-1)
    Cc = (op * op).sum(-1) - cy.radius ** 2
    disc = B * B - 4 * A * Cc
    sq = torch.sqrt(torch.clamp(disc, min=0))
    A2 = torch.where(A < 1e-12, torch.full_like(A, 1e-12), 2 * A)
    inf = torch.full_like(A, math.inf)
    best, nbest = inf.clone(), torch.zeros_like(d)
    for tt in ((-B - sq) / A2, (-B + sq) / A2):
        h = oa + tt * da
        ok = (disc >= 0) & (tt > 1e-6) & (h.abs() <= cy.half_height) & (tt < best)
        p = oc + d * tt.unsqueeze(-1).clamp(-1e9, 1e9)
        n = p - (p * a).sum(-1, keepdim=True) * a
        best = torch.where(ok, tt, best)
        nbest = torch.where(ok.unsqueeze(-1), n / cy.radius, nbest)
    for s in (-1.0, 1.0):
        tt = (s * cy.half_height - oa) / torch.where(da.abs() < 1e-12, torch.full_like(da, 1e-12), da)
        p = oc + d * tt.unsqueeze(-1).clamp(-1e9, 1e9)
        r2 = ((p - (p * a).sum(-1, keepdim=True) * a) ** 2).sum(-1)
        ok = (tt > 1e-6) & (r2 <= cy.radius ** 2) & (tt < best)
        best = torch.where(ok, tt, best)
        nbest = torch.where(ok.unsqueeze(-1), (s * a).expand_as(d), nbest)
    return best, nbest


_HIT = {Plane: _hit_plane, Sphere: _hit_sphere, Box: _hit_box, Cylinder: _hit_cylinder}


def _pattern(proj: Projector, device):
    g = torch.Generator(device="cpu").manual_seed(proj.seed)
    gw, gh = int(math.ceil(proj.width / proj.cell)) + 2, int(math.ceil(proj.height / proj.cell)) + 2
    return (torch.rand((gh, gw), generator=g, dtype=torch.float64) < proj.fill).to(torch.float64).to(device)


def _sample_pattern(grid, proj: Projector, P):
    """Projector pixel of world points P -> bilinear sample of the binary cell grid (0 outside)."""
    pp = P - torch.tensor(proj.position, dtype=torch.float64, device=P.device)
    if proj.R is not None:
        pp = pp @ torch.tensor(np.asarray(proj.R, np.float64), device=P.device).T
    z = pp[..., 2]
    u = proj.f * pp[..., 0] / z + proj.width / 2.0
    v = proj.f * pp[..., 1] / z + proj.height / 2.0
    gu, gv = u / proj.cell, v / proj.cell
    inside = (z > 1) & (u >= 0) & (v >= 0) & (u < proj.width) & (v < proj.height)
    x0, y0 = torch.floor(gu), torch.floor(gv)
    fx, fy = gu - x0, gv - y0
    gh, gw = grid.shape
    x0 = x0.clamp(0, gw - 2).long()
    y0 = y0.clamp(0, gh - 2).long()
    a, b = grid[y0, x0], grid[y0, x0 + 1]
    c, d = grid[y0 + 1, x0], grid[y0 + 1, x0 + 1]
    s = (a * (1 - fx) + b * fx) * (1 - fy) + (c * (1 - fx) + d * fx) * fy
    return torch.where(inside, s, torch.zeros_like(s))


def render(scene: Scene, cam: Camera, R_wc: np.ndarray, centre, *, noise_sigma=2.0, seed=0, device="cpu",
           distorted=True):
    """Renders the view of a camera with world->camera rotation R_wc and centre `centre` (world).

    Returns (image uint8 HxW, depth float32 HxW: camera-frame z of the hit, 0 where nothing is hit).
    """
    dev = torch.device(device)
    vs, us = torch.meshgrid(torch.arange(cam.height, dtype=torch.float64, device=dev),
                            torch.arange(cam.width, dtype=torch.float64, device=dev), indexing="ij")
    if distorted:
        x, y = cam.undistort(us, vs)
    else:
        x, y = (us - cam.cx) / cam.fx, (vs - cam.cy) / cam.fy
    rc = torch.stack([x, y, torch.ones_like(x)], -1)
    Rcw = torch.tensor(np.asarray(R_wc).T, dtype=torch.float64, device=dev)
    d = rc @ Rcw.T
    d = d / d.norm(dim=-1, keepdim=True)
    o = torch.tensor(np.asarray(centre, np.float64), device=dev).expand_as(d)
    best = torch.full(d.shape[:-1], math.inf, dtype=torch.float64, device=dev)
    nrm = torch.zeros_like(d)
    for prim in scene.primitives:
        t, n = _HIT[type(prim)](o, d, prim)
        closer = t < best
        best = torch.where(closer, t, best)
        nrm = torch.where(closer.unsqueeze(-1), n, nrm)
    hit = torch.isfinite(best)
    P = o + d * torch.where(hit, best, torch.zeros_like(best)).unsqueeze(-1)
    grid = _pattern(scene.projector, dev)
    pat = _sample_pattern(grid, scene.projector, P)
    L = P - torch.tensor(scene.projector.position, dtype=torch.float64, device=dev)
    L = L / L.norm(dim=-1, keepdim=True).clamp(min=1e-9)
    cosi = (nrm * L).sum(-1).abs().clamp(0.25, 1.0)
    img = 18.0 + 205.0 * pat * cosi
    img = torch.where(hit, img, torch.full_like(img, 6.0))
    g = torch.Generator(device=dev).manual_seed(int(seed))
    img = img + noise_sigma * torch.randn(img.shape, generator=g, dtype=torch.float64, device=dev)
    img = torch.clamp(torch.round(img), 0, 255).to(torch.uint8)
    Pc = (P - o) @ torch.tensor(np.asarray(R_wc), dtype=torch.float64, device=dev).T
    depth = torch.where(hit, Pc[..., 2], torch.zeros_like(best)).float()
    return img.cpu().numpy(), depth.cpu().numpy()


# --------------------------------------------------------------------------------------------------
# the benchmark workloads


@dataclass
class StereoPair:
    """One workload item: the images the hot path consumes plus what is needed to check it."""
    left: np.ndarray
    right: np.ndarray
    f: float
    baseline: float
    cx_offset: float
    min_disparity: int
    num_disparities: int
    depth_left: np.ndarray | None = None
    maps: tuple | None = None  # ((map_lx, map_ly), (map_rx, map_ry)) for raw pairs
    rectified: tuple | None = None
    meta: dict = field(default_factory=dict)

    @property
    def raw(self) -> bool:
        return self.maps is not None


def _rect_render(scene, f, baseline, w, h, seed, device):
    """An already rectified pair (identical pinholes, right centre at +baseline on x)."""
    cam = Camera(w, h, f, f, (w - 1) / 2.0, (h - 1) / 2.0)
    left, dl = render(scene, cam, np.eye(3), (0.0, 0.0, 0.0), seed=2 * seed + 1, device=device, distorted=False)
    right, _ = render(scene, cam, np.eye(3), (baseline, 0.0, 0.0), seed=2 * seed + 2, device=device, distorted=False)
    return left, right, dl


def plane_sphere_pair(seed=0, width=640, height=512, f=900.0, baseline=60.0, num_disparities=64, device="cpu",
                      plane_z=300.0, sphere_z=350.0, sphere_r=60.0) -> StereoPair:
    """A tilted plane at `plane_z` plus a sphere (radius sphere_r, centre depth sphere_z), speckle-lit,
    rendered by two rectified pinholes (principal point at the image centre), sigma 2 DN."""
    rng = np.random.default_rng(10_000 + seed)
    tilt_y, tilt_x = math.radians(rng.uniform(10, 18)), math.radians(rng.uniform(-10, 10))
    n = rot_axis((1, 0, 0), tilt_x) @ rot_axis((0, 1, 0), tilt_y) @ np.array([0.0, 0.0, -1.0])
    half_w = (width / 2) * plane_z / f
    sx = float(rng.uniform(0.25, 0.6)) * half_w
    scene = Scene([Plane((0.0, 0.0, plane_z), tuple(n)), Sphere((sx, float(rng.uniform(-0.2, 0.2)) * half_w, sphere_z), sphere_r)],
                  Projector((baseline / 2, 15.0, 0.0), f=f, seed=1000 + seed))
    left, right, dl = _rect_render(scene, f, baseline, width, height, seed, device)
    valid = dl > 0
    dmax = f * baseline / max(float(np.percentile(dl[valid], 1)), 1.0)
    dmin = f * baseline / float(np.percentile(dl[valid], 99))
    centre = 0.5 * (dmin + dmax)
    mind = int(math.floor(min(dmin - 4, centre - num_disparities / 2)))
    return StereoPair(left, right, f, baseline, 0.0, mind, num_disparities, dl, meta={"scene": "plane+sphere", "seed": seed})


def random_objects_scene(rng, n_objects, z_range, f, width, height, baseline, seed):
    prims = []
    for i in range(n_objects):
        z = float(rng.uniform(*z_range))
        hw, hh = 0.5 * width * z / f, 0.5 * height * z / f
        c = (float(rng.uniform(-0.85, 0.85) * hw), float(rng.uniform(-0.85, 0.85) * hh), z)
        if i % 2 == 0:
            q = rot_axis(rng.normal(size=3), rng.uniform(0, math.pi))
            prims.append(Box(c, q, tuple(float(v) for v in rng.uniform(8, 30, size=3))))
        else:
            ax = rng.normal(size=3)
            prims.append(Cylinder(c, tuple(ax / np.linalg.norm(ax)), float(rng.uniform(8, 25)), float(rng.uniform(15, 45))))
    back_z = z_range[1] + 20.0
    prims.append(Plane((0.0, 0.0, back_z), tuple(rot_axis((1, 0, 0), math.radians(rng.uniform(-8, 8))) @ np.array([0, 0, -1.0]))))
    return Scene(prims, Projector((baseline / 2, 15.0, 0.0), f=f, seed=2000 + seed))


def raw_objects_pair(seed=0, width=1280, height=1024, f=1100.0, baseline=60.0, k1=-0.08, k2=0.02, yaw_deg=1.5,
                     num_disparities=128, n_objects=20, z_range=(200.0, 600.0), device="cpu") -> StereoPair:
    """A raw (unrectified, distorted) pair of `n_objects` random boxes and cylinders in z_range before a
    back wall, plus float32 remap tables to the rectified frame. min_disparity is put at the far end of
    the range so the D window covers the densest depth band; nearer surfaces fall outside it."""
    rng = np.random.default_rng(20_000 + seed)
    rig = make_rig(width, height, f, baseline, k1=k1, k2=k2, yaw_deg=yaw_deg)
    scene = random_objects_scene(rng, n_objects, z_range, f, width, height, baseline, seed)
    # Right camera: world->camera rotation R, centre C = -R^T t.
    C = -rig.R.T @ rig.t
    left, dl = render(scene, rig.left, np.eye(3), (0.0, 0.0, 0.0), seed=2 * seed + 1, device=device)
    right, _ = render(scene, rig.right, rig.R, tuple(C), seed=2 * seed + 2, device=device)
    rect = compute_rectification(rig)
    ml = build_remap(rig.left, rect.R_left, rect, device)
    mr = build_remap(rig.right, rect.R_right, rect, device)
    d_far = rect.f * rect.baseline / (z_range[1] + 25.0)
    mind = int(math.floor(d_far)) - 2
    return StereoPair(left, right, rect.f, rect.baseline, 0.0, mind, num_disparities, None, maps=(ml, mr),
                      meta={"scene": "boxes+cylinders", "seed": seed, "rect": rect})


def batch_pairs(n=64, seed=0, device="cpu"):
    """Uneven batch: 24 x 640x512, 24 x 1280x1024, 16 x 960x768 rectified speckle pairs, each with its own
    calibration (f 800-1200 px, baseline 50-70 mm) and D drawn from {64, 96, 128, 192}."""
    rng = np.random.default_rng(30_000 + seed)
    sizes = [(640, 512)] * 24 + [(1280, 1024)] * 24 + [(960, 768)] * 16
    sizes = [sizes[i * 64 // n] for i in range(n)] if n != 64 else sizes
    out = []
    for i, (w, h) in enumerate(sizes):
        f = float(rng.uniform(800, 1200))
        b = float(rng.uniform(50, 70))
        nd = int(rng.choice([64, 96, 128, 192]))
        out.append(plane_sphere_pair(seed=seed * 1000 + i, width=w, height=h, f=f, baseline=b, num_disparities=nd,
                                     device=device))
    return out



# --------------------------------------------------------------------------------------------------
# offline recording: a handheld orbit around a small object


@dataclass
class Recording:
    """A synthetic raw IR recording: one rig, one object scene, a smooth handheld orbit of n_frames."""
    rig: Rig
    rect: Rectification
    maps: tuple
    primitives: list
    poses: list                  # (R_wc, centre) of the left camera per frame
    min_disparity: int
    num_disparities: int
    seed: int

    @property
    def n_frames(self) -> int:
        return len(self.poses)


def _look_at(centre: np.ndarray, target: np.ndarray, up=(0.0, -1.0, 0.0)) -> np.ndarray:
    """World -> camera rotation of a camera at `centre` looking at `target` (camera y points down)."""
    z = target - centre
    z = z / np.linalg.norm(z)
    x = np.cross(z, np.asarray(up, np.float64))
    x = x / np.linalg.norm(x)
    y = np.cross(z, x)
    return np.stack([x, y, z])


def recording(n_frames=2000, seed=0, width=1280, height=1024, f=1100.0, baseline=60.0, k1=-0.08, k2=0.02,
              yaw_deg=1.5, num_disparities=256, standoff=(250.0, 450.0), device="cpu") -> Recording:
    """A 150 mm object (12 random boxes, cylinders and spheres on a base plane) and a smooth handheld
    trajectory orbiting it at 250-450 mm. min_disparity brackets the object over the whole orbit."""
    rng = np.random.default_rng(40_000 + seed)
    prims: list = [Plane((0.0, 60.0, 0.0), (0.0, -1.0, 0.0))]  # base plane (world y points down)
    for _ in range(12):
        c = (float(rng.uniform(-55, 55)), float(rng.uniform(-20, 40)), float(rng.uniform(-55, 55)))
        kind = int(rng.integers(3))
        if kind == 0:
            prims.append(Box(c, rot_axis((0, 1, 0), float(rng.uniform(0, math.pi))),
                             tuple(float(v) for v in rng.uniform(8, 30, 3))))
        elif kind == 1:
            prims.append(Cylinder(c, (0.0, 1.0, 0.0), float(rng.uniform(8, 25)), float(rng.uniform(10, 40))))
        else:
            prims.append(Sphere(c, float(rng.uniform(10, 30))))
    rig = make_rig(width, height, f, baseline, k1=k1, k2=k2, yaw_deg=yaw_deg)
    rect = compute_rectification(rig)
    maps = (build_remap(rig.left, rect.R_left, rect, device), build_remap(rig.right, rect.R_right, rect, device))
    # smooth orbit: azimuth sweeps ~1.5 turns, elevation and standoff drift slowly, plus hand tremor
    t = np.linspace(0.0, 1.0, n_frames)
    ph = rng.uniform(0, 2 * math.pi, 4)
    az = 3.0 * math.pi * t + ph[0]
    el = np.radians(30.0 + 10.0 * np.sin(2 * math.pi * 1.3 * t + ph[1]))
    lo, hi = standoff
    r = lo + (hi - lo) * 0.5 * (1 + np.sin(2 * math.pi * 0.9 * t + ph[2]))
    tremor = 1.5 * np.stack([np.sin(2 * math.pi * 37 * t + ph[3]), np.cos(2 * math.pi * 29 * t),
                             np.sin(2 * math.pi * 23 * t)], -1)
    poses = []
    for i in range(n_frames):
        c = np.array([r[i] * math.cos(el[i]) * math.sin(az[i]), -r[i] * math.sin(el[i]),
                      -r[i] * math.cos(el[i]) * math.cos(az[i])]) + tremor[i]
        poses.append((_look_at(c, np.array([0.0, 10.0, 0.0])), c))
    z_far = hi + 110.0
    mind = int(math.floor(rect.f * rect.baseline / z_far)) - 2
    return Recording(rig, rect, maps, prims, poses, mind, num_disparities, seed)


def recording_frame(rec: Recording, i: int, device="cpu") -> tuple[np.ndarray, np.ndarray]:
    """The raw (distorted) left and right IR images of frame i; the projector moves with the rig."""
    R_wl, c_l = rec.poses[i]
    rig = rec.rig
    R_wr = rig.R @ R_wl                                   # world -> right camera
    c_r = c_l + R_wl.T @ (-rig.R.T @ rig.t)               # right centre in the world
    p_rig = np.array([0.5 * rig.baseline, 15.0, 0.0])     # projector between the cameras, as in the rigs above
    proj = Projector(tuple(c_l + R_wl.T @ p_rig), f=900.0, seed=1000 + rec.seed, R=R_wl)
    scene = Scene(rec.primitives, proj)
    left, _ = render(scene, rig.left, R_wl, tuple(c_l), seed=7 * i + 1, device=device)
    right, _ = render(scene, rig.right, R_wr, tuple(c_r), seed=7 * i + 2, device=device)
    return left, right


@dataclass
class MarkerLayout:
    """Stickers and distractors composited into an IR image (pixel coordinates)."""
    markers: list  # (cx, cy, a, b, angle): white disc semi-axes a >= b, angle of a
    glints: list   # (cx, cy, r): bright spots on a bright surround
    dots: list     # (cx, cy): small bright speckle-like dots


def add_markers(img: np.ndarray, n_markers: int = 20, seed: int = 0, radius=(3.0, 9.0), n_glints: int = 6, n_dots: int = 40,
                margin: int = 24) -> tuple[np.ndarray, MarkerLayout]:
    """Composites retro-reflective marker stickers into an 8-bit IR image, as the scanner sees them under its
    ring light: a saturated elliptical disc (a foreshortened circle) inside a dark ring of 1.8x its size,
    sigma 2 DN noise. Distractors: bright glints on a bright surround and small bright dots. Stickers do
    not overlap; every one lies at least `margin` pixels inside the image."""
    rng = np.random.default_rng(30_000 + seed)
    out = np.array(img, dtype=np.float32, copy=True)
    h, w = out.shape
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    placed = []

    def free(cx, cy, r):
        return all((cx - px) ** 2 + (cy - py) ** 2 > (r + pr + 4) ** 2 for px, py, pr in placed)

    markers, glints, dots = [], [], []
    tries = 0
    while len(markers) < n_markers and tries < 50 * n_markers:
        tries += 1
        a = float(rng.uniform(*radius))
        b = a * float(rng.uniform(0.45, 1.0))
        ang = float(rng.uniform(0, math.pi))
        cx, cy = float(rng.uniform(margin + 2 * a, w - margin - 2 * a)), float(rng.uniform(margin + 2 * a, h - margin - 2 * a))
        if not free(cx, cy, 2.0 * a):
            continue
        placed.append((cx, cy, 2.0 * a))
        c, s = math.cos(ang), math.sin(ang)
        u = (xx - cx) * c + (yy - cy) * s
        v = -(xx - cx) * s + (yy - cy) * c
        rho = np.sqrt((u / a) ** 2 + (v / b) ** 2)
        out[(rho >= 1.0) & (rho < 1.8)] = rng.uniform(8, 25)
        out[rho < 1.0] = 254.0
        markers.append((cx, cy, a, b, ang))
    for _ in range(n_glints):
        r = float(rng.uniform(3, 7))
        cx, cy = float(rng.uniform(margin, w - margin)), float(rng.uniform(margin, h - margin))
        if not free(cx, cy, 3 * r):
            continue
        placed.append((cx, cy, 3 * r))
        d2 = (xx - cx) ** 2 + (yy - cy) ** 2
        out[d2 < (3 * r) ** 2] = np.maximum(out[d2 < (3 * r) ** 2], 170.0)
        out[d2 < r * r] = 240.0
        glints.append((cx, cy, r))
    for _ in range(n_dots):
        cx, cy = float(rng.uniform(4, w - 4)), float(rng.uniform(4, h - 4))
        if not free(cx, cy, 3):
            continue
        d2 = (xx - cx) ** 2 + (yy - cy) ** 2
        out[d2 < 2.5 ** 2] = 200.0
        dots.append((cx, cy))
    out += rng.normal(0.0, 2.0, size=out.shape).astype(np.float32)
    return np.clip(np.rint(out), 0, 255).astype(np.uint8), MarkerLayout(markers, glints, dots)
