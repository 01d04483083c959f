"""Headless screen-space fluid rendering (the reference app's OpenGL passes as
CUDA kernels, pbf_b200/csrc/pbf_render.cu): cameras, the renderer and image
output.

The reference renders with glm matrices (src/renderapp.cpp:48-55) and its
camera class (include/camera.h); look_at and perspective restate glm::lookAt
and glm::perspective (right-handed, clip depth in [-1, 1]).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np

from ._lib import IMAGE, IMAGE_CHANNELS, Camera, check, lib

F = np.float32


def _normalize(v):
    v = np.asarray(v, np.float64)
    return v / np.linalg.norm(v)


def look_at(eye, center, up) -> np.ndarray:
    """glm::lookAt as a column-major float32[16]."""
    eye, center, up = (np.asarray(a, np.float64) for a in (eye, center, up))
    f = _normalize(center - eye)
    s = _normalize(np.cross(f, up))
    u = np.cross(s, f)
    m = np.eye(4)
    m[0, 0:3] = s
    m[1, 0:3] = u
    m[2, 0:3] = -f
    m[0, 3] = -s @ eye
    m[1, 3] = -u @ eye
    m[2, 3] = f @ eye
    return m.T.reshape(16).astype(np.float32)  # column-major


def perspective(fovy: float, aspect: float, near: float, far: float) -> np.ndarray:
    """glm::perspective (fovy in radians) as a column-major float32[16]."""
    t = math.tan(fovy / 2.0)
    m = np.zeros((4, 4))
    m[0, 0] = 1.0 / (aspect * t)
    m[1, 1] = 1.0 / t
    m[2, 2] = -(far + near) / (far - near)
    m[3, 2] = -1.0
    m[2, 3] = -(2.0 * far * near) / (far - near)
    return m.T.reshape(16).astype(np.float32)


def make_camera(eye, target, up, fovy: float, width: int, height: int, radius: float, near: float = 0.1,
                far: float = 1000.0, point_fov: Optional[float] = None, room=(-30.0, 0.0, -30.0, 30.0, 50.0, 30.0),
                light=(0.0, 50.0, -20.0), room_light=(0.0, 50.0, 0.0), smooth_iterations: int = 60) -> Camera:
    """A camera in the reference's conventions: the view looks from `eye` along
    eye -> target (include/camera.h re-orthogonalises `up`), the projection is
    glm::perspective(fovy), and the sprite size and the shading's surface
    reconstruction use tan(point_fov / 2) (the app's tanHalfFov)."""
    eye = np.asarray(eye, np.float64)
    inward = _normalize(eye - np.asarray(target, np.float64))
    right = _normalize(np.cross(up, inward))
    up2 = _normalize(np.cross(inward, right))
    cam = Camera()
    for i, v in enumerate(look_at(eye, eye - inward, up2)):
        cam.view[i] = float(v)
    for i, v in enumerate(perspective(fovy, width / height, near, far)):
        cam.proj[i] = float(v)
    for a in range(3):
        cam.cam_pos[a] = float(eye[a])
        cam.light_pos[a] = float(light[a])
        cam.light_diffuse[a] = 0.8
        cam.room_light_pos[a] = float(room_light[a])
        cam.room_light_diffuse[a] = 0.8
    tan_half = math.tan((fovy if point_fov is None else point_fov) / 2.0)
    cam.radius = float(radius)
    cam.tan_half_fov = float(np.float32(tan_half))
    cam.point_coeff = float(np.float32(height) / np.float32(tan_half))
    cam.roi = 1.3
    for i, v in enumerate(room):
        cam.room[i] = float(v)
    cam.smooth_iterations = int(smooth_iterations)
    return cam


def reference_app_camera(width: int = 800, height: int = 800, radius: float = 0.3) -> Camera:
    """The app's view (src/renderapp.cpp:48-55, 350-392): eye (0, 40, 85) looking
    at (0, 20, -1), glm::perspective(45, ...) -- the app passes 45 to a function
    that takes radians -- near 0.1, far 1000, sprites and shading with
    tanHalfFov = tan(22.5 degrees), the room of its background quads."""
    return make_camera((0.0, 40.0, 85.0), (0.0, 20.0, -1.0), (0.0, 1.0, 0.0), 45.0, width, height, radius,
                       point_fov=math.radians(45.0))


def box_camera(box: Sequence[float], width: int, height: int, radius: float, smooth_iterations: int = 60) -> Camera:
    """A view of a scene box (pMin xyz, pMax xyz) from the front, slightly above,
    with the box's left, right and back walls and floor as the room."""
    lo, hi = np.asarray(box[:3], np.float64), np.asarray(box[3:], np.float64)
    c = 0.5 * (lo + hi)
    ext = hi - lo
    fov = math.radians(45.0)
    t = math.tan(fov / 2.0)
    # the box's front face fills the view with a 10 % margin
    dist = 1.1 * max(ext[0] / (2.0 * t * (width / height)), ext[1] / (2.0 * t)) + 0.5 * ext[2]
    eye = (c[0], c[1] + 0.25 * ext[1], hi[2] + dist - 0.5 * ext[2])
    return make_camera(eye, c, (0.0, 1.0, 0.0), fov, width, height, radius, near=0.01 * dist, far=10.0 * dist,
                       room=tuple(lo) + tuple(hi), light=(c[0], hi[1] + ext[1], c[2] - 0.25 * ext[2]),
                       room_light=(c[0], hi[1] + ext[1], c[2]), smooth_iterations=smooth_iterations)


class Renderer:
    """A pbf_render handle: device images of width x height pixels."""

    def __init__(self, width: int, height: int):
        h = C.c_void_p()
        check(lib().pbf_render_create(int(width), int(height), C.byref(h)))
        self._h = h
        self.width, self.height = int(width), int(height)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pbf_render_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def frame(self, cam: Camera, positions=None, solver=None, stride: int = 3, stream=None) -> None:
        """Renders a solver's state, or n x stride device floats (a torch tensor or
        a device pointer with n given as positions.shape[0])."""
        st = None if stream is None else (stream if isinstance(stream, int) else int(stream.cuda_stream))
        if solver is not None:
            check(lib().pbf_render_frame_solver(self._h, solver.handle, C.byref(cam), st))
            return
        n = int(positions.shape[0])
        check(lib().pbf_render_frame(self._h, positions.data_ptr(), n, int(stride), C.byref(cam), st))

    def read(self, name: str) -> np.ndarray:
        """One image as (height, width) or (height, width, 4) float32, row 0 at the bottom."""
        ch = IMAGE_CHANNELS[name]
        out = np.empty((self.height, self.width, ch), np.float32)
        check(lib().pbf_render_read(self._h, IMAGE[name], out.ctypes.data, out.size))
        return out[:, :, 0] if ch == 1 else out


def to_rgb8(rgba: np.ndarray) -> np.ndarray:
    """float RGBA (row 0 at the bottom) -> uint8 RGB top-down, as the window shows it."""
    return (np.clip(rgba[::-1, :, :3], 0.0, 1.0) * 255.0 + 0.5).astype(np.uint8)


def save_png(path: str, rgba: np.ndarray) -> None:
    """8-bit RGB PNG (zlib from the standard library, no imaging package)."""
    import struct
    import zlib
    rgb = to_rgb8(rgba)
    h, w = rgb.shape[:2]
    raw = b"".join(b"\x00" + rgb[y].tobytes() for y in range(h))

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))


def save_ppm(path: str, rgba: np.ndarray) -> None:
    rgb = to_rgb8(rgba)
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (rgb.shape[1], rgb.shape[0]))
        f.write(rgb.tobytes())
