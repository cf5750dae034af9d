"""ORACLE — CPU restatement of the QSDVR render path.  Test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import this module.  The product (``qsdvr_b200``) never calls it; it has no CPU fallback.

Float arithmetic is float64 torch on the CPU so that autograd gives exact reference
gradients.  Sample counts and cell indices come from ``raygen.c`` (float32, bit-exact with
the reference's CUDA build).  Every function cites the reference lines it restates
(paths relative to the reference project root).

Two shading/indexing modes exist (see ``compat`` arguments):
  * compat — the reference exactly: the shader reads SH coefficient ``i`` from the
    overlapping channels ``i, i+1, i+2`` (kernel/render.cu:166-169) while its backward
    writes the data gradient packed at ``3i..3i+2`` (kernel/render.cu:212); the vertex
    grid is addressed with the sample's cell index (stride R) and neighbour strides
    R+1, (R+1)^2 (kernel/camera.cu:91 with kernel/render.cu:108-111).
  * fixed — the packed SH layout everywhere and the vertex index x + y(R+1) + z(R+1)^2,
    whose backward is the exact gradient of its forward.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")

# kernel/render.cu:5-15 (full-precision real SH normalisation constants, degree 2)
SH_FACTOR = (
    0.28209479177387814347403972578039,
    0.48860251190291992158638462283835,
    0.48860251190291992158638462283835,
    0.48860251190291992158638462283835,
    1.0925484305920790705433857058027,
    1.0925484305920790705433857058027,
    0.31539156525252000603089369029571,
    1.0925484305920790705433857058027,
    0.54627421529603953527169285290135,
)

DTYPE = torch.float64


# ----------------------------------------------------------------------------- raygen (C)

class _Camera(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("rotation", ctypes.c_float * 9), ("translation", ctypes.c_float * 3),
                ("fx", ctypes.c_float), ("fy", ctypes.c_float), ("cx", ctypes.c_float),
                ("cy", ctypes.c_float), ("near_", ctypes.c_float), ("far_", ctypes.c_float)]


_raygen = None


def raygen_library_path() -> str:
    return os.path.join(_BUILD, "liboracle_raygen.so")


def build_raygen() -> str:
    """Compile raygen.c with gcc (no contraction beyond the explicit fmaf calls)."""
    import subprocess
    os.makedirs(_BUILD, exist_ok=True)
    out = raygen_library_path()
    src = os.path.join(_HERE, "raygen.c")
    if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC",
                               "-o", out, src, "-lm"])
    return out


def _lib():
    global _raygen
    if _raygen is None:
        path = raygen_library_path()
        if not os.path.exists(path):
            build_raygen()
        lib = ctypes.CDLL(path)
        P = ctypes.c_void_p
        lib.oracle_ray_cut.argtypes = [ctypes.POINTER(_Camera), P, ctypes.c_uint32, ctypes.c_float, P, P, P, P]
        lib.oracle_generate_ray_points.argtypes = [P, P, P, ctypes.c_uint32, ctypes.c_float, ctypes.c_uint32,
                                                   P, P, P, P, P]
        lib.oracle_list_points.argtypes = [P, P, P, ctypes.c_uint32, P, ctypes.c_uint32, P, P, P, P, P]
        lib.oracle_ray_cut_pixels.argtypes = [ctypes.POINTER(_Camera), P, ctypes.c_uint32, ctypes.c_float, P, P, P]
        _raygen = lib
    return _raygen


@dataclass
class Camera:
    """kernel/camera.h:4-17 (CameraArgs): intrinsics, row-major c2w rotation, near/far depths."""
    width: int
    height: int
    rotation: tuple
    translation: tuple
    fx: float
    fy: float
    cx: float
    cy: float
    near: float
    far: float

    def _c(self) -> _Camera:
        c = _Camera()
        c.width, c.height = self.width, self.height
        for i in range(9):
            c.rotation[i] = float(np.float32(self.rotation[i]))
        for i in range(3):
            c.translation[i] = float(np.float32(self.translation[i]))
        c.fx, c.fy, c.cx, c.cy = self.fx, self.fy, self.cx, self.cy
        c.near_, c.far_ = self.near, self.far
        return c


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def ray_cut(cam: Camera, mask: np.ndarray, interval: float, rays_prev: np.ndarray | None = None):
    """kernel/camera.cu:98-130 (RayCut): per-pixel rays and the masked exclusive scan.

    Returns (rays [P,4] uint32, origin [P,3] f32, dir [P,3] f32, sdf_total, render_total).
    """
    P = cam.width * cam.height
    mask = np.ascontiguousarray(mask.reshape(-1).astype(np.uint8))
    assert mask.size >= P
    rays = np.zeros((P, 4), np.uint32) if rays_prev is None else np.ascontiguousarray(rays_prev.astype(np.uint32)).copy()
    origin = np.zeros((P, 3), np.float32)
    direction = np.zeros((P, 3), np.float32)
    totals = np.zeros(2, np.uint32)
    c = cam._c()
    _lib().oracle_ray_cut(ctypes.byref(c), _ptr(mask), P, ctypes.c_float(interval), _ptr(rays), _ptr(origin),
                          _ptr(direction), _ptr(totals))
    return rays, origin, direction, int(totals[0]), int(totals[1])


def ray_cut_pixels(cam: Camera, pixels: np.ndarray, interval: float):
    """kernel/camera.cu:12-58 for a list of pixel ids: (rays [n,4] uint32 with packed offsets
    in list order, counts < 2 zeroed; origin [n,3]; dir [n,3])."""
    pixels = np.ascontiguousarray(pixels, np.uint32)
    n = pixels.size
    rays = np.zeros((n, 4), np.uint32)
    origin = np.zeros((n, 3), np.float32)
    direction = np.zeros((n, 3), np.float32)
    c = cam._c()
    _lib().oracle_ray_cut_pixels(ctypes.byref(c), _ptr(pixels), n, ctypes.c_float(interval), _ptr(rays), _ptr(origin),
                                 _ptr(direction))
    return rays, origin, direction


def generate_ray_points(rays: np.ndarray, origin: np.ndarray, direction: np.ndarray, interval: float, reso: int):
    """kernel/camera.cu:60-96,132-147 (GenerateRayPoints) for already-masked rays."""
    rays = np.ascontiguousarray(rays.astype(np.uint32))
    origin = np.ascontiguousarray(origin.astype(np.float32))
    direction = np.ascontiguousarray(direction.astype(np.float32))
    n = rays.shape[0]
    S = int((rays[:, 1].astype(np.int64) + rays[:, 0]).max()) if n else 0
    M = int((rays[:, 3].astype(np.int64) + rays[:, 2]).max()) if n else 0
    out = dict(sdfPointList=np.zeros((S, 3), np.float32), sdfIndexList=np.zeros(S, np.int32),
               renderPointList=np.zeros((M, 3), np.float32), renderIndexList=np.zeros(M, np.int32),
               viewDirList=np.zeros((M, 3), np.float32))
    _lib().oracle_generate_ray_points(_ptr(rays), _ptr(origin), _ptr(direction), n, ctypes.c_float(interval), reso,
                                      _ptr(out["sdfPointList"]), _ptr(out["sdfIndexList"]),
                                      _ptr(out["renderPointList"]), _ptr(out["renderIndexList"]),
                                      _ptr(out["viewDirList"]))
    return out


def list_points(rays: np.ndarray, origin: np.ndarray, direction: np.ndarray, tlist: np.ndarray, reso: int):
    """Sample lists of the fused renderer's list sampling (33 SDF positions per ray from
    ``tlist``, 32 render samples at their midpoints; raygen.c oracle_list_points), with the
    matching ``rayList`` (rays with sdf_count < 2 keep no samples)."""
    rays = np.ascontiguousarray(rays.astype(np.uint32))
    origin = np.ascontiguousarray(origin.astype(np.float32))
    direction = np.ascontiguousarray(direction.astype(np.float32))
    tlist = np.ascontiguousarray(tlist.astype(np.float32))
    n = rays.shape[0]
    hit = rays[:, 0] >= 2
    k = int(hit.sum())
    out = dict(sdfPointList=np.zeros((33 * k, 3), np.float32), sdfIndexList=np.zeros(33 * k, np.int32),
               renderPointList=np.zeros((32 * k, 3), np.float32), renderIndexList=np.zeros(32 * k, np.int32),
               viewDirList=np.zeros((32 * k, 3), np.float32))
    _lib().oracle_list_points(_ptr(rays), _ptr(origin), _ptr(direction), n, _ptr(tlist), reso,
                              _ptr(out["sdfPointList"]), _ptr(out["sdfIndexList"]), _ptr(out["renderPointList"]),
                              _ptr(out["renderIndexList"]), _ptr(out["viewDirList"]))
    rank = np.cumsum(hit) - hit
    rl = np.zeros((n, 4), np.int32)
    rl[hit, 0] = 33
    rl[hit, 1] = 33 * rank[hit]
    rl[hit, 2] = 32
    rl[hit, 3] = 32 * rank[hit]
    out["rayList"] = rl
    return out


# ----------------------------------------------------------------------------- surface

def _t(x):
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(x)
    return x


def sample_sdf(grid7: torch.Tensor, points: torch.Tensor, index: torch.Tensor, reso: float):
    """kernel/surface.cu:54-72: f(u) / |grad_u f| / R for the quadric cell at ``index``."""
    g = grid7.reshape(-1, 7)[_t(index).long()]
    p = _t(points).to(g.dtype)
    a0, a1, a2 = g[:, 0] * p[:, 0], g[:, 1] * p[:, 1], g[:, 2] * p[:, 2]
    value = (a0 + g[:, 3]) * p[:, 0] + (a1 + g[:, 4]) * p[:, 1] + (a2 + g[:, 5]) * p[:, 2] + g[:, 6]
    norm = torch.sqrt((2 * a0 + g[:, 3]) ** 2 + (2 * a1 + g[:, 4]) ** 2 + (2 * a2 + g[:, 5]) ** 2)
    return value / norm / reso


MAX_SDF, MIN_GRAD2 = 4.0, 1e-30


def sdf_trusted(grid7: torch.Tensor, points: torch.Tensor, index: torch.Tensor, reso: float):
    """fixed mode's rule for a usable SDF sample (qsdvr_b200/csrc/fused.cu checked_sdf): |grad f|^2
    at least 1e-30 and |sdf| at most 4 (a degenerate quadric point otherwise); no counterpart
    in the reference."""
    with torch.no_grad():
        g = grid7.reshape(-1, 7)[_t(index).long()]
        p = _t(points).to(g.dtype)
        len2 = sum((2 * g[:, c] * p[:, c] + g[:, 3 + c]) ** 2 for c in range(3))
        sdf = sample_sdf(grid7, points, index, reso)
        return torch.isfinite(sdf) & (sdf.abs() <= MAX_SDF) & (len2 >= MIN_GRAD2)


def _bf16_bits(x: np.ndarray) -> np.ndarray:
    """float32 -> bf16 bit patterns, round to nearest even (finite inputs)."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def _bf16_value(b: np.ndarray) -> np.ndarray:
    return (b.astype(np.uint32) << 16).view(np.float32)


def sdf_cells_bf16(grid8: np.ndarray) -> np.ndarray:
    """The library's bf16 form of fp32 quadric cells [N,8] (no reference counterpart; the
    library's qsdvr_sdf_cells_bf16), in float32 numpy with the same rounding steps: a0..a5
    rounded to nearest, a6' = a6 (|bf16(a3..a5)| / |a3..a5|) split into bf16 hi and lo.
    Returns the [N,8] uint16 bit patterns."""
    a = np.ascontiguousarray(grid8, np.float32).reshape(-1, 8)
    out = np.zeros(a.shape, np.uint16)
    out[:, :6] = _bf16_bits(a[:, :6])
    b = _bf16_value(out[:, 3:6])
    with np.errstate(all="ignore"):
        n0 = np.sqrt((a[:, 3] * a[:, 3] + a[:, 4] * a[:, 4]) + a[:, 5] * a[:, 5])
        n1 = np.sqrt((b[:, 0] * b[:, 0] + b[:, 1] * b[:, 1]) + b[:, 2] * b[:, 2])
        use = (n0 > 0) & np.isfinite(n0) & np.isfinite(n1)
        c6 = np.where(use, a[:, 6] * np.where(use, n1 / np.where(use, n0, 1), 1), a[:, 6]).astype(np.float32)
        out[:, 6] = _bf16_bits(c6)
        lo = (c6 - _bf16_value(out[:, 6])).astype(np.float32)
        out[:, 7] = np.where(np.isfinite(c6), _bf16_bits(np.where(np.isfinite(lo), lo, 0)), 0)
    return out


def sdf_cells_decode(cells) -> torch.Tensor:
    """[N,7] float32 coefficients the render kernels read from bf16 cells [N,8] (bit patterns
    or a torch bfloat16 tensor): a0..a5 and a6 = slot 6 + slot 7."""
    if torch.is_tensor(cells):
        cells = cells.detach().cpu().contiguous().view(torch.int16).numpy().view(np.uint16)
    v = _bf16_value(np.ascontiguousarray(cells, np.uint16).reshape(-1, 8))
    out = v[:, :7].copy()
    out[:, 6] = v[:, 6] + v[:, 7]
    return torch.from_numpy(out)


def sample_normal(grid7: torch.Tensor, points: torch.Tensor, index: torch.Tensor):
    """kernel/surface.cu:104-115: normalize(2 a_k u_k + a_{k+3})."""
    g = grid7.reshape(-1, 7)[_t(index).long()]
    p = _t(points).to(g.dtype)
    v = torch.stack([2 * g[:, 0] * p[:, 0] + g[:, 3], 2 * g[:, 1] * p[:, 1] + g[:, 4],
                     2 * g[:, 2] * p[:, 2] + g[:, 5]], 1)
    return v / torch.sqrt((v * v).sum(1, keepdim=True))


def layer_to_grid(x: torch.Tensor, y: torch.Tensor, z: torch.Tensor, offset: torch.Tensor):
    """kernel/surface.cu:148-229 (LayerToGridForward): separable layers -> [R,R,R,7].

    a3[i] = 2 a0[i-1] + 2 a0[i] + a3[i-1] with a3[0] = offset[k];
    a6[i] = 3 a0[i-1] + a0[i] + 2 a3[i-1] + a6[i-1] with a6[0] = 0.
    Cell (x,y,z) = (X0[x], Y1[y], Z2[z], X3[x], Y4[y], Z5[z], X6[x]+Y6[y]+Z6[z]+offset[3]).
    """
    def axis(a0, off):
        zero = a0.new_zeros(1)
        inc3 = torch.cat([zero, 2 * a0[:-1] + 2 * a0[1:]])
        a3 = off + torch.cumsum(inc3, 0)
        inc6 = torch.cat([zero, 3 * a0[:-1] + a0[1:] + 2 * a3[:-1]])
        a6 = torch.cumsum(inc6, 0)
        return a3, a6

    R = x.shape[0]
    x3, x6 = axis(x, offset[0])
    y4, y6 = axis(y, offset[1])
    z5, z6 = axis(z, offset[2])
    X = lambda v: v.view(1, 1, R).expand(R, R, R)  # noqa: E731  index order [z][y][x]
    Y = lambda v: v.view(1, R, 1).expand(R, R, R)  # noqa: E731
    Z = lambda v: v.view(R, 1, 1).expand(R, R, R)  # noqa: E731
    return torch.stack([X(x), Y(y), Z(z), X(x3), Y(y4), Z(z5), X(x6) + Y(y6) + Z(z6) + offset[3]], -1)


def layer_to_grid_backward(grad7: torch.Tensor):
    """kernel/surface.cu:231-341 (LayerToGridBackward): adjoint of layer_to_grid.

    The gradient of offset[3] is the sum of all a6 gradients; offset[0..2] receive the
    reverse-recurrence gradient of a3[0], a4[0], a5[0].  (The reference copies R floats
    into the 4-float offset tensor there; only the first lands in offset[3].)
    """
    R = grad7.shape[0]
    x = torch.zeros(R, dtype=grad7.dtype, requires_grad=True)
    y = torch.zeros(R, dtype=grad7.dtype, requires_grad=True)
    z = torch.zeros(R, dtype=grad7.dtype, requires_grad=True)
    off = torch.zeros(4, dtype=grad7.dtype, requires_grad=True)
    out = layer_to_grid(x, y, z, off)
    gx, gy, gz, go = torch.autograd.grad(out, (x, y, z, off), grad7)
    return gx, gy, gz, go


# ----------------------------------------------------------------------------- render

def grid_interpolation(data: torch.Tensor, points: torch.Tensor, index: torch.Tensor, reso: int):
    """kernel/render.cu:93-119: trilinear fetch of 32 channels.

    ``data`` is the flat vertex array [V, C]; the 8 corners of a sample are
    index, +1, +reso, +reso+1, +reso^2, ... exactly as the reference addresses them.
    """
    C = data.shape[-1]
    d = data.reshape(-1, C)
    p = (_t(points).to(d.dtype) + 1.0) / 2.0
    i000 = _t(index).long()
    i010 = i000 + reso
    i100 = i000 + reso * reso
    i110 = i100 + reso
    px, py, pz = p[:, 0:1], p[:, 1:2], p[:, 2:3]
    lerp = lambda a, b, t: a * (1 - t) + b * t  # noqa: E731
    a0 = lerp(lerp(d[i000], d[i000 + 1], px), lerp(d[i010], d[i010 + 1], px), py)
    a1 = lerp(lerp(d[i100], d[i100 + 1], px), lerp(d[i110], d[i110 + 1], px), py)
    return lerp(a0, a1, pz)


def sh_basis(v: torch.Tensor):
    """kernel/render.cu:17-59: the 9 real SH basis values (with factors) at direction v."""
    x, y, z = v[:, 0], v[:, 1], v[:, 2]
    f = SH_FACTOR
    return torch.stack([torch.full_like(x, f[0]), f[1] * x, f[2] * y, f[3] * z, f[4] * x * z, f[5] * x * y,
                        f[6] * (2.0 * y * y - z * z - x * x), f[7] * y * z, f[8] * (z * z - x * x)], 1)


# Degree-3 extension (not in the reference): the reference's degree-2 basis treats y as the
# polar axis with (z, x) spanning the azimuthal plane; band 3 follows the same convention with
# the real-SH normalisations sqrt(35/(32 pi)), sqrt(105/(4 pi)), sqrt(21/(32 pi)),
# sqrt(7/(16 pi)), sqrt(105/(16 pi)).
SH3_A, SH3_B, SH3_C, SH3_D, SH3_E = (0.59004358992664351034, 2.89061144264055405538, 0.45704579946446573616,
                                     0.37317633259011539141, 1.44530572132027702769)


def sh_basis3(v: torch.Tensor):
    """16 basis values at v: the 9 of sh_basis plus band 3."""
    x, y, z = v[:, 0], v[:, 1], v[:, 2]
    b3 = torch.stack([SH3_A * x * (3 * z * z - x * x), SH3_B * x * y * z, SH3_C * x * (4 * y * y - z * z - x * x),
                      SH3_D * y * (2 * y * y - 3 * z * z - 3 * x * x), SH3_C * z * (4 * y * y - z * z - x * x),
                      SH3_E * y * (z * z - x * x), SH3_A * z * (z * z - 3 * x * x)], 1)
    return torch.cat([sh_basis(v), b3], 1)


def shader_sh3(normal, view, data):
    """Degree-3 shading: SH 16x3 packed at 0..47, diffuse 48..50, metallic 51, ao 52."""
    normal = _t(normal)
    view = _t(view).to(normal.dtype)
    vdotn = (view * normal).sum(1, keepdim=True)
    reflect = view - normal * (2.0 * vdotn)
    spec = (sh_basis3(reflect).unsqueeze(-1) * data[:, :48].reshape(-1, 16, 3)).sum(1)
    diffuse, metallic, ao = data[:, 48:51], data[:, 51:52], data[:, 52:53]
    return (diffuse * (1.0 - metallic) + spec * metallic) * ao


def sh_coefficients(data: torch.Tensor, compat: bool):
    """[M,9,3] SH coefficients: overlapping reads (render.cu:166-169) or packed."""
    if compat:
        return torch.stack([data[:, i:i + 3] for i in range(9)], 1)
    return data[:, :27].reshape(-1, 9, 3)


def shader(normal, view, data, compat: bool):
    """kernel/render.cu:154-179: reflection SH-2 shading.  Returns (rgb, specular)."""
    normal = _t(normal)
    view = _t(view).to(normal.dtype)
    vdotn = (view * normal).sum(1, keepdim=True)
    reflect = view - normal * (2.0 * vdotn)
    coef = sh_coefficients(data, compat)
    spec = (sh_basis(reflect).unsqueeze(-1) * coef).sum(1)
    diffuse, metallic, ao = data[:, 27:30], data[:, 30:31], data[:, 31:32]
    rgb = (diffuse * (1.0 - metallic) + spec * metallic) * ao
    return rgb, spec


def shader_backward_reference(grad, normal, view, data, specular, compat: bool):
    """kernel/render.cu:181-221 and :61-91 exactly as written (Q1 in compat mode).

    Normal gradient uses the coefficients the forward read; the data gradient of the SH
    block is always written packed at 3i..3i+2.
    """
    grad, normal, view, data, specular = (_t(a).to(DTYPE) for a in (grad, normal, view, data, specular))
    coef = sh_coefficients(data, compat)
    diffuse, metallic, ao = data[:, 27:30], data[:, 30:31], data[:, 31:32]
    vdotn = (view * normal).sum(1, keepdim=True)
    reflect = view - normal * (2.0 * vdotn)
    color = diffuse * (1.0 - metallic) + specular * metallic
    dg = torch.zeros_like(data)
    dg[:, 31] = (grad * color).sum(1)
    g = grad * ao
    dg[:, 30] = (g * (specular - diffuse)).sum(1)
    dg[:, 27:30] = g * (1.0 - metallic)
    gm = g * metallic
    basis = sh_basis(reflect)
    dg[:, :27] = (basis.unsqueeze(-1) * gm.unsqueeze(1)).reshape(-1, 27)
    f = SH_FACTOR
    gc = [f[i] * (coef[:, i] * gm).sum(1) for i in range(1, 9)]
    x, y, z = reflect[:, 0], reflect[:, 1], reflect[:, 2]
    rg = torch.stack([gc[0] + z * gc[3] + y * gc[4] - 2 * x * (gc[5] + gc[7]),
                      gc[1] + z * gc[6] + x * gc[4] + 4 * y * gc[5],
                      gc[2] + x * gc[3] + y * gc[6] + 2 * z * (gc[7] - gc[5])], 1)
    n, v = normal, view
    xx, yy, zz = n[:, 0] * v[:, 0], n[:, 1] * v[:, 1], n[:, 2] * v[:, 2]
    ng = torch.stack([
        -2.0 * (rg[:, 0] * (2 * xx + yy + zz) + v[:, 0] * (rg[:, 1] * n[:, 1] + rg[:, 2] * n[:, 2])),
        -2.0 * (rg[:, 1] * (xx + 2 * yy + zz) + v[:, 1] * (rg[:, 0] * n[:, 0] + rg[:, 2] * n[:, 2])),
        -2.0 * (rg[:, 2] * (xx + yy + 2 * zz) + v[:, 2] * (rg[:, 0] * n[:, 0] + rg[:, 1] * n[:, 1]))], 1)
    return ng, dg


class _CompatShader(torch.autograd.Function):
    """Forward with overlapping SH reads, backward = the reference's own formulas."""

    @staticmethod
    def forward(ctx, normal, view, data):
        rgb, spec = shader(normal, view, data, True)
        ctx.save_for_backward(normal, view, data, spec)
        return rgb

    @staticmethod
    def backward(ctx, grad):
        normal, view, data, spec = ctx.saved_tensors
        ng, dg = shader_backward_reference(grad, normal, view, data, spec, True)
        return ng, None, dg


def shade(normal, view, data, compat: bool):
    """Differentiable shader matching the reference's forward and backward."""
    if compat:
        return _CompatShader.apply(normal, view, data)
    return shader(normal, view, data, False)[0]


def _ray_matrix(rays: torch.Tensor):
    rays = _t(rays).long()
    n_s = rays[:, 0]
    n_r = torch.clamp(n_s - 1, min=0)
    L = int(n_r.max()) if rays.shape[0] else 0
    i = torch.arange(max(L, 1), device=rays.device)
    valid = i.unsqueeze(0) < n_r.unsqueeze(1)
    r_idx = torch.where(valid, rays[:, 3:4] + i, torch.zeros_like(valid, dtype=torch.long))
    s0 = torch.where(valid, rays[:, 1:2] + i, torch.zeros_like(valid, dtype=torch.long))
    return valid, r_idx, s0


def ray_aggregate(rgb, sdf, rays, k: float, sdf_ok=None):
    """kernel/render.cu:223-253: NeuS alpha and front-to-back compositing per ray.

    E_i = exp(-k sdf_i); alpha_i = max((E_{i+1} - E_i) / (1 + E_{i+1}), 0);
    T_0 = 1, T_{i+1} = T_i (1 - alpha_i); C = sum_i T_i alpha_i rgb_i.
    ``sdf_ok`` (fixed mode): intervals with an untrusted end sample are empty (alpha 0).
    Returns (color [N,3], alpha [M], T [M]) with alpha/T at each render sample.
    """
    rgb, sdf = _t(rgb), _t(sdf)
    valid, r_idx, s0 = _ray_matrix(rays)
    if sdf_ok is not None:
        valid = valid & sdf_ok[s0] & sdf_ok[s0 + valid.long()]
        sdf = torch.where(sdf_ok, sdf, torch.zeros_like(sdf))
    E0 = torch.exp(-k * sdf[s0])
    E1 = torch.exp(-k * sdf[s0 + valid.long()])
    x = (E1 - E0) / (1.0 + E1)
    alpha = torch.where(valid & (x > 0), x, torch.zeros_like(x))
    one_minus = 1.0 - alpha
    T = torch.cumprod(torch.cat([torch.ones_like(one_minus[:, :1]), one_minus[:, :-1]], 1), 1)
    w = (T * alpha).unsqueeze(-1)
    color = (w * rgb[r_idx] * valid.unsqueeze(-1)).sum(1)
    M = rgb.shape[0]
    alpha_list = torch.zeros(M, dtype=rgb.dtype, device=rgb.device)
    T_list = torch.zeros(M, dtype=rgb.dtype, device=rgb.device)
    alpha_list[r_idx[valid]] = alpha[valid].detach()
    T_list[r_idx[valid]] = T[valid].detach()
    return color, alpha_list, T_list


def ray_aggregate_backward_reference(grad, rgb, sdf, rays, alpha, T, k: float):
    """kernel/render.cu:255-315 with its division by (alpha - 1) (Q10), vectorised.

    dC/dalpha_i = T_i c_i + (sum_{m>i} T_m alpha_m c_m) / (alpha_i - 1);
    dalpha_i/dsdf_i = k E_i / (1 + E_{i+1}), dalpha_i/dsdf_{i+1} = -k E_{i+1} (1 + E_i) / (1 + E_{i+1})^2,
    both zero where alpha_i == 0.
    """
    grad, rgb, sdf, alpha, T = (_t(a).to(DTYPE) for a in (grad, rgb, sdf, alpha, T))
    valid, r_idx, s0 = _ray_matrix(rays)
    vf = valid.to(DTYPE)
    a = alpha[r_idx] * vf
    Tm = T[r_idx] * vf
    c = rgb[r_idx] * vf.unsqueeze(-1)
    Tac_incl = torch.flip(torch.cumsum(torch.flip((Tm * a).unsqueeze(-1) * c, [1]), 1), [1])
    Tac_after = Tac_incl - (Tm * a).unsqueeze(-1) * c
    dC_da = Tm.unsqueeze(-1) * c + Tac_after / (a - 1.0).unsqueeze(-1)
    g = grad.unsqueeze(1)
    dL_da = (g * dC_da).sum(-1) * vf
    E0 = torch.exp(-k * sdf[s0])
    E1 = torch.exp(-k * sdf[s0 + valid.long()])
    inv = 1.0 / (1.0 + E1)
    d_next = -k * E1 * (1.0 + E0) * inv * inv
    d_this = k * E0 * inv
    zero = a == 0
    d_next = torch.where(zero, torch.zeros_like(d_next), d_next)
    d_this = torch.where(zero, torch.zeros_like(d_this), d_this)
    sdf_grad = torch.zeros(sdf.shape[0], dtype=DTYPE, device=sdf.device)
    sdf_grad.index_add_(0, s0[valid], (dL_da * d_this)[valid])
    sdf_grad.index_add_(0, (s0 + 1)[valid], (dL_da * d_next)[valid])
    rgb_grad = torch.zeros(rgb.shape[0], 3, dtype=DTYPE, device=rgb.device)
    rgb_grad[r_idx[valid]] = (g * (Tm * a).unsqueeze(-1))[valid]
    return rgb_grad, sdf_grad


# ----------------------------------------------------------------------------- pipeline

def vertex_index(cell_index: torch.Tensor, R: int, compat: bool):
    """Base vertex of a cell in the (R+1)^3 grid: the cell index itself in compat mode
    (kernel/camera.cu:91 used with stride R+1 in kernel/render.cu:108-111), else
    x + y(R+1) + z(R+1)^2."""
    idx = _t(cell_index).long()
    if compat:
        return idx
    x, y, z = idx % R, (idx // R) % R, idx // (R * R)
    return x + y * (R + 1) + z * (R + 1) * (R + 1)


def render(sdf_grid7, data, inputs: dict, k: float, compat: bool = True, sh_degree: int = 2):
    """The reference RenderGrid.forward (models/render.py:225-234) on a dense quadric grid.

    sdf_grid7: [R,R,R,7] (or [R^3,7]); data: [(R+1)^3, 32]; inputs: the dict of sample
    lists produced by GenerateRayPoints plus ``rayList``.  Differentiable in float64.
    """
    g7 = sdf_grid7.reshape(-1, 7)
    R = round(g7.shape[0] ** (1.0 / 3.0))
    sdf = sample_sdf(g7, inputs["sdfPointList"], inputs["sdfIndexList"], R)
    sdf_ok = None if compat else sdf_trusted(g7, inputs["sdfPointList"], inputs["sdfIndexList"], R)
    normal = sample_normal(g7, inputs["renderPointList"], inputs["renderIndexList"])
    vidx = vertex_index(inputs["renderIndexList"], R, compat)
    d = grid_interpolation(data.reshape(-1, data.shape[-1]), inputs["renderPointList"], vidx, R + 1)
    if sh_degree == 3:
        rgb = shader_sh3(normal, _t(inputs["viewDirList"]).to(DTYPE), d)
    else:
        rgb = shade(normal, _t(inputs["viewDirList"]).to(DTYPE), d, compat)
    color, _, _ = ray_aggregate(rgb, sdf, inputs["rayList"], k, sdf_ok)
    return color
