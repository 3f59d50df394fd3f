"""Domain setups shared by the oracle and the CUDA path (test infrastructure).

A setup is a plain dict ("spec") describing blocks, vertex coordinates,
initial fields and boundary operations; ``build_oracle`` turns it into an FP64
``oracle.piso_oracle.ODomain`` and ``build_product`` into a prepared
``pict_b200.PISOtorch.Domain`` built through the same public API calls a
reference user makes (CreateBlock, CloseAllBoundaries, CloseBoundary,
MakePeriodic, ConnectBlock, PrepareSolve).

The cases follow the reference's test setups (tests/test_setups.py:30-300):
single closed blocks with a lid, periodic blocks, two connected blocks, 3D
blocks, stretched and distorted (rotated) grids.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if os.path.join(ROOT, "oracle") not in sys.path:
    sys.path.insert(0, os.path.join(ROOT, "oracle"))

import piso_oracle as po  # noqa: E402


# ------------------------------------------------------------------ grids

def tensor_grid(xs, ys, zs=None):
    """Vertex coordinates [1, D, (z), y, x] of a tensor-product grid from 1D vertex arrays."""
    if zs is None:
        Y, X = np.meshgrid(ys, xs, indexing="ij")
        return np.stack([X, Y])[None]
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack([X, Y, Z])[None]


def stretched(n, length=1.0, beta=1.5, both=True):
    """Vertex positions clustered towards the ends with tanh stretching."""
    s = np.linspace(-1.0, 1.0, n + 1) if both else np.linspace(0.0, 1.0, n + 1)
    if both:
        v = np.tanh(beta * s) / np.tanh(beta)
        return (v + 1.0) * 0.5 * length
    v = 1.0 - np.tanh(beta * (1.0 - s)) / np.tanh(beta)
    return v * length


def rotate_distort(coords, angle=0.3):
    """Rotate vertices around the grid centre with a smooth radial falloff (a non-orthogonal grid)."""
    c = coords.copy()
    x, y = c[0, 0], c[0, 1]
    cx, cy = x.mean(), y.mean()
    r = np.sqrt((x - cx) ** 2 + (y - cy) ** 2)
    rmax = 0.45 * min(x.max() - x.min(), y.max() - y.min())
    w = np.where(r < rmax, np.sin(0.5 * np.pi * (1 - r / rmax)), 0.0) * angle
    dx, dy = x - cx, y - cy
    c[0, 0] = cx + np.cos(w) * dx - np.sin(w) * dy
    c[0, 1] = cy + np.sin(w) * dx + np.cos(w) * dy
    return c


def _rand_field(rng, shape, scale=1.0):
    return (rng.standard_normal(shape) * scale).astype(np.float64)


# ------------------------------------------------------------------ cases

def case(name, seed=0):
    rng = np.random.default_rng(seed)
    if name == "cavity2d":
        n = 12
        coords = tensor_grid(np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1))
        return dict(dims=2, viscosity=1e-2, blocks=[dict(coords=coords, velocity=_rand_field(rng, (1, 2, n, n), 0.2))],
                    ops=[("close_all", 0), ("close", 0, "-y", np.array([[1.0, 0.0]]))])
    if name == "cavity2d_refined":
        nx, ny = 10, 14
        coords = tensor_grid(stretched(nx, 1.0, 1.2), stretched(ny, 1.5, 1.6))
        return dict(dims=2, viscosity=5e-3, blocks=[dict(coords=coords, velocity=_rand_field(rng, (1, 2, ny, nx), 0.3))],
                    ops=[("close_all", 0), ("close", 0, "+y", np.array([[1.0, 0.0]]))])
    if name == "distorted2d":
        n = 12
        coords = rotate_distort(tensor_grid(np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1)), 0.35)
        return dict(dims=2, viscosity=1e-2, blocks=[dict(coords=coords, velocity=_rand_field(rng, (1, 2, n, n), 0.2))],
                    ops=[("close_all", 0), ("close", 0, "-y", np.array([[1.0, 0.0]]))])
    if name == "periodic2d":
        nx, ny = 9, 7
        visc = np.abs(_rand_field(rng, (1, 1, ny, nx), 1e-2)) + 1e-3
        return dict(dims=2, viscosity=1e-2,
                    blocks=[dict(size=[nx, ny], velocity=_rand_field(rng, (1, 2, ny, nx), 0.5), viscosity=visc,
                                 source=np.array([[0.3, -0.1]]))],
                    ops=[("periodic", 0, "x"), ("close", 0, "-y"), ("close", 0, "+y")])
    if name == "fullperiodic2d":
        n = 8
        coords = tensor_grid(np.linspace(0, 2, n + 1), np.linspace(0, 1, n + 1))
        return dict(dims=2, viscosity=2e-2,
                    blocks=[dict(coords=coords, velocity=_rand_field(rng, (1, 2, n, n), 0.5),
                                 source=_rand_field(rng, (1, 2, n, n), 0.1))],
                    ops=[])
    if name == "inflow2d":
        nx, ny = 12, 8
        coords = tensor_grid(np.linspace(0, 3, nx + 1), np.linspace(0, 1, ny + 1))
        inflow = np.zeros((1, 2, ny, 1))
        inflow[0, 0, :, 0] = 1.0 + 0.1 * rng.standard_normal(ny)
        outflow = np.zeros((1, 2, ny, 1))
        outflow[0, 0, :, 0] = inflow[0, 0].sum() / ny
        return dict(dims=2, viscosity=1e-2, blocks=[dict(coords=coords, velocity=_rand_field(rng, (1, 2, ny, nx), 0.2))],
                    ops=[("close_all", 0), ("close", 0, "-x", inflow), ("close", 0, "+x", outflow)])
    if name == "twoblock2d":
        ny, n1, n2 = 8, 6, 7
        c1 = tensor_grid(np.linspace(0, 1, n1 + 1), np.linspace(0, 1, ny + 1))
        c2 = tensor_grid(np.linspace(1, 2.5, n2 + 1), np.linspace(0, 1, ny + 1))
        return dict(dims=2, viscosity=1e-2,
                    blocks=[dict(coords=c1, velocity=_rand_field(rng, (1, 2, ny, n1), 0.3)),
                            dict(coords=c2, velocity=_rand_field(rng, (1, 2, ny, n2), 0.3))],
                    ops=[("close_all", 0), ("close_all", 1), ("connect", 0, "+x", 1, "-x", "-y"),
                         ("close", 0, "+y", np.array([[1.0, 0.0]]))])
    if name == "twoblock2d_rotated":
        # block 1's +x face joins block 2's +y face with the tangential axis inverted: exercises the
        # connected-face axis permutation and the flux sign flip (extensions/PISO_multiblock_cuda_kernel.cu:1589-1606)
        n = 7
        c1 = tensor_grid(np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1))
        c2 = tensor_grid(np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1))
        return dict(dims=2, viscosity=1e-2,
                    blocks=[dict(coords=c1, velocity=_rand_field(rng, (1, 2, n, n), 0.3)),
                            dict(coords=c2, velocity=_rand_field(rng, (1, 2, n, n), 0.3))],
                    ops=[("close_all", 0), ("close_all", 1), ("connect", 0, "+x", 1, "+y", "-x"),
                         ("close", 0, "-y", np.array([[1.0, 0.0]]))])
    if name == "channel3d":
        nx, ny, nz = 6, 5, 4
        coords = tensor_grid(np.linspace(0, 2, nx + 1), stretched(ny, 1.0, 1.5), np.linspace(0, 1, nz + 1))
        return dict(dims=3, viscosity=1e-2,
                    blocks=[dict(coords=coords, velocity=_rand_field(rng, (1, 3, nz, ny, nx), 0.3),
                                 source=np.array([[0.2, 0.0, 0.0]]))],
                    ops=[("periodic", 0, "x"), ("periodic", 0, "z"), ("close", 0, "-y"), ("close", 0, "+y")])
    if name == "cavity3d":
        n = 5
        coords = tensor_grid(np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1))
        return dict(dims=3, viscosity=1e-2, blocks=[dict(coords=coords, velocity=_rand_field(rng, (1, 3, n, n, n), 0.2))],
                    ops=[("close_all", 0), ("close", 0, "+y", np.array([[1.0, 0.0, 0.0]]))])
    if name == "twoblock3d":
        nx1, nx2, ny, nz = 4, 5, 4, 3
        c1 = tensor_grid(np.linspace(0, 1, nx1 + 1), np.linspace(0, 1, ny + 1), np.linspace(0, 1, nz + 1))
        c2 = tensor_grid(np.linspace(1, 2, nx2 + 1), np.linspace(0, 1, ny + 1), np.linspace(0, 1, nz + 1))
        return dict(dims=3, viscosity=1e-2,
                    blocks=[dict(coords=c1, velocity=_rand_field(rng, (1, 3, nz, ny, nx1), 0.3)),
                            dict(coords=c2, velocity=_rand_field(rng, (1, 3, nz, ny, nx2), 0.3))],
                    ops=[("close_all", 0), ("close_all", 1), ("connect", 0, "+x", 1, "-x", "-y", "-z"),
                         ("close", 0, "+y", np.array([[1.0, 0.0, 0.0]]))])
    if name == "ring4_2d":
        # flow around a cylinder on an O-grid cut into four quarter blocks that connect in a ring (x clockwise
        # around the cylinder, y radial, tanh-stretched towards the wall), no-slip on the cylinder and a
        # uniform stream u = (1, 0) prescribed on the outer circle
        na, nr = 6, 5
        radii = 0.5 + stretched(nr, 1.5, 1.4, both=False)
        blocks = []
        for q in range(4):
            th = np.linspace(np.pi / 2 * (4 - q), np.pi / 2 * (3 - q), na + 1)
            R, TH = np.meshgrid(radii, th, indexing="ij")
            coords = np.stack([R * np.cos(TH), R * np.sin(TH)])[None]
            blocks.append(dict(coords=coords, velocity=_rand_field(rng, (1, 2, nr, na), 0.2)))
        ops = [("close_all", q) for q in range(4)]
        ops += [("connect", q, "+x", (q + 1) % 4, "-x", "-y") for q in range(4)]
        ops += [("close", q, "+y", np.array([[1.0, 0.0]])) for q in range(4)]
        return dict(dims=2, viscosity=2e-2, blocks=blocks, ops=ops)
    if name == "skewed_channel2d":
        # periodic in x, walls at +-y, skew growing with y (non-orthogonal at the upper wall)
        nx, ny = 10, 8
        c = tensor_grid(np.linspace(0, 2, nx + 1), np.linspace(0, 1, ny + 1))
        c[0, 0] = c[0, 0] + 0.35 * c[0, 1] ** 2
        return dict(dims=2, viscosity=1e-2,
                    blocks=[dict(coords=c, velocity=_rand_field(rng, (1, 2, ny, nx), 0.3), source=np.array([[0.2, 0.0]]))],
                    ops=[("periodic", 0, "x"), ("close", 0, "-y"), ("close", 0, "+y")])
    if name == "skewed_periodic2d":
        # uniformly sheared, periodic in both axes
        nx, ny = 9, 8
        c = tensor_grid(np.linspace(0, 1, nx + 1), np.linspace(0, 1, ny + 1))
        c[0, 0] = c[0, 0] + 0.3 * c[0, 1]
        return dict(dims=2, viscosity=1e-2, blocks=[dict(coords=c, velocity=_rand_field(rng, (1, 2, ny, nx), 0.3))],
                    ops=[])
    if name == "skewed_inflow2d":
        # inflow face with data varying along it (tangential gradient of the boundary data)
        nx, ny = 12, 8
        c = tensor_grid(np.linspace(0, 3, nx + 1), np.linspace(0, 1, ny + 1))
        c[0, 0] = c[0, 0] + 0.25 * c[0, 1]
        inflow = np.zeros((1, 2, ny, 1))
        inflow[0, 0, :, 0] = 1.0 + 0.2 * np.sin(np.linspace(0, np.pi, ny))
        outflow = np.zeros((1, 2, ny, 1))
        outflow[0, 0, :, 0] = inflow[0, 0].sum() / ny
        return dict(dims=2, viscosity=1e-2, blocks=[dict(coords=c, velocity=_rand_field(rng, (1, 2, ny, nx), 0.2))],
                    ops=[("close_all", 0), ("close", 0, "-x", inflow), ("close", 0, "+x", outflow)])
    if name == "skewed_twoblock2d":
        ny, n1, n2 = 8, 6, 7
        c1 = tensor_grid(np.linspace(0, 1, n1 + 1), np.linspace(0, 1, ny + 1))
        c2 = tensor_grid(np.linspace(1, 2.5, n2 + 1), np.linspace(0, 1, ny + 1))
        c1[0, 1] = c1[0, 1] + 0.15 * np.sin(np.pi * c1[0, 0]) * c1[0, 1] * (1 - c1[0, 1]) * 4
        c2[0, 1] = c2[0, 1] + 0.15 * np.sin(np.pi * c2[0, 0] / 2.5) * c2[0, 1] * (1 - c2[0, 1]) * 4
        return dict(dims=2, viscosity=1e-2,
                    blocks=[dict(coords=c1, velocity=_rand_field(rng, (1, 2, ny, n1), 0.3)),
                            dict(coords=c2, velocity=_rand_field(rng, (1, 2, ny, n2), 0.3))],
                    ops=[("close_all", 0), ("close_all", 1), ("connect", 0, "+x", 1, "-x", "-y"),
                         ("close", 0, "+y", np.array([[1.0, 0.0]]))])
    if name == "skewed_twoblock2d_rotated":
        n = 7
        c1 = rotate_distort(tensor_grid(np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1)), 0.3)
        c2 = tensor_grid(np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1))
        c2[0, 0] = c2[0, 0] + 0.2 * c2[0, 1] * (1 - c2[0, 1])
        return dict(dims=2, viscosity=1e-2,
                    blocks=[dict(coords=c1, velocity=_rand_field(rng, (1, 2, n, n), 0.3)),
                            dict(coords=c2, velocity=_rand_field(rng, (1, 2, n, n), 0.3))],
                    ops=[("close_all", 0), ("close_all", 1), ("connect", 0, "+x", 1, "+y", "-x"),
                         ("close", 0, "-y", np.array([[1.0, 0.0]]))])
    if name == "skewed_cavity3d":
        n = 5
        c = tensor_grid(np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1), np.linspace(0, 1, n + 1))
        c[0, 0] = c[0, 0] + 0.2 * c[0, 1] * c[0, 2]
        c[0, 2] = c[0, 2] + 0.15 * c[0, 1] ** 2
        return dict(dims=3, viscosity=1e-2, blocks=[dict(coords=c, velocity=_rand_field(rng, (1, 3, n, n, n), 0.2))],
                    ops=[("close_all", 0), ("close", 0, "+y", np.array([[1.0, 0.0, 0.0]]))])
    if name == "skewed_channel3d":
        nx, ny, nz = 6, 5, 4
        c = tensor_grid(np.linspace(0, 2, nx + 1), stretched(ny, 1.0, 1.5), np.linspace(0, 1, nz + 1))
        c[0, 0] = c[0, 0] + 0.3 * c[0, 1]
        c[0, 2] = c[0, 2] + 0.2 * c[0, 1]
        return dict(dims=3, viscosity=1e-2,
                    blocks=[dict(coords=c, velocity=_rand_field(rng, (1, 3, nz, ny, nx), 0.3),
                                 source=np.array([[0.2, 0.0, 0.0]]))],
                    ops=[("periodic", 0, "x"), ("periodic", 0, "z"), ("close", 0, "-y"), ("close", 0, "+y")])
    raise KeyError(name)


# non-orthogonal grids for the nonOrthoFlags paths (operators pinned on all of them; full steps where the
# pressure solve converges)
NONORTHO_CASES = ["distorted2d", "skewed_channel2d", "skewed_periodic2d", "skewed_inflow2d", "skewed_twoblock2d",
                  "skewed_twoblock2d_rotated", "skewed_cavity3d", "skewed_channel3d"]
NONORTHO_FLAG_SETS = [25, 27, 19]

# passive scalar setups: channels, scalar viscosity, block scalars, Dirichlet and Neumann faces per channel,
# static and varying boundary scalars, orthogonal and skewed grids, two blocks, 2D and 3D
SCALAR_CASES = ["scalar_cavity2d", "scalar_inflow2d", "scalar_twoblock2d_rotated", "scalar_distorted2d",
                "scalar_channel3d", "scalar_skewed_cavity3d"]


def scalar_case(name, seed=0):
    rng = np.random.default_rng(100 + seed)

    def add(spec, C, sv, extra_ops):
        spec["scalar_channels"] = C
        spec["scalar_viscosity"] = sv
        for b in spec["blocks"]:
            zyx = np.asarray(b["velocity"]).shape[2:]
            b["scalar"] = rng.random((1, C) + tuple(zyx))
        spec["ops"] = list(spec["ops"]) + extra_ops
        return spec

    if name == "scalar_cavity2d":
        return add(case("cavity2d"), 2, [2e-2, 5e-3],
                   [("close", 0, "-y", np.array([[1.0, 0.0]]), np.array([[1.0, 0.5]])),
                    ("close", 0, "+x", None, np.array([[0.2, 0.3]]), ["dirichlet", "neumann"])])
    if name == "scalar_inflow2d":
        spec = case("inflow2d")
        ny = np.asarray(spec["blocks"][0]["velocity"]).shape[2]
        inflow = [op for op in spec["ops"] if op[0] == "close" and op[2] == "-x"][0][3]
        outflow = [op for op in spec["ops"] if op[0] == "close" and op[2] == "+x"][0][3]
        s_in = np.zeros((1, 1, ny, 1))
        s_in[0, 0, :, 0] = np.linspace(0.0, 1.0, ny)
        return add(spec, 1, None, [("close", 0, "-x", inflow, s_in),
                                   ("close", 0, "+x", outflow, np.array([[0.0]]), ["neumann"])])
    if name == "scalar_twoblock2d_rotated":
        return add(case("twoblock2d_rotated"), 2, [1e-2],
                   [("close", 0, "-y", np.array([[1.0, 0.0]]), np.array([[1.0, -1.0]])),
                    ("close", 1, "+x", None, np.array([[0.1, 0.0]]), ["neumann"])])
    if name == "scalar_distorted2d":
        return add(case("distorted2d"), 1, [1e-2],
                   [("close", 0, "-y", np.array([[1.0, 0.0]]), np.array([[1.0]])),
                    ("close", 0, "+y", None, np.array([[0.0]]), ["neumann"])])
    if name == "scalar_channel3d":
        return add(case("channel3d"), 1, None,
                   [("close", 0, "-y", None, np.array([[1.0]])),
                    ("close", 0, "+y", None, np.array([[0.5]]), ["neumann"])])
    if name == "scalar_skewed_cavity3d":
        return add(case("skewed_cavity3d"), 2, [1e-2, 2e-2],
                   [("close", 0, "+y", np.array([[1.0, 0.0, 0.0]]), np.array([[1.0, 0.0]])),
                    ("close", 0, "-x", None, np.array([[0.2, 0.4]]), ["neumann", "dirichlet"])])
    raise KeyError(name)


CASES_2D = ["cavity2d", "cavity2d_refined", "distorted2d", "periodic2d", "fullperiodic2d", "inflow2d", "twoblock2d",
            "twoblock2d_rotated", "ring4_2d"]
CASES_3D = ["channel3d", "cavity3d", "twoblock3d"]
ALL_CASES = CASES_2D + CASES_3D


def lid_cavity(n, viscosity=1e-3, lid=1.0, dims=2):
    """The reference's minimal lid-driven cavity (minimal_lid_sample.py:33-66): uniform n^D vertex grid on [0,1]^D,
    all walls closed, lid velocity on -y."""
    xs = np.linspace(0, 1, n + 1)
    if dims == 2:
        coords = tensor_grid(xs, xs)
        lidv = np.array([[lid, 0.0]])
    else:
        coords = tensor_grid(xs, xs, xs)
        lidv = np.array([[lid, 0.0, 0.0]])
    return dict(dims=dims, viscosity=viscosity, blocks=[dict(coords=coords)],
                ops=[("close_all", 0), ("close", 0, "-y", lidv)])


def spectral_field(n, seed, kmax=8, dims=2):
    """Seeded Gaussian random vector field on an n^2 periodic grid with energy spectrum ~ k^-3 for
    1 <= |k| <= kmax (amplitude ~ k^-1.5), each component scaled to max |.| = 1: [1, 2, n, n]."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(n, 1.0 / n)
    KX, KY = np.meshgrid(kx, kx, indexing="xy")
    k = np.sqrt(KX ** 2 + KY ** 2)
    amp = np.where((k > 0) & (k <= kmax), np.power(np.maximum(k, 1e-9), -1.5), 0.0)
    comps = []
    for _ in range(dims):
        coef = amp * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
        f = np.real(np.fft.ifft2(coef))
        comps.append(f / np.abs(f).max())
    return np.stack(comps)[None]


def forcing_box(n=128, viscosity=1e-3, seed=3):
    """Periodic unit box (cell size 1/n) with a smooth random initial velocity and a zero per-cell
    velocity source: the differentiable forcing setup."""
    xs = np.linspace(0, 1, n + 1)
    return dict(dims=2, viscosity=viscosity,
                blocks=[dict(coords=tensor_grid(xs, xs), velocity=spectral_field(n, seed),
                             source=np.zeros((1, 2, n, n)))],
                ops=[])


# ------------------------------------------------------------------ builders

def build_oracle(spec) -> po.ODomain:
    d = po.ODomain(spec["dims"], spec["viscosity"], spec.get("scalar_channels", 0), spec.get("scalar_viscosity"))
    for b in spec["blocks"]:
        bi = d.create_block(size=b.get("size"), velocity=b.get("velocity"), pressure=b.get("pressure"),
                            coords=b.get("coords"))
        ob = d.blocks[bi]
        if d.scalar_channels:
            zyx = ob.velocity.shape[2:]
            ob.scalar = np.zeros((1, d.scalar_channels) + zyx) if b.get("scalar") is None else \
                np.asarray(b["scalar"], dtype=np.float64)
        if b.get("viscosity") is not None:
            ob.viscosity = np.asarray(b["viscosity"], dtype=np.float64)
        if b.get("source") is not None:
            ob.source = np.asarray(b["source"], dtype=np.float64)
    for op in spec["ops"]:
        if op[0] == "close_all":
            d.close_all(op[1])
        elif op[0] == "close":
            d.close_boundary(op[1], op[2], None if len(op) < 4 else op[3], None if len(op) < 5 else op[4],
                             None if len(op) < 6 else op[5])
        elif op[0] == "periodic":
            d.make_periodic(op[1], op[2])
        elif op[0] == "connect":
            d.connect(op[1], op[2], op[3], op[4], *op[5:])
        else:
            raise KeyError(op[0])
    d.prepare()
    return d


def build_product(spec, dtype=None, device="cuda", module=None, prepare=True):
    """Build through the PISOtorch API of `module` (default: pict_b200.PISOtorch; the reference's own
    compiled module has the same API and is used by tests/golden/make_ref_fixtures.py)."""
    import torch
    if module is None:
        from pict_b200 import PISOtorch
    else:
        PISOtorch = module
    dtype = torch.float64 if dtype is None else dtype
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=dtype, device=device).contiguous()
    C = spec.get("scalar_channels", 0)
    sv = spec.get("scalar_viscosity")
    dom = PISOtorch.Domain(spec["dims"], torch.tensor([spec["viscosity"]], dtype=dtype), name="test", dtype=dtype,
                           device=torch.device(device), passiveScalarChannels=C,
                           scalarViscosity=None if sv is None else t(np.asarray(sv, dtype=np.float64).reshape(-1)))
    blocks = []
    for b in spec["blocks"]:
        kw = {}
        if b.get("velocity") is not None:
            kw["velocity"] = t(b["velocity"])
        if C and b.get("scalar") is not None:
            kw["passiveScalar"] = t(b["scalar"])
        if b.get("coords") is not None:
            kw["vertexCoordinates"] = t(b["coords"])
        if not kw:
            size = list(b["size"]) + [1] * (3 - len(b["size"]))
            blk = dom.CreateBlockWithSize(PISOtorch.Int4(size[0], size[1], size[2], spec["dims"]), name="block")
        else:
            blk = dom.CreateBlock(name="block", **kw)
        if b.get("viscosity") is not None:
            blk.setViscosity(t(b["viscosity"]))
        if b.get("source") is not None:
            blk.setVelocitySource(t(b["source"]))
        blocks.append(blk)
    for op in spec["ops"]:
        if op[0] == "close_all":
            blocks[op[1]].CloseAllBoundaries()
        elif op[0] == "close":
            vel = None if len(op) < 4 or op[3] is None else t(op[3])
            if len(op) >= 5 and op[4] is not None:
                blocks[op[1]].CloseBoundary(op[2], vel, t(op[4]))
            else:
                blocks[op[1]].CloseBoundary(op[2], vel)
            if len(op) >= 6 and op[5] is not None:
                bct = PISOtorch.BoundaryConditionType
                types = [bct.NEUMANN if x == "neumann" else bct.DIRICHLET for x in op[5]]
                blocks[op[1]].getBoundary(po.face_index(op[2])).setPassiveScalarType(types if len(types) > 1 else types[0])
        elif op[0] == "periodic":
            blocks[op[1]].MakePeriodic(op[2])
        elif op[0] == "connect":
            blocks[op[1]].ConnectBlock(op[2], blocks[op[3]], op[4], *op[5:])
        else:
            raise KeyError(op[0])
    if prepare:
        dom.PrepareSolve()
    return dom


# ------------------------------------------------------------------ multi-block CNN structures

MBCNN_CASES = ["grid2x2_2d", "rotated_chain2d", "periodic_layers2d", "swapped3d", "chain1d"]
# 3D layouts whose connections cycle all three axes (the reference's MultiblockConv cannot pad these)
MBCNN_CYCLE_CASES = ["rotated3d"]


def mbcnn_case(name):
    """Block layouts for the multi-block convolution: sizes and boundary operations only (fields zero)."""
    def spec(dims, sizes, ops):
        return dict(dims=dims, viscosity=1e-3, blocks=[dict(size=s) for s in sizes], ops=ops)

    if name == "grid2x2_2d":
        return spec(2, [[6, 5], [4, 5], [6, 7], [4, 7]],
                    [("close_all", b) for b in range(4)] +
                    [("connect", 0, "+x", 1, "-x", "-y"), ("connect", 0, "+y", 2, "-y", "-x"),
                     ("connect", 1, "+y", 3, "-y", "-x"), ("connect", 2, "+x", 3, "-x", "-y")])
    if name == "rotated_chain2d":
        # +x of block 0 meets +y of block 1 with the axis inverted; -x of block 1 meets -y of block 2
        return spec(2, [[5, 6], [6, 4], [7, 4]],
                    [("close_all", b) for b in range(3)] +
                    [("connect", 0, "+x", 1, "+y", "+x"), ("connect", 1, "-x", 2, "+x", "-y")])
    if name == "periodic_layers2d":
        return spec(2, [[8, 4], [8, 5]],
                    [("periodic", 0, "x"), ("periodic", 1, "x"), ("close", 0, "-y"), ("close", 1, "+y"),
                     ("connect", 0, "+y", 1, "-y", "-x")])
    if name == "swapped3d":
        # +x of block 0 meets -z of block 1 with x and z swapped; +y of block 0 meets -y of block 2 with z inverted
        return spec(3, [[4, 5, 6], [6, 5, 3], [4, 3, 6]],
                    [("close_all", b) for b in range(3)] +
                    [("connect", 0, "+x", 1, "-z", "-y", "-x"), ("connect", 0, "+y", 2, "-y", "+z", "-x"),
                     ("periodic", 2, "z")])
    if name == "rotated3d":
        # +x of block 0 meets -y of block 1 with the axes cycled (y -> z inverted, z -> x)
        return spec(3, [[4, 5, 6], [6, 4, 5], [4, 4, 6]],
                    [("close_all", b) for b in range(3)] +
                    [("connect", 0, "+x", 1, "-y", "+z", "-x"), ("connect", 0, "+y", 2, "-y", "-z", "-x"),
                     ("periodic", 2, "z")])
    if name == "chain1d":
        return spec(1, [[6], [5], [7]],
                    [("close_all", b) for b in range(3)] +
                    [("connect", 0, "+x", 1, "-x"), ("connect", 1, "+x", 2, "-x"), ("connect", 2, "+x", 0, "-x")])
    raise KeyError(name)


class _StandInSizes:
    def __init__(self, size):
        s = list(size) + [1] * (3 - len(size))
        self.x, self.y, self.z, self.w = s[0], s[1], s[2], s[0] * s[1] * s[2]

    def __getitem__(self, i):
        return [self.x, self.y, self.z, self.w][i]


class _StandInBoundary:
    def __init__(self, btype, block=None, axes=None):
        self.type = btype
        self._block = block
        self.axes = axes

    def getConnectedBlock(self):
        return self._block


class _StandInBlock:
    def __init__(self, dims, size):
        self._dims = dims
        self._sizes = _StandInSizes(size)
        self.boundaries = []

    def getSpatialDims(self):
        return self._dims

    def getSizes(self):
        return self._sizes

    def getBoundaries(self):
        return list(self.boundaries)


class _StandInDomain:
    def __init__(self, dims, blocks):
        self._dims = dims
        self._blocks = blocks

    def getSpatialDims(self):
        return self._dims

    def getBlocks(self):
        return list(self._blocks)


def build_structure(spec, boundary_type):
    """Host-only object graph with the domain accessors a multi-block convolution reads (block sizes, boundary
    types, connected blocks and axes), built from the oracle's domain so that connection axes are those of
    ConnectBlock.  ``boundary_type`` is the BoundaryType enum whose FIXED / CONNECTED / PERIODIC tag the faces."""
    od = build_oracle(spec)
    blocks = [_StandInBlock(spec["dims"], ob.size) for ob in od.blocks]
    for blk, ob in zip(blocks, od.blocks):
        for bnd in ob.boundaries:
            if bnd.kind == "fixed":
                blk.boundaries.append(_StandInBoundary(boundary_type.FIXED))
            elif bnd.kind == "connected":
                blk.boundaries.append(_StandInBoundary(boundary_type.CONNECTED, blocks[bnd.block], list(bnd.axes)))
            else:
                blk.boundaries.append(_StandInBoundary(boundary_type.PERIODIC))
    return _StandInDomain(spec["dims"], blocks)
