"""The 2D cylinder vortex street: a unit-diameter cylinder in a 30 x 8 channel at Re 200.

Layout (all connections whole faces, as the PISOtorch block model requires):

* an O-grid around the cylinder (radius 0.5, centre at the origin) of four curvilinear quadrant
  blocks, ``n_ang`` angular x ``n_rad`` radial cells each (64 x 64: 256 angular x 64 radial in total),
  split on the diagonals so that each quadrant's outer face is one side of the square
  [-H, H]^2 (H = 4, the channel's half height); the angular index runs clockwise and the radial one
  outwards, vertices lie on rays from the centre, radially tanh-stretched towards the cylinder;
  the quadrants are connected in a ring;
* Cartesian far-field blocks with the quadrants' vertex rows at x = -H / x = H: one upstream block
  on [-8, -H] and ``n_wake`` blocks on [H, 22], uniform spacing ``dx`` in x;
* the top and bottom quadrants' outer faces and the far-field blocks' y faces are the channel
  walls, moving with the free stream (Dirichlet u = (1, 0)); the cylinder is a no-slip wall;
* inflow at x = -8: u = 1 + U(-0.01, 0.01) per face cell (seeded), v = 0;
* outflow at x = 22: a varying Dirichlet face updated every step by the advective outflow
  condition (``update_advective_boundaries`` with the characteristic velocity (1, 0)), its flux
  balanced against the inflow.

``make_cylinder_street`` builds the domain through the ``PISOtorch`` API of a module argument (this
package's by default; the reference's compiled module has the same API), so the same function
builds the domain for this package's step and for the reference's.

Why quadrants and not one ring block: a ring block that is periodic in its angular axis has one
closed outer face, and a face connects to exactly one face of one other block, which would then
have to be a ring as well; Cartesian far-field blocks can only meet an O-grid whose outer boundary
is cut into separate faces.
"""
from __future__ import annotations

import math

import numpy as np
import torch

X_IN, X_OUT, HALF_HEIGHT, RADIUS = -8.0, 22.0, 4.0, 0.5
VISCOSITY = 5e-3  # Re = U D / nu = 200
TIME_STEP = 0.005
INFLOW_SEED = 1


def radial_weights(n_rad, beta=2.0):
    """Radial vertex parameter in [0, 1], tanh-clustered towards 0 (the cylinder wall)."""
    s = np.arange(n_rad + 1, dtype=np.float64) / n_rad
    return 1.0 + np.tanh(beta * (s - 1.0)) / np.tanh(beta)


def quadrant_coords(k, n_ang, n_rad, beta=2.0, radius=RADIUS, half=HALF_HEIGHT):
    """Vertex coordinates [1, 2, n_rad+1, n_ang+1] of quadrant k (0: top, 1: right / downstream,
    2: bottom, 3: left / upstream); angles run clockwise from 135 - 90 k degrees."""
    theta0 = math.radians(135.0 - 90.0 * k)
    th = theta0 - np.arange(n_ang + 1, dtype=np.float64) * (0.5 * math.pi / n_ang)
    c, s = np.cos(th), np.sin(th)
    r_out = half / np.maximum(np.abs(c), np.abs(s))
    w = radial_weights(n_rad, beta)[:, None]
    r = radius + w * (r_out - radius)[None, :]
    xy = np.stack([r * c[None, :], r * s[None, :]])
    # exact square sides and corners on the outer row (rays hit them only up to rounding)
    if k in (0, 2):
        xy[1, -1, :] = half if k == 0 else -half
    else:
        xy[0, -1, :] = half if k == 1 else -half
    return xy[None]


def side_vertices(n_ang, beta=2.0):
    """y of the quadrant vertices on the square sides x = +-H, increasing from -H to H."""
    q = quadrant_coords(3, n_ang, 4, beta)  # left quadrant: outer row runs from (-H,-H) up to (-H,H)
    y = q[0, 1, -1, :].copy()
    y[0], y[-1] = -HALF_HEIGHT, HALF_HEIGHT
    return y


def cartesian_coords(xs, ys):
    Y, X = np.meshgrid(ys, xs, indexing="ij")
    return np.stack([X, Y])[None]


def street_layout(n_ang=64, n_rad=64, dx=0.125, n_wake=3, beta=2.0):
    """Block vertex coordinates and names: four quadrants, the upstream block, the wake blocks."""
    coords = [quadrant_coords(k, n_ang, n_rad, beta) for k in range(4)]
    names = ["QuadrantTop", "QuadrantDownstream", "QuadrantBottom", "QuadrantUpstream"]
    ys = side_vertices(n_ang, beta)
    n_up = int(round((-HALF_HEIGHT - X_IN) / dx))
    coords.append(cartesian_coords(np.linspace(X_IN, -HALF_HEIGHT, n_up + 1), ys))
    names.append("Upstream")
    wake_len = (X_OUT - HALF_HEIGHT) / n_wake
    n_w = int(round(wake_len / dx))
    for w in range(n_wake):
        x0 = HALF_HEIGHT + w * wake_len
        xs = np.linspace(x0, x0 + wake_len, n_w + 1)
        if w == n_wake - 1:
            xs[-1] = X_OUT
        coords.append(cartesian_coords(xs, ys))
        names.append("Wake%d" % w)
    return coords, names


def inflow_profile(n_cells, seed=INFLOW_SEED, amplitude=0.01):
    """Inflow u per face cell: 1 + U(-amplitude, amplitude), seeded."""
    g = torch.Generator().manual_seed(seed)
    return 1.0 + amplitude * (2.0 * torch.rand(n_cells, generator=g, dtype=torch.float64) - 1.0)


def street_spec(n_ang=64, n_rad=64, dx=0.125, n_wake=3, viscosity=VISCOSITY, beta=2.0, inflow_seed=INFLOW_SEED):
    """Plain description of the domain: {"dims", "viscosity", "blocks": [{"coords", "velocity", "name"}],
    "ops": [("close_all", b) | ("connect", b, face, other, other_face, axis) | ("close", b, face, velocity)],
    "outflow", "cylinder", "char_vel"}; arrays are float64 numpy.  The blocks start at the free stream."""
    coords, names = street_layout(n_ang, n_rad, dx, n_wake, beta)
    blocks = []
    for c, n in zip(coords, names):
        v = np.zeros((1, 2, c.shape[2] - 1, c.shape[3] - 1))
        v[:, 0] = 1.0
        blocks.append({"coords": c, "velocity": v, "name": n})
    nb = len(blocks)
    ops = [("close_all", b) for b in range(nb)]
    ops += [("connect", k, "+x", (k + 1) % 4, "-x", "-y") for k in range(4)]
    ops.append(("connect", 4, "+x", 3, "+y", "-x"))
    ops.append(("connect", 5, "-x", 1, "+y", "+x"))
    ops += [("connect", b, "+x", b + 1, "-x", "-y") for b in range(5, nb - 1)]
    free_stream = np.array([[1.0, 0.0]])
    for b, f in [(0, "+y"), (2, "+y")] + [(b, f) for b in range(4, nb) for f in ("-y", "+y")]:
        ops.append(("close", b, f, free_stream))
    ny = coords[4].shape[2] - 1
    inflow = np.zeros((1, 2, ny, 1))
    inflow[0, 0, :, 0] = inflow_profile(ny, inflow_seed).numpy()
    ops.append(("close", 4, "-x", inflow))
    outflow = np.zeros((1, 2, ny, 1))
    outflow[0, 0] = 1.0
    ops.append(("close", nb - 1, "+x", outflow))
    return {"dims": 2, "viscosity": viscosity, "blocks": blocks, "ops": ops, "outflow": [(nb - 1, 1)],
            "cylinder": [(k, 2) for k in range(4)], "char_vel": free_stream, "layout": names}


def build_street(spec, module=None, dtype=torch.float32, device="cuda", prepare=True):
    """Build `spec` (street_spec) through the PISOtorch API of `module` (default: this package's).
    Returns (domain, info) with info = {"outflow": [(block, face)], "cylinder": [(block, face)],
    "char_vel": [1,2] tensor on the device, "layout": block names}."""
    if module is None:
        from . import PISOtorch as module
    dev = torch.device(device)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=dtype, device=dev).contiguous()
    dom = module.Domain(spec["dims"], torch.tensor([spec["viscosity"]], dtype=dtype), name="CylinderStreet",
                        dtype=dtype, device=dev, passiveScalarChannels=0)
    blocks = [dom.CreateBlock(velocity=t(b["velocity"]), vertexCoordinates=t(b["coords"]), name=b["name"])
              for b in spec["blocks"]]
    for op in spec["ops"]:
        if op[0] == "close_all":
            blocks[op[1]].CloseAllBoundaries()
        elif op[0] == "connect":
            blocks[op[1]].ConnectBlock(op[2], blocks[op[3]], op[4], *op[5:])
        elif op[0] == "close":
            blocks[op[1]].CloseBoundary(op[2], t(op[3]))
        else:
            raise KeyError(op[0])
    if prepare:
        dom.PrepareSolve()
    info = {k: spec[k] for k in ("outflow", "cylinder", "layout")}
    info["char_vel"] = t(spec["char_vel"])
    return dom, info


def make_cylinder_street(module=None, dtype=torch.float32, device="cuda", prepare=True, **kwargs):
    """street_spec(**kwargs) built through `module`; see build_street."""
    return build_street(street_spec(**kwargs), module, dtype, device, prepare)


def outflow_bounds(domain, info):
    return [domain.getBlock(b).getBoundary(f) for b, f in info["outflow"]]


def street_prep_fn(info):
    """prep_fn for Simulation: the advective outflow update before every step, as the reference's
    vortex-street samples pass it (``{"PRE": fn}``)."""
    from .PISOtorch_simulation import update_advective_boundaries

    def prep(domain, time_step, **kwargs):
        update_advective_boundaries(domain, outflow_bounds(domain, info), info["char_vel"].to(domain.getDevice()),
                                    time_step.to(domain.getDevice()))
    return {"PRE": prep}


def cylinder_forces(domain, info, viscosity=VISCOSITY):
    """Force on the cylinder (per unit depth) from the block fields: pressure of the wall cell times the
    face normal, plus the viscous wall shear nu (u_cell - u_wall) / d over each wall face (u_wall = 0),
    d the distance of the cell centre from the face.  Returns (F_x, F_y) as floats; with U = D = 1 the
    drag and lift coefficients are 2 F_x and 2 F_y."""
    fx = fy = 0.0
    for bi, face in info["cylinder"]:
        b = domain.getBlock(bi)
        xy = b.vertexCoordinates.detach().double().cpu()[0]  # [2, ny+1, nx+1]
        u = b.velocity.detach().double().cpu()[0]  # [2, ny, nx]
        p = b.pressure.detach().double().cpu()[0, 0]
        assert face == 2
        v0 = xy[:, 0, :]  # wall vertices
        e = v0[:, 1:] - v0[:, :-1]  # face edge vectors along x
        length = torch.sqrt((e ** 2).sum(0))
        centre = 0.25 * (xy[:, 0, :-1] + xy[:, 0, 1:] + xy[:, 1, :-1] + xy[:, 1, 1:])
        mid = 0.5 * (v0[:, 1:] + v0[:, :-1])
        # outward normal of the fluid at the wall points into the cylinder: from the cell towards the face
        n = torch.stack([e[1], -e[0]]) / length
        s = ((mid - centre) * n).sum(0)
        n = n * torch.sign(s)
        d = ((mid - centre) * n).sum(0).abs()
        pw = p[0, :]
        uw = u[:, 0, :]
        # pressure pushes along the normal into the body; shear drags along the wall tangential velocity
        fpx, fpy = (pw * n[0] * length).sum(), (pw * n[1] * length).sum()
        un = (uw * n).sum(0)
        ut = uw - un * n
        fvx, fvy = (viscosity * ut[0] / d * length).sum(), (viscosity * ut[1] / d * length).sum()
        fx += float(fpx + fvx)
        fy += float(fpy + fvy)
    return fx, fy


def strouhal(lift, dt, every=1, skip=0.5):
    """Shedding frequency f D / U from the upward zero crossings of the lift series sampled every
    `every` steps of length dt, over its last (1 - skip) part; None with fewer than two periods."""
    y = np.asarray(lift, dtype=np.float64)
    y = y[int(len(y) * skip):]
    if len(y) < 4:
        return None
    y = y - y.mean()
    idx = np.nonzero((y[:-1] < 0) & (y[1:] >= 0))[0]
    if len(idx) < 3:
        return None
    # sub-sample position of each crossing
    tc = idx + (-y[idx]) / (y[idx + 1] - y[idx])
    period = np.mean(np.diff(tc)) * every * dt
    return 1.0 / period
