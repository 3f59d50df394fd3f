"""Multi-block convolution (pict_b200.multiblock_cnn, for lib/modules/multiblock_cnn.py).

* against fixtures computed by the reference's own ``MultiblockConv`` on the same layouts, inputs and
  weights (``tests/golden/make_ref_multiblock_cnn_fixtures.py``): outputs, input and weight gradients in FP64;
* the padding cells against the solver's topology: a cell ``o`` layers beyond a connected face is the cell
  the oracle's ``_conn_pos`` (computeConnectedPos) addresses, beyond a periodic face the wrapped cell, beyond
  a fixed face zero; edge regions follow the reference's walk order (lower axis first, the other path where
  that one ends at a fixed face).  This also covers the 3D layout whose connections cycle all three axes.
"""
import itertools
import os

import numpy as np
import pytest
import torch

import setups
import piso_oracle as po
from pict_b200 import PISOtorch as P
from pict_b200.multiblock_cnn import MultiblockConv, MultiblockConv_naive, MultiblockReLU

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = [(name, k) for name in setups.MBCNN_CASES for k in (3, 5)]


def _load(name, k):
    with np.load(os.path.join(GOLDEN, "ref_mbcnn_%s_k%d.npz" % (name, k))) as z:
        return {key: z[key] for key in z.files}


def _conv_from_fixture(domain, k, f, device="cpu"):
    conv = MultiblockConv(domain, "ZERO", f["weight"].shape[1], f["weight"].shape[0], k, dtype=torch.float64,
                          device=device)
    with torch.no_grad():
        conv.conv_layer.weight.copy_(torch.tensor(f["weight"]))
        conv.conv_layer.bias.copy_(torch.tensor(f["bias"]))
    return conv


def run_against_fixture(domain, name, k, device):
    f = _load(name, k)
    nb = int(f["num_blocks"])
    conv = _conv_from_fixture(domain, k, f, device)
    inputs = [torch.tensor(f["input_%d" % b], device=device, requires_grad=True) for b in range(nb)]
    out = conv(inputs, domain)
    loss = sum((o * torch.tensor(f["out_grad_%d" % b], device=device)).sum() for b, o in enumerate(out))
    loss.backward()
    for b in range(nb):
        np.testing.assert_allclose(out[b].detach().cpu().numpy(), f["output_%d" % b], rtol=0, atol=1e-12)
        np.testing.assert_allclose(inputs[b].grad.cpu().numpy(), f["input_grad_%d" % b], rtol=0, atol=1e-12)
    np.testing.assert_allclose(conv.conv_layer.weight.grad.cpu().numpy(), f["weight_grad"], rtol=0, atol=1e-10)


@pytest.mark.parametrize("name,k", FIXTURES)
def test_matches_reference_fixture(name, k):
    domain = setups.build_structure(setups.mbcnn_case(name), P.BoundaryType)
    run_against_fixture(domain, name, k, "cpu")


def _step(od, bi, q, axis):
    """Resolve the out-of-range coordinate ``axis`` of ``q`` through the face it leaves by: (block, q) or None."""
    b = od.blocks[bi]
    up = q[axis] >= b.size[axis]
    face = 2 * axis + int(up)
    bnd = b.boundaries[face]
    if bnd.kind == "fixed":
        return None
    if bnd.kind == "periodic":
        r = list(q)
        r[axis] %= b.size[axis]
        return bi, r
    offset = q[axis] - b.size[axis] if up else -1 - q[axis]
    nb, r = po._conn_pos(od, bi, face, list(q) + [0] * (3 - len(q)), offset)
    # the tangential coordinates map linearly, so out-of-range ones stay out of range in the neighbour's frame
    return nb, r[:od.dims]


def _resolve(od, bi, q):
    """The cell a padding position of block ``bi`` shows, following the walk: out-of-range axes in increasing
    order first, the reverse order for two axes where the first path ends at a fixed face."""
    out = [a for a in range(od.dims) if not 0 <= q[a] < od.blocks[bi].size[a]]
    assert len(out) <= 2
    for order in ([out] if len(out) < 2 else [out, out[::-1]]):
        cb, cq, ok = bi, list(q), True
        for _ in order:
            oob = [a for a in range(od.dims) if not 0 <= cq[a] < od.blocks[cb].size[a]]
            # the original axis order[i] is, in the current block's frame, the out-of-range axis reached by the path
            a = oob[0] if len(oob) == 1 else None
            if a is None:
                # two out of range: pick the one the current original axis maps to
                a = _mapped_axis(od, bi, q, cb, cq, order[len(order) - len(oob)])
            step = _step(od, cb, cq, a)
            if step is None:
                ok = False
                break
            cb, cq = step
        if ok:
            return cb, cq
    return None


def _mapped_axis(od, bi, q, cb, cq, orig_axis):
    if cb == bi:
        return orig_axis
    # probe: move the original position one cell further along orig_axis and see which coordinate moves
    q2 = list(q)
    q2[orig_axis] += 1 if q[orig_axis] >= 0 else -1
    b = od.blocks[bi]
    first = [a for a in range(od.dims) if not 0 <= q[a] < b.size[a] and a != orig_axis][0]
    step2 = _step(od, bi, q2, first)
    diff = [a for a in range(od.dims) if step2[1][a] != cq[a]]
    assert len(diff) == 1
    return diff[0]


@pytest.mark.parametrize("name", setups.MBCNN_CASES + setups.MBCNN_CYCLE_CASES)
@pytest.mark.parametrize("k", [3, 5])
def test_padding_follows_topology(name, k):
    spec = setups.mbcnn_case(name)
    od = setups.build_oracle(spec)
    domain = setups.build_structure(spec, P.BoundaryType)
    conv = MultiblockConv(domain, "ZERO", 1, 1, k, dtype=torch.float64)
    pad = k // 2
    dims = spec["dims"]
    ids = [torch.arange(1, 1 + int(np.prod(b.size)), dtype=torch.float64).reshape([1, 1] + list(reversed(b.size)))
           + od.offsets[i] for i, b in enumerate(od.blocks)]
    padded = conv.pad(ids)
    checked = 0
    for bi, b in enumerate(od.blocks):
        ranges = [range(-pad, s + pad) for s in b.size]
        P_ = padded[bi][0, 0].numpy()
        for q in itertools.product(*ranges):
            nout = sum(1 for a in range(dims) if not 0 <= q[a] < b.size[a])
            if nout == 0 or nout > 2:
                continue
            got = P_[tuple(q[a] + pad for a in reversed(range(dims)))]
            res = _resolve(od, bi, list(q))
            want = 0.0 if res is None else 1.0 + po._gidx(od, res[0], list(res[1]) + [0] * (3 - dims))
            assert got == want, (bi, q, got, want)
            checked += 1
    assert checked > 0


def test_cycle_layout_shapes():
    """On the 3-axis cycle layout every block is padded to its own size plus the padding on each side."""
    spec = setups.mbcnn_case("rotated3d")
    domain = setups.build_structure(spec, P.BoundaryType)
    conv = MultiblockConv(domain, "ZERO", 2, 3, 3, dtype=torch.float64)
    xs = [torch.randn([1, 2] + list(reversed(b["size"])), dtype=torch.float64) for b in spec["blocks"]]
    out = conv(xs, domain)
    assert [list(o.shape[2:]) for o in out] == [list(reversed(b["size"])) for b in spec["blocks"]]


def test_argument_checks():
    domain = setups.build_structure(setups.mbcnn_case("grid2x2_2d"), P.BoundaryType)
    with pytest.raises(NotImplementedError):
        MultiblockConv(domain, "ZERO", 1, 1, 4)
    with pytest.raises(NotImplementedError):
        MultiblockConv(domain, "ZERO", 1, 1, 3, dilation=2)
    with pytest.raises(ValueError):
        MultiblockConv(domain, ["ZERO"], 2, 1, 3)
    conv = MultiblockConv(domain, ["VEL_U", "S"], 2, 1, 3, dtype=torch.float64)
    shapes = [list(reversed(s["size"])) for s in setups.mbcnn_case("grid2x2_2d")["blocks"]]
    good = [torch.zeros([1, 2] + s, dtype=torch.float64) for s in shapes]
    with pytest.raises(ValueError):
        conv(good[:3], domain)
    with pytest.raises(ValueError):
        conv([torch.zeros([1, 3] + s, dtype=torch.float64) for s in shapes], domain)
    with pytest.raises(ValueError):
        conv([torch.zeros([1, 2] + s[::-1], dtype=torch.float64) for s in shapes], domain)
    assert len(conv(good, domain)) == 4


def test_naive_and_relu():
    naive = MultiblockConv_naive(2, 2, 3, 3, padding=1, dtype=torch.float64)
    xs = [torch.randn(1, 2, 5, 6, dtype=torch.float64), torch.randn(1, 2, 4, 4, dtype=torch.float64)]
    out = naive(xs)
    for x, o in zip(xs, out):
        torch.testing.assert_close(o, naive.conv_layer(x))
    r = MultiblockReLU()(out)
    for o, ro in zip(out, r):
        torch.testing.assert_close(ro, torch.relu(o))
