"""Multi-block convolution on CUDA tensors over domains built through the PISOtorch API, against the
reference's own ``MultiblockConv`` outputs and gradients (tests/golden/ref_mbcnn_*.npz)."""
import pytest
import torch

import setups
from test_multiblock_cnn import run_against_fixture, FIXTURES
from pict_b200.multiblock_cnn import MultiblockConv

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,k", FIXTURES)
def test_domain_matches_reference_fixture(name, k):
    domain = setups.build_product(setups.mbcnn_case(name), dtype=torch.float64, prepare=False)
    run_against_fixture(domain, name, k, "cuda")


def test_velocity_fields_through_layers():
    """A small multi-block network over a domain's block velocities: shapes per block, gradients reach every block."""
    spec = setups.mbcnn_case("grid2x2_2d")
    domain = setups.build_product(spec, dtype=torch.float32, prepare=False)
    net = torch.nn.ModuleList([MultiblockConv(domain, "ZERO", 2, 8, 3, device="cuda"),
                               MultiblockConv(domain, "ZERO", 8, 2, 5, device="cuda")])
    xs = [torch.randn_like(b.velocity).requires_grad_(True) for b in domain.getBlocks()]
    h = net[0](xs, domain)
    h = [torch.relu(t) for t in h]
    out = net[1](h, domain)
    assert [o.shape for o in out] == [x.shape for x in xs]
    sum(o.square().sum() for o in out).backward()
    assert all(x.grad is not None and torch.isfinite(x.grad).all() and x.grad.abs().sum() > 0 for x in xs)


@pytest.mark.parametrize("name", setups.MBCNN_CASES + setups.MBCNN_CYCLE_CASES)
@pytest.mark.parametrize("k", [3, 5])
def test_padding_kernels_equal_the_index_map(name, k):
    """The library's padding launch (pict_mb_pad_gather) equals the index map applied with index_select on
    CPU tensors, bitwise; its gradient (pict_mb_pad_scatter_sum, a fixed-order gather-sum) equals the
    index_add gradient of the CPU path to round-off."""
    from pict_b200 import _lib
    domain = setups.build_product(setups.mbcnn_case(name), dtype=torch.float64, prepare=False)
    layer = MultiblockConv(domain, "ZERO", 3, 2, k)
    g = torch.Generator().manual_seed(7)
    xs = [torch.randn([2, 3] + list(b.velocity.shape[2:]), generator=g, dtype=torch.float64) for b in domain.getBlocks()]
    ws = None
    grads = []
    outs = []
    for dev in ("cpu", "cuda"):
        layer = layer.to(dev)
        x = [t.detach().clone().to(dev).requires_grad_(True) for t in xs]
        pads = layer.pad(x)
        if ws is None:
            ws = [torch.randn(p.shape, generator=g, dtype=torch.float64) for p in pads]
        sum((p * w.to(dev)).sum() for p, w in zip(pads, ws)).backward()
        outs.append([p.detach().cpu() for p in pads])
        grads.append([t.grad.cpu() for t in x])
    for a, b in zip(*outs):
        assert torch.equal(a, b)
    for a, b in zip(*grads):
        assert torch.allclose(a, b, rtol=1e-13, atol=1e-13)
    assert _lib.load() is not None
