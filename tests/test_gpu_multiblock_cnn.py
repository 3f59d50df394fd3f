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
