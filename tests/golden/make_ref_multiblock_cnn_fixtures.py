"""Multi-block convolution fixtures computed by the reference's own ``MultiblockConv`` (run in a checkout that
has the reference sources; CPU only).

``lib/modules/multiblock_cnn.py`` is plain PyTorch over a domain's accessors, so it is run here on the
host-only object graph of ``tests/setups.py`` (``build_structure``: block sizes, boundary types, connected
blocks and axes of the layouts in ``MBCNN_CASES``) with a stand-in ``PISOtorch`` module that only provides
the ``BoundaryType`` enum.  For each layout and kernel size 3 / 5 the fixture ``ref_mbcnn_<layout>_k<k>.npz``
holds the seeded FP64 inputs per block, the convolution's weight and bias, the outputs, and the gradients
of ``sum(out_b * g_b)`` (seeded ``g_b``) with respect to the inputs and the weight.

Usage:  python tests/golden/make_ref_multiblock_cnn_fixtures.py --reference <reference checkout>
"""
import argparse
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)

import torch  # noqa: E402

from pict_b200 import PISOtorch  # noqa: E402  (BoundaryType only)
import setups  # noqa: E402

KERNELS = [3, 5]
IN_CH, OUT_CH, BATCH = 3, 2, 2


def block_shapes(spec):
    return [list(reversed(b["size"])) for b in spec["blocks"]]  # zyx


def make_case(name, k, module):
    spec = setups.mbcnn_case(name)
    domain = setups.build_structure(spec, PISOtorch.BoundaryType)
    rng = np.random.default_rng(1000 + 10 * setups.MBCNN_CASES.index(name) + k)
    shapes = block_shapes(spec)
    inputs = [torch.tensor(rng.standard_normal([BATCH, IN_CH] + s), requires_grad=True) for s in shapes]
    conv = module.MultiblockConv(domain, "ZERO", IN_CH, OUT_CH, k, dtype=torch.float64)
    with torch.no_grad():
        conv.conv_layer.weight.copy_(torch.tensor(rng.standard_normal(tuple(conv.conv_layer.weight.shape))))
        conv.conv_layer.bias.copy_(torch.tensor(rng.standard_normal(OUT_CH)))
    out = conv(inputs, domain)
    gs = [torch.tensor(rng.standard_normal(tuple(o.shape))) for o in out]
    loss = sum((o * g).sum() for o, g in zip(out, gs))
    loss.backward()
    arrays = {"weight": conv.conv_layer.weight.detach().numpy(), "bias": conv.conv_layer.bias.detach().numpy(),
              "weight_grad": conv.conv_layer.weight.grad.numpy(), "num_blocks": np.array(len(shapes))}
    for b in range(len(shapes)):
        arrays["input_%d" % b] = inputs[b].detach().numpy()
        arrays["output_%d" % b] = out[b].detach().numpy()
        arrays["out_grad_%d" % b] = gs[b].numpy()
        arrays["input_grad_%d" % b] = inputs[b].grad.numpy()
    return arrays


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="checkout of the reference (for lib/modules/multiblock_cnn.py)")
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    stub = types.ModuleType("PISOtorch")
    stub.BoundaryType = PISOtorch.BoundaryType
    stub.Domain = object  # annotation only
    sys.modules["PISOtorch"] = stub
    src = os.path.join(args.reference, "lib", "modules", "multiblock_cnn.py")
    spec = importlib.util.spec_from_file_location("ref_multiblock_cnn", src)
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    for name in setups.MBCNN_CASES:
        for k in KERNELS:
            np.savez_compressed(os.path.join(args.out, "ref_mbcnn_%s_k%d.npz" % (name, k)), **make_case(name, k, module))
            print("multi-block convolution fixture", name, k, flush=True)


if __name__ == "__main__":
    main()
