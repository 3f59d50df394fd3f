"""Convolutions over multi-block domains (the reference's lib/modules/multiblock_cnn.py).

A ``MultiblockConv`` applies one ``torch.nn.ConvNd`` to every block of a domain, padding each block with
the cells of the blocks it is connected to (across ``ConnectedBoundary`` faces, with their axis
permutations and inversions, and across periodic faces) and with zeros at fixed faces, so that a
network sees the domain as one field.  The padding of every block is a fixed gather, built once at
construction as a map from each padded cell to its source (block, cell) or zero.  On CUDA tensors it is one
launch of this library for all blocks, reading the blocks in place (``pict_mb_pad_gather``), and its gradient
is one gather-sum over the inverse map (``pict_mb_pad_scatter_sum``, deterministic).  On CPU tensors the same
map runs as ``index_select`` over the concatenated blocks.

Which block fills a padding region follows the reference's walk (lib/modules/multiblock_cnn.py:158-264):
from the block, each axis in order x, y, z, lower then upper face; a connected or periodic face makes
the cell region beyond it a block region (with the axis mapping of the connection composed along
the way) and continues the walk over the remaining axes from there; a fixed face makes a zero region
unless a block region reaches it; regions never reached are zero.  A region taken from another block
is that block's field flipped, permuted into this block's axes and sliced (:214-246).

One deliberate difference: the reference permutes with the inverse of the axis mapping
(``AxesMapping.make_inverted().get_permute_flip_args()``), which equals the mapping itself only when
the connections compose to a swap of axes.  That covers every 1D and 2D layout and 3D layouts whose
connections swap at most two axes, where the results here are the same as the reference's.  A 3D
connection that cycles all three axes makes the reference concatenate mis-shaped regions (an error)
or, on cubic blocks, pad with transposed data; here the permutation follows the mapping itself, so
such layouts are padded with the cells across the connection (the cells ``computeConnectedPos``
addresses in the solver's stencils).
"""
from __future__ import annotations

import ctypes
from typing import List

import numpy as np
import torch

from . import PISOtorch as P
from . import _lib

__all__ = ["MultiblockConv", "MultiblockConv_naive", "MultiblockReLU"]


def _zyx(d, dims):
    return dims - 1 - d


def _spatial_shape(block):
    dims = block.getSpatialDims()
    s = block.getSizes()
    xyz = [s.x, s.y, s.z][:dims]
    return [xyz[_zyx(d, dims)] for d in range(dims)]  # zyx


# An axis mapping is a tuple of directions: entry i = 2 * (target axis) + (inverted) for source axis i.
def _map_identity(dims):
    return tuple(2 * d for d in range(dims))


def _map_direction(m, direction):
    a, up = direction >> 1, direction & 1
    return (m[a] >> 1) * 2 + int(up != (m[a] & 1))


def _map_from_face(face, axes, dims):
    a, up = face >> 1, face & 1
    m = [0] * dims
    m[a] = (axes[0] >> 1) * 2 + int(up == (axes[0] & 1))
    for i in range(1, dims):
        m[(a + i) % dims] = axes[i]
    return tuple(m)


def _map_compose(m, other):
    return tuple((other[m[i] >> 1] >> 1) * 2 + int((other[m[i] >> 1] & 1) != (m[i] & 1)) for i in range(len(m)))


def _map_invert(m):
    inv = [0] * len(m)
    for i, t in enumerate(m):
        inv[t >> 1] = 2 * i + (t & 1)
    return tuple(inv)


def _permute_flip(m):
    """torch.flip dims (applied first) and torch.permute dims that bring a neighbour's zyx tensor into this
    block's axes, for the mapping ``m`` from this block's axes to the neighbour's.  The flips are those of
    the inverse mapping (the neighbour's axes that run against this block's) and the permutation takes
    this block's axis i from the neighbour's axis m[i]."""
    dims = len(m)
    inv = _map_invert(m)
    permute = [0, 1] + [_zyx(m[_zyx(d, dims)] >> 1, dims) + 2 for d in range(dims)]
    flip = [_zyx(d, dims) + 2 for d in range(dims) if inv[d] & 1]
    return permute, flip


class MultiblockConv(torch.nn.Module):
    def __init__(self, domain, fixed_boundary_padding, in_channels: int, out_channels: int, kernel_size: int,
                 stride: int = 1, padding="same", dilation: int = 1, groups: int = 1, bias: bool = True,
                 padding_mode: str = "zeros", device=None, dtype=None):
        super().__init__()
        dims = domain.getSpatialDims()
        conv = {1: torch.nn.Conv1d, 2: torch.nn.Conv2d, 3: torch.nn.Conv3d}.get(dims)
        if conv is None:
            raise ValueError
        ok_list = isinstance(fixed_boundary_padding, (list, tuple)) and len(fixed_boundary_padding) == in_channels and \
            all(p in ["VEL_U", "VEL_V", "VEL_W", "S", "ZERO"] for p in fixed_boundary_padding)
        if not (ok_list or fixed_boundary_padding in ["ZERO"]):
            raise ValueError
        if kernel_size not in [3, 5, 7]:
            raise NotImplementedError("kernel_size must be 3, 5, or 7.")
        if padding not in [kernel_size // 2, "same"]:
            raise NotImplementedError("padding must be 1 or 'same'")
        if dilation != 1:
            raise NotImplementedError("dilation is not supported")
        self.dims = dims
        self.fixed_boundary_padding = fixed_boundary_padding
        self.in_channels = in_channels
        self.kernel_size = kernel_size
        self.padding = kernel_size // 2
        self.device = device
        self.dtype = dtype
        blocks = domain.getBlocks()
        self._shapes = [_spatial_shape(b) for b in blocks]
        offsets, n = [], 0
        for s in self._shapes:
            offsets.append(n)
            n += int(torch.tensor(s).prod())
        self._zero_index = n
        idx = [self._gather_index(bi, blocks, offsets) for bi in range(len(blocks))]
        for bi, t in enumerate(idx):  # moved with the module by .to() / .cuda()
            self.register_buffer("_gather_%d" % bi, t if device is None else t.to(device), persistent=False)
        self._build_device_map(idx, offsets, n)
        self.conv_layer = conv(in_channels, out_channels, kernel_size, stride=stride, padding=0, dilation=dilation,
                               groups=groups, bias=bias, padding_mode=padding_mode, device=device, dtype=dtype)

    # ---- padding structure ----
    def _slot(self, pos):
        return sum(p * 3 ** a for a, p in enumerate(pos))

    def _regions(self, block, blocks):
        """Per 3^D region (axis-wise lower / centre / upper, x fastest): ('BORDER',), ('CENTER',) or
        ('BLOCK', block index, axis mapping)."""
        dims = self.dims
        info = [None] * 3 ** dims

        def walk(blk, pos, m, axes):
            for a in axes:
                rest = [x for x in axes if x != a]
                for up in (0, 1):
                    npos = list(pos)
                    npos[a] += 1 if up else -1
                    k = self._slot(npos)
                    face = _map_direction(m, 2 * a + up)
                    bnd = blk.getBoundaries()[face]
                    if bnd.type == P.BoundaryType.FIXED:
                        if info[k] is None:
                            info[k] = ("BORDER",)
                    elif bnd.type in (P.BoundaryType.CONNECTED, P.BoundaryType.PERIODIC):
                        if info[k] is None or info[k][0] == "BORDER":
                            if bnd.type == P.BoundaryType.CONNECTED:
                                nb = bnd.getConnectedBlock()
                                nm = _map_compose(m, _map_from_face(face, bnd.axes, dims))
                            else:
                                nb, nm = blk, m
                            info[k] = ("BLOCK", blocks.index(nb), nm)
                            walk(nb, npos, nm, rest)
                    else:
                        raise TypeError("Boundary type not supported.")

        walk(block, [1] * dims, _map_identity(dims), list(range(dims)))
        info = [("BORDER",) if x is None else x for x in info]
        info[self._slot([1] * dims)] = ("CENTER",)
        return info

    def _gather_index(self, bi, blocks, offsets):
        dims, pad = self.dims, self.padding
        shape = self._shapes[bi]
        own = torch.arange(int(torch.tensor(shape).prod())).reshape([1, 1] + shape) + offsets[bi]
        grid = []
        for k, reg in enumerate(self._regions(blocks[bi], blocks)):
            pos = [(k // 3 ** a) % 3 for a in range(dims)]  # xyz
            if reg[0] == "CENTER":
                grid.append(own)
            elif reg[0] == "BORDER":
                size = [pad if pos[_zyx(d, dims)] != 1 else shape[d] for d in range(dims)]
                grid.append(torch.full([1, 1] + size, self._zero_index, dtype=torch.long))
            else:
                _, nb, m = reg
                permute, flip = _permute_flip(m)
                nshape = self._shapes[nb]
                t = torch.arange(int(torch.tensor(nshape).prod())).reshape([1, 1] + nshape) + offsets[nb]
                pshape = [nshape[permute[d + 2] - 2] for d in range(dims)]
                if flip:
                    t = torch.flip(t, flip)
                t = t.permute(permute)
                sl = [slice(None), slice(None)]
                for d in range(dims):
                    p = pos[_zyx(d, dims)]
                    sl.append(slice(pshape[d] - pad, pshape[d]) if p == 0 else (slice(pad) if p == 2 else slice(None)))
                grid.append(t[tuple(sl)])
        for cat_dim in range(dims - 1, -1, -1):  # zyx tensors, regions in xyz order
            grid = [torch.cat(grid[i * 3:i * 3 + 3], dim=cat_dim + 2) for i in range(len(grid) // 3)]
        return grid[0].reshape(-1).contiguous()

    def _build_device_map(self, idx, offsets, n):
        """The map of the library's padding kernels: per padded cell (output block, position) <- (source block,
        cell) or -1, and its inverse (the padded cells reading each source cell, CSR)."""
        nb = len(idx)
        starts = np.asarray(offsets + [n], dtype=np.int64)
        ob, pos, sb, loc = [], [], [], []
        for bi, t in enumerate(idx):
            g = t.cpu().numpy().astype(np.int64)
            b = np.searchsorted(starts, g, side="right") - 1
            zero = g >= n
            ob.append(np.full(g.size, bi, np.int32))
            pos.append(np.arange(g.size, dtype=np.int32))
            sb.append(np.where(zero, -1, b).astype(np.int32))
            loc.append(np.where(zero, 0, g - starts[np.minimum(b, nb - 1)]).astype(np.int32))
        ob, pos, sb, loc = (np.concatenate(a) for a in (ob, pos, sb, loc))
        gsrc = np.concatenate([t.cpu().numpy() for t in idx]).astype(np.int64)
        keep = gsrc < n
        order = np.argsort(gsrc[keep], kind="stable")
        readers = np.nonzero(keep)[0][order]
        counts = np.bincount(gsrc[keep], minlength=n)
        rptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
        cell_block = np.repeat(np.arange(nb, dtype=np.int32), np.diff(starts))
        cell_loc = (np.arange(n, dtype=np.int64) - starts[cell_block]).astype(np.int32)
        t32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32))
        maps = {"ob": ob, "pos": pos, "sb": sb, "loc": loc, "cb": cell_block, "cl": cell_loc, "rptr": rptr,
                "rob": ob[readers], "rpos": pos[readers]}
        for k, v in maps.items():
            self.register_buffer("_pad_%s" % k, t32(v) if self.device is None else t32(v).to(self.device),
                                 persistent=False)
        pad = self.padding
        self._src_cells = [int(np.prod(s)) for s in self._shapes]
        self._out_cells = [int(np.prod([x + 2 * pad for x in s])) for s in self._shapes]

    def _pad_device(self, tensor_list):
        return _PadFunction.apply(self, *tensor_list)

    # ---- forward ----
    def forward(self, tensor_list: List[torch.Tensor], domain=None):
        if domain is not None:
            if domain.getSpatialDims() != self.dims:
                raise ValueError("domain dimensionality does not match this layer.")
            blocks = domain.getBlocks()
            if not (isinstance(tensor_list, (list, tuple)) and all(isinstance(t, torch.Tensor) for t in tensor_list)):
                raise TypeError("tensor_list must be a list of torch.Tensor.")
            if len(tensor_list) != len(blocks):
                raise ValueError("length of tensor_list must match domain blocks.")
            if len(blocks) == 0:
                raise ValueError("no input tensors.")
            if any(t.dim() != self.dims + 2 for t in tensor_list):
                raise ValueError("tensors must have shape NCDHW.")
            batch = tensor_list[0].size(0)
            if any(t.size(0) != batch for t in tensor_list):
                raise ValueError("tensors have inconsistent batch size.")
            if any(t.size(1) != self.in_channels for t in tensor_list):
                raise ValueError("channel dimension of tensors must match in_channels.")
            if any(list(t.shape[2:]) != s for t, s in zip(tensor_list, self._shapes)):
                raise ValueError("tensor spatial dimensions must match block sizes")
        return [self.conv_layer(t) for t in self.pad(tensor_list)]

    def pad(self, tensor_list: List[torch.Tensor]) -> List[torch.Tensor]:
        """Every block's tensor with ``padding`` cells added on each side from its neighbours (zeros at fixed
        faces and unreachable corners)."""
        if all(t.is_cuda for t in tensor_list) and tensor_list[0].dtype in (torch.float32, torch.float64) and \
                len(tensor_list) <= 64:
            return list(self._pad_device(tensor_list))
        batch, ch = tensor_list[0].size(0), tensor_list[0].size(1)
        ref = tensor_list[0]
        flat = torch.cat([t.reshape(batch, ch, -1) for t in tensor_list] +
                         [torch.zeros(batch, ch, 1, dtype=ref.dtype, device=ref.device)], dim=2)
        out = []
        for bi in range(len(tensor_list)):
            idx = getattr(self, "_gather_%d" % bi)
            if idx.device != ref.device:
                idx = idx.to(ref.device)
            shape = [s + 2 * self.padding for s in self._shapes[bi]]
            out.append(flat.index_select(2, idx).reshape([batch, ch] + shape))
        return out


def _host_ptrs(tensors):
    return (ctypes.c_void_p * len(tensors))(*[t.data_ptr() for t in tensors])


def _host_cells(cells):
    return (ctypes.c_int64 * len(cells))(*cells)


class _PadFunction(torch.autograd.Function):
    """The padding of all blocks in one launch (pict_mb_pad_gather) and its gradient in one launch
    (pict_mb_pad_scatter_sum); the blocks' pointers travel in the kernel parameters."""

    @staticmethod
    def forward(ctx, layer, *tensors):
        lib = _lib.load()
        dev = tensors[0].device
        dtype = tensors[0].dtype
        batch, ch = tensors[0].size(0), tensors[0].size(1)
        srcs = [t.contiguous() for t in tensors]
        pad = layer.padding
        outs = [torch.empty([batch, ch] + [x + 2 * pad for x in s], dtype=dtype, device=dev) for s in layer._shapes]
        for k in ("ob", "pos", "sb", "loc"):
            if getattr(layer, "_pad_" + k).device != dev:
                setattr(layer, "_pad_" + k, getattr(layer, "_pad_" + k).to(dev))
        code = _lib.PICT_F64 if dtype == torch.float64 else _lib.PICT_F32
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(lib.pict_mb_pad_gather(int(layer._pad_ob.numel()), batch * ch, code, len(srcs),
                                          layer._pad_ob.data_ptr(), layer._pad_pos.data_ptr(), layer._pad_sb.data_ptr(),
                                          layer._pad_loc.data_ptr(), _host_ptrs(srcs), _host_cells(layer._src_cells),
                                          _host_ptrs(outs), _host_cells(layer._out_cells), stream),
                   "multi-block padding")
        ctx.layer = layer
        ctx.meta = (batch, ch, dtype, dev, [t.shape for t in srcs])
        return tuple(outs)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, *gouts):
        layer = ctx.layer
        batch, ch, dtype, dev, shapes = ctx.meta
        lib = _lib.load()
        g = [torch.zeros([batch, ch] + [x + 2 * layer.padding for x in s], dtype=dtype, device=dev) if x is None
             else x.contiguous() for x, s in zip(gouts, layer._shapes)]
        gs = [torch.empty(sh, dtype=dtype, device=dev) for sh in shapes]
        for k in ("cb", "cl", "rptr", "rob", "rpos"):
            if getattr(layer, "_pad_" + k).device != dev:
                setattr(layer, "_pad_" + k, getattr(layer, "_pad_" + k).to(dev))
        code = _lib.PICT_F64 if dtype == torch.float64 else _lib.PICT_F32
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(lib.pict_mb_pad_scatter_sum(int(layer._pad_cb.numel()), batch * ch, code, len(gs),
                                               layer._pad_cb.data_ptr(), layer._pad_cl.data_ptr(),
                                               layer._pad_rptr.data_ptr(), layer._pad_rob.data_ptr(),
                                               layer._pad_rpos.data_ptr(), _host_ptrs(g), _host_cells(layer._out_cells),
                                               _host_ptrs(gs), _host_cells(layer._src_cells), stream),
                   "multi-block padding gradient")
        return (None, *gs)


class MultiblockConv_naive(torch.nn.Module):
    """One convolution per block with the convolution's own padding (lib/modules/multiblock_cnn.py:336-359)."""

    def __init__(self, dims, *conv_args, **conv_kwargs):
        super().__init__()
        conv = {1: torch.nn.Conv1d, 2: torch.nn.Conv2d, 3: torch.nn.Conv3d}.get(dims)
        if conv is None:
            raise ValueError
        self.conv_layer = conv(*conv_args, **conv_kwargs)

    def forward(self, tensor_list, domain=None):
        return [self.conv_layer(t) for t in tensor_list]


class MultiblockReLU(torch.nn.Module):
    def forward(self, tensor_list, domain=None):
        return [torch.nn.functional.relu(t) for t in tensor_list]
