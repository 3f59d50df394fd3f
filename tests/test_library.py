"""CPU checks of the C-ABI library: it loads, exports every symbol declared in include/pict_b200.h,
its struct layouts match the ctypes binding, and the host-side topology builder agrees with the
oracle's neighbour tables.  No GPU compute calls."""
import ctypes
import os
import re

import numpy as np
import pytest

from setups import ALL_CASES, build_oracle, case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    src = open(os.path.join(ROOT, "include", "pict_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pict_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_all_declared_symbols():
    from pict_b200 import _lib
    lib = _lib.load()
    syms = _declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert set(syms) <= set(_lib.SIGNATURES), set(syms) - set(_lib.SIGNATURES)
    assert lib.pict_version().decode().startswith("pict_b200")
    assert lib.pict_sizeof_block() == ctypes.sizeof(_lib.BlockDesc)
    assert lib.pict_sizeof_domain() == ctypes.sizeof(_lib.DomainDesc)


def test_binding_argument_counts_match_the_header():
    """Every prototype of include/pict_b200.h has as many parameters as its ctypes signature."""
    from pict_b200 import _lib
    src = open(os.path.join(ROOT, "include", "pict_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    bad = {}
    for name, params in re.findall(r"\b(pict_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", src):
        params = params.strip()
        n = 0 if params in ("", "void") else params.count(",") + 1
        if name in _lib.SIGNATURES and len(_lib.SIGNATURES[name][1]) != n:
            bad[name] = (n, len(_lib.SIGNATURES[name][1]))
    assert not bad, bad


def _pack_from_oracle(od):
    from pict_b200 import _lib
    arr = (_lib.BlockDesc * len(od.blocks))()
    for bi, b in enumerate(od.blocks):
        d = arr[bi]
        s = list(b.size) + [1] * (3 - od.dims)
        d.size[0], d.size[1], d.size[2] = s
        d.offset = od.offsets[bi]
        for f, bnd in enumerate(b.boundaries):
            F = d.face[f]
            if bnd.kind == "fixed":
                F.type = _lib.PICT_FACE_FIXED
            elif bnd.kind == "periodic":
                F.type = _lib.PICT_FACE_PERIODIC
            else:
                F.type = _lib.PICT_FACE_CONNECTED
                F.conn_block = bnd.block
                for k, a in enumerate(bnd.axes):
                    F.conn_axes[k] = a
    return arr


@pytest.mark.parametrize("name", ALL_CASES)
def test_topology_matches_oracle(name):
    from pict_b200 import _lib
    od = build_oracle(case(name))
    arr = _pack_from_oracle(od)
    nbr = np.empty((2 * od.dims, od.N), dtype=np.int32)
    cb = np.empty(od.N, dtype=np.int32)
    st = _lib.load().pict_build_topology(arr, len(od.blocks), od.dims, od.N, nbr.ctypes.data, cb.ctypes.data)
    assert st == 0, _lib.load().pict_last_error()
    assert np.array_equal(nbr, od.nb)
    assert np.array_equal(cb, od.blk)


def test_topology_rejects_inconsistent_connections():
    from pict_b200 import _lib
    od = build_oracle(case("twoblock2d"))
    arr = _pack_from_oracle(od)
    arr[1].face[0].conn_axes[0] = 0  # break the back-connection
    nbr = np.empty((4, od.N), dtype=np.int32)
    cb = np.empty(od.N, dtype=np.int32)
    st = _lib.load().pict_build_topology(arr, 2, 2, od.N, nbr.ctypes.data, cb.ctypes.data)
    assert st != 0
    assert b"not mutual" in _lib.load().pict_last_error()
    arr = _pack_from_oracle(build_oracle(case("periodic2d")))
    arr[0].face[1].type = _lib.PICT_FACE_FIXED  # periodic -x without periodic +x
    od2 = build_oracle(case("periodic2d"))
    nbr = np.empty((4, od2.N), dtype=np.int32)
    cb = np.empty(od2.N, dtype=np.int32)
    assert _lib.load().pict_build_topology(arr, 1, 2, od2.N, nbr.ctypes.data, cb.ctypes.data) != 0


def test_non_ortho_flags_enum():
    """NonOrthoFlags carries the bits of extensions/PISO_multiblock_cuda.h:9-13 and is accepted wherever
    the operators take nonOrthoFlags; the driver's mode is the same int."""
    from pict_b200 import PISOtorch as P
    from pict_b200.PISOtorch_simulation import Simulation
    F = P.NonOrthoFlags
    assert (F.DIRECT_MATRIX, F.DIRECT_RHS, F.DIAGONAL_MATRIX, F.DIAGONAL_RHS, F.CENTER_MATRIX) == (1, 2, 4, 8, 16)
    mode = F.CENTER_MATRIX | F.DIRECT_MATRIX | F.DIAGONAL_RHS
    assert int(mode) == Simulation._NON_ORTHO_MODE == 25
    assert P._non_ortho(mode) == 25 and P._non_ortho(F.NONE) == 0


def test_bicg_preconditioner_switch():
    """SetBiCGPreconditioner selects the preconditioned BiCGStab's operator and returns the previous one;
    the default is the operator the reference's build applies."""
    from pict_b200 import PISOtorch as P
    from pict_b200 import _lib
    B = P.BiCGPreconditioner
    assert (int(B.AS_REFERENCE), int(B.ILU0)) == (_lib.PICT_PRECOND_AS_REFERENCE, _lib.PICT_PRECOND_ILU0)
    assert P.GetBiCGPreconditioner() == B.AS_REFERENCE
    prev = P.SetBiCGPreconditioner(B.ILU0)
    try:
        assert prev == B.AS_REFERENCE and P.GetBiCGPreconditioner() == B.ILU0
        with pytest.raises(ValueError):
            P.SetBiCGPreconditioner(7)
    finally:
        P.SetBiCGPreconditioner(prev)
    assert P.GetBiCGPreconditioner() == B.AS_REFERENCE


def test_two_sweep_stage_fit():
    """Host check of the multigrid levels that take two smoothing sweeps: 2D, not y-periodic, every tile's
    stage (rows plus two halo rows; the prolongation's three) within the shared-memory stage."""
    import numpy as np
    from pict_b200.multigrid import level_tiles, two_sweep_fits

    def case(nx, ny, per_y=0, dims=2, tile=512):
        fine = np.array([[nx, ny, 1]])
        coarse = np.array([[(nx + 1) // 2, (ny + 1) // 2, 1]])
        per = np.array([[0, per_y, 0]])
        sh = np.array([[1, 1, 0]])
        ct = level_tiles([0], [coarse[0, 0] * coarse[0, 1]], [0], tile)
        ft = level_tiles([0], [nx * ny], [0], tile)
        return two_sweep_fits(fine, per, np.array([0]), coarse, sh, ct, ft, dims)

    assert case(256, 256)
    assert case(181, 200)
    assert not case(256, 256, per_y=1)
    assert not case(256, 256, dims=3)
    assert not case(1024, 64)
