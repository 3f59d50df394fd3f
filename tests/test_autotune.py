"""Autotuner: candidate table, workload signature and cache (CPU); tuning a small batch (GPU)."""
import os

import pytest
import torch

from pict_b200 import autotune as at


class _B:
    def __init__(self, shape):
        self.velocity = torch.zeros(shape)


class _D:
    def __init__(self, shapes, dtype=torch.float32):
        self._b = [_B(s) for s in shapes]
        self._dt = dtype

    def getBlocks(self):
        return self._b

    def getSpatialDims(self):
        return 2

    def getDtype(self):
        return self._dt


def test_candidates_and_signature():
    c = at.candidates()
    assert len(c) == len(at.DEFAULT_TILES) * len(at.DEFAULT_CAPS) * len(at.DEFAULT_VARIANTS)
    assert all(set(x) == {"tile_cells", "cap", "cg_variant"} for x in c)
    d = _D([(1, 2, 32, 32), (1, 2, 64, 64)])
    s1 = at.workload_signature(d, {"pressure_tol": 1e-6}, "B200")
    assert s1 == at.workload_signature(_D([(1, 2, 64, 64), (1, 2, 32, 32)]), {"pressure_tol": 1e-6}, "B200")
    assert s1 != at.workload_signature(d, {"pressure_tol": 1e-7}, "B200")
    assert s1 != at.workload_signature(d, {"pressure_tol": 1e-6}, "H100")


def test_cache_roundtrip(tmp_path):
    p = os.path.join(tmp_path, "sub", "tune.json")
    assert at.load_cache(p) == {}
    at.save_cache(p, {"k": {"best": {"tile_cells": 1024}, "table": []}})
    assert at.load_cache(p)["k"]["best"]["tile_cells"] == 1024


@pytest.mark.gpu
def test_autotune_small_batch(tmp_path):
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    from setups import build_product, lid_cavity
    doms = [build_product(lid_cavity(n, viscosity=1e-3), torch.float32) for n in (40, 64, 96)]
    b = BatchDomain(doms, time_steps=[0.5 / n for n in (40, 64, 96)])
    v0 = [d.getBlock(0).velocity.clone() for d in doms]
    kw = dict(time_step=0.01, advection_tol=1e-6, pressure_tol=1e-6)
    cache = os.path.join(tmp_path, "tune.json")
    best, table = at.autotune(b, kw, cache_path=cache)
    assert len(table) == len(at.candidates()) and best["ms_per_step"] == min(r["ms_per_step"] for r in table)
    assert b.tile_cells == best["tile_cells"]
    assert all(torch.equal(d.getBlock(0).velocity, v) for d, v in zip(doms, v0))
    best2, _ = at.autotune(b, kw, cache_path=cache)   # cache hit
    assert best2 == best
    st = PISOStepper(b, p_group_size=best["p_group_size"], adv_group_size=best["adv_group_size"],
                     cg_variant=best["cg_variant"], **kw)
    st.step()
    st.check()
