"""Autotuner: picks launch shapes for a context by timing them on the model's own state.

The knobs are the tile shape of the tiled 3D right-hand side (sf_ctx_set_tile: 32 x 8, 32 x 4,
64 x 4, 32 x 16 rho points per block), which trades halo re-reads (smaller tiles stage relatively more
halo) against blocks per SM and, for ensembles, against the ragged edges of small members; and,
for single grids, its marching forms (sf_ctx_tune SF_TUNE_RHS_MARCH: each thread walks a few
rows of one column, 31 output columns per block).  Results do not depend on the choice (FP64:
bit for bit; FP32: to FP32 rounding); only the time does.
"""
import ctypes

import torch

from ._lib import check, lib
from .model import stream_handle

TILES = {0: (32, 8), 1: (32, 4), 2: (64, 4), 3: (32, 16)}
# marching forms: rows per thread x warps per block (blocks per SM)
MARCH = {1: "march 4x4", 2: "march 2x8 (2 blocks/SM)", 3: "march 2x8"}
TUNE_RHS_MARCH = 3


def variant_name(v):
    """A printable name of a variant key of tune_rhs3d's result."""
    return str(TILES[v]) if isinstance(v, int) else MARCH[int(v[5:])]


def _time(fn, reps):
    s = torch.cuda.current_stream()
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(reps):
        fn()
    b.record(s)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def tune_rhs3d(model, reps=5, variants=tuple(TILES), marching=None):
    """Times sf_rhs3d on `model` (a Model or Ensemble) for each tile variant (keys 0..3) and, on
    single grids unless `marching` is False, each marching form (keys "march1".."march3");
    leaves the fastest set on its context (model.rhs_tile, model.rhs_march) and returns
    {variant: ms}."""
    c, p = model.ctx.ptr, model._p
    st = stream_handle()
    if marching is None:
        marching = lib.sf_ctx_members(c) == 1

    def run():
        check(lib.sf_rhs3d(c, p(model.u), p(model.v), p(model.Huon), p(model.Hvom), p(model.W),
                           p(model.Hz), p(model.ru), p(model.rv), st), "sf_rhs3d")

    times = {}
    if marching:
        check(lib.sf_ctx_tune(c, TUNE_RHS_MARCH, 0), "sf_ctx_tune")
    for v in variants:
        check(lib.sf_ctx_set_tile(c, v), "sf_ctx_set_tile")
        times[v] = _time(run, reps)
    if marching:
        for mv in MARCH:
            check(lib.sf_ctx_tune(c, TUNE_RHS_MARCH, mv), "sf_ctx_tune")
            times["march%d" % mv] = _time(run, reps)
    best = min(times, key=times.get)
    tile, mv = (best, 0) if isinstance(best, int) else (0, int(best[5:]))
    check(lib.sf_ctx_set_tile(c, tile), "sf_ctx_set_tile")
    if marching:
        check(lib.sf_ctx_tune(c, TUNE_RHS_MARCH, mv), "sf_ctx_tune")
    model.rhs_tile, model.rhs_march = tile, mv
    return times
