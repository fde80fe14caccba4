"""uint16 material index of the 3D engine: per material array a set of value levels, the joint level combinations
ranked into ids, and per-id float32 tables -- open_sol's scheme (physics/em3d/material_index3d.py:1-179).

Levels of an array are its exact distinct values when there are at most `limit` of them, else bins of a width found
by geometric bisection (representative = the mean of the member cells, error = max |value - representative|).  The
id of a cell is the rank of its tuple of levels (arrays in order, single-valued arrays left out) among the occurring
tuples in lexicographic order, computed stage by stage over x-slab chunks as codes rank(previous) * count + level, so
no full-grid temporary beyond one chunk is made.  When the joint count exceeds `limit`, every array with more than 256
levels is re-binned at half its level count, up to 12 times; ValueError when that is not enough.
"""
from __future__ import annotations

import math

import numpy as np

from .constants import DTYPE

_MIN_REDUCIBLE_LEVELS = 256
_MAX_ATTEMPTS = 12
_BISECTION_RATIO = 1.1
_SEARCH_DEPTH = 2.0 ** 24
_CHUNK_CELLS = 1 << 22


class Levels:
    """Levels of one array: exact sorted values (bins None) or occupied bin numbers of width delta above minimum."""

    def __init__(self, values, bins=None, minimum=0.0, delta=0.0, error=0.0):
        self.values, self.bins, self.minimum, self.delta, self.error = values, bins, minimum, delta, error

    @property
    def count(self) -> int:
        return int(self.values.size)

    def index(self, values):
        flat = values.ravel()
        if self.bins is None:
            return np.searchsorted(self.values, flat)
        return np.searchsorted(self.bins, _bin_numbers(flat, self.minimum, self.delta))


def _bin_numbers(flat, minimum, delta):
    return np.floor((flat.astype(np.float64) - minimum) / delta).astype(np.int64)


def x_chunks(shape, chunk_cells=_CHUNK_CELLS):
    per_chunk = max(1, chunk_cells // (shape[1] * shape[2]))
    return [(slice(start, min(start + per_chunk, shape[0])),) for start in range(0, shape[0], per_chunk)]


def _merged_unique(parts, limit):
    merged = None
    for part in parts:
        values = np.unique(part)
        merged = values if merged is None else np.union1d(merged, values)
        if merged.size > limit:
            return None
    return merged


def _exact(array, chunks, limit):
    values = _merged_unique((array[c] for c in chunks), limit)
    if values is None:
        return None
    if not bool(np.isfinite(values).all()):
        raise ValueError(f'non-finite material values ({float(values[0])}, {float(values[-1])}) in the em_fdtd_3d '
                         'material arrays')
    return Levels(values.astype(DTYPE, copy=False))


def _binned(array, chunks, budget, delta_hint=None):
    minimum = min(float(array[c].min()) for c in chunks)
    maximum = max(float(array[c].max()) for c in chunks)
    if not (math.isfinite(minimum) and math.isfinite(maximum)):
        raise ValueError(f'non-finite material values ({minimum}, {maximum}) in the em_fdtd_3d material arrays')

    def occupied(delta):
        return _merged_unique((_bin_numbers(array[c].ravel(), minimum, delta) for c in chunks), budget)

    upper = max(maximum - minimum, 1e-30) / max(budget - 1, 1)
    lower = upper / _SEARCH_DEPTH if delta_hint is None else min(max(delta_hint / 4.0, upper / _SEARCH_DEPTH), upper)
    if occupied(lower) is not None:
        upper = lower
    while upper / lower > _BISECTION_RATIO:
        middle = math.sqrt(upper * lower)
        if occupied(middle) is None:
            lower = middle
        else:
            upper = middle
    bins = occupied(upper)
    n = int(bins.size)
    sums, counts = np.zeros(n), np.zeros(n)
    for c in chunks:
        flat = array[c].ravel()
        rank = np.searchsorted(bins, _bin_numbers(flat, minimum, upper))
        sums += np.bincount(rank, weights=flat.astype(np.float64), minlength=n)
        counts += np.bincount(rank, minlength=n)
    levels = Levels((sums / counts).astype(DTYPE), bins, minimum, upper)
    levels.error = max(float(np.abs(array[c].ravel() - levels.values[levels.index(array[c])]).max()) for c in chunks)
    return levels


def _stage_code(arrays, levels, order, keys, chunk, stage):
    code = levels[order[0]].index(arrays[order[0]][chunk])
    for position in range(1, stage + 1):
        name = order[position]
        code = np.searchsorted(keys[position - 1], code) * levels[name].count + levels[name].index(arrays[name][chunk])
    return code


def _stage_keys(arrays, levels, order, chunks, limit):
    keys = []
    for stage in range(len(order)):
        stage_keys = _merged_unique((_stage_code(arrays, levels, order, keys, c, stage) for c in chunks), limit)
        if stage_keys is None:
            return None
        keys.append(stage_keys)
    return keys


def build_material_index(arrays, shape, limit=65534, delta_hints=None):
    """(uint16 ids (shape), {name: float32 table}, {name: quantisation error}, {name: bin width}) of the material
    arrays (dict name -> float32 array of `shape`)."""
    delta_hints = delta_hints or {}
    chunks = x_chunks(shape)
    levels = {}
    for name, array in arrays.items():
        exact = _exact(array, chunks, limit)
        levels[name] = exact if exact is not None else _binned(array, chunks, limit, delta_hints.get(name))
    keys = []
    order = []
    for _ in range(_MAX_ATTEMPTS):
        order = [name for name in arrays if levels[name].count > 1]
        keys = _stage_keys(arrays, levels, order, chunks, limit) if order else []
        if keys is not None:
            break
        reducible = [name for name in order if levels[name].count > _MIN_REDUCIBLE_LEVELS]
        if not reducible:
            break
        for name in reducible:
            levels[name] = _binned(arrays[name], chunks, levels[name].count // 2,
                                   levels[name].delta or delta_hints.get(name))
    if keys is None:
        raise ValueError(f'em_fdtd_3d stores materials as a uint16 index: more than {limit} distinct material '
                         f'combinations remain after re-quantising {", ".join(arrays)} (arrays varying together in '
                         f'many independent ways); use fewer field-dependent material properties')
    n_ids = int(keys[-1].size) if order else 1
    ids = np.empty(shape, dtype=np.uint16)
    for c in chunks:
        if order:
            code = _stage_code(arrays, levels, order, keys, c, len(order) - 1)
            ids[c] = np.searchsorted(keys[-1], code).astype(np.uint16).reshape(ids[c].shape)
        else:
            ids[c] = 0
    level_of_id = {}
    if order:
        key = keys[-1]
        for position in range(len(order) - 1, 0, -1):
            count = levels[order[position]].count
            level_of_id[order[position]] = key % count
            key = keys[position - 1][key // count]
        level_of_id[order[0]] = key
    tables = {name: (levels[name].values[level_of_id[name]] if name in level_of_id
                     else np.repeat(levels[name].values[:1], n_ids)).astype(DTYPE) for name in arrays}
    errors = {name: levels[name].error for name in arrays if levels[name].bins is not None}
    deltas = {name: levels[name].delta for name in arrays if levels[name].bins is not None}
    return ids, tables, errors, deltas
