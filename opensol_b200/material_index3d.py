"""uint16 material ids of the 3D engine and the per-id float32 value tables.

The ids are part of the engine's contract with open_sol (physics/em3d/material_index3d.py:110-179,
engine3d.py:337-369): a cell's id is the position, in lexicographic order, of its tuple of value levels -- one level
number per material array that takes more than one value, arrays in the order given -- among the tuples that occur
in the grid.  An array's levels are its distinct values when there are at most `limit` of them, otherwise quantised
levels (equal-width bins above the array's minimum; the narrowest width that leaves at most `limit` occupied bins,
searched geometrically; each occupied bin represented by the float64 mean of its members).  When the joint count
exceeds `limit`, every array with more than 256 levels is quantised again at half its level count, at most 12 times.

The joint ids are computed here from a radix code: every level number is below 2^16 (a count never exceeds the uint16
limit), so the levels of up to three arrays pack into one int64 whose numeric order is the tuples' lexicographic
order; a longer tuple packs the dense rank of its leading digits' code (again below 2^16) ahead of the next ones.  The
sorted distinct codes of the grid are the id table: a cell's id is its code's position in it, and a table row
unpacks into the level numbers of its id.  Every pass walks x-slabs of the grid, so no full-grid temporary is made.
"""
from __future__ import annotations

import math

import numpy as np

from .constants import DTYPE

DIGIT_BITS = 16
DIGITS_PER_WORD = 3                     # 48 bits of level digits per int64 word
REQUANTISE_ABOVE = 256                  # arrays with more levels are quantised again when the joint count is too large
REQUANTISE_ROUNDS = 12
WIDTH_SEARCH_RATIO = 1.1                # geometric width search stops once the bracket is this narrow
WIDTH_SEARCH_SPAN = 2.0 ** 24           # without a hint the search starts this far below the guaranteed width
SLAB_CELLS = 1 << 22


def x_slabs(shape, cells=SLAB_CELLS):
    """Index tuples of consecutive x-planes holding about `cells` cells each."""
    planes = max(1, cells // (int(shape[1]) * int(shape[2])))
    return [(slice(x, min(x + planes, shape[0])),) for x in range(0, shape[0], planes)]


def _distinct_upto(blocks, cap):
    """Sorted distinct values over the blocks, or None once more than cap are seen."""
    seen = None
    for block in blocks:
        values = np.unique(block)
        seen = values if seen is None else np.union1d(seen, values)
        if seen.size > cap:
            return None
    return seen


class ValueLevels:
    """The levels of one material array.

    Exact levels: `table` holds the sorted distinct values, `occupied` is None.  Quantised levels: values map to bin
    floor((v - origin) / width), `occupied` holds the sorted occupied bins and `table` their members' means; `error`
    is the largest |value - its level's table value|."""

    def __init__(self, table, occupied=None, origin=0.0, width=0.0):
        self.table, self.occupied, self.origin, self.width = table, occupied, origin, width
        self.error = 0.0

    @property
    def count(self) -> int:
        return int(self.table.size)

    @property
    def quantised(self) -> bool:
        return self.occupied is not None

    def bins(self, values):
        return np.floor((values.astype(np.float64) - self.origin) / self.width).astype(np.int64)

    def numbers(self, block):
        """int64 level number of every value of the block (flattened)."""
        flat = block.ravel()
        if self.occupied is None:
            return np.searchsorted(self.table, flat)
        return np.searchsorted(self.occupied, self.bins(flat))

    @classmethod
    def exact(cls, array, slabs, cap):
        values = _distinct_upto((array[s] for s in slabs), cap)
        if values is None:
            return None
        if not np.isfinite(values).all():
            raise ValueError(f'non-finite material values ({float(values[0])}, {float(values[-1])}) in the '
                             'em_fdtd_3d material arrays')
        return cls(values.astype(DTYPE, copy=False))

    @classmethod
    def quantised_to(cls, array, slabs, budget, width_hint=None):
        """At most `budget` occupied bins of the narrowest width the geometric search finds."""
        low = min(float(array[s].min()) for s in slabs)
        high = max(float(array[s].max()) for s in slabs)
        if not (math.isfinite(low) and math.isfinite(high)):
            raise ValueError(f'non-finite material values ({low}, {high}) in the em_fdtd_3d material arrays')
        probe = cls(None, origin=low)

        def occupied_at(width):
            probe.width = width
            return _distinct_upto((probe.bins(array[s].ravel()) for s in slabs), budget)

        # a width of range / (budget - 1) always fits; search below it (from a quarter of the last width, if known)
        wide = max(high - low, 1e-30) / max(budget - 1, 1)
        narrow = wide / WIDTH_SEARCH_SPAN
        if width_hint is not None:
            narrow = min(max(width_hint / 4.0, narrow), wide)
        if occupied_at(narrow) is not None:
            wide = narrow
        while wide / narrow > WIDTH_SEARCH_RATIO:
            middle = math.sqrt(wide * narrow)
            if occupied_at(middle) is None:
                narrow = middle
            else:
                wide = middle
        levels = cls(None, occupied_at(wide), low, wide)
        n = levels.occupied.size
        sums, members = np.zeros(n), np.zeros(n)
        for s in slabs:
            flat = array[s].ravel()
            number = levels.numbers(flat)
            sums += np.bincount(number, weights=flat.astype(np.float64), minlength=n)
            members += np.bincount(number, minlength=n)
        levels.table = (sums / members).astype(DTYPE)
        levels.error = max(float(np.abs(array[s].ravel() - levels.table[levels.numbers(array[s])]).max())
                           for s in slabs)
        return levels


class JointCode:
    """Radix codes of the level tuples of the varying arrays (see the module docstring): the first three arrays'
    digits pack into one code; each further group of at most two arrays is packed behind the dense rank of the code
    so far, whose sorted distinct values (never more than the full tuples') are found in one pass over the slabs."""

    def __init__(self, arrays, levels, names, slabs, cap):
        self.arrays, self.levels = arrays, levels
        self.groups = [names[:DIGITS_PER_WORD]] + [names[i:i + DIGITS_PER_WORD - 1]
                                                   for i in range(DIGITS_PER_WORD, len(names), DIGITS_PER_WORD - 1)]
        self.prefix_keys = []           # sorted distinct codes of the tuples up to the end of each group but the last
        self.ok = True
        for g in range(len(self.groups) - 1):
            keys = _distinct_upto((self._code(s, g) for s in slabs), cap)
            if keys is None:
                self.ok = False
                return
            self.prefix_keys.append(keys)

    def _pack(self, names, slab, code=None):
        for name in names:
            digit = self.levels[name].numbers(self.arrays[name][slab])
            code = digit if code is None else (code << DIGIT_BITS) | digit
        return code

    def _code(self, slab, last_group):
        code = self._pack(self.groups[0], slab)
        for g in range(1, last_group + 1):
            code = self._pack(self.groups[g], slab, np.searchsorted(self.prefix_keys[g - 1], code))
        return code

    def codes(self, slab):
        return self._code(slab, len(self.groups) - 1)

    def unpack(self, keys):
        """{name: level number} of every key."""
        out = {}
        for g in range(len(self.groups) - 1, -1, -1):
            for name in reversed(self.groups[g]):
                out[name] = keys & ((1 << DIGIT_BITS) - 1)
                keys = keys >> DIGIT_BITS
            if g:
                keys = self.prefix_keys[g - 1][keys]
        return out


def build_material_index(arrays, shape, limit=65534, width_hints=None):
    """(uint16 ids of `shape`, {name: float32 per-id table}, {name: quantisation error}, {name: bin width}) of the
    material arrays (name -> float32 array of `shape`, in the order that ranks the tuples).  ValueError when no
    quantisation within the rounds brings the joint count to `limit`."""
    width_hints = width_hints or {}
    slabs = x_slabs(shape)
    levels = {}
    for name, array in arrays.items():
        levels[name] = (ValueLevels.exact(array, slabs, limit)
                        or ValueLevels.quantised_to(array, slabs, limit, width_hints.get(name)))
    keys, joint, varying = None, None, []
    for _ in range(REQUANTISE_ROUNDS):
        varying = [name for name in arrays if levels[name].count > 1]
        if not varying:
            break
        joint = JointCode(arrays, levels, varying, slabs, limit)
        keys = _distinct_upto((joint.codes(s) for s in slabs), limit) if joint.ok else None
        if keys is not None:
            break
        coarse = [name for name in varying if levels[name].count > REQUANTISE_ABOVE]
        if not coarse:
            break
        for name in coarse:
            levels[name] = ValueLevels.quantised_to(arrays[name], slabs, levels[name].count // 2,
                                                    levels[name].width or width_hints.get(name))
    if varying and keys is None:
        raise ValueError(f'em_fdtd_3d stores materials as a uint16 index: more than {limit} distinct material '
                         f'combinations remain after re-quantising {", ".join(arrays)} (arrays varying together in '
                         f'many independent ways); use fewer field-dependent material properties')
    ids = np.zeros(shape, dtype=np.uint16)
    n_ids = 1
    numbers = {}
    if varying:
        keys = keys.astype(np.int64)
        n_ids = int(keys.size)
        for s in slabs:
            ids[s] = np.searchsorted(keys, joint.codes(s)).astype(np.uint16).reshape(ids[s].shape)
        numbers = joint.unpack(keys)
    tables = {name: (levels[name].table[numbers[name]] if name in numbers
                     else np.full(n_ids, levels[name].table[0])).astype(DTYPE) for name in arrays}
    quantised = [name for name in arrays if levels[name].quantised]
    return (ids, tables, {name: levels[name].error for name in quantised},
            {name: levels[name].width for name in quantised})
