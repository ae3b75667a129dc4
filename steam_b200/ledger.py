"""The realized per-class scalars of a run (steam/ledger.py:46-270).

The cascade is local except for a handful of per-class, per-level scalars
realized from the data (flux means, product norms, bounded-add constants,
projections).  They are stored additively -- (total, count) pairs with
float64 totals -- so partial sums from tiles or ranks combine exactly.  The
device path produces every total with float64 accumulators in a fixed
reduction order, so a total is reproducible on the same device.
"""

from __future__ import annotations

import numpy as np

N_RESCALE_DEFAULT = 10


class MeanReduction:
    """Additive (total, count) pair; ``mean`` divides in float64
    (steam/ledger.py:46-84)."""

    __slots__ = ('total', 'count')

    def __init__(self, total, count):
        self.total = total
        self.count = int(count)

    @property
    def mean(self):
        return float(self.total) / max(self.count, 1)

    def __add__(self, other):
        return MeanReduction(self.total + other.total, self.count + other.count)

    def __repr__(self):
        return f"MeanReduction(total={self.total!r}, count={self.count})"


class PatternLedger:
    """Per-level sum |W S g| and turbulon-centre count (steam/ledger.py:87-112)."""

    __slots__ = ('level_total', 'level_count')

    def __init__(self, level_total, level_count):
        self.level_total = np.asarray(level_total, dtype=np.float64)
        self.level_count = np.asarray(level_count, dtype=np.int64)

    @property
    def level_mean(self):
        return (self.level_total / np.maximum(self.level_count, 1)).astype(np.float32)

    def __add__(self, other):
        return PatternLedger(self.level_total + other.level_total,
                             self.level_count + other.level_count)


class FluxAdvanceLedger:
    """Entering / noise / realized means of one flux advance and its clip count
    (steam/ledger.py:115-142)."""

    __slots__ = ('entering', 'noise_abs', 'realized', 'n_clipped')

    def __init__(self, entering, noise_abs, realized, n_clipped):
        self.entering = entering
        self.noise_abs = noise_abs
        self.realized = realized
        self.n_clipped = int(n_clipped)

    @property
    def rescale(self):
        realized = self.realized.mean
        if realized > 0:
            return np.float32(self.entering.mean / realized)
        return None


class BoundedAddLedger:
    """Per-level results of one bounded-add solve (steam/ledger.py:145-194):
    the target amplitude a0, the loop's demeans and scales, the loop length
    n_loop and rescale count n_scale, the final demean and the zero-mean
    shift mu (NaN where none was needed) -- the sequence that replays the
    solve with no reduction (steam/simulate.py:3196-3213) -- plus how many
    field sweeps the device solve took.

    ``demean`` and ``scale`` (nz, n_rescale) hold the values the device's
    chain applied, in the working dtype (exact in float64); a step that was
    not rescaled carries scale 1, which multiplies exactly.
    """

    __slots__ = ('a0', 'demean', 'scale', 'n_loop', 'n_scale', 'final_demean', 'mu',
                 'n_sweeps', 'n_steps', 'has_final')

    def __init__(self, nz, n_rescale=10):
        self.a0 = np.zeros(nz, dtype=np.float64)
        self.demean = np.zeros((nz, n_rescale), dtype=np.float64)
        self.scale = np.ones((nz, n_rescale), dtype=np.float64)
        self.n_loop = np.zeros(nz, dtype=np.int32)
        self.n_scale = np.zeros(nz, dtype=np.int32)
        self.final_demean = np.zeros(nz, dtype=np.float64)
        self.mu = np.full(nz, np.nan, dtype=np.float64)
        self.n_sweeps = 0
        self.n_steps = np.zeros(nz, dtype=np.int32)
        self.has_final = np.zeros(nz, dtype=np.int32)

    @staticmethod
    def record_doubles(n_rescale):
        """Doubles per level of the device record (the C-ABI's
        steam_bounded_add_ledger_doubles)."""
        return 7 + 2 * int(n_rescale)

    @classmethod
    def from_device(cls, packed, n_rescale=10):
        R = int(n_rescale)
        packed = np.asarray(packed, dtype=np.float64).reshape(-1, cls.record_doubles(R))
        out = cls(packed.shape[0], R)
        out.a0[:] = packed[:, 0]
        out.n_loop[:] = packed[:, 1].astype(np.int32)
        out.final_demean[:] = packed[:, 2]
        out.mu[:] = packed[:, 3]
        out.n_sweeps = int(packed[0, 4]) if packed.shape[0] else 0
        out.n_steps[:] = packed[:, 5].astype(np.int32)
        out.has_final[:] = packed[:, 6].astype(np.int32)
        out.demean[:] = packed[:, 7:7 + R]
        out.scale[:] = packed[:, 7 + R:7 + 2 * R]
        steps = np.arange(R)[None, :]
        out.n_scale[:] = np.count_nonzero((out.scale != 1.0) & (steps < out.n_steps[:, None]),
                                          axis=1)
        return out

    def to_device(self):
        """The packed per-level record the replay entry points read."""
        nz, R = self.demean.shape
        packed = np.zeros((nz, self.record_doubles(R)), dtype=np.float64)
        packed[:, 0] = self.a0
        packed[:, 1] = self.n_loop
        packed[:, 2] = self.final_demean
        packed[:, 3] = self.mu
        packed[:, 4] = self.n_sweeps
        packed[:, 5] = self.n_steps
        packed[:, 6] = self.has_final
        packed[:, 7:7 + R] = self.demean
        packed[:, 7 + R:7 + 2 * R] = self.scale
        return packed

    @property
    def n_rescale(self):
        return self.demean.shape[1]

    @property
    def clip_only(self):
        return self.a0 <= 0.0

    @property
    def bisected(self):
        return ~np.isnan(self.mu)


class ProjectionLedger:
    """Per-level projection shift, NaN where untouched (steam/ledger.py:197-212)."""

    __slots__ = ('mu',)

    def __init__(self, mu):
        self.mu = np.asarray(mu, dtype=np.float64)

    @property
    def violating(self):
        return ~np.isnan(self.mu)


class FluxOutputLedger:
    """Clip-and-restore of the composed flux (steam/ledger.py:215-229)."""

    __slots__ = ('entering', 'realized')

    def __init__(self, entering, realized):
        self.entering = entering
        self.realized = realized

    @property
    def rescale(self):
        realized = self.realized.mean
        if realized > 0:
            return np.float32(self.entering.mean / realized)
        return None


class ClassLedger:
    __slots__ = ('flux', 'pattern', 'bounded_add')

    def __init__(self):
        self.flux = None
        self.pattern = {}
        self.bounded_add = {}


class RunLedger:
    """One ClassLedger per size class plus the composition (steam/ledger.py:240-270)."""

    __slots__ = ('classes', 'projection', 'flux_output')

    def __init__(self, n_classes):
        self.classes = [ClassLedger() for _ in range(n_classes)]
        self.projection = {}
        self.flux_output = None
