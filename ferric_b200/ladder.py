"""The SCF precision ladder for the mixed DF-J / DF-K device builds.

Restates ``JkLadder`` (ferric-scf/src/jk_ladder.rs:312-430) and the density
step of ``PrecisionLadder::step_with`` (ferric-core/src/precision_ladder.rs:150-190):

* a build may run mixed only when mixed was requested, a previous build of the
  same SCF exists, and some spin density moved by more than ``thresh`` (RMS
  over the AO matrix) since it -- the first build of every SCF is FP64;
* one way: the first build that finds the density settled (moved by at most
  ``thresh``) or not contracting (change >= the previous mixed build's) after a
  mixed build latches the SCF to FP64 for good;
* the FP64 exit: a converged exit whose last build ran mixed is refused
  (``REDO_IN_F64``); the ladder latches and the solver must reset DIIS,
  invalidate its deltas and rebuild J/K in FP64 at the same density.

Host control only; the device builders take the decision through
``DfJK.set_precision`` (``fc_dfjk_set_precision``).
"""
from __future__ import annotations

import math

import numpy as np

JK_LADDER_THRESH = 1e-5
REDO_IN_F64 = "redo_in_f64"


def rms_diff(a, b):
    """RMS of a - b over all elements (``rms_diff``, precision_ladder.rs:226-233)."""
    a = np.asarray(a)
    n = max(a.size, 1)
    return math.sqrt(float(np.sum((a - np.asarray(b)) ** 2)) / n)


class JkLadder:
    def __init__(self, has_df=True, mixed_requested=True, thresh=JK_LADDER_THRESH):
        self.has_df = bool(has_df)
        self.mixed_requested = bool(mixed_requested)
        self.thresh = float(thresh)
        self._prev_ds = None
        self.last_change = None
        self.latched_f64 = False
        self._allowed_mixed = False
        self._prev = (False, None)
        self._ran_mixed = None   # which kernels of the current build ran mixed

    # -- density step (PrecisionLadder::step_with) -------------------------
    def _step(self, ds):
        self._ran_mixed = None
        self.last_change = None
        prev = self._prev_ds
        same = prev is not None and len(prev) == len(ds) and all(p.shape == d.shape for p, d in zip(prev, ds))
        moving = False
        if same:
            diffs = [rms_diff(p, d) for p, d in zip(prev, ds)]
            self.last_change = float("nan") if any(math.isnan(x) for x in diffs) else max(diffs)
            moving = any(x > self.thresh for x in diffs)
        self._prev_ds = [np.array(d, dtype=np.float64, copy=True) for d in ds]
        return moving

    # -- the decision (JkLadder::decide) -----------------------------------
    def decide(self, moving, change):
        prev_mixed, prev_change = self._prev
        stalled = prev_mixed and prev_change is not None and change is not None and change >= prev_change
        if (not moving or stalled) and self._allowed_mixed:
            self.latched_f64 = True
        mixed = bool(moving) and not self.latched_f64
        if mixed:
            self._allowed_mixed = True
        self._prev = (mixed, change)
        return mixed

    def begin_build(self, ds):
        """Step with this build's spin densities; True = this build may run mixed."""
        if not self.has_df or not self.mixed_requested:
            return False
        moving = self._step(ds)
        return self.decide(moving, self.last_change)

    def note_mixed_build(self, dfj=False, dfk=False):
        """A device kernel of the current build ran mixed (the dispatchers' record)."""
        if self.latched_f64:
            raise AssertionError("a J/K build ran mixed after the ladder latched to f64")
        if dfj or dfk:
            prev = self._ran_mixed or (False, False)
            self._ran_mixed = (prev[0] or dfj, prev[1] or dfk)

    def veto_mixed_exit(self, conv):
        """``conv``: the solver's converged-exit decision (None = not converged).
        Returns ``conv`` to proceed, or ``REDO_IN_F64`` when the build ran mixed."""
        if conv is None:
            return None
        ran, self._ran_mixed = self._ran_mixed, None
        if ran is None:
            return conv
        self.latched_f64 = True
        return REDO_IN_F64
