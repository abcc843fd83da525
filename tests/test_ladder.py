"""SCF precision ladder (CPU): the reference's JkLadder unit tests
(ferric-scf/src/jk_ladder.rs:502-610), restated."""
import numpy as np

from ferric_b200.ladder import REDO_IN_F64, JkLadder, rms_diff


def test_a_settled_density_latches_f64_one_way():
    l = JkLadder()
    assert not l.decide(False, None)          # first build: f64
    assert not l.latched_f64
    assert l.decide(True, 1e-2) and l.decide(True, 1e-3)
    assert not l.decide(False, 1e-6)          # settled after mixed: latched
    assert l.latched_f64
    assert not l.decide(True, 1e-4)           # moving again: still f64
    assert not l.decide(False, 1e-7)


def test_a_density_change_that_stops_shrinking_latches_f64():
    l = JkLadder()
    assert not l.decide(False, None)
    assert l.decide(True, 1e-2)
    assert l.decide(True, 3e-3)
    assert l.decide(True, 2.9e-3)             # barely shrinking is still shrinking
    assert not l.latched_f64
    assert not l.decide(True, 2.9e-3)         # not shrinking: f64
    assert l.latched_f64
    assert not l.decide(True, 1e-3)
    m = JkLadder()
    assert not m.decide(False, None)
    assert m.decide(True, 1e-3)
    assert not m.decide(False, float("nan")) and m.latched_f64


def test_only_a_mixed_build_vetoes_the_exit():
    l = JkLadder()
    assert l.veto_mixed_exit(1) == 1           # no kernel ran mixed: the exit stands
    l.note_mixed_build(dfj=True)
    assert l.veto_mixed_exit(None) is None     # a non-exit is untouched
    assert not l.latched_f64
    l.note_mixed_build(dfj=True)
    assert l.veto_mixed_exit(2) == REDO_IN_F64
    assert l.latched_f64
    assert l.veto_mixed_exit(3) == 3


def test_first_build_is_f64_and_density_step():
    l = JkLadder(thresh=1e-5)
    d0 = np.eye(4)
    assert not l.begin_build([d0])             # first build of the SCF
    assert l.begin_build([d0 + 1e-3])          # moved by 1e-3 > tau
    assert abs(l.last_change - 1e-3) < 1e-15
    assert not l.begin_build([d0 + 1e-3 + 1e-7])   # settled: latched
    assert l.latched_f64
    assert rms_diff(np.zeros(4), np.full(4, 2.0)) == 2.0


def test_inert_without_df_or_request():
    assert not JkLadder(has_df=False).begin_build([np.eye(2)])
    l = JkLadder(mixed_requested=False)
    l.begin_build([np.eye(2)])
    assert not l.begin_build([np.eye(2) * 2])
