"""Host logic of the drag API that needs no GPU: the hysteretic regime controller
(drag.jl:5-76, checked as in test/inherited/test_terminal_ct.jl:387-411)."""
import pytest

import pmfmhd


def test_drag_regime_default_thresholds():
    c = pmfmhd.DragRegimeController()
    assert c.exit_drag_over_omega == 1 and c.enter_drag_over_omega == 2
    assert pmfmhd.update_drag_regime(c, 3, 0.1)[0]


def test_drag_regime_hysteresis_is_one_way_by_default():
    c = pmfmhd.DragRegimeController(exit_drag_over_omega=8, enter_drag_over_omega=16, confirm_checks=2)
    assert pmfmhd.update_drag_regime(c, 20, 0.1) == (True, "none")
    assert pmfmhd.update_drag_regime(c, 7.9, 0.1) == (True, "none")
    assert pmfmhd.update_drag_regime(c, 8.1, 0.1) == (True, "none")
    assert pmfmhd.update_drag_regime(c, 7.9, 0.1) == (True, "none")
    assert pmfmhd.update_drag_regime(c, 7.8, 0.1) == (False, "terminal_to_full")
    assert pmfmhd.update_drag_regime(c, 32, 0.1) == (False, "none")


def test_drag_regime_reentry_needs_consecutive_votes():
    c = pmfmhd.DragRegimeController(exit_drag_over_omega=8, enter_drag_over_omega=16, confirm_checks=2,
                                    reenter_terminal=True)
    assert pmfmhd.update_drag_regime(c, 4, 0.1)[0] is False
    assert pmfmhd.update_drag_regime(c, 17, 0.1) == (False, "none")
    assert pmfmhd.update_drag_regime(c, 18, 0.1) == (True, "full_to_terminal")


def test_drag_regime_magnetisation_gate_and_errors():
    c = pmfmhd.DragRegimeController(min_va_over_cs=1.0)
    assert pmfmhd.update_drag_regime(c, 50, 0.5) == (False, "none")
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.DragRegimeController(exit_drag_over_omega=2, enter_drag_over_omega=1)
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.DragRegimeController(confirm_checks=0)
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.DragRegimeController(min_va_over_cs=-1)
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.update_drag_regime(c, float("nan"), 0.1)
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.update_drag_regime(c, 1.0, -0.1)
