"""Host-side Grover logic (no GPU): optimal_iterations against the reference's
unit tests (grover.rs:205-228) and test_algorithms.rs:273-305."""
import pytest

from ruqu_b200.grover import optimal_iterations


def test_optimal_iterations_known_answers():
    assert optimal_iterations(3, 1) == 2            # grover.rs:210-212
    assert optimal_iterations(2, 2) >= 1            # grover.rs:218-219
    assert optimal_iterations(1, 1) >= 1            # grover.rs:225-226
    assert 10 <= optimal_iterations(8, 1) <= 15     # test_algorithms.rs:277-282
    assert 7 <= optimal_iterations(8, 2) <= 11      # test_algorithms.rs:288-293
    assert 1 <= optimal_iterations(2, 1) <= 2       # test_algorithms.rs:299-304


def test_optimal_iterations_rounds_halves_away_from_zero():
    # N = 4, M = 2: pi/4 / (pi/4) - 1/2 = 0.5 (to rounding) -> max(round, 1) = 1
    assert optimal_iterations(2, 2) == 1
    assert optimal_iterations(8, 1) == 12


def test_no_targets_is_rejected():
    with pytest.raises(ValueError):
        optimal_iterations(4, 0)
