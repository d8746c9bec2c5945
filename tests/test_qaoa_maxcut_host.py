"""ruqu-wasm's qaoa_maxcut mirror (ruqu_b200.qaoa.qaoa_maxcut): the argument checks of
crates/ruqu-wasm/src/lib.rs:416-441 need no GPU and raise before any state exists."""
import pytest

from ruqu_b200.qaoa import qaoa_maxcut


def test_argument_checks():
    with pytest.raises(ValueError, match="Qubit limit exceeded"):
        qaoa_maxcut(26, [0, 1], 1, [0.1], [0.2])
    with pytest.raises(ValueError, match="gammas length mismatch"):
        qaoa_maxcut(4, [0, 1], 2, [0.1], [0.2, 0.3])
    with pytest.raises(ValueError, match="betas length mismatch"):
        qaoa_maxcut(4, [0, 1], 1, [0.1], [0.2, 0.3])
    with pytest.raises(ValueError, match="even number"):
        qaoa_maxcut(4, [0, 1, 2], 1, [0.1], [0.2])
