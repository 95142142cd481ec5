"""The random-gather probe that bench.py sets the search kernels against."""
import pytest

pytestmark = pytest.mark.gpu


def test_gather_probe_measures_and_checks_arguments(bt, cuda):
    r64 = bt.measure_gather(64 << 20, 1 << 20, 64)
    assert 1e8 < r64 < 1e12  # reads per second, a plausible range for any GPU
    with pytest.raises(bt.BTreeError):
        bt.measure_gather(64 << 20, 1 << 20, 48)
    with pytest.raises(bt.BTreeError):
        bt.measure_gather(0, 1 << 20, 64)
