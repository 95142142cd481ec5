"""The memory-system probes that bench.py sets the search kernels against
(lib/libbt_probe.so, a separate library the engine does not link)."""
import pytest

pytestmark = pytest.mark.gpu


def test_gather_probe_measures_and_checks_arguments(bt, cuda):
    r64 = bt.measure_gather(64 << 20, 1 << 20, 64)
    assert 1e8 < r64 < 1e12  # reads per second, a plausible range for any GPU
    with pytest.raises(bt.BTreeError):
        bt.measure_gather(64 << 20, 1 << 20, 48)
    with pytest.raises(bt.BTreeError):
        bt.measure_gather(0, 1 << 20, 64)


def test_chain_probe_measures_and_checks_arguments(bt, cuda):
    for lines in (0, 1, 2):
        r = bt.measure_chain(8 << 20, 256 << 20, 1 << 20, 128, lines, 2)
        assert 1e8 < r < 1e12
    with pytest.raises(bt.BTreeError):
        bt.measure_chain(8 << 20, 256 << 20, 1 << 20, 96, 1, 2)
    with pytest.raises(bt.BTreeError):
        bt.measure_chain(8 << 20, 256 << 20, 1 << 20, 128, 3, 2)


@pytest.mark.parametrize("form", ["lane", "pair", "bulk", "quad", "pair_quad"])
def test_hop_probe_measures_and_checks_arguments(bt, cuda, form):
    for hops in (0, 1, 2, 3):
        r = bt.measure_hops(8 << 20, 256 << 20, 1 << 20, hops, form)
        assert 1e8 < r < 1e12
    with pytest.raises(bt.BTreeError):
        bt.measure_hops(8 << 20, 256 << 20, 1 << 20, 4, form)
