"""Host logic of the multi-problem driver (no GPU)."""
import pytest

from isg.multi import level_of


def test_level_of_grid_sizes():
    assert [level_of(n * n) for n in (32, 64, 128, 256, 512, 1024, 4096)] == [3, 4, 5, 6, 7, 8, 10]
    for bad in (100, 24 * 24, 96 * 96):
        with pytest.raises(ValueError):
            level_of(bad)
