"""One solve over several GPUs, host side: the x partition into slabs (as
even as possible, at least three cells each) and argument checks.  No device
is touched."""
import pytest

from sams_b200 import lare


def test_partition_is_even_and_covers_the_grid():
    assert lare.dist_partition(12, 2) == [0, 6, 12]
    assert lare.dist_partition(16, 3) == [0, 6, 11, 16]
    assert lare.dist_partition(256, 8) == [32 * q for q in range(9)]
    off = lare.dist_partition(1001, 7)
    sizes = [b - a for a, b in zip(off, off[1:])]
    assert off[0] == 0 and off[-1] == 1001 and max(sizes) - min(sizes) <= 1


def test_partition_needs_three_cells_per_slab():
    assert lare.dist_partition(9, 3) == [0, 3, 6, 9]
    with pytest.raises(lare.LareError):
        lare.dist_partition(8, 3)
    with pytest.raises(lare.LareError):
        lare.dist_partition(100, 0)
