"""Host logic of the autotuner's table (no GPU)."""
from traceon_b200 import autotune


def test_size_buckets():
    assert [autotune._bucket(x) for x in (0, 1, 2, 3, 1000, 1024, 1025)] == [0, 1, 2, 4, 1024, 1024, 2048]


def test_table_is_copied_and_cleared():
    autotune.clear()
    with autotune._lock:
        autotune._table[('k',)] = 4
    t = autotune.table()
    t[('k',)] = 8
    assert autotune.table() == {('k',): 4}
    autotune.clear()
    assert autotune.table() == {}
