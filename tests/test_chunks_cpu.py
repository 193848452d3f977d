"""The staged filter kernel's row chunks on the CPU (no GPU): the host
function the matrix set-up runs (pEVSL_B200_ChunkLayout).  The chunks tile
the rows in order, start on multiples of 4 rows (so that the bulk copies of
row pointers and vector rows start on 16-byte boundaries), hold at most 256
rows and, unless one 4-row group alone exceeds it, at most 4096 entries (the
size of a stage's entry buffers); every entry belongs to exactly one chunk.
"""
import ctypes as C

import numpy as np
import pytest


def layout(n, ia):
    import pevsl_b200
    L = pevsl_b200.load()
    nc = C.c_int()
    ia = np.ascontiguousarray(ia, np.int32)
    P = lambda x: x.ctypes.data_as(C.c_void_p)  # noqa: E731
    assert L.pEVSL_B200_ChunkLayout(n, P(ia), C.byref(nc), None) == 0
    ch = np.zeros(2 * nc.value + 2, np.int32)
    assert L.pEVSL_B200_ChunkLayout(n, P(ia), C.byref(nc), P(ch)) == 0
    return ch.reshape(-1, 2)


@pytest.mark.parametrize("n,per_row,heavy", [(10007, 7, ()), (3000, 40, ()),
                                             (20001, 17, ((7000, 3000), (7001, 3000))),
                                             (5, 2, ()), (1, 1, ()), (4096, 0, ())])
def test_chunks_tile_rows_within_stage_limits(n, per_row, heavy):
    rng = np.random.default_rng(n + per_row)
    counts = rng.integers(max(0, per_row - 3), per_row + 4, size=n)
    for h, cnt in heavy:
        counts[h] = cnt
    ia = np.zeros(n + 1, np.int64)
    ia[1:] = np.cumsum(counts)
    ch = layout(n, ia)
    starts, first = ch[:, 0], ch[:, 1]
    assert starts[0] == 0 and starts[-1] == n and np.all(np.diff(starts) > 0)
    assert np.all(starts[:-1] % 4 == 0) and np.all(np.diff(starts) <= 256)
    assert np.array_equal(first, ia[starts])
    entries, rows = np.diff(first), np.diff(starts)
    assert np.all((entries <= 4096) | (rows <= 4))   # only a lone 4-row group may exceed
    if heavy:
        assert np.any(entries > 4096)                 # the heavy group is its own chunk
    # a chunk stops only when the next 4-row group would exceed a limit
    for c in range(len(starts) - 2):
        nxt = min(n, starts[c + 1] + 4)
        assert rows[c] == 256 or ia[nxt] - ia[starts[c]] > 4096 or rows[c] <= 4
