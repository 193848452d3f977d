"""The wavefront filter's layout and schedule on the CPU (no GPU): the host
functions the kernels run (pEVSL_B200_WaveLayout / WaveItem / WaveTerms).

* Layout: chunks tile the rows, start on multiples of 4 rows, hold at most
  256 rows and (unless one 4-row group alone exceeds it) 4096 entries; for
  every entry (row r, column j) the chunk of j lies in the dependency range
  of r's chunk and vice versa -- the wavefront waits on those ranges before
  gathering from a chunk or overwriting it.
* Schedule: the claim index -> (degree offset, chunk) map is a bijection,
  and every item's dependencies (the previous degree on the chunks within
  the reach) have smaller claim indices, which is what makes the wait of the
  smallest unfinished item always end.
* Deferral: the closed-form schedule equals the degree loop's (update at
  degree min(defer, 2), then every `defer` degrees, and at the last).
"""
import ctypes as C

import numpy as np
import pytest


def lib():
    import pevsl_b200
    return pevsl_b200.load()


def layout(n, ia, ja):
    L = lib()
    nc, reach = C.c_int(), C.c_int()
    ia = np.ascontiguousarray(ia, np.int32)
    ja = np.ascontiguousarray(ja, np.int32)
    P = lambda x: x.ctypes.data_as(C.c_void_p)  # noqa: E731
    assert L.pEVSL_B200_WaveLayout(n, P(ia), P(ja), C.byref(nc), None, None, C.byref(reach)) == 0
    ch = np.zeros(2 * nc.value + 2, np.int32)
    dep = np.zeros(2 * nc.value, np.int32)
    assert L.pEVSL_B200_WaveLayout(n, P(ia), P(ja), C.byref(nc), P(ch), P(dep), C.byref(reach)) == 0
    return nc.value, ch.reshape(-1, 2), dep.reshape(-1, 2), reach.value


def random_pattern(n, seed, band, heavy=()):
    rng = np.random.default_rng(seed)
    rows, cols = [np.arange(n)], [np.arange(n)]
    for _ in range(3):
        off = rng.integers(-band, band + 1, size=n)
        c = np.arange(n) + off
        keep = (c >= 0) & (c < n)
        rows.append(np.arange(n)[keep])
        cols.append(c[keep])
    for h, cnt in heavy:
        rows.append(np.full(cnt, h))
        cols.append(rng.integers(0, n, size=cnt))
    r, c = np.concatenate(rows), np.concatenate(cols)
    key = np.unique(r.astype(np.int64) * n + c)   # unsymmetric on purpose
    r, c = key // n, key % n
    ia = np.zeros(n + 1, np.int64)
    np.add.at(ia, r + 1, 1)
    return np.cumsum(ia).astype(np.int32), c.astype(np.int32)


@pytest.mark.parametrize("n,band,heavy", [(10007, 40, ()), (3000, 1500, ()),
                                          (20001, 300, ((7000, 3000), (7001, 3000))),
                                          (5, 2, ()), (1, 0, ())])
def test_layout_covers_every_dependency(n, band, heavy):
    ia, ja = random_pattern(n, n + band, band, heavy)
    nc, ch, dep, reach = layout(n, ia, ja)
    starts = ch[:, 0]
    assert starts[0] == 0 and starts[-1] == n and np.all(np.diff(starts) > 0)
    assert np.all(starts[:-1] % 4 == 0) and np.all(np.diff(starts) <= 256)
    assert np.array_equal(ch[:, 1], ia[starts])
    big = np.diff(ch[:, 1]) > 4096
    assert np.all(np.diff(starts)[big] <= 4)  # only a lone 4-row group may exceed
    rows = np.repeat(np.arange(n), np.diff(ia))
    rc = np.searchsorted(starts[:-1], rows, side="right") - 1
    cc = np.searchsorted(starts[:-1], ja, side="right") - 1
    assert np.all((dep[rc, 0] <= cc) & (cc <= dep[rc, 1]))  # gathers
    assert np.all((dep[cc, 0] <= rc) & (rc <= dep[cc, 1]))  # readers of rows it overwrites
    assert reach == max(np.max(np.arange(nc) - dep[:, 0]), np.max(dep[:, 1] - np.arange(nc)))


@pytest.mark.parametrize("nc,D,reach,grid", [(3907, 8, 40, 444), (275, 8, 119, 444),
                                             (10, 3, 9, 5), (1, 1, 0, 1), (5, 8, 2, 100),
                                             (977, 4, 10, 296)])
def test_claim_order_is_a_bijection_and_respects_dependencies(nc, D, reach, grid):
    L = lib()
    Lp = reach + 1 + grid // D
    j, c = C.c_int(), C.c_int()
    index = {}
    for idx in range(nc * D):
        assert L.pEVSL_B200_WaveItem(nc, D, Lp, idx, C.byref(j), C.byref(c)) == 0
        key = (j.value, c.value)
        assert 0 <= key[0] < D and 0 <= key[1] < nc and key not in index
        index[key] = idx
    assert len(index) == nc * D
    for (jj, cc), idx in index.items():
        if jj:
            lo, hi = max(0, cc - reach), min(nc - 1, cc + reach)
            assert max(index[(jj - 1, q)] for q in range(lo, hi + 1)) < idx
    assert L.pEVSL_B200_WaveItem(nc, D, Lp, nc * D, C.byref(j), C.byref(c)) != 0


def test_deferral_schedule_matches_the_degree_loop():
    L = lib()
    fresh = C.c_int()
    for defer in (1, 2, 3):
        for maxdeg in range(1, 80):
            lastw = 0
            for k in range(1, maxdeg + 1):
                span = min(defer, 2) if lastw == 0 else defer
                ny = k - lastw if (k == maxdeg or k - lastw == span) else 0
                got = L.pEVSL_B200_WaveTerms(k, maxdeg, defer, C.byref(fresh))
                assert (got, fresh.value) == (ny, int(ny > 0 and lastw == 0)), (defer, maxdeg, k)
                if ny:
                    lastw = k
