"""Owen-scrambled Sobol / ZSobol of the oracle against the reference's own
CPU sampler oracle (restated in tests/golden/make_sobol_golden.py) and the
properties of tests/unit/sobol.test.ts:15-90."""
import json
import os

import numpy as np

from tests import oracle_lib
from tests.golden import make_sobol_golden as ref

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sobol_golden.json")
EPS = np.float32(0.0005)
SCALE = np.float32(0.999)


def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def oracle_sobol2d_bits(i, s):
    L = oracle_lib.lib()
    ii = L.oracle_owen(i, L.oracle_sample_seed(s, 0))
    x = L.oracle_owen(L.oracle_reverse_bits(ii), L.oracle_sample_seed(s, 1))
    y = L.oracle_owen(L.oracle_sobol_d1(ii), L.oracle_sample_seed(s, 2))
    return x >> 8, y >> 8


def test_golden_file_is_reproducible():
    g = golden()
    for x, h in g["hash"]:
        assert ref.hash32(x) == h


def test_hash_and_owen_match_golden():
    L = oracle_lib.lib()
    g = golden()
    for x, h in g["hash"]:
        assert L.oracle_sample_hash(x) == h
    for x, s, o in g["owen"]:
        assert L.oracle_owen(x, s) == o


def test_sobol2d_matches_golden():
    for i, s, x, y in golden()["sobol2d"]:
        assert oracle_sobol2d_bits(i, s) == (x, y)


def test_zsobol_index_matches_golden():
    L = oracle_lib.lib()
    for m, dim, lg, want in golden()["zindex"]:
        assert L.oracle_zsobol_index(m, dim, lg) == want


def test_structured_samples_match_reference_sample():
    import ctypes as C
    L = oracle_lib.lib()
    out = (C.c_float * 2)()
    for pattern, px, py, width, index, dim, lg, seq, bx, by in golden()["samples"]:
        L.oracle_structured_sample(px, py, width, index, dim, seq, 1 if pattern == "zsobol" else 0, lg, out)
        want = EPS + SCALE * (np.float32([bx, by]) * np.float32(1.0 / 16777216.0))
        assert np.array_equal(np.float32([out[0], out[1]]), want.astype(np.float32)), (pattern, px, py, index, dim)


def _net(points, k):
    pts = np.asarray(points)
    assert ((pts >= 0) & (pts < 1)).all()
    for a in range(k + 1):
        cells = np.floor(pts[:, 0] * 2 ** a).astype(np.int64) + np.floor(pts[:, 1] * 2 ** (k - a)).astype(np.int64) * 2 ** a
        counts = np.bincount(cells, minlength=2 ** k)
        assert (counts == 1).all()


def test_progressive_nets():
    # sobol.test.ts:15-20: every elementary interval of each 2^k prefix holds one point.
    for s in (0, 1, 12345, 0xFFFFFFFF):
        for k in range(0, 9):
            pts = [np.array(oracle_sobol2d_bits(i, s)) / 16777216.0 for i in range(2 ** k)]
            _net(pts, k)
    assert oracle_sobol2d_bits(0, 1) != oracle_sobol2d_bits(0, 2)


def test_owen_bijective_and_nested():
    L = oracle_lib.lib()
    values = [L.oracle_owen(i, 77) for i in range(4096)]
    assert len(set(values)) == len(values)
    assert len({v >> 12 for v in values}) == 1


def test_butterfly_equals_direction_recurrence():
    L = oracle_lib.lib()

    def naive(index):
        r, v = 0, 0x80000000
        while index:
            if index & 1:
                r ^= v
            index >>= 1
            v ^= v >> 1
        return r

    inputs = [0, 0xFFFFFFFF] + [(1 << i) & 0xFFFFFFFF for i in range(32)] + \
        [(i * 0x9E3779B9) & 0xFFFFFFFF for i in range(2048)]
    for i in inputs:
        assert L.oracle_sobol_d1(i) == naive(i)


def test_zsobol_pixel_nets_and_first_sample_policy():
    # Each pixel's ZSobol indices form a 2D net; sample 0 is independent of the
    # planned budget (sobol.test.ts:24-35, 53-62).
    L = oracle_lib.lib()
    for k in range(0, 5):
        for dim in (0, 1, 9):
            idx = [L.oracle_zsobol_index((L.oracle_morton2(3, 2) << k) | i, dim, k) for i in range(2 ** k)]
            mask = (1 << k) - 1
            low = sorted(v & mask for v in idx)
            assert low == list(range(2 ** k))
    import ctypes as C
    out = (C.c_float * 2)()
    firsts = set()
    for lg in (0, 1, 4, 16):
        L.oracle_structured_sample(255, 256, 1024, 0, 14, 11, 1, lg, out)
        firsts.add((out[0], out[1]))
    assert len(firsts) == 1
    L.oracle_structured_sample(255, 256, 1024, 1, 14, 11, 1, 4, out)
    assert (out[0], out[1]) not in firsts
