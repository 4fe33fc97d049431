"""Generates tests/golden/sobol_golden.json.

A Python restatement of the reference's own CPU sampler oracle,
tests/unit/sobolReference.ts:1-63 (hash, seed, reverse, owen, sobol2D, morton2,
zIndex, referenceSample), evaluated on fixed inputs.  The C++ oracle and the
CUDA sampler are checked against these vectors; the properties asserted by
tests/unit/sobol.test.ts:15-90 are re-checked in tests/test_sampler_golden.py.

Run: python tests/golden/make_sobol_golden.py
"""
import json
import os

M = 0xFFFFFFFF
Z_PERMS = [[0, 1, 2, 3], [0, 1, 3, 2], [0, 2, 1, 3], [0, 2, 3, 1], [0, 3, 2, 1], [0, 3, 1, 2], [1, 0, 2, 3],
           [1, 0, 3, 2], [1, 2, 0, 3], [1, 2, 3, 0], [1, 3, 2, 0], [1, 3, 0, 2], [2, 1, 0, 3], [2, 1, 3, 0],
           [2, 0, 1, 3], [2, 0, 3, 1], [2, 3, 0, 1], [2, 3, 1, 0], [3, 1, 2, 0], [3, 1, 0, 2], [3, 2, 1, 0],
           [3, 2, 0, 1], [3, 0, 2, 1], [3, 0, 1, 2]]
Z_PERM_VALUES = [sum(d << (2 * i) for i, d in enumerate(p)) for p in Z_PERMS]


def imul(a, b):
    return (a * b) & M


def hash32(x):
    x &= M
    x = imul(x ^ (x >> 16), 0x7FEB352D)
    x = imul(x ^ (x >> 15), 0x846CA68B)
    return (x ^ (x >> 16)) & M


def seed(a, b):
    return hash32(a ^ hash32((b + 0x9E3779B9) & M))


def reverse(x):
    x &= M
    x = ((x & 0x55555555) << 1 | (x >> 1) & 0x55555555) & M
    x = ((x & 0x33333333) << 2 | (x >> 2) & 0x33333333) & M
    x = ((x & 0x0F0F0F0F) << 4 | (x >> 4) & 0x0F0F0F0F) & M
    x = ((x & 0x00FF00FF) << 8 | (x >> 8) & 0x00FF00FF) & M
    return ((x << 16) | (x >> 16)) & M


def owen(x, s):
    x = (reverse(x) + s) & M
    for c in (0x6C50B47C, 0xB82F1E52, 0xC7AFE638, 0x8D22F6E6):
        x ^= imul(x, c)
    return reverse(x)


def sobol2d_bits(index, s):
    i = owen(index, seed(s, 0))
    x = owen(reverse(i), seed(s, 1))
    y, v = 0, 0x80000000
    while i:
        if i & 1:
            y ^= v
        i >>= 1
        v ^= v >> 1
    return x >> 8, owen(y, seed(s, 2)) >> 8


def morton2(x, y, bits=8):
    r = 0
    for b in range(bits):
        r |= ((x >> b) & 1) << (2 * b) | ((y >> b) & 1) << (2 * b + 1)
    return r & M


def z_index(m, dim, log_spp, tile_bits=8):
    odd = log_spp & 1
    digits = tile_bits + ((log_spp + 1) >> 1)
    r = 0
    for d in range(digits - 1, odd - 1, -1):
        shift = 2 * d - odd
        higher = (m >> (shift + 2)) if shift < 30 else 0
        p = (hash32(higher ^ imul(0x55555555, dim)) >> 24) % 24
        r |= ((Z_PERM_VALUES[p] >> (2 * ((m >> shift) & 3))) & 3) << shift
    if odd:
        r |= (m & 1) ^ (hash32((m >> 1) ^ imul(0x55555555, dim)) & 1)
    return r & M


def reference_sample_bits(pattern, px, py, width, index, dim, log, seq_seed):
    s = seed(seed((px + py * width) & M, dim), seq_seed)
    if pattern == "zsobol":
        first = index == 0
        lg = 0 if first else log
        ordinal = 0 if first else (index - 1) & M
        block = (ordinal >> lg) + (0 if first else 1)
        index = z_index(((morton2(px, py) << lg) | (ordinal & ((1 << lg) - 1))) & M, dim, lg)
        s = seed(seed(dim, seq_seed), seed(px >> 8, py >> 8))
        s = seed(s, block)
    return sobol2d_bits(index, s)


def main():
    out = {"hash": [], "owen": [], "sobol2d": [], "zindex": [], "samples": []}
    for x in [0, 1, 2, 77, 12345, 0x9E3779B9, 0xFFFFFFFF, 0x80000000]:
        out["hash"].append([x, hash32(x)])
    for x, s in [(0, 0), (1, 77), (4095, 77), (12345, 0xDEADBEEF), (0xFFFFFFFF, 5)]:
        out["owen"].append([x, s, owen(x, s)])
    for s in [0, 1, 12345, 0xFFFFFFFF]:
        for i in [0, 1, 2, 3, 7, 100, 1023, 65535]:
            out["sobol2d"].append([i, s, *sobol2d_bits(i, s)])
    for m, dim, lg in [(0, 0, 0), (5, 1, 3), (0x1234, 9, 4), (0xFFFFFFFF, 0, 16), (777, 0x80000001, 7)]:
        out["zindex"].append([m, dim, lg, z_index(m, dim, lg)])
    for pattern in ("sobol", "zsobol"):
        for px, py in [(0, 0), (255, 256), (512, 91)]:
            for index in [0, 1, 17, 65536]:
                for dim in [0, 14, 0x80001234]:
                    out["samples"].append([pattern, px, py, 1024, index, dim, 6, 11,
                                           *reference_sample_bits(pattern, px, py, 1024, index, dim, 6, 11)])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sobol_golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=0)
    print(path)


if __name__ == "__main__":
    main()
