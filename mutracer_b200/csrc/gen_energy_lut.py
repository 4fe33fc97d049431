"""Writes openpbr_energy_lut.f32: the OpenPBR energy-compensation table the
reference's BSDF samples (32 x 2177 R32F, little-endian float32, row-major).

The numbers are Adobe's OpenPBR tabulations (adobe/openpbr-bsdf, Apache
License 2.0, Copyright 2026 Adobe): the opaque-dielectric albedo complement,
the ideal-metal complement and its averages, and the ideal-dielectric loss,
averages and reflection ratio.  The reference (src/renderer/openPbrEnergyLut.ts)
stores them re-quantised and delta-coded in base64 strings and decodes them
when its module loads (src/renderer/decodeOpenPbrEnergyLut.ts:35-83).  This
script reads those strings from the reference's source file and decodes them
with the same arithmetic, so the committed table holds exactly the float32
values the reference uploads:

* rows 0..2176 except the averaged ones: per row a little-endian u16 min and
  max (added modulo 65536 to the previous row's) and 32 u8 samples (added
  modulo 256 to the previous row's), the value being
  (min + (max - min) * sample / 255) / 65535 in float64, stored as float32;
* the metal averages (row 1088, 32 values) and dielectric averages (rows
  2113..2144) from exact u16 values / 65535;
* then row 1088 replaced by the exact integral of 2*mu times each
  piecewise-linear metal row (decodeOpenPbrEnergyLut.ts:72-81), accumulated in
  float64 in the reference's order.

tests/test_energy_lut.py checks the committed file against the SHA-256 digests
and UNORM anchors of the reference's tests/unit/openPbrEnergyLut.test.ts.

Run (needs the reference source tree):
  python mutracer_b200/csrc/gen_energy_lut.py /root/reference/src/renderer/openPbrEnergyLut.ts
"""
import base64
import os
import re
import sys

import numpy as np

WIDTH = 32
HEIGHT = 2177
METAL_ROW = 1056
METAL_AVERAGE_ROW = 1088
DIELECTRIC_AVERAGE_ROW = 2113
REFLECTION_RATIO_ROW = 2145

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "openpbr_energy_lut.f32")

NAMES = ("OPENPBR_ENERGY_LUT_ROW_DELTA_BASE64", "OPENPBR_METAL_ENERGY_LUT_ROW_DELTA_BASE64",
         "OPENPBR_DIELECTRIC_ENERGY_LUT_ROW_DELTA_BASE64", "OPENPBR_METAL_AVERAGE_U16_BASE64",
         "OPENPBR_DIELECTRIC_AVERAGE_U16_BASE64")


def read_strings(path):
    """The five base64 constants of openPbrEnergyLut.ts, each the
    concatenation of the string literals in its initialiser."""
    text = open(path, encoding="utf-8").read()
    out = {}
    for name in NAMES:
        m = re.search(r"const\s+" + name + r"\s*=(.*?);", text, re.S)
        if not m:
            raise ValueError(f"{name} not found in {path}")
        out[name] = "".join(re.findall(r'"([A-Za-z0-9+/=]*)"', m.group(1)))
    return out


def decode(strings):
    encoded = b"".join(base64.b64decode(strings[n]) for n in NAMES[:3])
    averages = base64.b64decode(strings[NAMES[3]]) + base64.b64decode(strings[NAMES[4]])
    data = np.zeros(WIDTH * HEIGHT, dtype=np.float32)
    lo = hi = 0
    samples = [0] * WIDTH
    encoded_row = 0
    for row in range(HEIGHT):
        if row == METAL_AVERAGE_ROW or DIELECTRIC_AVERAGE_ROW <= row < REFLECTION_RATIO_ROW:
            continue
        at = encoded_row * (WIDTH + 4)
        encoded_row += 1
        lo = (lo + (encoded[at] | (encoded[at + 1] << 8))) & 65535
        hi = (hi + (encoded[at + 2] | (encoded[at + 3] << 8))) & 65535
        for column in range(WIDTH):
            samples[column] = (samples[column] + encoded[at + 4 + column]) & 255
            data[row * WIDTH + column] = np.float32((lo + (hi - lo) * samples[column] / 255) / 65535)
    if encoded_row * (WIDTH + 4) != len(encoded):
        raise ValueError("encoded row count does not match the table shape")
    for index in range(32 + 32 * 32):
        value = (averages[index * 2] | (averages[index * 2 + 1] << 8)) / 65535
        offset = (METAL_AVERAGE_ROW * 32 + index if index < 32
                  else DIELECTRIC_AVERAGE_ROW * 32 + index - 32)
        data[offset] = np.float32(value)
    h = 1 / (WIDTH - 1)
    for row in range(WIDTH):
        offset = (METAL_ROW + row) * WIDTH
        average = 0.0
        for i in range(WIDTH - 1):
            a, b = float(data[offset + i]), float(data[offset + i + 1])
            average += h * (i * h * (a + b) + h * (a + 2 * b) / 3)
        data[METAL_AVERAGE_ROW * WIDTH + row] = np.float32(average)
    return data


def main(argv):
    if len(argv) != 2:
        print(__doc__)
        return 2
    data = decode(read_strings(argv[1]))
    data.astype("<f4").tofile(OUT)
    print(f"wrote {OUT}: {data.size} float32 values")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
