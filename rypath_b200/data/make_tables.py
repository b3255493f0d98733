"""Extract the fixed data tables the spectral path needs from a rypath checkout.

The tables are third-party data that must be bit-identical to what rypath compiles in,
because the integer sample words, the sensor response and the RGB reconstruction are pinned
to them:

* ``pbrt_sobol_tables.bin`` -- the 234,208-byte ``sobol::Tables`` block (direction
  matrices, interval and inverse tables) that rypath includes from
  ``third_party/pbrt/sobol_tables.inc`` (PBRT v4, Apache-2.0; Joe & Kuo 2008 direction
  numbers as prepared by L. Gruenschloss).  Layout follows ``src/sobol_shared.h:36-52``:
  ``uint32 directions[1024*52]; uint64 intervals[25*52]; uint64 inverse[26*52]``,
  little endian.
* ``cie_xyz_1931.bin`` -- the CIE 1931 2-degree colour matching functions at 1 nm from
  360 to 830 nm (471 rows of x, y, z as float64), from ``third_party/cie`` (CIE 2019,
  CC BY-SA 4.0), i.e. the table rypath generates in ``cmake/CieData.cmake``.
* ``srgb_spectrum.xz`` -- PBRT v4's sRGB-to-spectrum table (Jakob & Hanika 2019
  coefficients; Apache-2.0) that rypath embeds from ``third_party/pbrt/srgb.bin``
  (``cmake/RgbSpectrumData.cmake``): 64 z nodes then 3 x 64^3 cells of 3 quadratic
  coefficients, binary32.  Stored byte-planed (every float's byte 0, then byte 1, ...) and
  xz-compressed; ``rgb_table()`` in ``rypath_b200/images.py`` restores it and checks the
  SHA-256 that rypath's extraction script pins.
* ``ewa_weights.bin`` -- PBRT v4's 128-entry EWA filter table (``MIPFilterLUT`` of
  ``src/pbrt/util/mipmap.cpp``; Apache-2.0), as rypath carries it in ``src/ewa_weights.h``:
  128 binary32.
* ``d65_dense.bin`` -- PBRT's luminance-normalised stdillum-D65 at 360..830 nm in 1 nm
  steps (471 binary32), the ``pbrt_d65()`` table of ``src/rgb_spectrum.hpp``, from
  ``third_party/pbrt/d65.inc``.

Usage: ``python make_tables.py /path/to/rypath`` (writes next to this script).
"""

import lzma
import os
import re
import struct
import sys
from pathlib import Path

SOBOL_WORDS = 1024 * 52
INTERVAL_WORDS = 25 * 52
INVERSE_WORDS = 26 * 52
SOBOL_BYTES = 234208


def _strip_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def sobol_tables(reference: Path) -> bytes:
    text = _strip_comments((reference / "third_party/pbrt/sobol_tables.inc").read_text())
    literals = re.findall(r"\b(0[xX][0-9a-fA-F]+|\d+)(?:[uU]?[lL]{0,2}|[lL]{1,2}[uU]?)\b", text)
    values = [int(v, 0) for v in literals]
    expected = SOBOL_WORDS + INTERVAL_WORDS + INVERSE_WORDS
    if len(values) != expected:
        raise SystemExit(f"expected {expected} integers in sobol_tables.inc, found {len(values)}")
    directions = values[:SOBOL_WORDS]
    rest = values[SOBOL_WORDS:]
    blob = struct.pack(f"<{SOBOL_WORDS}I", *directions)
    blob += struct.pack(f"<{INTERVAL_WORDS + INVERSE_WORDS}Q", *rest)
    if len(blob) != SOBOL_BYTES:
        raise SystemExit("unexpected Sobol table size")
    return blob


def cie_table(reference: Path) -> bytes:
    rows = (reference / "third_party/cie/CIE_xyz_1931_2deg.csv").read_text().split()
    values = []
    for expected_nm, row in zip(range(360, 831), rows):
        fields = row.split(",")
        if int(fields[0]) != expected_nm:
            raise SystemExit("CIE table rows are not 360..830 nm at 1 nm")
        values.extend(float(v) for v in fields[1:4])
    if len(values) != 471 * 3:
        raise SystemExit("CIE table must have 471 rows")
    return struct.pack("<1413d", *values)


SRGB_SHA256 = "6adffc41eefcf064b6524606cb8734941aa69ac962ac268fd9276f440cef61d5"
SRGB_BYTES = 4 * (64 + 3 * 64 ** 3 * 3)


def srgb_table(reference: Path) -> bytes:
    import hashlib

    blob = (reference / "third_party/pbrt/srgb.bin").read_bytes()
    if len(blob) != SRGB_BYTES or hashlib.sha256(blob).hexdigest() != SRGB_SHA256:
        raise SystemExit("srgb.bin is not the pinned PBRT sRGB table")
    planes = b"".join(blob[k::4] for k in range(4))
    return lzma.compress(planes, preset=9 | lzma.PRESET_EXTREME)


def d65_table(reference: Path) -> bytes:
    text = _strip_comments((reference / "third_party/pbrt/d65.inc").read_text())
    values = [float.fromhex(v) for v in re.findall(r"([-+]?0x[0-9a-fA-F.]+p[-+]?\d+)f", text)]
    if len(values) != 471:
        raise SystemExit(f"expected 471 D65 values in d65.inc, found {len(values)}")
    return struct.pack("<471f", *values)


def ewa_table(reference: Path) -> bytes:
    text = _strip_comments((reference / "src/ewa_weights.h").read_text())
    body = text[text.index("weights[128] = {"):]
    values = [float(v) for v in re.findall(r"([0-9.]+(?:e[-+]?\d+)?)f", body[: body.index("};")])]
    if len(values) != 128:
        raise SystemExit(f"expected 128 EWA weights, found {len(values)}")
    return struct.pack("<128f", *values)


def main() -> None:
    # the rypath checkout: the first argument, else the RYPATH_REFERENCE environment variable
    source = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RYPATH_REFERENCE")
    if not source:
        raise SystemExit("usage: name a rypath checkout as the argument or in RYPATH_REFERENCE")
    reference = Path(source)
    out = Path(__file__).resolve().parent
    (out / "pbrt_sobol_tables.bin").write_bytes(sobol_tables(reference))
    (out / "cie_xyz_1931.bin").write_bytes(cie_table(reference))
    (out / "srgb_spectrum.xz").write_bytes(srgb_table(reference))
    (out / "d65_dense.bin").write_bytes(d65_table(reference))
    (out / "ewa_weights.bin").write_bytes(ewa_table(reference))


if __name__ == "__main__":
    main()
