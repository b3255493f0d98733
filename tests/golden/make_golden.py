"""Extract rypath's own known-answer vectors for the spectral path into JSON fixtures.

Reads the reference's test sources as text (nothing is executed):

* ``tests/sampling_tests.cpp`` -- PBRT v4 Sobol known answers (interval index, signed-seed
  dimension hash, words for the four randomisations, binary32 pixel remap), generated by
  the reference from PBRT v4 b0bdf461.
* ``tests/replay_tests.cpp`` -- Random123 v1.14.0 Philox4x32-10 known-answer vectors.
* ``tests/qmc_sampling_tests.cpp`` -- PBRT v4 Halton and ZSobol known answers (index, camera
  samples and scrambled radical inverse / ZSobol words for four randomisations), generated
  by the reference from PBRT v4 b0bdf461.
* ``tests/gaussian_filter_tests.cpp`` -- FNV-1a digests of the Gaussian filter tables (every
  CDF entry) and of 33x33 filter samples for three (x radius, y radius, sigma)
  configurations, obtained by the reference from PBRT v4 b0bdf461.

Usage: ``python tests/golden/make_golden.py /path/to/rypath`` (writes next to this file).
"""

import json
import os
import re
import sys
from pathlib import Path

INT_MIN, INT_MAX = -(2**31), 2**31 - 1


def _int(token: str) -> int:
    token = token.strip()
    if "numeric_limits<std::int32_t>::min()" in token:
        return INT_MIN
    if "numeric_limits<std::int32_t>::max()" in token:
        return INT_MAX
    return int(re.sub(r"(?<=[0-9a-fA-F])[uUlL]+$", "", token), 0)


def _float(token: str) -> float:
    token = token.strip().rstrip("fF")
    return float.fromhex(token) if "0x" in token.lower() else float(token)


def sobol_answers(text: str):
    answers = []
    for body in re.findall(r"KnownAnswer\{(.*?)\}\s*\}", text, flags=re.S):
        body = re.sub(r"//[^\n]*", "", body)
        words_match = re.search(r"\{([^{}]*)\}\s*,\s*\{([^{}]*)$", body.strip(), flags=re.S)
        head = body[: words_match.start()]
        scalars = [t for t in head.replace("\n", " ").split(",") if t.strip()]
        words = [_int(t) for t in words_match.group(1).split(",")]
        camera = [_float(t) for t in words_match.group(2).split(",")]
        m, x, y, sample, dimension, seed, index, hash_ = scalars
        answers.append(
            {
                "m": _int(m), "x": _int(x), "y": _int(y), "sample": _int(sample),
                "dimension": _int(dimension), "seed": _int(seed), "index": _int(index),
                "hash": _int(hash_), "words": words, "camera": [c.hex() for c in camera],
            }
        )
    return answers


def philox_answers(text: str):
    out = []
    pattern = (r"rr::philox\(\{([^}]*)\},\s*\{([^}]*)\}\)\)\s*==\s*"
               r"std::array<rr::Word, 4>\{([^}]*)\}")
    for counter, key, expected in re.findall(pattern, text, flags=re.S):
        out.append(
            {
                "counter": [_int(t) for t in counter.split(",")],
                "key": [_int(t) for t in key.split(",")],
                "expected": [_int(t) for t in expected.split(",")],
            }
        )
    return out


def qmc_answers(text: str):
    out = []
    for q, a in re.findall(r"\{\{([-0-9, ]+)\},\s*\{([0-9ul, ]+)\}\}", text):
        out.append({"q": [int(t) for t in q.split(",")], "a": [_int(t) for t in a.split(",")]})
    return out


def gaussian_answers(text: str):
    configs = re.findall(r"Configuration\{([^}]*)\}", text)
    configs = [[_float(t) for t in c.split(",")] for c in configs]
    block = re.search(r"expected\{(.*?)\};", text, flags=re.S).group(1)
    pairs = re.findall(r"\{(0x[0-9a-fA-F]+ULL),\s*(0x[0-9a-fA-F]+ULL)\}", block)
    return [{"x_radius": c[0], "y_radius": c[1], "sigma": c[2], "cdf_hash": _int(a), "sample_hash": _int(b)}
            for c, (a, b) in zip(configs, pairs)]


def main() -> None:
    # the rypath checkout: the first argument, else the RYPATH_REFERENCE environment variable
    source = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RYPATH_REFERENCE")
    if not source:
        raise SystemExit("usage: name a rypath checkout as the argument or in RYPATH_REFERENCE")
    reference = Path(source)
    here = Path(__file__).resolve().parent
    sobol = sobol_answers((reference / "tests/sampling_tests.cpp").read_text())
    philox = philox_answers((reference / "tests/replay_tests.cpp").read_text())
    gaussian = gaussian_answers((reference / "tests/gaussian_filter_tests.cpp").read_text())
    qmc = qmc_answers((reference / "tests/qmc_sampling_tests.cpp").read_text())
    if len(sobol) != 8 or len(philox) != 3 or len(gaussian) != 3 or len(qmc) != 28:
        raise SystemExit(f"unexpected vector counts: sobol {len(sobol)}, philox {len(philox)}, "
                         f"gaussian {len(gaussian)}, qmc {len(qmc)}")
    (here / "sobol_known_answers.json").write_text(json.dumps(sobol, indent=1) + "\n")
    (here / "philox_known_answers.json").write_text(json.dumps(philox, indent=1) + "\n")
    (here / "gaussian_filter_known_answers.json").write_text(json.dumps(gaussian, indent=1) + "\n")
    (here / "qmc_known_answers.json").write_text(json.dumps(qmc, indent=1) + "\n")


if __name__ == "__main__":
    main()
