"""Record rypath's demo-model reference answers into tests/golden/demo_reference.json.

Runs rypath's own CPU demo code compiled from a rypath checkout into
oracle/_ref/libref_demo.so (oracle/ref.mk; tests/render_reference.cpp and src/render.cpp):

* ``analytic`` -- analytic_xyz: mean and variance of XYZ of the unit demo sky and of the
  unobstructed Lambertian floor for the reflectances used by the tests;
* ``estimator`` -- reference_image on make_demo_scene: the image mean XYZ of each replicate
  (8 x 6 pixels, 128 samples, seeds 0x56DA2309 + k) and the largest scattering count.

The GPU tests read the JSON, so nothing of rypath is needed where they run.
Usage: ``python tests/golden/make_demo_golden.py`` after ``make -f oracle/ref.mk REF=...``.
"""

import ctypes as C
import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE.parent.parent / "oracle" / "_ref" / "libref_demo.so"
FLOOR = (0.54, 0.54, 0.55, 0.58, 0.61, 0.63, 0.65, 0.65)
ESTIMATOR = {"width": 8, "height": 6, "samples": 128, "seed": 0x56DA2309, "replicates": 8}


def main() -> None:
    lib = C.CDLL(str(LIB))
    lib.ref_demo_analytic.argtypes = [C.c_void_p, C.c_void_p]
    lib.ref_demo_reference_image.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p]
    analytic = {}
    for name, refl in (("sky", None), ("floor", FLOOR), ("grey", (0.5,) * 8)):
        out = np.zeros(6)
        r = None if refl is None else np.asarray(refl, np.float32)
        lib.ref_demo_analytic(None if r is None else r.ctypes.data, out.ctypes.data)
        analytic[name] = {"reflectance": refl, "mean": out[:3].tolist(), "variance": out[3:].tolist()}
    means, deepest = [], 0
    for k in range(ESTIMATOR["replicates"]):
        out = np.zeros(4)
        lib.ref_demo_reference_image(ESTIMATOR["width"], ESTIMATOR["height"], ESTIMATOR["samples"],
                                     ESTIMATOR["seed"] + k, out.ctypes.data)
        means.append(out[:3].tolist())
        deepest = max(deepest, int(out[3]))
    record = {"analytic": analytic, "estimator": dict(ESTIMATOR, means=means, max_scatterings=deepest)}
    (HERE / "demo_reference.json").write_text(json.dumps(record, indent=1) + "\n")


if __name__ == "__main__":
    main()
