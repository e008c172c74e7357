"""Writes the golden fixtures under tests/golden/.

    python tests/golden/make_goldens.py

What it records, and from where:
  * gradient_{0,1,2}.npy -- the reference test suite's 32x32 8-bit sRGB
    gradient images, rebuilt from their definition (MakeGradient,
    tests/support.h:93-103, 259-289 of GreatValueCreamSoda/vqm).
  * goldens.json
      - "vqm_pins": the scores the reference's own tests pin for those pairs
        (tests/metrics/ssimulacra2/pipeline_test.cc:172-173, +-5e-3), the
        identity rule (:120-144) and the scale counts (:760-783), and the
        RequiredBytes values its pool tests pin (:573, :692).
      - "oracle": the CPU oracle's FP32 and FP64 norms and scores on the
        gradient pairs and on the seeded 256x256 pair, as regression pins of
        the oracle itself (regenerate only on a deliberate oracle change).
"""

from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests import helpers  # noqa: E402
from oracle import binding as ob  # noqa: E402


def main() -> None:
    images = {}
    for v in range(3):
        img = helpers.gradient(v)
        np.save(os.path.join(HERE, f"gradient_{v}.npy"), img.data)
        images[v] = img
    pins = {
        "gradient_scores": [
            {"original": 0, "distorted": 1, "score": 93.17505696, "tolerance": 5e-3,
             "source": "tests/metrics/ssimulacra2/pipeline_test.cc:172"},
            {"original": 0, "distorted": 2, "score": 92.12553218, "tolerance": 5e-3,
             "source": "tests/metrics/ssimulacra2/pipeline_test.cc:173"},
        ],
        "identity_score": 100.0,
        "scale_counts": [[8, 8, 2], [13, 9, 2], [64, 64, 5], [65, 65, 5], [129, 97, 5],
                         [32, 32, 4]],
        "required_bytes": [
            {"format": "srgb8", "width": 33, "height": 17, "bytes": 1692,
             "source": "tests/metrics/ssimulacra2/pipeline_test.cc:573"},
            {"format": "grey8", "width": 8, "height": 8, "bytes": 64,
             "source": "tests/metrics/ssimulacra2/pipeline_test.cc:692"},
        ],
    }
    oracle = {}
    for v in (1, 2):
        for prec in (32, 64):
            norms, score = ob.compute(helpers.to_oracle(images[0]),
                                      helpers.to_oracle(images[v]), precision=prec)
            oracle[f"gradient_0_{v}_f{prec}"] = {"score": score, "norms": norms.tolist()}
    o, d = helpers.plain_256_pair()
    digest = hashlib.sha256(o.data.tobytes() + d.data.tobytes()).hexdigest()
    for prec in (32, 64):
        norms, score = ob.compute(helpers.to_oracle(o), helpers.to_oracle(d), precision=prec)
        oracle[f"plain_256_f{prec}"] = {"score": score, "norms": norms.tolist(),
                                        "sha256": digest}
    with open(os.path.join(HERE, "goldens.json"), "w") as f:
        json.dump({"vqm_pins": pins, "oracle": oracle}, f, indent=1)
    print("wrote", os.path.join(HERE, "goldens.json"))


if __name__ == "__main__":
    main()
