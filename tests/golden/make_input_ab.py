"""Writes tests/golden/input_ab.npz: the FP64 values of the input-format A/B
cases (tests/input_ab.py), evaluated by the reference's own
tests/input/input_reference.h compiled into oracle/_ref/libvqm_ref.so.

    make -C oracle ref VQM_REFERENCE=<reference checkout>
    python tests/golden/make_input_ab.py
"""

from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from tests import input_ab  # noqa: E402


def main() -> int:
    ref = input_ab.live_reference()
    if ref is None:
        print("oracle/_ref/libvqm_ref.so with the input_reference.h shim is not built",
              file=sys.stderr)
        return 1
    values = input_ab.reference_values(ref)
    np.savez_compressed(input_ab.FIXTURE, **values)
    print(f"wrote {len(values)} arrays to {input_ab.FIXTURE}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
