"""Batch scorers on a caller's stream.

A batch scorer moves its tables up and its results down on a copy stream of
its own and runs its kernels on the stream the caller set, ordered by
events. These checks drive two scorers in turn on one caller stream, the
way a pipeline overlaps host work with the device, with each step's input
planes written on that stream just before the submit: every step's results
must equal a standalone scoring of the same pairs bit for bit, so the
kernels saw the new planes and each step read its own tables and results.
"""

import numpy as np
import pytest

from tests import synthetic
from vqm_b200 import ss2

pytestmark = pytest.mark.gpu


def test_two_scorers_in_turn_on_a_caller_stream():
    import torch
    steps = [[synthetic.rgb_pair(640, 360, 950 + 2 * k + i)[:2] for i in range(2)]
             for k in range(6)]
    alone = ss2.Ssimulacra2Batch()
    expected = [alone.compute_many(pairs) for pairs in steps]
    alone.close()

    nbytes = steps[0][0][0].data.nbytes
    fmt = steps[0][0][0].format
    stream = torch.cuda.Stream()
    # Per scorer: device planes for its two pairs, rewritten every other step.
    slots = [[(torch.empty(nbytes, dtype=torch.uint8, device="cuda"),
               torch.empty(nbytes, dtype=torch.uint8, device="cuda")) for _ in range(2)]
             for _ in range(2)]
    batches = [ss2.Ssimulacra2Batch(), ss2.Ssimulacra2Batch()]
    for b in batches:
        b.set_stream(stream.cuda_stream)
    got, pending = [None] * len(steps), [None, None]
    try:
        for k, pairs in enumerate(steps):
            w = k % 2
            if pending[w] is not None:
                j, token = pending[w]
                got[j] = batches[w].finish(token)
            dev = []
            with torch.cuda.stream(stream):
                for (o, d), (to, td) in zip(pairs, slots[w]):
                    to.copy_(torch.from_numpy(o.data).pin_memory(), non_blocking=True)
                    td.copy_(torch.from_numpy(d.data).pin_memory(), non_blocking=True)
                    dev.append((ss2.DeviceImage.packed(o.width, o.height, fmt, to.data_ptr(), to),
                                ss2.DeviceImage.packed(d.width, d.height, fmt, td.data_ptr(), td)))
            pending[w] = (k, batches[w].submit(dev))
        for w in (0, 1):
            if pending[w] is not None:
                j, token = pending[w]
                got[j] = batches[w].finish(token)
    finally:
        for b in batches:
            b.close()
    for k in range(len(steps)):
        for g, e in zip(got[k], expected[k]):
            assert np.array_equal(g.norms, e.norms), k
            assert g.score() == e.score(), k
