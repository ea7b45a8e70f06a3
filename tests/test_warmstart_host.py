"""Host-side logic of the learned-warm-start protocol, without a GPU: the objective-tolerance count
and the subject stream (phantoms synthesised on spawned host processes, in seed order, with the
same k-space as a direct synthesis)."""
import numpy as np

from llr_b200 import warmstart as W
from llr_b200.phantom import make_dataset


def test_iterations_to_objective_tolerance():
    obj = np.array([5.0, 3.0, 2.0003, 2.0002, 2.0001, 2.0])
    assert W.iterations_to(obj, 2.0, 1e-4) == 4          # first F_k <= F* (1 + 1e-4): the 4th iterate
    assert W.iterations_to(obj, 2.0, 1e-6) == 6
    assert W.iterations_to(obj, 1.0, 1e-4) is None       # never within the run


def test_subject_stream_order_and_content():
    proto = W.Protocol(vol=(12, 12, 12), centre=4)
    seeds = [3, 1, 2]
    got = list(W.subject_stream(proto, seeds, 2))
    assert [s for s, _ in got] == seeds
    for s, y in got:
        ref = make_dataset(proto.vol, proto.shells, proto.accel, s, centre=proto.centre,
                           protocol_seed=proto.protocol_seed).y
        np.testing.assert_array_equal(y, ref)
    single = list(W.subject_stream(proto, seeds[:1], 1))
    np.testing.assert_array_equal(single[0][1], got[0][1])
