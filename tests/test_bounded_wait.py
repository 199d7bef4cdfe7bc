"""GPU: a bounded device-side wait that runs out is reported as
GE_ERR_TIMEOUT, and the context works again after a fresh upload.

The reference has no counterpart (its GL compute path only prints shader
errors, GalaxyEngine/src/globalLogic.cpp:601-615).  Here every wait on
another block is bounded; the test makes one run out without faulting or
hanging anything: the test hook ge_set_sort_wait_test caps the radix sort's
look-back polls and makes the sort's first tile keep its digit counts to
itself (a flag that nothing sets), so the look-back waits of the tiles after
it give up, set the device error word and carry on with in-bounds writes.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TIMEOUT = 6   # GE_ERR_TIMEOUT


def _params(ge):
    return ge.default_params(2, G=1.0, theta=0.7, eps2=1e-4, leaf_cap=4, dt=1e-3,
                             precision=ge.PREC_EXACT)


def test_sort_wait_runs_out_and_the_context_recovers(ge, ics):
    st = ics.disk2d(10000, seed=5)   # three sort tiles of 4096 keys
    with ge.Simulation(_params(ge)) as ref:
        ref.upload(st)
        ref.step(2)
        want = ref.download()
    with ge.Simulation(_params(ge)) as s:
        s.upload(st)
        s.set_sort_wait_test(spin_limit=2000, withhold=True)
        for _ in range(2):   # gives up again on a second try
            s.compute_morton_keys()
            with pytest.raises(ge.GeError) as e:
                s.sort_particles_by_morton_key()
            assert e.value.code == TIMEOUT
        # the frame calls never withhold: a capped but healthy sort still works
        s.set_sort_wait_test(spin_limit=2000, withhold=False)
        s.upload(st)
        s.step(2)
        out = s.download()
    for k in want:
        assert np.array_equal(out[k], want[k]), k


def test_withheld_tile_leaves_the_frame_calls_alone(ge, ics):
    """The hook applies to the stage sort only: ge_step with it set still
    sorts normally (a frame would otherwise build on an unsorted order)."""
    st = ics.disk2d(9000, seed=6)
    with ge.Simulation(_params(ge)) as ref:
        ref.upload(st)
        ref.step(1)
        want = ref.download()
    with ge.Simulation(_params(ge)) as s:
        s.upload(st)
        s.set_sort_wait_test(spin_limit=0, withhold=True)
        s.step(1)
        out = s.download()
    for k in want:
        assert np.array_equal(out[k], want[k]), k
