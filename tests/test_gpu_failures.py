"""Failure paths on the device, driven without faulting the GPU.

  * A bounded device wait that runs out: the wait-test hook makes one thread
    block of the block-sigma kernel wait on a shared-memory barrier that
    nothing completes, with a 2 ms limit.  The search returns CS_ERR_TIMEOUT,
    and the same handle's next search (hook off) gives the normal result:
    the context stays usable.
  * An allocation cap: a memory limit below one block's working set makes the
    search fail with CS_ERR_OUT_OF_MEMORY on the host side, before any device
    work; a limit that holds only a few blocks splits the search into many
    waves whose records equal the uncapped search's.
"""
import numpy as np
import pytest

from tests.fixtures import multi_spectrum

pytestmark = pytest.mark.gpu

CS_ERR_OUT_OF_MEMORY = 5
CS_ERR_TIMEOUT = 6


def _engine(synth="fp16"):
    import cohsearch as cs
    amps, N, dt = multi_spectrum()
    eng = cs.Engine(cs.SearchParams(nharms=32, m=16, decimations=cs.decimation_set(32, 4), threshold=7.0,
                                    synth=synth))
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    return eng


@pytest.mark.parametrize("synth", ["fp32", "fp16"])
def test_device_wait_runs_out_and_the_handle_recovers(synth):
    import cohsearch as cs
    eng = _engine(synth)
    want = eng.search_raw(1.0, 60.0, 100, 2048, 7.0)
    assert len(want) > 0
    eng.set_wait_test(2_000_000)    # 2 ms
    with pytest.raises(cs.CohSearchError) as ei:
        eng.search_raw(1.0, 60.0, 100, 2048, 7.0)
    assert ei.value.status == CS_ERR_TIMEOUT
    eng.set_wait_test(0)
    assert np.array_equal(eng.search_raw(1.0, 60.0, 100, 2048, 7.0), want)


def test_memory_cap_fails_cleanly_or_splits_into_waves():
    import cohsearch as cs
    eng = _engine()
    want = eng.search_raw(1.0, 60.0, 100, 2048, 7.0)
    blocks = eng.stats()["blocks"]
    assert eng.stats()["waves"] == 1 and blocks > 8
    eng.set_memory_limit(1 << 20)   # below one block's working set beside the spectrum
    with pytest.raises(cs.CohSearchError) as ei:
        eng.search_raw(1.0, 60.0, 100, 2048, 7.0)
    assert ei.value.status == CS_ERR_OUT_OF_MEMORY
    eng.set_memory_limit(24 << 20)  # a few blocks per wave
    got = eng.search_raw(1.0, 60.0, 100, 2048, 7.0)
    assert eng.stats()["waves"] > 1
    assert np.array_equal(got, want)
    eng.set_memory_limit(0)
    assert np.array_equal(eng.search_raw(1.0, 60.0, 100, 2048, 7.0), want)
