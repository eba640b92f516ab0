"""The launch-shape autotuner (cs_autotune): it times the interpolation
kernels and, in the tensor modes, the epilogue's segment size per profile bin
count, the base level's TMEM double buffer and the split epilogue on a sample
of the band, keeps the fastest, and every shape it may choose computes the
same values.

Checked: the tuned search returns exactly the untuned search's records and
agrees with the C port of the reference search (tolerances of
test_gpu_configs); every forced shape the tuner may pick gives the same
records; the report names a shape for every level.
"""
import numpy as np
import pytest

from tests.fixtures import multi_spectrum

pytestmark = pytest.mark.gpu


def _engine(synth):
    import cohsearch as cs
    amps, N, dt = multi_spectrum()
    eng = cs.Engine(cs.SearchParams(nharms=60, m=16, decimations=cs.decimation_set(60, 6), threshold=8.0,
                                    synth=synth))
    eng.set_diagnostics(1)
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    return eng, amps, N, dt


@pytest.mark.parametrize("synth", ["fp16", "fp32"])
def test_tuned_search_equals_untuned_and_the_port(synth):
    from tests.test_gpu_configs import check_against_port, _port
    band = (0.2, 120.0)
    ref, amps, N, dt = _engine(synth)
    want = ref.search_raw(band[0], band[1], 100, 2048, 8.0)
    eng, _, _, _ = _engine(synth)
    rep = eng.autotune(band[0], band[1], 100, 2048, nsample=48)
    print(f"\nautotune ({synth}): {rep}")
    assert rep["sample_blocks"] == 48
    assert rep["interp_kernel"] in ("persistent", "per-item")
    assert len(rep["units_per_level"]) == 6
    if synth != "fp32":
        assert all(u >= 1 for u in rep["units_per_level"].values())
        assert rep["ms_synth_tuned"] <= rep["ms_synth_model"]
    got = eng.search_raw(band[0], band[1], 100, 2048, 8.0)
    assert np.array_equal(got, want)
    sig, nv = eng.block_values()
    port = _port(amps, N, dt, 60, eng.params.decimations, band[0], band[1])
    matched, _ = check_against_port(got, sig, nv, port, N, dt, 60, band[0], band[1], 6)
    assert matched > 0
    # an engine created afterwards with the same parameters starts with the tuned shapes
    import cohsearch as cs
    again = cs.Engine(eng.params)
    again.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    assert np.array_equal(again.search_raw(band[0], band[1], 100, 2048, 8.0), want)


@pytest.mark.parametrize("synth", ["fp16", "bf16_split", "fp32"])
def test_every_launch_shape_gives_the_same_records(synth):
    """Each kernel form and epilogue plan the tuner can choose, pinned by
    cs_set_launch_shapes: identical records and block sigmas."""
    band = (0.2, 120.0)
    ref, _, _, _ = _engine(synth)
    ref.set_launch_shapes(0, 0, 0, (0, 0))
    want = ref.search_raw(band[0], band[1], 100, 2048, 8.0)
    wsig, wnv = ref.block_values()
    assert len(want) > 0
    shapes = [(1, 0, 1, (0, 0)), (0, 1, 1, (4, 4)), (1, 1, 0, (2, 0)), (0, 0, 1, (16, 3)), (1, 1, 1, (8, 12)),
              (0, 0, 2, (2, 2)), (1, 1, 2, (3, 4)), (0, 0, 2, (0, 0))]
    for sh in shapes:
        eng, _, _, _ = _engine(synth)
        eng.set_launch_shapes(*sh)
        got = eng.search_raw(band[0], band[1], 100, 2048, 8.0)
        sig, nv = eng.block_values()
        assert np.array_equal(got, want), sh
        assert np.array_equal(sig, wsig) and np.array_equal(nv, wnv), sh
    import cohsearch as cs
    with pytest.raises(ValueError):
        ref.set_launch_shapes(0, 0, 1, (7, 0))


@pytest.mark.parametrize("synth", ["fp16", "bf16"])
def test_split_epilogue_gates_equal_the_phased_form(synth):
    """The split epilogue (warpgroups 0-1 on the base level's two TMEM slots,
    2-3 on the decimated levels, each pair issuing its own products) and the
    phased one (all warpgroups on the decimated levels, then the base level)
    read the same accumulators through the same segments: every gate value
    and record bit for bit."""
    band = (0.2, 120.0)
    out = []
    for db in (1, 2):
        eng, _, _, _ = _engine(synth)
        eng.set_diagnostics(2)
        eng.set_launch_shapes(0, 0, db, (2, 2))
        got = eng.search_raw(band[0], band[1], 100, 2048, 8.0)
        out.append((got, eng.gate_values().copy()))
    assert len(out[0][0]) > 0
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1].view(np.uint32), out[1][1].view(np.uint32))
