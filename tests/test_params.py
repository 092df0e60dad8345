"""Parameter derivation and output columns (src/gpu_setup.rs:528-580,
src/execute_gpu.rs:482-519, gpu_tracking_macros/src/lib.rs defaults)."""
import numpy as np
import pytest

from gpu_tracking_b200._params import column_names, derived, log_params, trackpy_params


@pytest.mark.parametrize("diam,sep,dil,margin", [(9, 9, 12, 4), (11, 12, 16, 5), (9, None, 14, 4), (5, 1, 1, -1)])
def test_trackpy_derived(oracle, diam, sep, dil, margin):
    kw = {} if sep is None else {"separation": sep}
    p = trackpy_params(diam, **kw)
    d = derived(p, 64, 64)
    assert d["dilation"] == dil and d["margin"] == margin and d["smoothing"] == diam
    g = np.frombuffer(bytes(oracle.gpu_params(p, 64, 64)), np.int32)
    assert g[7] == dil and g[12] == margin and g[2] == diam


def test_log_derived(oracle):
    p = log_params(2.0, 8.0)
    assert derived(p, 10, 10)["smoothing"] == 17
    r = oracle.log_radii(log_params(2.0, 8.0, n_radii=10, log_spacing=True))
    assert len(r) == 10 and abs(r[0] - 2.0) < 1e-5 and abs(r[-1] - 8.0) < 1e-4


def test_defaults_follow_python_layer():
    p = trackpy_params(9)
    assert p.separation == 10 and p.characterize == 1 and p.doughnut_correction == 1 and p.filter_close == 1
    assert p.has_search_range == 0 and p.memory == 0 and p.has_gap_radius == 0
    p = trackpy_params(9, bg_radius=8.0)
    assert p.has_gap_radius == 1 and p.gap_radius == 0.0
    with pytest.raises(TypeError):
        trackpy_params(9, bogus=1)
    trackpy_params(9, maxsize=3, threshold=1, invert=False, percentile=1, topn=3, preprocess=True)


def test_column_names():
    assert [c for c, _ in column_names(trackpy_params(9))] == [
        "frame", "y", "x", "mass", "Rg", "raw", "signal", "ecc", "raw_mass", "raw_bg_median",
        "raw_mass_corrected"]
    cols = [c for c, _ in column_names(log_params(2, 5, search_range=3, characterize=False,
                                                  doughnut_correction=False))]
    assert cols == ["frame", "y", "x", "mass", "r", "particle", "duration"]
