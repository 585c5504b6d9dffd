"""The product's vectorised partition builder reproduces the oracle's
restatement of class_partition.cpp exactly (coordinates bit for bit, indices,
order inside regions)."""
import numpy as np

import mra_oracle as oracle
from nonstationary_mra_b200 import refio


def test_structure_bit_exact(case_dir):
    for mode in ("likelihood", "prediction"):
        a, _, _ = oracle.load_case(case_dir, mode=mode)
        b, _, _ = refio.load_case(case_dir, mode=mode)
        assert (a.J, a.M, a.r, a.n_interior) == (b.J, b.M, b.r, b.n_interior)
        for name in ("finest_parent", "obs_offset", "obs_index"):
            np.testing.assert_array_equal(getattr(a, name), getattr(b, name))
        for name in ("knots", "obs", "obs_value"):
            assert np.array_equal(getattr(a, name), getattr(b, name)), name
        if mode == "prediction":
            np.testing.assert_array_equal(a.pred_offset, b.pred_offset)
            assert np.array_equal(a.pred, b.pred)


def test_coincident_observation_is_dropped():
    # an observation sitting exactly on an ancestor knot is skipped (class_partition.cpp:533-551)
    from nonstationary_mra_b200 import partition
    rng = np.random.default_rng(0)
    lon, lat = rng.uniform(0, 1, 400), rng.uniform(0, 1, 400)
    lo0, hi0, lo1, hi1 = partition.boxes(4, 3, lon, lat)
    klon, klat, r = partition.knots_in_boxes(lo0, hi0, lo1, hi1, 5, 4, np.exp(1) / 100)
    lon2 = np.concatenate([lon, klon[7:8]])
    lat2 = np.concatenate([lat, klat[7:8]])
    st = partition.build_by_program(lon2, lat2, np.zeros(401), 4, 3, 4, np.exp(1) / 100, all_lon=lon2, all_lat=lat2)
    ost = oracle.build_structure_by_program(lon2, lat2, np.zeros(401), 4, 3, 4, np.exp(1) / 100,
                                            all_lon=lon2, all_lat=lat2)
    assert 400 not in set(st.obs_index.tolist())
    np.testing.assert_array_equal(st.obs_index, ost.obs_index)
