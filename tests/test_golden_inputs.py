"""The regenerated r = 64 golden cases rebuild bitwise the inputs the
reference's outputs were recorded on (digests in each case's spec.json), and
their partitions have the shape the cases are meant to exercise."""
import json
import os

import numpy as np
import pytest

import large_cases


@pytest.mark.parametrize("name", large_cases.names())
def test_inputs_reproduce_digests(name):
    spec = json.load(open(os.path.join(large_cases.HERE, name, "spec.json")))
    cfg, xy, pred, theta, y = large_cases.generate(name)
    assert large_cases.digests(xy, pred, y) == spec["digests"]
    assert spec["config"]["r"] == 64 and cfg.r == 64


def test_c2s_case_has_uneven_regions():
    st, md, _ = large_cases.load("r64_c2s_nu12", mode="likelihood")
    n = np.diff(st.obs_offset)
    assert st.r == 64 and st.M == 7
    # clustered: empty finest regions next to regions of hundreds of observations,
    # so that some level M-2 groups exceed the factored-form threshold (2r)
    assert (n == 0).sum() > 0 and n.max() > 128
    groups = np.bincount(st.finest_parent - st.finest_parent.min(), weights=n)
    assert groups.max() > 2 * st.r
