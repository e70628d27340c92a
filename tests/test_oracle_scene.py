"""The oracle's own set-up of the benchmark workloads (oracle.params,
oracle/scene_oracle.c), which bench.py's CPU arm uses so that it loads no
product library, against the product's (icm_params_parse_string,
icm_scene_block): parameter blocks and particle arrays bit-identical."""
import numpy as np
import pytest

import icempm_b200 as im
from icempm_b200 import configs
from oracle import oracle as orc


@pytest.mark.parametrize("name", ["c1_70k", "c2_250k"])
def test_oracle_workload_is_the_products(name):
    p, soa = orc.workload(name)
    q, ref = configs.make_scene(name)
    diff = [f for f, _ in im.SimParams._fields_ if getattr(p, f) != getattr(q, f)]
    assert not diff, diff
    assert bytes(p) == bytes(q)
    assert np.array_equal(soa, ref)


def test_oracle_params_follow_the_reference_reset_and_parser():
    import json

    q = im.SimParams()
    q.Reset()
    p = orc.params({})
    assert bytes(p) == bytes(q)
    over = dict(GridX=300, GridY=90, GridXDimension=3.0, InitialTimeStep=1.5e-6, DP_phi=55, YoungsModulus=2.5e9,
                IceTensileStrength=7e6, SortPointsByGridCell=0)
    q = im.SimParams()
    q.Reset()
    q.ParseString(json.dumps(dict(over, InputRawPoints="x")))
    assert bytes(orc.params(over)) == bytes(q)
