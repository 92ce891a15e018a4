"""The field map on the CPU: the oracle's restatement of the reference's CMS
map reader against the reader itself (golden tests/golden/field.npz from
make_golden_field.py), and the map format checks of the library's loader."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAP = os.path.join(os.path.dirname(HERE), "geantexascalepilot_b200", "data", "field", "cmsmagfield2015.txt")


def test_oracle_field_map_matches_reference(oracle):
    z = np.load(os.path.join(HERE, "golden", "field.npz"))
    h = oracle.field_map_load(MAP)
    B = oracle.field_map_value(h, z["pos"])
    assert np.array_equal(B, z["B"])
    # the solenoid: ~3.8 T along z at the centre, falling outside
    c = oracle.field_map_value(h, [[0.0, 0.0, 0.0], [0.0, 0.0, 15000.0]])
    assert abs(c[0, 2] - 3.811) < 0.01 and abs(c[1, 2]) < 0.5
