"""The polar driver's host-side semantics against the reference's own code
(golden vectors from tests/golden/make_polar_golden.py): sweepAngles
(Polar.cpp:36-77) through the C ABI, bit for bit and with the reference's
refusals, and the polar CSV writer byte for byte against toCsv
(Polar.cpp:126-164)."""
import math

import numpy as np
import pytest

import cfd_b200 as cb
from helpers import golden

G = golden("polar")
SWEEPS = sorted({int(k.split("/")[0][5:]) for k in G if k.startswith("sweep")})
CSVS = sorted({int(k.split("/")[0][3:]) for k in G if k.startswith("csv")})


@pytest.mark.parametrize("k", SWEEPS)
def test_sweep_angles_match_the_reference(k):
    start, end, step = G[f"sweep{k}/request"]
    if f"sweep{k}/angles" in G:
        got = np.array(cb.sweep_angles(start, end, step))
        assert np.array_equal(got, G[f"sweep{k}/angles"])
    else:
        with pytest.raises(cb.CfdError) as err:
            cb.sweep_angles(start, end, step)
        assert err.value.code == 1
        assert str(err.value).endswith(str(G[f"sweep{k}/error"]))


def _results(points):
    out = []
    for v in points:
        r = cb.Result()
        r.alpha_deg = v[0]
        r.lift_coefficient, r.drag_coefficient = v[1], v[2]
        r.pressure_drag_coefficient, r.friction_drag_coefficient, r.moment_coefficient = v[3], v[4], v[5]
        r.separation_upper_chord_fraction, r.separation_lower_chord_fraction = v[7], v[8]
        r.status = 0 if v[9] else (2 if v[10] else 1)
        r.iterations = int(v[11])
        r.continuity = v[12]
        out.append(r)
    return out


@pytest.mark.parametrize("k", CSVS)
def test_polar_csv_matches_the_reference_byte_for_byte(k):
    pts = G[f"csv{k}/points"]
    section, mesh = (str(x) for x in G[f"csv{k}/header"])
    re, speed, chord, mref, cont = G[f"csv{k}/numbers"]
    text = cb.polar_csv(_results(pts), None, section, mesh, re, speed, chord, mref, bool(cont))
    assert text == str(G[f"csv{k}/text"])


def test_l_over_d_is_zero_where_drag_is_not_positive():
    """AerodynamicForces::liftToDrag (Forces.cpp:50-56) inside the writer."""
    rows = cb.polar_csv(_results(G["csv0/points"][:2]), None, "s", "m", 1e6, 1.0).splitlines()[11:]
    assert all(row.split(",")[6] == "0.000000" for row in rows)
    assert math.isnan(G["csv0/points"][1, 2])
