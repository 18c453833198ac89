"""CollisionValidator on a hand-built contact list, without a GPU.

The reference pins its validator with two known-answer cases
(tests/test_collision_validator.cpp:30-126): an empty list, and a mixed list on
a two-triangle quad whose four vertices move at (0, -1, 0), (0, 0.25, 0),
(0, -0.4, 0) and (0, 0.1, 0): a point-triangle contact 0.5 mm inside, an
edge-edge contact 0.2 mm apart and a wall contact 1.5 mm inside, all with
normal +y, judged with gap_max = 2 mm. The same expectations hold for this
module's validator (the host path: a list built by hand is always read on
the host), plus the exact values the formulas give for that list.
"""
from __future__ import annotations

import numpy as np
import pytest


def quad(core):
    m = core.Mesh()
    m.initialize(np.array([[0.0, 0, 0], [1, 0, 0], [0, 0, 1], [1, 0, 1]]), np.array([[0, 1, 2], [1, 3, 2]]), core.Material())
    st = core.State()
    st.initialize(m)
    return m, st


def test_empty_list(core):
    m, st = quad(core)
    met = core.CollisionValidator.compute_metrics(m, st, [], 0.002, True)
    assert met.num_total_contacts == 0 and met.num_penetrations == 0
    assert met.is_stable and met.ccd_effectiveness == 0.0 and met.quality_level() == 0
    assert not core.CollisionValidator.has_penetrations([])
    assert core.CollisionValidator.max_penetration_depth([]) == 0.0


def test_mixed_list(core):
    m, st = quad(core)
    v = np.array([[0.0, -1.0, 0.0], [0.0, 0.25, 0.0], [0.0, -0.4, 0.0], [0.0, 0.1, 0.0]])
    st.set_velocities64(v)
    up = np.array([0.0, 1.0, 0.0])
    C = core.Contact
    contacts = [C(core.ContactType.POINT_TRIANGLE, 0, 1, 2, 3, gap=-5.0e-4, normal=up),
                C(core.ContactType.EDGE_EDGE, 0, 1, 2, 3, gap=2.0e-4, normal=up),
                C(core.ContactType.WALL, 2, gap=-1.5e-3, normal=up)]
    assert [c.type for c in contacts] == [core.ContactType.POINT_TRIANGLE, core.ContactType.EDGE_EDGE, core.ContactType.WALL]
    met = core.CollisionValidator.compute_metrics(m, st, contacts, 0.002, True)
    # the reference's expectations
    assert (met.num_total_contacts, met.num_point_triangle, met.num_edge_edge, met.num_wall) == (3, 1, 1, 1)
    assert met.num_penetrations == 2
    assert abs(met.max_penetration - 1.5e-3) < 1e-6
    assert met.has_major_penetration and met.has_tunneling
    assert met.ccd_enabled and met.num_ccd_contacts == 3 and met.ccd_effectiveness > 99.0
    assert met.max_relative_velocity > 0.5 and met.avg_relative_velocity > 0.0
    assert met.quality_level() == 3
    assert core.CollisionValidator.has_penetrations(contacts)
    assert abs(core.CollisionValidator.max_penetration_depth(contacts) - 1.5e-3) < 1e-6
    # the values the formulas give: relative normal speeds |v0 - mean(v1..v3)|, |mean(v0,v1) - mean(v2,v3)|, |v2|
    rv = [abs(-1.0 - (0.25 - 0.4 + 0.1) / 3.0), abs((-1.0 + 0.25) / 2 - (-0.4 + 0.1) / 2), 0.4]
    assert met.max_relative_velocity == pytest.approx(max(rv), rel=1e-6)
    assert met.avg_relative_velocity == pytest.approx(sum(rv) / 3, rel=1e-6)
    assert met.min_gap == pytest.approx(-1.5e-3, rel=1e-6) and met.max_gap == pytest.approx(2.0e-4, rel=1e-6)
    assert met.avg_gap == pytest.approx((-5.0e-4 + 2.0e-4 - 1.5e-3) / 3, rel=1e-5)
    assert met.avg_penetration == pytest.approx(1.0e-3, rel=1e-5)
    assert not met.is_stable
    # without CCD the CCD figures are zero and the penetration figures unchanged
    off = core.CollisionValidator.compute_metrics(m, st, contacts, 0.002, False)
    assert not off.ccd_enabled and off.ccd_effectiveness == 0.0 and off.num_ccd_contacts == 0
    assert off.num_penetrations == met.num_penetrations and off.num_broad_phase_contacts == 3
