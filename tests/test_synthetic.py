"""The seeded benchmark surveys: per-shot apertures of the batching configuration and the
geometries, costs and CPU-baseline samples derived from them (host only)."""
import numpy as np

import gubingluo_b200 as G
from gubingluo_b200 import shards, synthetic


def test_apertures_are_seeded_uniform_and_give_layout1_windows():
    s, shots, v, vm, rho, meta = synthetic.config(4)
    again = synthetic.config(4)[5]
    assert meta["apertures"] == again["apertures"]
    ap = np.array([meta["apertures"][k] for k in shots])
    assert len(ap) == 256 and ap.min() >= 201 and ap.max() <= 801 and np.all(ap % 2 == 1)
    # roughly uniform over the 301 odd widths: every sixth of the range is populated
    assert len(np.unique((ap - 201) // 101)) == 6
    sm = G.SurveyConfig(**{**s.__dict__, "mode": 1})
    geos = synthetic.shot_geometries(sm, shots, meta)
    for ishot, g in zip(shots, geos):
        w = meta["apertures"][ishot]
        isrc = int(s.spx0 / s.dx) + (ishot - 1) * int(s.dspx / s.dx)   # the reference's layout-1 source column
        half = (w - 1) // 2
        assert g.nx1 == max(isrc - half, 0) and g.nx2 == min(isrc + half, s.nx - 1)
        assert g.nxlength == g.nx2 - g.nx1 + 1 == g.nrec
        assert g.nsx == s.npml + isrc - g.nx1          # the source sits at its own column
        assert g.nxpad == g.nxlength + 2 * s.npml
        if 0 < isrc - half and isrc + half < s.nx - 1:
            assert g.nxlength == w                      # uncut inside the model


def test_fixed_layouts_have_no_per_shot_geometry():
    for n in (1, 2, 5):
        s, shots, _, _, _, meta = synthetic.config(n)
        assert "apertures" not in meta
        assert synthetic.shot_geometries(G.SurveyConfig(**s.__dict__), shots, meta) is None


def test_shot_costs_follow_the_given_geometries():
    s, shots, _, _, _, meta = synthetic.config(4, nshots=12)
    sm = G.SurveyConfig(**{**s.__dict__, "mode": 1})
    geos = synthetic.shot_geometries(sm, shots, meta)
    costs = shards.shot_costs(sm, shots, geos)
    assert costs == [float(s.nt) * g.nxpad * g.nzpad for g in geos]
    assert len(set(costs)) > 1
    # the survey's own layout-1 windows (offsetmax 8 km) are wider than the drawn ones
    own = shards.shot_costs(sm, shots)
    assert all(c <= o for c, o in zip(costs, own))
    parts = shards.lpt_shards(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(12))
