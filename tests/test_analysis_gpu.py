"""The GPU radial distribution function against the reference's O(n^2) NumPy rdf (accusim/analysis.py:7-24)
on a perturbed 1000-ion rock-salt box: identical g(r), all ions and one species."""
import numpy as np
import pytest

from tests.test_dropin_gpu import product_system

pytestmark = pytest.mark.gpu


def test_rdf_matches_reference(golden):
    from devinproj_b200.analysis import rdf
    g = golden("analysis_melt1000")
    s = product_system(g)
    r, gr = rdf(s, float(g["rmax"]), bins=120)
    assert np.array_equal(r, g["r_all"]) and np.array_equal(gr, g["g_all"])
    r, gr = rdf(s, float(g["rmax"]), bins=60, species="Na")
    assert np.array_equal(r, g["r_na"]) and np.array_equal(gr, g["g_na"])
    with pytest.raises(ValueError):
        rdf(s, 0.6 * float(s.box[0]))
