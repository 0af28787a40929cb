"""granite_b200.amr.AMRHierarchy on the GPU, driven like the reference's main
loop: a tracking sphere, initialize, Brill-Lindquist data written into the
host blocks, setLevelDt(0), then subcycle(0) with an in-step regrid at every
level step (the sphere's boxes exist already, so nothing is added)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_amr_hierarchy_steps_on_the_device():
    from granite_b200.amr import AMRHierarchy, AMRParams, SimulationParams, gradientChiTagger
    from granite_b200.initial_data import brill_lindquist
    h = AMRHierarchy(AMRParams(max_levels=3, regrid_interval=1),
                     SimulationParams(ncells=(16, 16, 16), domain_lo=(-8.0,) * 3, domain_hi=(8.0,) * 3))
    h.addTrackingSphere((0.5, 0.0, 0.0), 2.0, 2)
    h.initialize(gradientChiTagger(0.1))
    for b in h.getAllBlocks():
        brill_lindquist(b, [1.0], [(0.5, 0.0, 0.0)], r_floor=0.5 * b.dx(0))
    h.setLevelDt(0, 0.25 * h.effectiveResolution())
    assert (h.numLevels(), h.numBlocks()) == (3, 3)
    for s in range(2):
        assert h.subcycle(0, None, gradientChiTagger(0.1)) == []
        assert h.currentTime(0) == 0.25 * (s + 1)
    assert all(np.isfinite(b.array).all() for b in h.getAllBlocks())
    assert all(np.isfinite(x) for x in h.evolver().constraint_norms())
    h.close()
