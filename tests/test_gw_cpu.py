"""Host analysis of the Psi4 time series (granite_b200.gw.Psi4Extractor) on the
CPU: the reference's formulas (postprocess.cpp:316-475) checked on series with
known integrals, and the recording rules of extract (a new entry per time, the
same time accumulates, radii without points inside the block record nothing)."""
import numpy as np

from granite_b200.gw import GWExtractionParams, Psi4Extractor, mode_list


def extractor(series, radii=(10.0, 20.0)):
    ex = Psi4Extractor(GWExtractionParams(extraction_radii=list(radii), l_max=2, n_theta=4, n_phi=8))
    for t, v in series:
        modes = np.full((len(radii), 5), v, dtype=complex)
        modes[1] *= 2.0
        ex._record(t, np.array(radii), modes, [1] * len(radii))
    return ex


def test_mode_order():
    assert mode_list(3)[:6] == [(2, -2), (2, -1), (2, 0), (2, 1), (2, 2), (3, -3)]
    assert len(mode_list(4)) == 21


def test_strain_of_a_constant_mode():
    # Psi4 = c: h_dot = c t, h = c t^2 / 2 (trapezoid sums, exact for these on a uniform grid up to O(dt))
    c = 0.3 - 0.1j
    ts = np.linspace(0.0, 2.0, 201)
    ex = extractor([(t, c) for t in ts])
    h = ex.computeStrain(2, 2, 10.0)
    dt = ts[1] - ts[0]
    want = sum(c * (i * dt) * dt for i in range(1, 201))
    assert abs(h - want) < 1e-12
    assert abs(h - c * 2.0) < 2e-2  # c t^2 / 2 at t = 2


def test_energy_extrapolation_and_recording():
    ts = np.linspace(0.0, 1.0, 11)
    ex = extractor([(t, 1.0) for t in ts])
    E = ex.computeRadiatedEnergy(10.0)
    # five modes with |h_dot| = t: sum_i t_i^2 dt over the grid, times r^2 / (16 pi)
    dt = 0.1
    want = 5 * sum((i * dt) ** 2 * dt for i in range(1, 11)) * 100.0 / (16.0 * np.pi)
    assert abs(E - want) < 1e-12 * want
    assert ex.extrapolateToInfinity(2, 0) == (100.0 * 2.0 - 400.0 * 1.0) / (100.0 - 400.0)
    assert ex.computeRadiatedMomentum(10.0) == (0.0, 0.0, 0.0)
    # the same time accumulates, a radius without points records nothing
    ex2 = Psi4Extractor(GWExtractionParams(extraction_radii=[10.0, 20.0], l_max=2))
    m = np.ones((2, 5), dtype=complex)
    ex2._record(0.5, np.array([10.0, 20.0]), m, [3, 0])
    ex2._record(0.5, np.array([10.0, 20.0]), m, [3, 0])
    assert ex2.getTimeSeries(2, 1, 10.0) == [(0.5, 2.0 + 0j)]
    assert ex2.getTimeSeries(2, 1, 20.0) == [] and ex2.getMode(2, 1, 20.0) == 0j


def test_energy_spectrum_peaks_at_the_mode_frequency():
    # the DFT kernel is exp(-2 pi i f t) over f >= 0, so a mode exp(+2 pi i f0 t) shows at f0
    f0 = 2.0
    ts = np.linspace(0.0, 4.0, 161)
    ex = extractor([(t, np.exp(2j * np.pi * f0 * t)) for t in ts])
    spec = ex.computeEnergySpectrum(2, 2, 10.0)
    assert len(spec) == 80
    f = np.array([s[0] for s in spec])
    S = np.array([s[1] for s in spec])
    assert f[np.argmax(S[1:]) + 1] == f0


def test_analysis_matches_compiled_reference(reference_lib):
    """The reference's Psi4Extractor records a noisy puncture at 13 unevenly spaced
    times; fed the same series, strain, energy, extrapolation and spectrum here
    equal the compiled postprocess.cpp:316-475 bit for bit, and a radius whose
    sphere leaves the block records nothing on either side."""
    import oracle
    from oracle import Geom
    g = Geom((24, 24, 24), (-3.0, -3.0, -3.0), (3.0, 3.0, 3.0))
    base = reference_lib.init_brill_lindquist(g, [0.5], [[0.1, -0.05, 0.0]])
    dts = [0.1, 0.12, 0.08, 0.1, 0.15, 0.05, 0.1, 0.1, 0.11, 0.09, 0.1, 0.13]
    times = np.concatenate([[0.0], np.cumsum(dts)])
    states = [base + 1e-4 * (1 + t) * oracle.hash_noise(g.shape, 100 + t) for t in range(len(times))]
    radii = [1.0, 1.5, 2.25, 6.0]
    l_max = 3
    ref = reference_lib.psi4_series(g, states, times, radii, 6, 12, l_max, (2, 2, 1))
    ex = Psi4Extractor(GWExtractionParams(extraction_radii=list(radii), l_max=l_max, n_theta=6, n_phi=12))
    keys = mode_list(l_max)
    for r, rad in enumerate(radii):
        for q, key in enumerate(keys):
            s = ref["series"][(r, q)]
            assert len(s) == (0 if rad == 6.0 else len(times))
            if s:
                ex.data.setdefault(float(rad), {})[key] = list(s)
    assert 6.0 not in ex.data
    for r, rad in enumerate(radii):
        assert ex.computeRadiatedEnergy(rad) == ref["energy"][r]
        for q, (l, m) in enumerate(keys):
            assert ex.computeStrain(l, m, rad) == ref["strain"][r, q]
    for q, (l, m) in enumerate(keys):
        assert ex.extrapolateToInfinity(l, m) == ref["extrap"][q]
    spec = ex.computeEnergySpectrum(2, 2, radii[1])
    assert len(spec) == len(ref["spectrum"]) == len(times) // 2
    assert spec == ref["spectrum"]
    assert any(e > 0.0 for e in ref["energy"][:3])
