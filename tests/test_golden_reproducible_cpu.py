"""The committed golden vectors are what tests/golden/make_golden.py makes from
the compiled reference: regenerated into a temporary directory, every array of
every fixture is equal. Skipped where the compiled reference is absent."""
import importlib.util
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_golden_vectors_regenerate_identically(tmp_path):
    oracle.build()
    if not oracle.reference_available("strict"):
        pytest.skip("compiled reference (oracle/_ref) not available on this host")
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    mg.OUT = str(tmp_path)
    mg.main()
    made = sorted(f for f in os.listdir(tmp_path) if f.endswith(".npz"))
    assert len(made) >= 18
    for f in made:
        a, b = np.load(tmp_path / f), np.load(os.path.join(GOLD, f))
        assert sorted(a.files) == sorted(b.files), f
        for k in a.files:
            assert np.array_equal(a[k], b[k]), (f, k)
