"""bench.py keeps its command-line contract (no GPU needed): every workload
the parser accepts has a runner, and the reference arm prints one JSON line."""
import importlib.util
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(HERE, "..", "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_every_workload_has_a_runner():
    b = _bench()
    assert callable(b.run_dense)
    assert callable(b.main)
    assert callable(b.run_reference_arm)
    assert b.make_matrix(0.02).nr > 0
