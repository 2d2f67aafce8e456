"""The build entry's smoke check (one small Ros2 step, the rate build and one
adaptive-loop attempt on cuda:0, each against the oracle) runs clean."""
import importlib
import os
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_smoke_entry_point():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    entry = importlib.import_module("__graft_entry__")
    entry.smoke()
