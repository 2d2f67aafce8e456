"""The runner slots of the reference ``RunState`` (`state.py:106-160`): the
field names of ``runstate.py`` must equal the reference NamedTuples' (read
from the reference source as text; skipped without a reference checkout).
The device round trip is in tests/test_gpu_loop.py."""
import ast
import os

import pytest

from conftest import ROOT, load_pkg

rs = load_pkg("runstate")


def _reference_state_py():
    for cand in (os.environ.get("VULCAN_REFERENCE"), os.path.join(os.path.dirname(ROOT), "reference")):
        if cand and os.path.exists(os.path.join(cand, "state.py")):
            return os.path.join(cand, "state.py")
    return None


def _namedtuple_fields(path, name):
    tree = ast.parse(open(path).read())
    for node in tree.body:
        if isinstance(node, ast.ClassDef) and node.name == name:
            return tuple(st.target.id for st in node.body if isinstance(st, ast.AnnAssign))
    raise KeyError(name)


@pytest.mark.parametrize("name,fields", [("StepInputs", rs.STEP_FIELDS), ("ParamInputs", rs.PARAM_FIELDS),
                                         ("AtomInputs", rs.ATOM_FIELDS), ("PhotoRuntimeInputs", rs.PHOTO_FIELDS)])
def test_slot_fields_match_the_reference(name, fields):
    path = _reference_state_py()
    if path is None:
        pytest.skip("reference checkout not available")
    assert _namedtuple_fields(path, name) == fields
