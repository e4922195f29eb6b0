"""The constant tables are regenerated from their closed forms and must match the
committed header exactly (and the reference header, when it is present)."""
import importlib.util
import os

import pytest

from conftest import ROOT

GEN = os.path.join(ROOT, "multifloats_b200", "csrc", "gen_dd_tables.py")
HEADER = os.path.join(ROOT, "multifloats_b200", "csrc", "dd_tables.h")
# the reference source tree: $MULTIFLOATS_REFERENCE, else a checkout named
# "reference" beside this repository (absent on machines without it: skipped)
REF_DIR = os.environ.get("MULTIFLOATS_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")
REF_HEADER = os.path.join(REF_DIR, "src", "dd_constants.hh")


def _gen():
    spec = importlib.util.spec_from_file_location("gen_dd_tables", GEN)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_header_is_regenerable():
    g = _gen()
    assert g.emit(g.build()) == open(HEADER).read()


@pytest.mark.skipif(not os.path.exists(REF_HEADER), reason="reference sources not present")
def test_tables_match_reference_header():
    g = _gen()
    assert g.check(g.build(), REF_HEADER) == 0
