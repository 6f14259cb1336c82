"""Plan compiler parity: product (C++) == oracle (C) == the reference's own
PatternPreprocessor output (tests/golden/plans.jsonl, made by
tests/golden/make_golden.py from the reference's untouched src/pattern.h)."""
import glob
import json
import os
import subprocess

import pytest

import pm_oracle as orc
import pumatch_b200 as pm
from pumatch_b200 import patterns as P

GOLD = os.path.join(os.path.dirname(__file__), "golden")
KEYS = ["nnodes", "multiplicity", "nslots", "level_begin", "degree", "partial", "slot_labels", "set_ops"]


def _records():
    with open(os.path.join(GOLD, "plans.jsonl")) as f:
        return [json.loads(line) for line in f]


PATTERNS = json.load(open(os.path.join(GOLD, "patterns.json")))


@pytest.mark.parametrize("rec", _records(), ids=lambda r: f"{r['pattern']}-{'lab' if r['labeled'] else 'unl'}")
def test_plan_matches_reference(rec):
    text = PATTERNS[rec["pattern"]]
    labeled = bool(rec["labeled"])
    mine = pm.PatternPreprocessor(text=text, labeled=labeled).describe()
    ora = orc.plan(text, labeled).as_dict()
    for k in KEYS:
        assert mine[k] == rec[k], (k, mine[k], rec[k])
        assert ora[k] == rec[k], (k, ora[k], rec[k])
    if labeled:
        assert mine["vertex_label"] == rec["vertex_label"]


def test_known_multiplicities():
    for k in range(3, 8):
        assert pm.PatternPreprocessor(text=P.to_g(*P.clique(k)), labeled=False).PatternMultiplicity == \
            [1, 1, 2, 6, 24, 120, 720, 5040][k]
        assert pm.PatternPreprocessor(text=P.to_g(*P.cycle(k)), labeled=False).PatternMultiplicity == 2 * k
        assert pm.PatternPreprocessor(text=P.to_g(*P.path(k)), labeled=False).PatternMultiplicity == 2
    assert pm.PatternPreprocessor(text=P.to_g(*P.star(5)), labeled=False).PatternMultiplicity == 24


def test_c7_plan_shape():
    d = pm.PatternPreprocessor(text=P.to_g(*P.cycle(7)), labeled=False).describe()
    # five levels; the last one intersects N(v5) with the carried N(v0) slot
    assert d["level_begin"] == [0, 1, 3, 5, 7, 9, 10]
    assert d["set_ops"][9] & 0x40 and (d["set_ops"][9] & 0x1F) == 8
    assert d["partial"][0] == 1  # root edges keep v1 < v0


def test_bad_pattern_text():
    with pytest.raises(pm.PmError) as e:
        pm.PatternPreprocessor(text="v 0 1\nv 1 1\ne 0 1 1\n", labeled=False)
    assert e.value.status == pm.PM_ERR_FORMAT
    with pytest.raises(pm.PmError):
        pm.PatternPreprocessor(text="v 0 1\nv 1 1\nv 2 1\ne 0 9 1\n", labeled=False)
    with pytest.raises(pm.PmError) as e:
        pm.PatternPreprocessor("/nonexistent/p.g")
    assert e.value.status == pm.PM_ERR_IO


# the reference checkout, when one is named (PM_REF_DIR); skipped otherwise
REF_DIR = os.environ.get("PM_REF_DIR", "")
REF_PAT = sorted(glob.glob(os.path.join(REF_DIR, "pattern", "*.g"))) if REF_DIR else []
REF_PROBE = os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref")


@pytest.mark.skipif(not REF_PAT or not os.path.exists(os.path.join(REF_PROBE, "ref_plan_dump_labeled")),
                    reason="PM_REF_DIR unset, or the reference-built probe is missing")
@pytest.mark.parametrize("path", REF_PAT, ids=os.path.basename)
def test_reference_pattern_files(path):
    """The reference's own 20 pattern files, where a reference checkout is named."""
    for mode in ("labeled", "unlabeled"):
        ref = json.loads(subprocess.run([os.path.join(REF_PROBE, f"ref_plan_dump_{mode}"), path],
                                        capture_output=True, text=True, check=True).stdout)
        mine = pm.PatternPreprocessor(path, labeled=mode == "labeled").describe()
        for k in KEYS:
            assert mine[k] == ref[k], (mode, k)
