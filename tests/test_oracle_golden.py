"""Pin the CPU oracle against the reference's own pathMIS known answers:
scene/pa5/tests/test-direct.xml and test-furnace.xml, evaluated with the
reference's Student-t procedure (src/core/StudentTTest.cpp:143-190)."""
import os

import pytest

from hikari_b200.scenedesc import parse_xml
from oracle.oracle import OracleScene, students_t_test


@pytest.mark.parametrize("fname", ["test-direct.xml", "test-furnace.xml"])
def test_pathmis_golden_ttest(golden_dir, fname):
    scenes = parse_xml(os.path.join(golden_dir, "pa5", fname))
    mis = [s for s in scenes if s.integrator == "pathMIS"]
    assert mis, "no pathMIS scenes in the golden file"
    for sd in mis:
        o = OracleScene(sd)
        mean, var = o.ttest_scene(100000)
        ok, p = students_t_test(mean, var, sd.reference, 100000, 0.01, len(scenes))
        assert ok, f"{fname}: mean {mean} vs reference {sd.reference} (p={p})"
