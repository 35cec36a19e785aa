"""The pre/post-pursuit fixtures are what the reference's own functions
return on the seeded inputs (re-run here when the reference package is
staged under baseline/_ref); no GPU needed."""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import reference_harness as RH

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(not os.path.isdir(os.path.join(RH.REF_STAGED, "spikesorting_fullpursuit")),
                    reason="reference package not staged")
def test_prepost_fixtures_are_the_references_outputs(tmp_path):
    gold = np.load(os.path.join(HERE, "golden", "prepost", "prepost.npz"))
    src = open(os.path.join(HERE, "golden", "make_prepost_golden.py")).read()
    src = src.replace('os.path.join(HERE, "prepost", "prepost.npz")', repr(str(tmp_path / "p.npz")))
    script = tmp_path / "gen.py"
    script.write_text(src.replace("HERE = os.path.dirname(os.path.abspath(__file__))",
                                  "HERE = %r" % os.path.join(HERE, "golden")))
    subprocess.run([sys.executable, str(script)], check=True, capture_output=True)
    fresh = np.load(tmp_path / "p.npz")
    assert sorted(fresh.files) == sorted(gold.files)
    for k in gold.files:
        assert np.array_equal(fresh[k], gold[k]), k
