"""The results matrix (CPU): `python -m dynlplus_b200.matrix <dir>` writes the same matrix.csv and
matrix.md as the reference's scripts/matrix.py for the same benchmark CSVs (fixture made by running
the reference's script, tests/golden/make_golden.py)."""
import os
import shutil

import pandas as pd

from conftest import GOLDEN
from dynlplus_b200 import matrix


def test_matrix_matches_the_reference(tmp_path, capsys):
    src = os.path.join(GOLDEN, "matrix")
    for f in ("sbm-20k.csv", "er-50k.csv"):
        shutil.copy(os.path.join(src, f), tmp_path / f)
    d = str(tmp_path)
    matrix.main(d)
    capsys.readouterr()
    got_csv = pd.read_csv(tmp_path / "matrix.csv")
    want_csv = pd.read_csv(os.path.join(src, "expected_matrix.csv"))
    pd.testing.assert_frame_equal(got_csv, want_csv)
    got_md = (tmp_path / "matrix.md").read_text(encoding="utf-8").replace(d, "RESULTS_DIR")
    want_md = open(os.path.join(src, "expected_matrix.md"), encoding="utf-8").read()
    assert got_md == want_md
