"""The GPU error lab produces its CSV / markdown, with the numbers the refinement
contract implies: every tier ends at the fp64 backward error, fp32 refines
well-conditioned matrices without fallback, and the emulated formats' factorization
errors sit at their unit roundoff."""
import csv

import pytest

from conftest import load_pkg

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

lab = load_pkg("lab")


def test_lab_rows_and_report(tmp_path):
    rows = lab.mixed_rows(16, 1e2, 128, 0) + lab.emulated_rows(8, 1e2, 16, 0)
    lab.write(tmp_path, rows)
    text = (tmp_path / "gpu_lab.md").read_text()
    assert "Mixed precision" in text and "Emulated" in text
    with open(tmp_path / "gpu_lab.csv") as f:
        got = list(csv.DictReader(f))
    assert len(got) == len(rows) == 8 + 4
    for r in rows:
        if r["section"] == "mixed":
            assert r["backward_max"] <= 1e-15, r
            if r["tier"] == "fp32":
                assert r["refined_frac"] == 1.0
        else:
            u = 2.0 ** -11 if r["tier"] == "fp16" else 2.0 ** -8
            assert r["fail_frac"] == 0.0 and 1e-3 * u < r["backward_med"] < 16 * u, r
