"""Host-side helpers of bench.py that shape its JSON line: the split form's
per-part error report, the count of slice products behind its roofline, and
the labels of the roofline peaks (measured when the peaks file is present,
fallback otherwise)."""
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402
import qd_imsrg_b200 as qd  # noqa: E402


def test_split_errors_per_part():
    P = qd.Layout(6, 4, device=qd.HOST_ONLY)
    ref = qd.random_operator(P, 1, 3)
    got = ref.copy()
    assert bench.split_errors(P, got, ref)["max"] == 0.0
    q = int(np.argmax(P.dims[:, 2] * P.dims[:, 0]))  # a block with a Vpphh part
    s = int(P.offs[q, 2])
    got[s] += 1e-6
    err = bench.split_errors(P, got, ref)
    assert err["Vpphh"] > 0.0 and err["max"] == err["Vpphh"]
    assert all(v == 0.0 for k, v in err.items() if k not in ("Vpphh", "max"))


def test_slice_pairs_and_form():
    assert [bench.slice_pairs(s) for s in (1, 2, 4, 8)] == [1, 3, 10, 36]
    assert bench.form_name(0) == "plain FP64"
    assert "4 BF16 slices" in bench.form_name(4)


def test_peak_labels(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert "fallback" in bench.hbm_source() and bench.hbm_peak_gbs() == 6650.0
    assert "fallback" in bench.bf16_source()
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6500.0, "bf16_tflops": 1600.0}))
    assert "of measured" in bench.hbm_source() and bench.hbm_peak_gbs() == 6500.0
    assert bench.bf16_peak_tflops() == 1600.0 and "of measured" in bench.bf16_source()
