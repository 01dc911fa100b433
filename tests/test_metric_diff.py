"""The metric difference forms used by the mixed-precision line search
(dmu2 / dmu3 in egg_b200/csrc/metric*.cuh), compiled for the host: exact to
fp64 round-off against extended-precision differences, and in fp32 far more
accurate than subtracting two fp32 metric values, which loses the change
entirely where mu ~ 1 (the size term at small cells)."""

from __future__ import annotations

import shutil
import subprocess

import pytest

from tests.conftest import ROOT

KIND = {0: "shape", 1: "untangle", 2: "shape_size"}


@pytest.fixture(scope="module")
def report(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path_factory.mktemp("metric_diff") / "check"
    subprocess.run([gxx, "-O1", "-std=c++17", f"-I{ROOT / 'egg_b200' / 'csrc'}",
                    str(ROOT / "tests" / "native" / "metric_diff_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    rows = {}
    for line in out.split("\n"):
        if line.strip():
            k, d, e64, e32, naive = line.split()
            rows[(KIND[int(k)], int(d))] = (float(e64), float(e32), float(naive))
    return rows


@pytest.mark.parametrize("kind", list(KIND.values()))
@pytest.mark.parametrize("dim", [2, 3])
def test_difference_form_accuracy(report, kind, dim):
    e64, e32, naive = report[(kind, dim)]
    assert e64 < 1e-8
    assert e32 < 0.1
    assert naive > 10 * e32


def test_forms_without_zero_terms_match_the_general_forms(tmp_path):
    """dmu2_col, role3 / line_sample3 / line_norms3 with an axis hint leave
    out terms with an exact-zero factor; they agree with the general forms to
    rounding."""
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "axis"
    subprocess.run([gxx, "-O1", "-std=c++17", f"-I{ROOT / 'egg_b200' / 'csrc'}",
                    str(ROOT / "tests" / "native" / "axis_forms_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    worst = {k: float(v) for k, v in (line.split() for line in out.strip().split("\n"))}
    assert set(worst) == {"dmu2_col", "role3_ax", "line_sample3_ax", "line_norms3_ax"}
    for name, w in worst.items():
        assert w < 1e-13, (name, w)


@pytest.fixture(scope="module")
def x2_report(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path_factory.mktemp("x2") / "check"
    subprocess.run([gxx, "-O1", "-std=c++17", "-ffp-contract=off", f"-I{ROOT / 'egg_b200' / 'csrc'}",
                    str(ROOT / "tests" / "native" / "x2_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    rows = {}
    for line in out.split("\n"):
        if line.strip():
            what, k, err = line.split()
            rows[(what, KIND[int(k)])] = float(err)
    return rows


@pytest.mark.parametrize("kind", list(KIND.values()))
def test_packed_pair_forms_match_fp64(x2_report, kind):
    """The two-lane fp32 forms of the packed 2D sweep (x2.cuh): role
    contributions of a sample pair and the metric change of a trial pair,
    against the fp64 metric, at fp32 accuracy (the scalar fp32 forms reach
    1.0e-5 / 2.8e-6 / 1.6e-5 for shape / untangle / shape_size here); an index
    or sign slip would show as an O(1) error."""
    assert x2_report[("roles", kind)] < 1e-4
    assert x2_report[("dmu", kind)] < 3e-4
