"""Extract the golden vectors of the ExaGeoStatCPP unit tests into a JSON fixture.

Run once, in a checkout that has the reference source tree, as
``python tests/golden/extract_reference_goldens.py /path/to/ExaGeoStatCPP``.
It reads the reference test sources as text (nothing is compiled or run) and
writes ``reference_goldens.json`` beside this script.  The tests only read the
JSON file, so they also run where the reference tree is absent.
"""
from __future__ import annotations

import json
import os
import re
import sys


def _numbers(text: str) -> list[float]:
    return [float(v) for v in re.findall(r"-?\d+\.\d+(?:[eE][-+]?\d+)?", text)]


def _array_after(src: str, marker: str, start: int = 0) -> tuple[list[float], int]:
    i = src.index(marker, start)
    j = src.index("{", i)
    k = src.index("}", j)
    return _numbers(src[j:k]), k


def _line_of(src: str, pos: int) -> int:
    return src.count("\n", 0, pos) + 1


def main(ref: str) -> None:
    out: dict = {}
    p = "tests/cpp-tests/data-generators/concrete/TestSyntheticGenerator.cpp"
    src = open(os.path.join(ref, p)).read()
    i = src.index("vector<double> x = {")
    x, _ = _array_after(src, "vector<double> x = {")
    y, _ = _array_after(src, "vector<double> y = {")
    out["locations_n9_seed0"] = {"source": f"{p}:{_line_of(src, i)}", "n": 9, "seed": 0,
                                 "x": x, "y": y, "margin": 1e-6}

    p = "tests/cpp-tests/kernels/concrete/TestUnivariateMaternStationary.cpp"
    src = open(os.path.join(ref, p)).read()
    i = src.index("expected_output_data[] =")
    z, _ = _array_after(src, "expected_output_data[] =")
    out["z_n9_dts5_seed0"] = {"source": f"{p}:{_line_of(src, i)}", "n": 9, "dts": 5, "seed": 0,
                              "theta": [1.0, 0.1, 0.5], "z": z, "margin": 1e-6}

    p = "tests/cpp-tests/api/TestExaGeoStatApi.cpp"
    src = open(os.path.join(ref, p)).read()
    i = src.index("expected_output_data[] =")
    z, _ = _array_after(src, "expected_output_data[] =")
    out["z_n16_dts9_seed0"] = {"source": f"{p}:{_line_of(src, i)}", "n": 16, "dts": 9, "seed": 0,
                               "theta": [1.0, 0.1, 0.5], "z": z, "margin": 1e-6}
    i = src.index("auto *z_matrix = new double[N]")
    zf, _ = _array_after(src, "auto *z_matrix = new double[N]", i)
    xf, _ = _array_after(src, "auto *location_x = new double[N]", i)
    yf, _ = _array_after(src, "auto *location_y = new double[N]", i)
    out["fixture_n16"] = {"source": f"{p}:{_line_of(src, i)}", "n": 16, "z": zf, "x": xf, "y": yf}
    m = re.search(r"expected = (-?\d+\.\d+);\s*\n\s*\} else if \(aComputation == DIAGONAL_APPROX\)", src)
    md = re.search(r"DIAGONAL_APPROX\) \{\s*\n\s*expected = (-?\d+\.\d+);", src)
    out["modeling_loglik_n16"] = {
        "source": f"{p}:{_line_of(src, m.start())}", "exact_dense": float(m.group(1)),
        "diag_approx_band1": float(md.group(1)), "dts": 8, "lb": [0.1, 0.1, 0.1],
        "ub": [5.0, 5.0, 5.0], "max_mle_iterations": 3, "tolerance_exponent": 4, "margin": 1e-6}

    p = "tests/cpp-tests/prediction/TestPrediction.cpp"
    src = open(os.path.join(ref, p)).read()
    m = re.search(r"GetMSPEError\(\) == Catch::Approx\((\d+\.\d+)\)", src)
    et = re.search(r"estimated_theta\{([^}]*)\}", src)
    out["prediction_mspe_n16"] = {
        "source": f"{p}:{_line_of(src, m.start())}", "mspe": float(m.group(1)), "z_miss_number": 4,
        "estimated_theta": _numbers(et.group(1)), "dts": 8,
        "note": "Catch::Approx default relative epsilon is ~1.19e-5 (float epsilon * 100)"}
    # MLOE/MMOM: the third PickRandomPoints split of the test case (Catch re-runs the
    # body for each SECTION; the MSPE and IDW sections split first), truth theta =
    # the initial theta, estimated theta = (0.9, 0.09, 0.4)
    m1 = re.search(r"GetMLOE\(\) == Catch::Approx\((-?\d+\.\d+)\)\.margin\((\d+\.\d+)\)", src)
    m2 = re.search(r"GetMMOM\(\) == Catch::Approx\((-?\d+\.\d+)\)\.margin\((\d+\.\d+)\)", src)
    out["prediction_mloe_mmom_n16"] = {
        "source": f"{p}:{_line_of(src, m1.start())}", "mloe": float(m1.group(1)), "mmom": float(m2.group(1)),
        "margin": float(m1.group(2)), "z_miss_number": 4, "split_index": 2,
        "truth_theta": [1.0, 0.1, 0.5], "estimated_theta": [0.9, 0.09, 0.4]}
    i = src.index("required_fisher = {")
    fisher, _ = _array_after(src, "required_fisher = {")
    out["prediction_fisher_n16"] = {
        "source": f"{p}:{_line_of(src, i)}", "fisher_inverse": fisher, "margin": 1e-6,
        "estimated_theta": [0.9, 0.09, 0.4], "n": 16,
        "note": "inverse of the 3x3 Fisher information at the estimated theta on all 16 fixture locations"}

    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_goldens.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EXAGEOSTAT_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: extract_reference_goldens.py <ExaGeoStatCPP source tree> "
                 "(or set EXAGEOSTAT_REFERENCE_ROOT)")
    main(root)
