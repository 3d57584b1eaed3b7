"""The C++ binding shown in INTEGRATION.md is the header the tests compile.

Every code line of the first C++ block of section 2 (an excerpt of CudaDense.hpp)
must appear, whitespace aside, in the compiled host headers, so the document
cannot drift from the binding that tests/cpp/test_exageostat_api.cpp runs."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "exageostatcpp_b200", "host", "include", "linear-algebra-solvers")


def test_integration_snippet_lines_are_in_the_compiled_binding():
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    sec = doc[doc.index("## 2."):]
    block = re.search(r"```cpp\n(.*?)```", sec, re.S).group(1)
    src = ""
    for name in ("LinearAlgebraMethods.hpp", os.path.join("concrete", "CudaDense.hpp")):
        src += open(os.path.join(HDR, name)).read()
    norm = lambda t: re.sub(r"\s+", " ", t).strip()  # noqa: E731
    body = norm(src)
    lines = [norm(line) for line in block.splitlines() if norm(line) and norm(line) not in ("}", "};")]
    assert len(lines) > 20
    missing = [line for line in lines if line not in body]
    assert not missing, missing
