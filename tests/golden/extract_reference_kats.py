"""Extracts the known-answer tests of the reference's marching-step sampler
(unittests/marching_steps.cpp, DensityArray sections) into
tests/golden/marching_steps_kats.json.

Run once where the reference is available:

    python tests/golden/extract_reference_kats.py /path/to/reference

The fixture holds, per SECTION, the operations and expected values exactly as
written in the reference test (numeric literals are kept as text, with their
C++ type suffix, so the test can convert them to float32 / float64 the way the
C++ compiler does).  Sections whose statements are not plain put / CHECK
sequences (the randomised section, the sampler property checks) are not
extracted; tests/test_oracle_kats.py covers those separately.
"""
from __future__ import annotations

import json
import os
import re
import sys

NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?f?"


def lit(tok: str) -> str:
    tok = tok.strip()
    m = re.fullmatch(r"scalar_t\((.*)\)", tok)
    if m:
        tok = m.group(1).strip()
    if not re.fullmatch(NUM, tok):
        raise ValueError(f"not a literal: {tok!r}")
    return tok


def triple(text: str) -> list[str]:
    parts = [p for p in text.split(",")]
    if len(parts) != 3:
        raise ValueError(text)
    return [lit(p) for p in parts]


def extract(path: str) -> dict:
    src = open(path).read()
    start = src.index('TEMPLATE_TEST_CASE("dgmr marching step DensityArray"')
    end = src.index('TEST_CASE("dgmr marching step Array")')
    body = src[start:end]
    sections = []
    current = None
    re_section = re.compile(r'SECTION\("([^"]+)"\)')
    re_combine = re.compile(r"auto v = DensityArray::combine\(\{([^}]*)\},\s*\{([^}]*)\}\);")
    re_arr = re.compile(r"DensityArray<(\d+), scalar_t> arr\(([^)]*)\);")
    re_put = re.compile(r"arr\.put\(\{([^}]*)\}\);")
    re_size = re.compile(r"CHECK\(arr\.size\(\) == (\d+)\);")
    re_field = re.compile(r"CHECK\(arr\[(\d+)\]\.(start|end|delta_t) == (" + NUM + r")\);")
    re_vfield = re.compile(r"CHECK\(v\[(\d+)\]\.(start|end|delta_t) == (" + NUM + r")\);")
    for line in body.splitlines():
        line = line.strip()
        m = re_section.search(line)
        if m:
            current = {"name": m.group(1), "ops": []}
            sections.append(current)
            continue
        if current is None or line.startswith("//"):
            continue
        if "std::srand" in line or "for (" in line or "smallest" in line:
            current["unsupported"] = True
        if current.get("unsupported"):
            continue
        if (m := re_combine.search(line)):
            current["ops"].append({"op": "combine", "a": triple(m.group(1)), "b": triple(m.group(2))})
        elif (m := re_arr.search(line)):
            current["ops"].append({"op": "array", "capacity": int(m.group(1)), "start": lit(m.group(2))})
        elif (m := re_put.search(line)):
            current["ops"].append({"op": "put", "entry": triple(m.group(1))})
        elif (m := re_size.search(line)):
            current["ops"].append({"op": "size", "value": int(m.group(1))})
        elif (m := re_field.search(line)):
            current["ops"].append({"op": "field", "index": int(m.group(1)), "field": m.group(2), "value": m.group(3)})
        elif (m := re_vfield.search(line)):
            current["ops"].append({"op": "vfield", "index": int(m.group(1)), "field": m.group(2), "value": m.group(3)})
    kept = [s for s in sections if not s.get("unsupported") and s["ops"]]
    return {"source": "unittests/marching_steps.cpp (TEMPLATE_TEST_CASE \"dgmr marching step DensityArray\")",
            "sections": kept}


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: extract_reference_kats.py <path of the reference project checkout>")
    ref = sys.argv[1]
    data = extract(os.path.join(ref, "unittests", "marching_steps.cpp"))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "marching_steps_kats.json")
    with open(out, "w") as f:
        json.dump(data, f, indent=1)
    n_checks = sum(1 for s in data["sections"] for o in s["ops"] if o["op"] in ("size", "field", "vfield"))
    print(f"{len(data['sections'])} sections, {n_checks} checks -> {out}")


if __name__ == "__main__":
    main()
