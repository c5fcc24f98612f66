"""The shipped C ABI of libqmb200.so as a plain-text inventory, the C counterpart of the .NET
PublicAPI.Shipped.txt files: every exported prototype, every struct's field list and every
#define of include/qm_b200.h, whitespace-normalised, one per line, sorted.

    python include/shipped_abi.py          # prints the inventory of the current header
    python include/shipped_abi.py --write  # rewrites include/qm_b200.shipped.txt

tests/test_abi.py fails when the header and the committed inventory differ, so an entry point or
a struct layout cannot change without the inventory (and the ABI version) changing with it.
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
HEADER = HERE / "qm_b200.h"
SHIPPED = HERE / "qm_b200.shipped.txt"


def _norm(text: str) -> str:
    return re.sub(r"\s+", " ", text).replace("( ", "(").replace(" )", ")").replace(" ,", ",").strip()


def inventory(header: str) -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", header, flags=re.S)
    lines = []
    for m in re.finditer(r"#define\s+(QM_\w+)\s+(\S+)", text):
        if m.group(1) != "QM_B200_H":
            lines.append(f"define {m.group(1)} {m.group(2)}")
    for m in re.finditer(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*\w+\s*;", text, flags=re.S):
        fields = [_norm(f) for f in m.group(2).split(";") if f.strip()]
        lines.append(f"struct {m.group(1)} {{ {'; '.join(fields)}; }}")
    for m in re.finditer(r"typedef\s+[^;{}]*\(\s*\*\s*(qm_\w+)\s*\)\s*\([^;]*\)\s*;", text):
        lines.append(_norm(m.group(0)).rstrip(";"))
    for m in re.finditer(r"(?<![\w*])((?:int32_t|int64_t|void|double)\s*\*?\s*qm_\w+\s*\([^;{}]*\))\s*;", text):
        lines.append("function " + _norm(m.group(1)))
    return sorted(set(lines))


def main() -> None:
    inv = inventory(HEADER.read_text())
    if "--write" in sys.argv:
        SHIPPED.write_text("".join(l + "\n" for l in inv))
    else:
        print("\n".join(inv))


if __name__ == "__main__":
    main()
