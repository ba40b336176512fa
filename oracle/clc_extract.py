"""Turns one of the reference's OpenCL kernel files into C the host compiler
can build with oracle/clc_shim.h -- part of the oracle's reference build
(test infrastructure only; its output goes to oracle/_ref/).

The reference stores each kernel file as one or more C++ raw-string literals
(src/library/kernels/*.cl, wrapped in R"( ... )" so that
src/library/internal/kernel-cache.cpp can embed the text). This script:

  * drops the raw-string delimiter lines, leaving the OpenCL C text as is;
  * turns each work-group-local array declared in a kernel body
    (``__local T name[N];`` / ``local volatile T name[N];``) into a function
    static, which the shim's threads of one work-group share.

Nothing else in the kernel text is changed.

    python clc_extract.py <reference .cl file> <output .c.inc file>
"""
from __future__ import annotations

import re
import sys

DECL = re.compile(r"^(\s*)(?:__local|local)\s+((?:volatile\s+)?\w+)\s+(\w+)\s*\[([^\]]+)\]\s*;")


def extract(text: str) -> str:
    out = []
    for line in text.splitlines():
        if line.strip() in ('R"(', ')"'):
            out.append("")  # keep line numbers
            continue
        m = DECL.match(line)
        if m:
            line = f"{m.group(1)}static {m.group(2)} {m.group(3)}[{m.group(4)}];"
        out.append(line)
    return "\n".join(out) + "\n"


def main(argv):
    src, dst = argv[1], argv[2]
    with open(src) as f:
        text = f.read()
    with open(dst, "w") as f:
        f.write(f'#line 1 "{src}"\n')
        f.write(extract(text))


if __name__ == "__main__":
    main(sys.argv)
