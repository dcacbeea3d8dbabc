"""Generate the committed fixtures under tests/golden from the reference tree.

The reference (gargantua, Swift + Metal) cannot run here, so its acceptance
data is carried over as files:

  goldens/*.json      the 11 golden definitions, copied verbatim
                      (gargantua/goldens/*.json: claim, kind, expected,
                      tolerance, method, parameters)
  constants.json      every #define of the reference's generated constants
                      header (Sources/Gargantua/Shaders/Constants.h:8-216),
                      symbol -> numeric value, so a CPU test can check that
                      include/gargantua_constants.h carries the same numbers

Usage: python tests/golden/make_fixtures.py /path/to/gargantua
"""
import json
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(reference: str) -> None:
    goldens_src = os.path.join(reference, "goldens")
    goldens_dst = os.path.join(HERE, "goldens")
    os.makedirs(goldens_dst, exist_ok=True)
    for name in sorted(os.listdir(goldens_src)):
        if name.endswith(".json"):
            shutil.copyfile(os.path.join(goldens_src, name), os.path.join(goldens_dst, name))

    header = os.path.join(reference, "Sources", "Gargantua", "Shaders", "Constants.h")
    constants = {}
    pattern = re.compile(r"^#define\s+([A-Z0-9_]+)\s+\(([-+0-9.eE]+)([fu])\)\s*$")
    with open(header) as fh:
        for line in fh:
            m = pattern.match(line.strip())
            if m:
                symbol, number, suffix = m.groups()
                constants[symbol] = float(number) if suffix == "f" else int(number)
    with open(os.path.join(HERE, "constants.json"), "w") as fh:
        json.dump(constants, fh, indent=1, sort_keys=True)
        fh.write("\n")
    print(f"{len(os.listdir(goldens_dst))} goldens, {len(constants)} constants")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py /path/to/gargantua (the reference's source tree)")
    main(sys.argv[1])
