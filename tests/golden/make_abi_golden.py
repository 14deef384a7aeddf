"""Writes tests/golden/tapp_abi.json: the prototypes, constant values and
DLPack struct sizes of the reference's pinned C headers
(crates/tprims-capi/include/tapp.h and include/tprims/tprims.h, with the
DLPack header they include), read in place and seen through the C compiler
(abi_extract.py). tests/test_abi_cpu.py compares include/tprims_b200.h with it.

Run: python tests/golden/make_abi_golden.py <reference-root>
"""
import glob
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from abi_extract import extract  # noqa: E402


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_abi_golden.py <reference-root>")
    inc = os.path.join(sys.argv[1], "crates", "tprims-capi", "include")
    files = sorted(glob.glob(os.path.join(inc, "tapp", "*.h")) + glob.glob(os.path.join(inc, "tprims", "*.h")))
    facts = extract([inc], ["tapp.h", "tprims/tprims.h"], files + [os.path.join(inc, "tapp.h")])
    facts["source"] = ("crates/tprims-capi/include/{tapp.h,tapp/*.h,tprims/*.h} of the reference, through "
                       "gcc -aux-info and a compiled value dump")
    with open(os.path.join(HERE, "tapp_abi.json"), "w") as f:
        json.dump(facts, f, indent=1, sort_keys=True)
        f.write("\n")
    print(f"{len(facts['prototypes'])} prototypes, {len(facts['values'])} values")


if __name__ == "__main__":
    main()
