"""Extracts the reference's golden values for its 1-D bar test into runtest1.json.

Source: ValidationTests/results/runtest1.out of bourdin/VPFHF (the output of
ValidationTests/test1.c run by `make runtest1`, arguments at
ValidationTests/makefile:196-198).  Run from the repository root:

    python tests/golden/make_runtest1.py /path/to/VPFHF

(or with the path of the VPFHF source tree in the VPFHF_REFERENCE environment variable).
"""
import json
import os
import re
import sys

ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("VPFHF_REFERENCE")
if not ref:
    sys.exit("usage: make_runtest1.py /path/to/VPFHF (or set VPFHF_REFERENCE)")
text = open(f"{ref}/ValidationTests/results/runtest1.out").read()
steps = []
for block in re.split(r"==== time step ", text)[1:]:
    t = float(re.search(r"t = ([-+.\deE]+)", block).group(1))
    rec = {"t": t, "am_its": len(re.findall(r"^Step \d+ / \d+", block, re.M))}
    for key, pat in [("cov", r"Total crack opening: ([-+.\deE]+)"),
                     ("elastic", r"Elastic Energy:\s+([-+.\deE]+)"),
                     ("surface", r"Surface  energy:\s+([-+.\deE]+)")]:
        m = re.search(pat, block)
        if m:
            rec[key] = float(m.group(1))
    steps.append(rec)
json.dump({"source": "ValidationTests/results/runtest1.out",
           "args": "-n 101,5,5 -l 10,1,1 -nu 0 -epsilon 0.5 -eta 1e-8 -gc .1 -altmintol 1.e-3 "
                   "-maxtimestep 11 -maxtimevalue 4 -atnum 1 -V_X0_BC ONE -U_X0_BC_0 FIXED "
                   "-U_X0_0 -1. -U_X0_BC_1 ZERO -U_X0_BC_2 ZERO -V_X1_BC ONE -U_X1_BC_0 FIXED "
                   "-U_X1_0 1. -U_X1_BC_1 ZERO -U_X1_BC_2 ZERO -alpha 0 -beta 0 -pressure 0",
           "steps": steps}, open("tests/golden/runtest1.json", "w"), indent=1)
print(len(steps), "steps")
