"""Extract the far-field term sequence pinned by the reference's own unrolled kernel.

fast_rap_src_dfpt_gpu_eval/sum_up_far_dist_potential_dot.hpp:12-210 spells out,
for l_max <= 6, one line per table row n:
    acc += pA(x) * pB(y) * pC(z) * Fp[nn] * multipole_c[n];
with the early return after each l.  This script reads that file AS TEXT and
writes tests/golden/index_cc_l6.json: the (i, j, k, nn) of every row and the
cumulative row count at each l.  It runs only where the reference tree exists;
the JSON it wrote is committed.
"""
import json
import os
import re
import sys

# the reference checkout: $FR_REF, else the directory `reference` beside this repository
ref = os.environ.get("FR_REF") or os.path.join(
    os.path.dirname(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))), "reference")
path = os.path.join(ref, "fast_rap_src_dfpt_gpu_eval", "sum_up_far_dist_potential_dot.hpp")
src = open(path).read()
body = src[src.index("sum_up_far_dist_potential_dot_spec"):]
body = body[: body.index("\n}\n")]
rows, counts = [], []
term = re.compile(r"acc \+= p(\d)\(x\) \* p(\d)\(y\) \* p(\d)\(z\) \* Fp\[(\d+)\] \* multipole_c\[(\d+)\];")
for line in body.splitlines():
    m = term.search(line)
    if m:
        i, j, k, nn, n = map(int, m.groups())
        assert n == len(rows), (n, len(rows))
        rows.append([i, j, k, nn])
    elif "if constexpr (l_max ==" in line:
        counts.append(len(rows))
if not counts or counts[-1] != len(rows):
    counts.append(len(rows))
out = {"source": "fast_rap_src_dfpt_gpu_eval/sum_up_far_dist_potential_dot.hpp:12-210",
       "rows_ijk_nn": rows, "n_cc_lm_ijk": counts}
dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "index_cc_l6.json")
json.dump(out, open(dst, "w"))
print(len(rows), counts, file=sys.stderr)
