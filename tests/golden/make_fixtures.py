"""Make the small input fixtures of the drop-in CLI tests from the reference's
own input files (run in the development container, where the reference tree
exists; the outputs are committed):

* panda_problems_small.json -- the first 3 valid problems of every family of
  scripts/panda_problems.json (same structure: {"problems": {family: [...]}});
* scene_small.txt -- scripts/scene.txt restricted to the OBJECT lines, every
  group's mean line and the first 8 samples of every sampled group.

Usage: python tests/golden/make_fixtures.py <reference>/scripts
"""
import json
import os
import sys

here = os.path.dirname(os.path.abspath(__file__))
src = sys.argv[1]

d = json.load(open(os.path.join(src, "panda_problems.json")))
small = {"robot": d.get("robot"), "problems": {}}
for fam in sorted(d["problems"]):
    keep = [p for p in d["problems"][fam] if p.get("valid")][:3]
    for p in keep:
        p.pop("goals", None)
        p.pop("start", None)
    small["problems"][fam] = keep
json.dump(small, open(os.path.join(here, "panda_problems_small.json"), "w"), indent=0)

seen = {}
out = []
for line in open(os.path.join(src, "scene.txt")):
    f = line.split()
    if not f:
        continue
    cat = f[0]
    if cat.endswith("_"):
        seen[cat] = seen.get(cat, 0) + 1
        if seen[cat] > 8:
            continue
    out.append(line.rstrip("\n"))
open(os.path.join(here, "scene_small.txt"), "w").write("\n".join(out) + "\n")
print("wrote", len(small["problems"]), "families,", len(out), "scene lines")
