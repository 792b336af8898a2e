"""Make tests/golden/halton_reference.txt: the output of tests/cpp/halton_draws.cpp
compiled against the reference's own src/random/halton.hh (standard library
only), to pin the drop-in header include/src/random/halton.hh bit for bit.
Run in the development container, where the reference tree exists; the output
is committed.

Usage: python tests/golden/make_halton.py <reference project root>
"""
import os
import subprocess
import sys
import tempfile

here = os.path.dirname(os.path.abspath(__file__))
src = os.path.join(os.path.dirname(here), "cpp", "halton_draws.cpp")
tree = sys.argv[1]
with tempfile.TemporaryDirectory() as d:
    exe = os.path.join(d, "halton_draws")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", tree, src, "-o", exe])
    out = subprocess.check_output([exe], text=True)
open(os.path.join(here, "halton_reference.txt"), "w").write(out)
