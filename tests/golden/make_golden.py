"""Copy the reference's own golden vectors for this path into tests/golden/.

Usage: python make_golden.py <path of the WannierNLQG source tree>.  The files are
data fixtures of the reference's test suite (not source):
  test/fixtures/third_order/jerk_input.dat, jerk_reference.dat   (third_order_unit.jl:210-253)
  examples/fixtures/synthetic_runtime/synthetic_tb.dat            (4-orbital _tb.dat fixture)
  test/fixtures/second_harmonic/*.dat                             (second_harmonic_unit.jl:13-100)
"""
import os
import shutil
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py <WannierNLQG source tree>")
REF = sys.argv[1]
HERE = os.path.dirname(os.path.abspath(__file__))

FILES = {
    "jerk_input.dat": "test/fixtures/third_order/jerk_input.dat",
    "jerk_reference.dat": "test/fixtures/third_order/jerk_reference.dat",
    "synthetic_tb.dat": "examples/fixtures/synthetic_runtime/synthetic_tb.dat",
}

if __name__ == "__main__":
    for dst, src in FILES.items():
        shutil.copyfile(os.path.join(REF, src), os.path.join(HERE, dst))
    shg_src = os.path.join(REF, "test/fixtures/second_harmonic")
    os.makedirs(os.path.join(HERE, "second_harmonic"), exist_ok=True)
    for name in sorted(os.listdir(shg_src)):
        if name.endswith(".dat"):
            shutil.copyfile(os.path.join(shg_src, name), os.path.join(HERE, "second_harmonic", name))
    print("golden fixtures written to", HERE)
