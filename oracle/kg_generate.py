"""Generate the reference's optimised ADER-DG kernels with its own KernelGenerator. CHECKER /
BASELINE ONLY: nothing of the product links the output.

The KernelGenerator (KernelGenerator/kernelgenerator/controller.py:51-286 in the reference checkout)
is imported from the checkout and run in its plain-loop mode: its Configuration.useLibxsmm is set
to False in this process (the libxsmm submodule is empty in the checkout, so the libxsmm variant
cannot be generated). Nothing is written to the checkout; the generated sources go to
oracle/_ref/kg/<name>/kernels/, beside the compiled reference kernels.

    python oracle/kg_generate.py [--ref PATH_TO_EXAHYPE_CHECKOUT]

Generates Euler 3D order 5 (the benchmark configuration) and order 3 (the parity test's), both
nVar 5, no parameters, flux only, arch skx (AVX-512 padding), Gauss-Legendre nodes.
"""
import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [("euler_o5", 5), ("euler_o3", 3)]


def generate(ref, name, order):
    out = os.path.join(HERE, "_ref", "kg", name)
    os.makedirs(out, exist_ok=True)
    sys.path.insert(0, os.path.join(ref, "KernelGenerator"))
    from kernelgenerator.configuration import Configuration
    Configuration.useLibxsmm = False
    from kernelgenerator import Controller
    argv = sys.argv
    sys.argv = ["kernelgenerator", "aderdg", out, "kernels", "kg::" + name, "Euler::EulerSolver_ADERDG", "5", "0",
                str(order), "3", "nonlinear", "skx", "--useFlux"]
    try:
        Controller().generateCode()
    finally:
        sys.argv = argv
    return os.path.join(out, "kernels")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("EXAHYPE_REF", "/root/reference"))
    args = ap.parse_args()
    for name, order in CASES:
        print(generate(args.ref, name, order))


if __name__ == "__main__":
    main()
