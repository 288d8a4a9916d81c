"""Generate the solver glue Abstract<Solver>.{h,cpp} of an application for the B200 C ABI.

The reference's toolkit generates Abstract<App>Solver_ADERDG from the application's specification:
a class whose kernel methods call kernels::aderdg::generic::c templated on the user's solver
(Toolkit/exahype/toolkit/templates/solvers/AbstractGenericADERDGSolverImplementation.template
:104-361, AbstractGenericADERDGSolverHeader.template:34-68). This generator emits the same methods
calling include/exa_aderdg.h instead, from a small JSON specification:

    {"project": "Euler", "solver": "EulerSolver_ADERDG", "pde": 0, "dimension": 3, "order": 3,
     "variables": 5, "parameters": 0, "cfl": 0.9, "maxPicardIterations": false,
     "precision": "FP64"}

"pde" is an exa_pde id: a built-in system (EXA_PDE_EULER ...) or an application functor registered
with include/exa_aderdg_user.cuh (>= EXA_PDE_USER_BASE).

    python exahype-engine_b200/glue/generate_glue.py spec.json OUTDIR
"""
import json
import os
import sys

import jinja2

HERE = os.path.dirname(os.path.abspath(__file__))
# ADER-DG PNPM by order (Toolkit/exahype/toolkit/solverController.py:17-23)
PNPM = [1.0, 0.33, 0.17, 0.1, 0.069, 0.045, 0.038, 0.03, 0.02, 0.015]


def generate(spec, outdir, spec_name="<dict>"):
    ctx = dict(project=spec["project"], solver=spec["solver"], pde=int(spec["pde"]), dim=int(spec["dimension"]),
               order=int(spec["order"]), nvar=int(spec["variables"]), npar=int(spec.get("parameters", 0)),
               cfl=repr(float(spec.get("cfl", 0.9))), pnpm=repr(float(spec.get("pnpm", PNPM[int(spec["order"])]))),
               fixed_picard=bool(spec.get("maxPicardIterations", False)),
               precision=str(spec.get("precision", "FP64")).upper(), spec=spec_name)
    if ctx["dim"] not in (2, 3) or ctx["precision"] not in ("FP64", "MIXED"):
        raise ValueError("dimension must be 2 or 3 and precision FP64 or MIXED")
    env = jinja2.Environment(loader=jinja2.FileSystemLoader(HERE), keep_trailing_newline=True,
                             undefined=jinja2.StrictUndefined)
    os.makedirs(outdir, exist_ok=True)
    out = []
    for tmpl, ext in (("AbstractSolver.h.template", ".h"), ("AbstractSolver.cpp.template", ".cpp")):
        path = os.path.join(outdir, "Abstract%s%s" % (ctx["solver"], ext))
        with open(path, "w") as f:
            f.write(env.get_template(tmpl).render(**ctx))
        out.append(path)
    return out


def main():
    if len(sys.argv) != 3:
        sys.stderr.write(__doc__)
        return 2
    with open(sys.argv[1]) as f:
        spec = json.load(f)
    for p in generate(spec, sys.argv[2], os.path.basename(sys.argv[1])):
        print(p)
    return 0


if __name__ == "__main__":
    sys.exit(main())
