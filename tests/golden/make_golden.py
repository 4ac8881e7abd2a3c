"""Generate the golden fixtures of this directory from the reference itself.

The reference ParMooN hot path is compiled from its own sources by
``oracle/ref/Makefile`` into ``oracle/_ref/pmg_ref`` (a driver of ours that
calls TSquareStructure3D, TAssembleMat3D::Assemble3D, TMultiGrid3D,
TFgmresIte, Prolongate/DefectRestriction and TSystemTCD3D).  This script runs
that binary on small cases and packs its dumps into ``<case>.npz``:

  L<l>_{rowptr,kcol,entries,rhs,elem_dof,cell_vert,dof_xyz}  per level
  L<l>_{N,active_bound,n_cells,n_loc}                         per level
  L<l>_parent                                                  parent cells (l >= 1)
  T<l>_{coarse_in,fine_in,prolongated,restricted}             transfer probes
  solution, solve_iterations, res0, res_final                 FGMRES + GMG solve
  params                                                      the driver options

``tcd3d_amc.npz`` additionally holds the L2 / H1-semi errors the recorded
reference run printed (ReadIn/tcd3d_GMG.out), so the compiled reference can be
checked against the reference's own log without the source tree.

Run from the repository root after ``make -C oracle/ref``:
    python tests/golden/make_golden.py [--ref /root/reference]
"""
import argparse
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BIN = os.path.join(ROOT, "oracle", "_ref", "pmg_ref")

# name -> (mode, driver options)
# the solves stop at |r| <= 1e-14 |r0| (red), near the FP64 rounding floor, so
# the stored solution is the discrete solution to ~cond(A) * 1e-14
TIGHT = dict(red=1e-14, maxit=300)
CASES = {
    "q1_laplace": ("cd3d", dict(order=1, levels=3, coarse_steps=1, problem="laplace", **TIGHT)),
    "q1_supg": ("cd3d", dict(order=1, levels=3, coarse_steps=1, problem="cdsupg",
                             eps=1e-3, b1=1, b2=0.5, b3=0.25, **TIGHT)),
    "q2_supg": ("cd3d", dict(order=2, levels=2, coarse_steps=1, problem="cdsupg",
                             eps=1e-6, b1=1, b2=0.5, b3=0.25, **TIGHT)),
    # (an assembly pin only: Galerkin at this mesh Peclet number is not a solve case)
    "q2_galerkin": ("cd3d", dict(order=2, levels=2, coarse_steps=1, problem="cdsupg", disc=1,
                                 eps=1e-2, b1=1, b2=0.5, b3=0.25)),
    "p2tet_supg": ("cd3d", dict(order=2, levels=2, coarse_steps=1, problem="cdsupg",
                                eps=1e-3, b1=1, b2=0.5, b3=0.25, geo="SixTetras", **TIGHT)),
    "p1tet_laplace": ("cd3d", dict(order=1, levels=2, coarse_steps=1, problem="laplace",
                                   geo="SixTetras", **TIGHT)),
    # the C1 configuration exactly: Poisson, Q1, 4^3 -> 32^3 cells over 4 levels,
    # Gauss2; the solution and the finest dof positions only (no matrices)
    "c1_poisson_q1_32": ("cd3d", dict(order=1, levels=4, coarse_steps=2, problem="laplace", dump=0,
                                      dump_solution=1, **TIGHT)),
    "tcd3d_amc": ("tcd3d", dict(order=1, levels=3, coarse_steps=2, endtime=0.5)),
    # SC_MG_TYPE_SCALAR = 1: N_Q1 on the 2^3, 4^3, 8^3 meshes, then the conforming
    # space on the 8^3 mesh (4 multigrid levels); L<l>_parent = Prolongate's parent cells
    "mdml_q1_laplace": ("cd3d", dict(order=1, levels=3, coarse_steps=1, problem="laplace", mg_type=1, **TIGHT)),
    "mdml_q1_supg": ("cd3d", dict(order=1, levels=3, coarse_steps=1, problem="cdsupg", eps=1e-3, b1=1, b2=0.5,
                                  b3=0.25, mg_type=1, **TIGHT)),
    "mdml_q2_supg": ("cd3d", dict(order=2, levels=2, coarse_steps=1, problem="cdsupg", eps=1e-6, b1=1, b2=0.5,
                                  b3=0.25, mg_type=1, **TIGHT)),
}


# Smoother variants of TMultiGrid3D::Smooth / Cycle on the q1_supg problem
# (same mesh, space and numbering as q1_supg.npz): only the solutions and
# iteration counts are kept; the matrices are those of q1_supg.npz.
SMOOTHER_BASE = dict(order=1, levels=3, coarse_steps=1, problem="cdsupg", eps=1e-3, b1=1, b2=0.5, b3=0.25,
                     red=1e-12, dump=0, dump_solution=1, restart=30)
SMOOTHER_VARIANTS = [dict(smoother=1, omega=0.8), dict(smoother=2, omega=1.0), dict(smoother=2, omega=1.2, slc_fine=1),
                     dict(smoother=3, omega=1.0, slc_all=1), dict(smoother=1, omega=0.7, slc_all=1)]


def make_smoothers():
    out = {}
    for k, v in enumerate(SMOOTHER_VARIANTS):
        opt = dict(SMOOTHER_BASE, **v)
        with tempfile.TemporaryDirectory() as td:
            subprocess.run([BIN, "cd3d", td] + [f"{a}={b}" for a, b in opt.items()], check=True,
                           stdout=subprocess.DEVNULL)
            data = load_dump(td)
        out[f"V{k}_solution"] = data["solution"]
        out[f"V{k}_iterations"] = data["solve_iterations"]
        out[f"V{k}_rel_res"] = data["res_final"] / data["res0"]
        out[f"V{k}_params"] = np.array([f"{a}={b}" for a, b in opt.items()])
    np.savez_compressed(os.path.join(HERE, "q1_supg_smoothers.npz"), **out)
    print("q1_supg_smoothers", {k: v for k, v in out.items() if k.endswith("_iterations")})


def load_dump(d):
    out = {}
    with open(os.path.join(d, "meta.txt")) as f:
        for line in f:
            name, kind, val = line.split()
            if kind == "scalar":
                out[name] = np.float64(val)
            else:
                dt = {"i4": np.int32, "f8": np.float64}[kind]
                out[name] = np.fromfile(os.path.join(d, name + ".bin"), dtype=dt)
    return out


def recorded_log(ref):
    """(time, L2, H1) triples printed by the recorded GMG run."""
    path = os.path.join(ref, "ReadIn", "tcd3d_GMG.out")
    rows = []
    with open(path) as f:
        for line in f:
            m = re.match(r"time:\s+(\S+)\s+L2:\s+(\S+)\s+H1-semi:\s+(\S+)", line)
            if m:
                rows.append([float(m.group(i)) for i in (1, 2, 3)])
    return np.array(rows)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PMG_REFERENCE_DIR"),
                    help="the ParMooN source tree (default: $PMG_REFERENCE_DIR)")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if not args.ref or not os.path.isdir(args.ref):
        raise SystemExit("give the ParMooN source tree with --ref or PMG_REFERENCE_DIR")
    if not os.path.exists(BIN):
        raise SystemExit("build the reference oracle first: make -C oracle/ref")
    if args.only in (None, "q1_supg_smoothers"):
        make_smoothers()
    for name, (mode, opt) in CASES.items():
        if args.only and name != args.only:
            continue
        with tempfile.TemporaryDirectory() as td:
            cmd = [BIN, mode, td] + [f"{k}={v}" for k, v in opt.items()]
            subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
            data = load_dump(td)
        for k in [k for k in data if k.startswith("t_") or k.endswith("t_assemble")]:
            data.pop(k)  # timings are not golden data
        data["params"] = np.array([f"{k}={v}" for k, v in opt.items()])
        if name == "tcd3d_amc":
            data["recorded_log"] = recorded_log(args.ref)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **data)
        print(name, {k: getattr(v, "shape", ()) for k, v in data.items() if k.startswith("L1_") or k == "solution"})


if __name__ == "__main__":
    main()
