"""The reference's own main programs 3DPrograms/CD3D_ParMooN.C (example
Laplace.h) and 3DPrograms/TCD3D_ParMooN.C (example amc.h), compiled
unmodified, run twice: linked with the reference's system classes
(*_program_ref) and with the link-time replacements SystemCD3D_pmg.C /
SystemTCD3D_pmg.C on libpmg_b200 (*_program_pmg).  The L2 and H1-semi errors
they print (6 significant digits) must agree; the time-dependent run must also
reproduce the L2 column of the reference's recorded log ReadIn/tcd3d_GMG.out.
Needs the binaries of `make -C oracle/ref programs`."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden

pytestmark = pytest.mark.gpu
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

SOLVER = dict(SOLVER_TYPE=1, SC_SOLVER_SCALAR=16, SC_PRECONDITIONER_SCALAR=5, SC_SMOOTHER_SCALAR=3,
              SC_PRE_SMOOTH_SCALAR=2, SC_POST_SMOOTH_SCALAR=2, SC_COARSE_SMOOTHER_SCALAR=3,
              SC_COARSE_MAXIT_SCALAR=10, SC_COARSE_RED_FACTOR_SCALAR=0.1, SC_LIN_MAXIT_SCALAR=1000,
              SC_GMRES_RESTART=20, SC_MG_TYPE_SCALAR=0, SC_MG_CYCLE_SCALAR=1, SC_SMOOTH_DAMP_FACTOR_SCALAR=1.0,
              SC_GMG_DAMP_FACTOR_SCALAR=1.0, SC_STEP_LENGTH_CONTROL_FINE_SCALAR=0,
              SC_STEP_LENGTH_CONTROL_ALL_SCALAR=0, SC_VERBOSE=0)


def write_dat(path, geo, **kw):
    d = os.path.join(REF_DIR, "data")
    lines = ["VERSION: 1", f"GEOFILE: {d}/{geo}.GEO", f"BNDFILE: {d}/Wuerfel.PRM", "OUTFILE: run.out",
             "LOGFILE: run.log", "MESH_TYPE: 0", "WRITE_VTK: 0", "MEASURE_ERRORS: 1", "DISCTYPE: 1"]
    lines += [f"{k}: {v}" for k, v in {**SOLVER, **kw}.items()]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def run_program(exe, workdir, dat):
    path = os.path.join(REF_DIR, exe)
    if not os.path.exists(path):
        pytest.skip(f"{exe} not built (needs the reference sources)")
    os.makedirs(workdir, exist_ok=True)
    p = subprocess.run([path, dat], cwd=workdir, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    l2 = [float(v) for v in re.findall(r"^L2: (\S+)", p.stdout, re.M)]
    h1 = [float(v) for v in re.findall(r"^H1-semi: (\S+)", p.stdout, re.M)]
    assert l2 and len(l2) == len(h1), p.stdout[-3000:]
    return np.array(l2), np.array(h1)


# (the unmodified CD3D main program crashes in the reference's own mesh set-up on
# SixTetras.GEO, CPU build included, so tetrahedra are covered by test_gpu_dropin)
@pytest.mark.parametrize("geo,order,levels,steps,mg_type", [("Wuerfel", 1, 3, 2, 0), ("Wuerfel", 2, 3, 1, 0),
                                                             ("Wuerfel", 1, 4, 2, 0), ("Wuerfel", 1, 3, 2, 1),
                                                             ("Wuerfel", 2, 3, 1, 1)])
def test_cd3d_program_on_device_matches_reference(tmp_path, geo, order, levels, steps, mg_type):
    """mg_type 1: SC_MG_TYPE_SCALAR = 1, N_Q1 levels under the conforming one."""
    dat = str(tmp_path / "cd3d.dat")
    write_dat(dat, geo, ANSATZ_ORDER=order, LEVELS=levels, UNIFORM_STEPS=steps, SC_LIN_RED_FACTOR_SCALAR=1e-10,
              SC_LIN_RES_NORM_MIN_SCALAR=0, SC_MG_TYPE_SCALAR=mg_type)
    l2r, h1r = run_program("cd3d_program_ref", str(tmp_path / "ref"), dat)
    l2p, h1p = run_program("cd3d_program_pmg", str(tmp_path / "pmg"), dat)
    assert np.allclose(l2p, l2r, rtol=2e-6, atol=0) and np.allclose(h1p, h1r, rtol=2e-6, atol=0), (l2r, l2p, h1r, h1p)


@pytest.mark.parametrize("mg_type", [0, 1])
def test_tcd3d_program_on_device_reproduces_recorded_log(tmp_path, mg_type):
    """mg_type 1 is the multilevel type of the recorded run (SC_MG_TYPE_SCALAR = 1:
    an N_Q1 level on every mesh under the Q1 level, tcd3d_GMG.out:388-396)."""
    dat = str(tmp_path / "tcd3d.dat")
    write_dat(dat, "Wuerfel", ANSATZ_ORDER=1, LEVELS=3, UNIFORM_STEPS=2, SC_LIN_RED_FACTOR_SCALAR=0.0,
              SC_LIN_RES_NORM_MIN_SCALAR=1e-13, TIME_DISC=2, STARTTIME=0, ENDTIME=0.5,
              TIMESTEPLENGTH=0.1082532, STEPS_PER_IMAGE=100, SC_MG_TYPE_SCALAR=mg_type)
    l2r, h1r = run_program("tcd3d_program_ref", str(tmp_path / "ref"), dat)
    l2p, h1p = run_program("tcd3d_program_pmg", str(tmp_path / "pmg"), dat)
    assert l2p.size == l2r.size == 6
    assert np.allclose(l2p, l2r, rtol=2e-6, atol=0) and np.allclose(h1p, h1r, rtol=2e-6, atol=0), (l2r, l2p)
    rec = golden("tcd3d_amc")["recorded_log"][:l2p.size]  # rows: time, L2, H1 of the recorded run
    assert np.allclose(l2p, rec[:, 1], rtol=2e-6, atol=0), (l2p, rec[:, 1])
