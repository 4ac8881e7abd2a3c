"""TPmgSystemCD3D (parmoon_b200/shim) dropped into a ParMooN-style program in
place of the reference's TSystemCD3D, on the reference's own domain, FE spaces,
CSR structures and callbacks (oracle/ref/dropin_driver.C, linked against the
compiled reference).  Matrices on every level and the finest rhs agree to
1e-12 relative; both solves stop at |r| <= 1e-14 |r0| (near the FP64
rounding floor), and the solutions agree to 1e-10 relative.  Needs oracle/_ref/pmg_dropin (make -C oracle/ref dropin)."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "oracle", "_ref", "pmg_dropin")


def run(tmp_path, **kw):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/pmg_dropin not built (needs the reference sources)")
    args = [EXE, str(tmp_path)] + [f"{k}={v}" for k, v in kw.items()]
    p = subprocess.run(args, capture_output=True, text=True, timeout=600)
    line = [l for l in p.stdout.splitlines() if l.startswith("dropin ")]
    assert p.returncode == 0 and line, p.stdout[-2000:] + p.stderr[-2000:]
    return {k: float(v) for k, v in re.findall(r"(\w+)=([-+0-9.eE]+)", line[-1])}


@pytest.mark.parametrize("order,geo,problem,dev", [
    (1, "Wuerfel", "laplace", 0), (2, "Wuerfel", "cd", 0), (1, "SixTetras", "cd", 0),
    (2, "SixTetras", "laplace", 0), (2, "Wuerfel", "laplace", 1)])
def test_dropin_matches_reference_system(tmp_path, order, geo, problem, dev):
    r = run(tmp_path, order=order, geo=geo, problem=problem, device_coeffs=dev, levels=3, coarse_steps=1, red=1e-14)
    assert r["mat_rel"] <= 1e-12 and r["rhs_rel"] <= 1e-12, r
    assert r["sol_rel"] <= 1e-10, r
    assert r["res_pmg"] <= 10 * max(r["res_ref"], 1e-14), r
