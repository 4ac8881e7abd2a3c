"""Region sweeps (csrc/region_sweep.cu): the SSOR phases of the mid-size
levels as one cooperative launch each, with neighbour-only waits, against the
colour-by-colour launches (PMG_REGION_SWEEP=0, read once per process, hence
the subprocesses).  One FP64 V-cycle on the Q2 32^3 hierarchy (level 2, 29,791
active rows, runs as regions) agrees with the colour launches to rounding
(1e-12 relative), the FP32 one to 1e-5, and the solves reach the same
solution (both to 1e-12: 1e-9 relative)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
import parmoon_b200 as P
out = {}
levels = P.struct_hierarchy(P.Q2_HEX, 32, 4)
for prec in (0, 1):
    h = P.Handle(4, P.default_params(precision=prec, lin_red=1e-12, lin_maxit=200))
    h.set_coefficients(P.coeff(kind=P.COEF_CONST, eps=1e-3, b=(1.0, 0.5, 0.25), f=1.0))
    P.load_hierarchy(h, levels, dirichlet=lambda x, y, z: (x < 1e-12).astype(float))
    h.assemble(-1, P.FORM_SUPG, copy_out=False)
    _, st, rc = h.solve()
    out[f"sol{prec}"] = h.get_solution().tolist()
    out[f"it{prec}"] = st.iterations
    out[f"rc{prec}"] = rc
    N = levels[-1]["N"]
    v = torch.from_numpy(np.random.default_rng(1).standard_normal(N)).cuda()
    z = torch.empty_like(v)
    h.vcycle(v.data_ptr(), z.data_ptr())
    torch.cuda.synchronize()
    out[f"z{prec}"] = z.cpu().numpy().tolist()
    h.close()
print(json.dumps(out))
"""


def run(env_value):
    env = dict(os.environ)
    if env_value is not None:
        env["PMG_REGION_SWEEP"] = env_value
    p = subprocess.run([sys.executable, "-c", SCRIPT, ROOT], capture_output=True, text=True, timeout=900, env=env)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-3000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_region_sweeps_match_colour_launches():
    a, b = run(None), run("0")
    for prec, tol in ((0, 1e-12), (1, 1e-5)):
        za, zb = np.array(a[f"z{prec}"]), np.array(b[f"z{prec}"])
        assert np.linalg.norm(za - zb) <= tol * np.linalg.norm(zb), (prec, np.linalg.norm(za - zb) / np.linalg.norm(zb))
        assert a[f"rc{prec}"] == 0 and b[f"rc{prec}"] == 0
        xa, xb = np.array(a[f"sol{prec}"]), np.array(b[f"sol{prec}"])
        assert np.linalg.norm(xa - xb) <= 1e-9 * np.linalg.norm(xb)
        assert abs(a[f"it{prec}"] - b[f"it{prec}"]) <= 1
