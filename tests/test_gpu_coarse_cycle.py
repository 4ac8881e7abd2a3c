"""The coarse end of the V-cycle as one launch (one CTA for the smallest
levels, PMG_COARSE_CLUSTER=1; a 16-CTA thread-block cluster, =16; an 8-CTA
cluster on the levels of at most 8192 rows, =8:8192, the default) gives the
same solve as the level-by-level launches (=0): same
FGMRES iteration count (+-1) and solutions within 1e-8 relative (both stop at
|r| <= 1e-10 |r0|; the two paths differ only in the order of partial sums
inside a row).  Each configuration runs in its own process because the switch
is read once per process."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import json, sys, numpy as np
sys.path.insert(0, {root!r})
import parmoon_b200 as P
elem, n, nl, prec, coarse = {args}
levels = P.struct_hierarchy(elem, n, nl)
h = P.Handle(nl, P.default_params(precision=prec, coarse_smoother=coarse))
h.set_coefficients(P.coeff(kind=P.COEF_CONST, eps=1e-3, b=(1.0, 0.5, 0.25), f=1.0))
P.load_hierarchy(h, levels, dirichlet=lambda x, y, z: (abs(x) < 1e-12).astype(float))
h.assemble(-1, P.FORM_SUPG, copy_out=False)
_, st, rc = h.solve()
x = h.get_solution()
np.save({out!r}, x)
print(json.dumps(dict(rc=rc, its=st.iterations, rel=st.rel_res)))
"""


def run(tmp_path, tag, args, mode):
    out = str(tmp_path / f"{tag}.npy")
    env = dict(os.environ)
    env["PMG_COARSE_CLUSTER"] = mode if mode is not None else "0"
    p = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, args=args, out=out)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    return json.loads(p.stdout.strip().splitlines()[-1]), np.load(out)


@pytest.mark.parametrize("mode", ["1", "16", "8:8192"])  # one CTA, 16-CTA cluster, 8-CTA cluster on small levels
@pytest.mark.parametrize("elem,n,nl,prec,coarse", [(2, 16, 3, 1, 17), (1, 32, 4, 1, 17), (1, 32, 4, 0, 17),
                                                   (2, 16, 3, 0, 3)])
def test_coarse_cycle_launch_matches_level_launches(tmp_path, elem, n, nl, prec, coarse, mode):
    args = (elem, n, nl, prec, coarse)
    a, xa = run(tmp_path, "one", args, mode)
    b, xb = run(tmp_path, "levels", args, None)
    assert a["rc"] == 0 and b["rc"] == 0 and a["rel"] <= 1e-10 and b["rel"] <= 1e-10
    assert abs(a["its"] - b["its"]) <= 1, (a, b)
    assert np.linalg.norm(xa - xb) <= 1e-8 * np.linalg.norm(xb)


GIVEUP = r"""
import json, os, sys, numpy as np
os.environ["PMG_NO_GRAPH"] = "1"  # launch the V-cycle kernels directly, so the test switch is read per launch
sys.path.insert(0, {root!r})
import parmoon_b200 as P
levels = P.struct_hierarchy(2, 16, 3)
h = P.Handle(3, P.default_params(precision=1, lin_maxit=2))
h.set_coefficients(P.coeff(kind=P.COEF_CONST, eps=1e-3, b=(1.0, 0.5, 0.25), f=1.0))
P.load_hierarchy(h, levels, dirichlet=lambda x, y, z: (abs(x) < 1e-12).astype(float))
h.assemble(-1, P.FORM_SUPG, copy_out=False)
os.environ["PMG_TEST_CC_EXTRA_TX"] = "8"  # every pass waits for 8 bytes nobody sends
_, st, rc_fail = h.solve(raise_on_error=False)
del os.environ["PMG_TEST_CC_EXTRA_TX"]
h.set_params(P.default_params(precision=1))
_, st, rc_ok = h.solve(raise_on_error=False)
print(json.dumps(dict(rc_fail=rc_fail, rc_ok=rc_ok, rel=st.rel_res, its=st.iterations)))
"""


def test_coarse_cycle_wait_gives_up_and_recovers():
    """The give-up path of the one-launch coarse cycle: with every pass of the
    8-CTA cluster (levels of at most 8192 rows) expecting bytes no CTA sends,
    each wait runs out after 0.2 s, the launch ends, and the solve reports
    PMG_ERR_STATE; the flag is cleared and the next solve converges on the same
    handle and context."""
    env = dict(os.environ)
    env["PMG_COARSE_CLUSTER"] = "8:8192"
    p = subprocess.run([sys.executable, "-c", GIVEUP.format(root=ROOT)], env=env, capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stderr[-3000:]
    r = json.loads(p.stdout.strip().splitlines()[-1])
    assert r["rc_fail"] == -3, r
    assert r["rc_ok"] == 0 and r["rel"] <= 1e-10, r
