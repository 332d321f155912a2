"""The bounded waits of the TMA line-FFT passes give up and report instead
of hanging.  In a child process with the test hook MLG_TEST_WAIT_TIMEOUT=1
the producer of CTA 0 never loads its first bundle: that CTA's transform
threads wait 2 s, give up together, the kernel finishes, the plan's status
reports MLG_ERR_TIMEOUT once (the flag is then clear), and the CUDA context
keeps working."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
import monalisa_b200 as mb
from monalisa_b200 import traj, _native as N
n, Ng = 64, 128
t = traj.golden_angle_radial2(128, 64, 1.0)
Gu, Gut = mb.bmTraj2SparseMat(t, np.ones(t.shape[1]), [Ng, Ng], [1, 1])
rec = mb.SensaRecon(Gu, Gut, traj.coil_maps([n, n], 4, 1), [n, n])
rec.plan.variant = {"pass_buffers": 2}
x = torch.ones(n * n, dtype=torch.complex64, device="cuda")
y = rec.plan.shanna(x)
try:
    rec.plan.status()
    print("NO_TIMEOUT")
except N.MonalisaError as e:
    print("TIMEOUT", e)
rec.plan.status()
print("CLEARED")
print("CONTEXT_OK", float((torch.ones(8, device="cuda") * 2).sum()))
rec.plan.close()
"""


def test_tma_wait_runs_out_and_reports():
    env = dict(os.environ, MLG_TEST_WAIT_TIMEOUT="1")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "TIMEOUT" in r.stdout and "NO_TIMEOUT" not in r.stdout, r.stdout
    assert "CLEARED" in r.stdout and "CONTEXT_OK 16.0" in r.stdout, r.stdout
