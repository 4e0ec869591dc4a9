"""The reference's own apps compile unchanged against the drop-in header.

FunDEM's tutorial apps (FunDEM/apps/tutorial/*.cpp + globalDamping.cu) include
"kernel/LSSolver.h" and the reference's host-only helper headers; with this
repository's include/ first on the include path they build against
include/kernel/LSSolver.h and link liblsdem_b200.so. Needs the reference tree
(present where the repository is developed, absent on GPU hosts).
"""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT

REF = Path(os.environ.get("REF", "/root/reference")) / "FunDEM"  # the reference tree, where it is present
APPS = ["tutorial1-LSParticleFalling", "tutorial2-LSParticleRolling", "tutorial3-bondedLSParticleBeam",
        "tutorial4-PeriodicBoundary"]


@pytest.mark.skipif(not REF.is_dir() or shutil.which("nvcc") is None, reason="reference tree or nvcc not available")
@pytest.mark.parametrize("app", APPS)
def test_tutorial_app_builds(app, tmp_path):
    out = tmp_path / app
    cmd = ["nvcc", "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", str(ROOT / "include"), "-I", str(ROOT / "include" / "kernel"),
           "-I", str(REF), "-I", str(REF / "kernel"), "-I", str(REF / "apps" / "tutorial"),
           str(REF / "apps" / "tutorial" / f"{app}.cpp"), str(REF / "apps" / "tutorial" / "globalDamping.cu"),
           "-L", str(ROOT / "lsdem2.0_b200"), "-llsdem_b200", "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    assert out.exists()
