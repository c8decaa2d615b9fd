"""The reference's own driver and V&V tests (src/main.cpp, TestCG.cpp,
TestSymmetry.cpp, TestNorms.cpp), unchanged, linked with the drop-in
translation unit hpcg_b200/dropin/hpcg_dropin.cpp (oracle/_ref/xhpcg_b200,
built by `make -C oracle dropin` where the reference tree is present)."""
import glob
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "xhpcg_b200")


def run_driver(tmp_path, n):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/xhpcg_b200 not built")
    out = subprocess.run([EXE, f"--nx={n}", f"--ny={n}", f"--nz={n}", "--rt=0"], cwd=tmp_path,
                         capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    reports = glob.glob(os.path.join(tmp_path, "HPCG-Benchmark*.txt"))
    logs = glob.glob(os.path.join(tmp_path, "hpcg*.txt"))
    assert reports, os.listdir(tmp_path)
    return open(reports[0]).read(), (open(logs[0]).read() if logs else "")


@pytest.mark.parametrize("n", [32, 64])
def test_reference_driver_validates_with_dropin(tmp_path, n):
    report, log = run_driver(tmp_path, n)
    assert "failed with status" not in log, log[-3000:]
    assert "HPCG result is VALID" in report, report[-3000:]
    fields = dict(re.findall(r"^([^=\n]+)=(.*)$", report, re.M))
    assert int(fields["Spectral Convergence Tests::Unpreconditioned::Maximum iteration count"]) <= 12
    assert int(fields["Spectral Convergence Tests::Preconditioned::Maximum iteration count"]) <= 2
    assert float(fields["Departure from Symmetry |x'Ay-y'Ax|/(2*||x||*||A||*||y||)/epsilon::Departure for SpMV"]) <= 1
    assert float(fields["Departure from Symmetry |x'Ay-y'Ax|/(2*||x||*||A||*||y||)/epsilon::Departure for MG"]) <= 1
    assert float(fields["Reproducibility Information::Scaled residual variance"]) < 1e-6
    # the optimised CG must reach the reference's 50-iteration residual in few extra iterations
    assert int(fields["Iteration Count Information::Optimized CG iterations per set"]) <= 60
    assert float(fields["Memory Use Information::Memory used for OptimizeProblem data (Gbytes)"]) > 0
