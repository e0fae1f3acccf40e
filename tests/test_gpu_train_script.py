"""The reference's GA training script runs unchanged on top of this package.

scripts/train-singleshot.py of the reference (train-singleshot.py:1-154) imports qmtools.GAEngine,
qmtools.automaton_nn_singleshot, qmtools.cidhelper and the facade, builds ten molecules
(density with subgrid 2, the VNe pseudo-field) and evolves a population of single-shot
automata.  The test runs the file itself, unmodified, in a subprocess with this package first on
PYTHONPATH, and stops it once the GA has logged two generations.  Point QMTOOLS_TRAIN_SCRIPT at
the reference's scripts/train-singleshot.py to run it (skipped otherwise: the script is not part
of this repository).
"""
import os
import shutil
import subprocess
import sys
import time
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "qmtools-pycuda_b200"


def test_reference_training_script_runs_unchanged(tmp_path):
    script = os.environ.get("QMTOOLS_TRAIN_SCRIPT")
    if not script or not Path(script).exists():
        pytest.skip("QMTOOLS_TRAIN_SCRIPT does not name the reference's scripts/train-singleshot.py")
    # the script reads ../data/cc-pvdz.bin and keeps its molecules in ./data
    (tmp_path / "data").mkdir()
    shutil.copy(PKG / "qmtools" / "data" / "cc-pvdz.bin", tmp_path / "data" / "cc-pvdz.bin")
    run = tmp_path / "run"
    (run / "data").mkdir(parents=True)
    env = dict(os.environ, PYTHONPATH=str(PKG) + os.pathsep + os.environ.get("PYTHONPATH", ""))
    log = run / "ga.log"
    with open(run / "stdout.txt", "w") as out:
        proc = subprocess.Popen([sys.executable, script, "--populationSize", "4"], cwd=run, env=env,
                                stdout=out, stderr=subprocess.STDOUT)
        try:
            deadline = time.time() + 900
            while time.time() < deadline and proc.poll() is None:
                if log.exists() and len(log.read_text().splitlines()) >= 2:
                    break
                time.sleep(1)
        finally:
            still_running = proc.poll() is None
            if still_running:
                proc.terminate()
                try:
                    proc.wait(timeout=30)
                except subprocess.TimeoutExpired:
                    proc.kill()
                    proc.wait()
    text = (run / "stdout.txt").read_text()
    assert still_running, "the script ended early:\n" + text[-3000:]
    lines = log.read_text().splitlines()
    assert len(lines) >= 2, text[-3000:]
    for line in lines[:2]:
        best, worst, mean = (float(v) for v in line.split())
        assert best >= mean >= worst
    assert len(list((run / "data").glob("molecule.*.pickle"))) == 10
    assert (run / "ga.restart.bin").exists()
