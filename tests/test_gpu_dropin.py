"""The drop-in, end to end: the reference's own command-line program
(main.cpp and the rest of its sources, unchanged) built with GPU_BATCH::rcm
replaced by the shim over libpbrcm (`make -C oracle dropin`).  Run as a user of
the reference would run it, `-i GPU_BATCH -w`, on the golden MatrixMarket
inputs: it must exit 0 (the reference's checkPermutation passed) and report
the bandwidth of the reference's own output."""
import os
import subprocess

import pytest

from conftest import load_golden
from test_oracle_golden import MTX_NAMES, golden_mtx_path

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "oracle", "_ref", "CuthillMcKee_pbrcm")


@pytest.mark.parametrize("name", MTX_NAMES)
def test_reference_cli_with_pbrcm_gpu_batch(name, tmp_path):
    if not os.path.exists(CLI):
        pytest.skip("drop-in CLI not built (make -C oracle dropin)")
    g = load_golden(name)
    csv = tmp_path / "perf.csv"
    r = subprocess.run([CLI, golden_mtx_path(name, tmp_path), "-i", "GPU_BATCH", "-w", "--perffile", str(csv)],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "GPU-DYN-RCM" in r.stdout
    fields = [f.strip() for f in csv.read_text().strip().splitlines()[-1].split(",")]
    # name, initial bandwidth, max valency, start (the reference's own CPU
    # search), GPU_BATCH time (reported by the shim), bandwidth
    assert int(fields[-1]) == int(g["bandwidth"]), fields
    assert float(fields[-2]) >= 0.0
    assert int(fields[-3]) == int(g["start"]), fields
    assert int(fields[1]) == int(g["initial_bandwidth"]), fields
