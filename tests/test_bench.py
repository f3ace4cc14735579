"""bench.py's own logic on the CPU: the constants it reads from the committed profiles, its
L2 note, the FP64-oracle accuracy record, and the reference arm's JSON line (the reference's
CPU build runs here, so that arm needs no GPU)."""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def bench():
    import bench as b  # importing parses no arguments; main() does
    return b


def test_constants_from_committed_profiles(bench):
    assert bench.traffic_from_profiles("chained") == pytest.approx(8.45e8)
    assert bench.traffic_from_profiles("restart") == pytest.approx(1.42e8)
    assert bench.fp64_flop_per_update() == pytest.approx(3698)


def test_l2_note_follows_the_input_size(bench):
    assert "larger than the 126 MB L2" in bench.l2_note(100)
    assert "profiling size" in bench.l2_note(8)


def test_accuracy_record_is_symmetric(p2r, bench):
    """Fed the reference's own output as this library's, both error records are identical."""
    from oracle.oracle import RefTBB, ref_available
    if not ref_available(32, "kf"):
        pytest.skip("reference build not present")
    cfg = p2r.Config(bsize=32, nlayer=20, nevts=1, nb=10, bz=3.8)
    trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=3.8, seed=3))
    ref = RefTBB(32, "kf")
    ref.set_bz(3.8)
    rout = ref.run(trk, hit, 1, cfg.nb, 20, True)
    r = bench.accuracy_vs_fp64(trk.reshape(-1), hit.reshape(-1), rout, cfg.nb, 32, 3.8, 2)
    assert r["this_library"] == r["reference_cpu"]
    assert 0 < r["this_library"]["par"]["p50"] < 1e-5 and r["this_library"]["cov"]["max"] < 1


@pytest.mark.parametrize("mode", ["chained", "restart"])
def test_reference_arm_line(mode):
    from oracle.oracle import host_isa, ref_available
    if not ref_available(32, host_isa()):
        pytest.skip("reference build not present")
    res = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1", "--nevts", "2", "--ref-budget", "3", "--mode", mode],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    line = json.loads(res.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "track-layer updates/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["config"]["mode"] == mode and line["steps"] == 2 and line["warmup"] == 1
    assert mode in line["cpu_baseline"]["sample"]
