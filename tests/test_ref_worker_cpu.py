"""Host side of the reference-side binding (integration/): the reference's
DBmaker builds its DB from a FASTA file with whole 128-record batches, and
without a device the B200 worker reports the library's SW_ERR_NO_DEVICE
through the reference's error path (a const char* thrown from alloc() and
printed by Worker::threadControl) and the driver exits 1 with nothing
scored."""
import os
import subprocess

import numpy as np
import pytest

from swhybrid_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "integration", "_ref")
ALPHA = "ABCDEFGHIKLMNPQRSTVWXYZ"


def _gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(not os.path.exists(os.path.join(BIN, "ref_worker_pool")),
                    reason="integration/_ref not built (needs the reference sources at build time)")
@pytest.mark.skipif(_gpu(), reason="checks the no-device path")
def test_dbmaker_db_and_worker_without_device(tmp_path):
    rng = np.random.default_rng(5)
    with open(tmp_path / "db.fa", "w") as f:
        for b, L in enumerate((40, 120, 300)):
            for i in range(128):
                r = synth.residues(rng, L - int(rng.integers(0, 4)))
                f.write(f">r{b}_{i}\n{''.join(ALPHA[c] for c in r)}\n")
    (tmp_path / "q.fa").write_text(">q\n" + "ACDEFGHIKLMNPQRSTVWY" * 5 + "\n")
    out = subprocess.run([os.path.join(BIN, "dbmaker"), str(tmp_path / "db.fa"),
                          str(tmp_path / "db")], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "total sequence num is 384" in out.stdout
    for ext in ("seq", "map", "title"):
        assert (tmp_path / f"db.{ext}").stat().st_size > 0
    out = subprocess.run([os.path.join(BIN, "ref_worker_pool"), "-q", str(tmp_path / "q.fa"),
                          "-db", str(tmp_path / "db"), "-t", "10", "-g", "1"],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 1
    assert "B200Worker(0): sw_ctx_create failed (status 9)" in out.stdout
    assert "records 0 recalc 0" in out.stdout
