"""The bench's N > 1 path on CPU: two gloo ranks under torchrun (the same
launcher and rendezvous as a multi-GPU run, 127.0.0.1). Checks the
max-over-ranks step time, the whole-job value (weak scaling: every rank's
bytes over the slowest rank's time), per-rank stripes from distinct seeds,
and that only rank 0 prints."""
import json
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_account_like_the_gpu_job():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "tests" / "_gloo_ranks.py")]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=180, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout  # rank 0 alone prints
    r = json.loads(lines[0])
    assert r["world"] == 2
    assert r["slowest_ms"] == 13.5  # max of 10.0 and 13.5
    per_rank = 256 * 2 * 10 * (1 << 20)
    assert abs(r["value"] - 2 * per_rank / (13.5 / 4 / 1e3) / 1e9) < 1e-9
    ranks = sorted(r["ranks"], key=lambda x: x["rank"])
    assert [x["rank"] for x in ranks] == [0, 1]
    assert ranks[0]["seeds"] != ranks[1]["seeds"]
    assert ranks[0]["patterns"] != ranks[1]["patterns"]
    for x in ranks:
        for p in x["patterns"]:
            assert len(p) == 4 and len(set(p)) == 4 and all(0 <= i < 14 for i in p)
