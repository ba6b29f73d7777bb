"""Worker for tests/test_multirank.py: one rank of a CPU (gloo) job launched
by torchrun, exercising the bench's multi-rank accounting the way a GPU run
uses it: every rank has its own stripes (seeds), the step time is the
slowest rank's, the value is the whole job's, and rank 0 alone prints."""
import datetime
import json
import os
import sys

import torch.distributed as dist

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def main() -> int:
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 3.5 * rank  # this rank's device time for 4 steps
        slowest = bench.max_over_ranks(ms, dist, "cpu")
        seeds = bench.rank_seeds(rank)
        pats = bench.erasure_patterns(8, seed=seeds[1])
        everyone = [None] * world
        dist.all_gather_object(everyone, {"rank": rank, "seeds": seeds, "patterns": pats, "ms": ms})
        per_rank_bytes = 256 * 2 * 10 * (1 << 20)
        value = bench.job_source_gbps(per_rank_bytes, world, slowest / 4)
        dist.barrier()
        if rank == 0:
            print(json.dumps({"world": world, "slowest_ms": slowest, "value": value, "ranks": everyone}))
    finally:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
