"""Child script of test_replica_aggregation_gloo (run under torch.distributed.run)."""
import os
import sys

import torch.distributed as dist

sys.path.insert(0, os.environ["ROOT"])
import bench  # noqa: E402

dist.init_process_group("gloo")
r = dist.get_rank()
total = bench.combine_ranks(100.0 + 50.0 * r, steps=4, backend="gloo")
assert abs(total["ms"] - 150.0) < 1e-9, total
assert abs(total["value"] - 2 * 4 / 0.150) < 1e-9, total
print("ok", r, flush=True)
dist.destroy_process_group()
