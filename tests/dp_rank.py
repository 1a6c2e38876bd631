"""One rank of the data-parallel learner test (tests/test_gpu_data_parallel.py):
    python tests/dp_rank.py RANK WORLD PORT WORKDIR
Reads WORKDIR/case.npz (rows, labels, gradient sets, shard bounds) and
WORKDIR/params.json, trains one tree per gradient set on its shard with the
reductions going through host memory over a gloo process group, and writes
WORKDIR/rank<RANK>.pkl with the trees."""
import datetime
import json
import os
import pickle
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "lightgbm-rust_b200"))


class _Binned:
    def __init__(self, b):
        self.b = b

    def construct(self, params=None):
        return self

    def binned(self):
        return self.b


def main():
    rank, world, port, work = int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4]
    import numpy as np
    import torch
    import torch.distributed as dist

    import lgbm_b200 as lgb
    from lgbm_b200 import data_parallel

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    d = np.load(os.path.join(work, "case.npz"))
    params = json.load(open(os.path.join(work, "params.json")))
    X, y, bounds = d["X"], d["y"], d["bounds"]
    ds = lgb.Dataset(X, y, params=params)  # every rank bins all rows: the same mappers everywhere
    b = ds.binned()
    off, end = int(bounds[rank]), int(bounds[rank + 1])
    shard = dict(b, bins=np.ascontiguousarray(b["bins"][off:end]), num_data=end - off)
    learner = lgb.Learner(_Binned(shard), params)
    learner.set_data_parallel(off, len(y), data_parallel.torch_allreduce_host(torch.device("cuda", 0)))
    trees = [learner.train(g[off:end], h[off:end])[0] for g, h in zip(d["g"], d["h"])]
    with open(os.path.join(work, f"rank{rank}.pkl"), "wb") as f:
        pickle.dump(trees, f)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
