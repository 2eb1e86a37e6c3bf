"""Times the reference's own CUDA build on the secondary workloads.

Measurement infrastructure, like the rest of oracle/: nothing in the library
calls it.  It drives oracle/_ref/libpoggers_refcuda.so (the reference's
tables compiled from its own sources by oracle/Makefile, one tile per key in
the reference's launch shape) through oracle/pyrefcuda.py, on the inputs and
with the phase timers that poggers_b200.bench_configs uses for this library,
so the two JSON lines compare the same keys on the same GPU:

    python -m poggers_b200.bench_configs --config del    # this library
    python -m oracle.time_refcuda --config del           # the reference's build
    python -m poggers_b200.bench_configs --config tcf
    python -m oracle.time_refcuda --config tcf
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def time_del(args):
    from oracle import pyrefcuda as rc
    from poggers_b200 import bench_configs as bc

    d = bc.del_flow(args.log2)
    ms = []
    for step in range(args.steps + 2):
        r = rc.RefTable(rc.KIND_DEL_TCF, d["n0"], d["n1"], 42)

        def run(op, k, v, fl, out=None):
            r.bbulk(op if op != 3 else rc.OP_INSERT_DELETE, k, v, fl, out)

        m = bc.del_phases(run, d)
        r.close()
        if step >= 2:
            ms.append(m)
    return {"config": "del", "impl": "reference_cuda", "keys": d["n"], "reference_cuda": bc.del_summary(ms, d)}


def time_tcf(args):
    from oracle import pyrefcuda as rc
    from poggers_b200 import bench_configs as bc

    res = {"config": "tcf", "impl": "reference_cuda"}
    for name, log2, backing, load, values in bc.TCF_WORKLOADS:
        d = bc.tcf_inputs(log2, load, values)
        n0 = 1 << log2
        kind = rc.KIND_TCF if backing else rc.KIND_TCQF
        runs = []
        for step in range(args.steps + 2):
            r = rc.RefTable(kind, n0, n0 // backing if backing else 0, 42)

            def run(op, k, v, fl):
                r.bulk(op, k, v, fl)

            out = bc.tcf_phases(run, d)
            r.close()
            if step >= 2:
                runs.append(out)
        res[name] = bc.tcf_summary(runs, d)
        del d
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", choices=["del", "tcf"], required=True)
    ap.add_argument("--log2", type=int, default=28, help="config del: log2 of the primary slot count")
    ap.add_argument("--steps", type=int, default=5)
    a = ap.parse_args()
    from oracle import pyrefcuda as rc
    if not rc.available():
        print(json.dumps({"config": a.config, "impl": "reference_cuda",
                          "unavailable": "oracle/_ref/libpoggers_refcuda.so is not built (make -C oracle refcuda)"}))
        return
    print(json.dumps(time_del(a) if a.config == "del" else time_tcf(a)))


if __name__ == "__main__":
    main()
