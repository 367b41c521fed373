"""Run extraction jobs through the multi-job server and print its statistics.

    python -m deeprwcap_b200.serve [--structure dense_stack|two_layer_crossing]
        [--walks 65536] [--N 16] [--net none|random|PATH] [--uniform-table 0|1]
        [--stream JOBS] [--walks-max 1e6] [--net-sizes 16,21,23]

One job of --walks walks on the named structure (or, with --stream, a
seeded Poisson stream of that many jobs, 50 jobs/s, as in the serving
benchmark) is submitted to a server created with the given options; the job
results and the server's counters are printed as one JSON line. --net random
uses untrained networks, one per size in --net-sizes (the cost of the
learned path does not depend on the weights); PATH loads a network saved by
deeprwcap_b200.train.
"""
from __future__ import annotations

import argparse
import json
import time

from . import engine
from . import workloads as W


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--structure", default="dense_stack",
                    choices=["dense_stack", "two_layer_crossing"])
    ap.add_argument("--walks", type=int, default=65536)
    ap.add_argument("--N", type=int, default=16)
    ap.add_argument("--net", default="none")
    ap.add_argument("--net-sizes", default="16",
                    help="with --net random: the cube resolutions to build networks for, e.g. 16,21,23")
    ap.add_argument("--uniform-table", type=int, default=0)
    ap.add_argument("--slots", type=int, default=0,
                    help="walks in flight (0: 65536)")
    ap.add_argument("--stream", type=int, default=0)
    ap.add_argument("--walks-max", type=float, default=1e6)
    a = ap.parse_args()
    ctx = engine.default_context(0)
    net = None
    if a.net == "random":
        net = [engine.Net(seed=1, ctx=ctx, N=int(n)) for n in a.net_sizes.split(",")]
    elif a.net != "none":
        from . import train
        net = train.load(a.net, ctx=ctx)
    opts = dict(slots=a.slots, uniform_table=a.uniform_table)
    if net is not None:
        opts.update(conf_threshold=1e9 if a.net == "random" else -1.5, audit_frac=0.01)
    if a.stream:
        jobs = [(j.arrival, j.structure, W.serve_params(j))
                for j in W.serving_stream(n_jobs=a.stream, seed=1, walks=(1e5, a.walks_max))]
    else:
        s = W.dense_stack(seed=3) if a.structure == "dense_stack" else W.two_layer_crossing()
        jobs = [(0.0, s, W.job_params_plain(N=a.N, seed=4242, tol=1e-8, min_walks=a.walks,
                                            max_walks=a.walks, batch_walks=1 << 16))]
    with engine.Server(ctx, net=net, **opts) as srv:
        t0 = time.perf_counter()
        ids = []
        for arrival, s, p in jobs:
            dt = t0 + arrival - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            ids.append(srv.submit(s, p))
        res = [srv.wait(i, timeout=3600) for i in ids]
        wall = time.perf_counter() - t0
        lat = [srv.times(i)[1] for i in ids]
        st = srv.stats()
    hops = sum(r.hops for r in res)
    print(json.dumps({"jobs": len(jobs), "hops": hops, "seconds": wall, "hops_per_s": hops / wall,
                      "latency_s": lat, "self_cap_fF": [float(r.cap[0]) for r in res],
                      "stats": st}))


if __name__ == "__main__":
    main()
