"""Benchmark of the FRW transition engine: plain FRW capacitance extraction
with an FDM surface-Green's-function solve on every hop (N = 16), on the
8-conductor two-layer crossing structure (two orthogonal layers of 4 wires,
w = s = t = 0.1 um, L = 2 um, 3-layer dielectric 3.9/2.7/4.2, grounded box
with 1 um margin, Gaussian surface 0.05 um, master = wire 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

A step is one batch of walks (``--walks`` per GPU, default 32768) of that job
on the device; every hop of every walk voxelises its transition cube, solves
the cube's FDM system on chip (FP32 CG + FP64 refinement to 1e-8), draws the
next point and hit-tests it. Walk ids advance across steps and ranks, so no
step repeats work. Prints one JSON line (rank 0).

--impl reference times the reference's CPU implementation of the path on the
host cores: the restated CPU walk loop (the reference walker ships compiled
only) calling the reference ggft solver, compiled from its own sources, for
every hop.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "hops/s & job time at 1% cap error: learned+served vs FDM-per-hop, 1 B200"
N_CUBE = 16
FDM_TOL = 1e-8


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


def sustained_bf16():
    """Dense BF16 peak under the power cap, for work timed inside a long step:
    (TFLOP/s, source)."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        if "bf16_tflops_sustained" in d:
            return float(d["bf16_tflops_sustained"]), "measured sustained"
    return 1400.0, "fallback sustained"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self._t = None

    def __enter__(self):
        # one nvidia-smi process printing a line every 50 ms (a process per
        # sample takes longer to start than a short timed region lasts)
        self._p = None
        try:
            self._p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            return self

        def run():
            for line in self._p.stdout:
                if line.strip():
                    self.rows.append([x.strip() for x in line.split(",")])
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        if self._p is None:
            return
        self._p.terminate()
        try:
            self._p.wait(timeout=5)
        except Exception:
            self._p.kill()
        self._t.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def workload():
    from deeprwcap_b200 import workloads as W
    s = W.two_layer_crossing()
    p = W.job_params_plain(N=N_CUBE, seed=20261203, tol=FDM_TOL)
    return s, p


def cpu_walks(nthreads: int, budget_s: float, walk0: int, batch: int, records=None):
    """Reference CPU path: restated walk loop + reference ggft per hop. With
    records = [] the per-walk (end net, weight) arrays are appended to it."""
    from oracle import oracle as O
    s, p = workload()
    sc = s.to_c()
    kind = "reference" if O.ref_available(N_CUBE) else "port"
    fdm = "ggft" if kind == "reference" else "oracle"
    hops = walks = 0
    t0 = time.perf_counter()
    w0 = walk0
    while time.perf_counter() - t0 < budget_s:
        e, h, w, _ = O.frw_walks(sc, p, w0, batch, fdm=fdm, fdm_tol=FDM_TOL, nthreads=nthreads)
        if records is not None:
            records.append((e, w))
        hops += int(h.sum())
        walks += batch
        w0 += batch
    dt = time.perf_counter() - t0
    return hops, walks, dt, kind


def run_reference(args, world, rank):
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_walks(nthreads, 0.0, 10_000_000, nthreads)
    tot_h = tot_w = 0
    tot_t = 0.0
    kind = "reference"
    for k in range(args.steps):
        h, w, dt, kind = cpu_walks(nthreads, args.cpu_step_s, 20_000_000 + k * 100_000,
                                   2 * nthreads)
        tot_h += h; tot_w += w; tot_t += dt
    v = tot_h / tot_t
    sample = (f"{tot_w} walks ({tot_h} hops) of the two-layer crossing job per run, "
              f"{args.steps} steps of ~{args.cpu_step_s:.0f} s; restated CPU walk loop with the "
              f"reference ggft (compiled from its sources, N={N_CUBE}, tol {FDM_TOL:g}) per hop")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "hops/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": "two_layer_crossing_frw_fdm_per_hop",
                                        "N": N_CUBE, "fdm_tol": FDM_TOL},
        "cpu_baseline": {"value": v, "unit": "hops/s", "cores": nthreads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": v, "unit": "hops/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def walk_roofline(prof, hops_tot, t_dev, steps, clocks, streamed_gbs, hbm, src):
    """Roofline of the walk kernel. The kernel keeps each cube in shared
    memory and registers, so its bound is the shared-memory pipe: achieved =
    the ncu shared-memory wavefronts per hop x 128 B x the hops per second
    measured here; peak = 148 SMs x 128 B per clock at the sampled median SM
    clock; traffic = ncu DRAM bytes per hop x hops per launch. The streamed-
    PCG figure (the HBM bytes an HBM-resident solver would move for the same
    iterations) is kept as a secondary field."""
    mhz = clocks.get("sm_mhz") or 1965.0
    wf = prof.get("smem_wavefronts_per_hop")
    dram = prof.get("dram_bytes_per_hop")
    hps = hops_tot / t_dev
    out = {"bound": "smem", "unit": "GB/s", "peak": smem_peak_gbs(mhz),
           "peak_source": f"148 SMs x 128 B/clk x {mhz:.0f} MHz (sampled median)",
           "achieved": None, "frac": None,
           "traffic": None if dram is None else dram * hops_tot / steps,
           "smem_wavefronts_per_hop": wf, "dram_bytes_per_hop": dram,
           "fma_pipe_frac_profiled": prof.get("fma_pipe_frac"),
           "fp64_pipe_frac_profiled": prof.get("fp64_pipe_frac"),
           "issue_frac_profiled": prof.get("issue_active_frac"),
           "streamed_pcg_hbm_equivalent": {"achieved": streamed_gbs, "peak": hbm,
                                           "frac": streamed_gbs / hbm, "peak_source": src},
           "note": "achieved = ncu shared-memory wavefronts per hop x 128 B x live hops/s; "
                   "*_profiled are fractions from the ncu capture (a 2048-walk launch)"}
    if wf:
        out["achieved"] = wf * 128.0 * hps / 1e9
        out["frac"] = out["achieved"] / out["peak"]
    return out


def profile_figures():
    """Per-hop figures of the walk kernel from the committed ncu summary
    (profiles/walk_kernel_two_layer_crossing_N16.txt): lines "key: value"."""
    p = ROOT / "profiles" / "walk_kernel_two_layer_crossing_N16.txt"
    out = {}
    if not p.exists():
        return out
    for line in p.read_text().splitlines():
        if ":" in line and not line.startswith(" "):
            k, v = line.split(":", 1)
            try:
                out[k.strip()] = float(v.split()[0])
            except (ValueError, IndexError):
                pass
    return out


def smem_peak_gbs(sm_mhz):
    """Shared-memory pipe bandwidth of the GPU: 148 SMs x 128 B (one wavefront)
    per SM clock at the sampled SM clock."""
    return 148 * 128 * float(sm_mhz) * 1e6 / 1e9


def learned_section(ctx, args):
    """Train the network on engine-generated FDM data (untimed), then run the
    same walks with the learned transition kernels and with the FDM per hop,
    on the dense structure (3 orthogonal layers x 8 wires, 5 stratified
    dielectric layers, 10 dielectric blocks), and time the network alone."""
    import torch
    from deeprwcap_b200 import engine, train
    from deeprwcap_b200 import workloads as W
    t0 = time.perf_counter()
    X, T, TG = train.build_dataset(ctx, args.train_samples, seed=0, log=lambda *a: None)
    Xt, Tt, TGt, Xv, Tv, TGv = train.split(X, T, TG)
    net = engine.Net(seed=1, ctx=ctx)
    tsec = train.train(net, Xt, Tt, TGt, epochs=args.train_epochs, batch=512, lr=1e-3,
                       log=lambda *a: None)
    ev = train.evaluate(net, Xv, Tv, TGv)
    t_train = time.perf_counter() - t0
    s = W.dense_stack(seed=3)
    p = W.job_params_plain(N=16, seed=4242, tol=FDM_TOL)
    nw = args.learned_walks
    o = engine.learned_opts(slots=65536, conf_threshold=-1.5, audit_frac=0.01)
    engine.frw_walks_learned(s, p, net, 50_000_000, 20000, o)  # warm-up
    l0 = ctx.launches
    e1, h1, w1, st = engine.frw_walks_learned(s, p, net, 0, nw, o)
    l_launch = ctx.launches - l0
    t1 = time.perf_counter()
    e0, h0, w0 = engine.frw_walks(s, p, 0, nw, ctx=ctx)
    t_fdm = time.perf_counter() - t1
    cap = lambda e, w: [float(w[e == j].sum() / len(w)) for j in range(s.n_nets + 1)]
    c1, c0 = cap(e1, w1), cap(e0, w0)
    # the same job through the server: network + uniform-permittivity table
    served = {}
    for name, kw in (("served_learned", {}), ("served_learned_table", {"uniform_table": 1})):
        pj = W.job_params_plain(N=16, seed=4242, tol=FDM_TOL, min_walks=nw, max_walks=nw,
                                batch_walks=1 << 16)
        dev = torch.device("cuda", ctx.device)
        rec_e = torch.full((nw,), -2, dtype=torch.int32, device=dev)
        rec_w = torch.zeros(nw, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        with engine.Server(ctx, net=net, timing=1 if not kw else 0, **kw) as srv:
            t2 = time.perf_counter()
            r = srv.wait(srv.submit(s, pj, records=(rec_e, rec_w)), timeout=3600)
            dt = time.perf_counter() - t2
            sst = srv.stats()
        torch.cuda.synchronize()
        acc = paired_accuracy(rec_e.cpu().numpy(), rec_w.cpu().numpy(), e0, w0, s.n_nets + 1)
        if not kw:
            # network stage of the served step (voxeliser + conv1, conv2, conv3, heads,
            # sampler) timed by graph event nodes; one gradient-head row per walk
            flop = sst["net_rows"] * 2.0 * (512 * 16 * 27 + 64 * 32 * 432 + 8 * 64 * 864 +
                                             512 * net.out_row) + nw * 2.0 * 512 * net.grad_row
            served_nn = {"rows": sst["net_rows"], "seconds": sst["net_seconds"],
                         "tflops": flop / max(sst["net_seconds"], 1e-12) / 1e12}
        served[name] = {"seconds": dt, "hops": int(r.hops), "hops_per_s": r.hops / dt,
                        "net_hops": sst["net_hops"], "fdm_hops": sst["fdm_hops"],
                        "table_hops": sst["table_hops"], "fallbacks": sst["fallbacks"],
                        "audits": sst["audits"], "audit_kl_mean": sst["audit_kl_mean"],
                        "cap_fF": [float(x) for x in r.cap],
                        "self_rel_diff_vs_fdm": abs(r.cap[0] - c0[0]) / abs(c0[0]),
                        "self_rel_stderr": float(r.stderr[0] / abs(r.cap[0])),
                        "accuracy": acc}
    # the network alone on a fixed batch (tensor-core fraction)
    B = 65536
    dev = torch.device("cuda", ctx.device)
    Xb = X[:B].contiguous()
    O = torch.empty(B, net.out_row, device=dev)
    torch.cuda.synchronize()
    net.forward(Xb, O)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    reps = 5
    ev0.record(stream)
    for _ in range(reps):
        ctx.lib.drwc_net_forward(net.h, B, Xb.data_ptr(), O.data_ptr(), None)
    ev1.record(stream)
    torch.cuda.synchronize()
    t_nn = ev0.elapsed_time(ev1) / 1e3 / reps
    flop = B * 2.0 * (512 * 16 * 27 + 64 * 32 * 432 + 8 * 64 * 864 + 512 * engine.NET_OUT)
    _, bf16, src = peaks()
    sus, sus_src = sustained_bf16()
    hl, hf = h1.sum() / st["seconds"], h0.sum() / t_fdm
    return net, {"structure": "dense_stack (24 conductors, 5 layers, 10 blocks)", "walks": nw,
            "train": {"samples": int(X.shape[0]), "epochs": args.train_epochs,
                      "seconds": t_train, "train_step_seconds": tsec, **ev},
            "learned_hops_per_s": hl, "fdm_hops_per_s": hf, "gain": hl / hf,
            **served,
            "gain_served_learned_table": served["served_learned_table"]["hops_per_s"] / hf,
            "gain_served_learned": served["served_learned"]["hops_per_s"] / hf,
            "net_hops": st["net_hops"], "fdm_hops": st["fdm_hops"],
            "fallbacks": st["fallbacks"], "audits": st["audits"],
            "audit_kl_mean": st["audit_kl"], "learned_launches": int(l_launch),
            "cap_learned_fF": c1, "cap_fdm_fF": c0,
            "self_rel_diff": abs(c1[0] - c0[0]) / abs(c0[0]),
            "accuracy": paired_accuracy(e1, w1, e0, w0, s.n_nets + 1),
            "nn_forward": {"cubes": B, "seconds": t_nn, "tflops": flop / t_nn / 1e12,
                           "peak_tflops": bf16, "frac": flop / t_nn / 1e12 / bf16,
                           "peak_source": src, "path": "drwc_net_forward (conv1 as a GEMM)"},
            "nn_served_stage": {**served_nn, "peak_tflops": sus,
                                "frac": served_nn["tflops"] / sus, "peak_source": sus_src,
                                "note": "server network stage incl. voxelisation and sampling, "
                                        "timed inside a long step (sustained peak)"}}


def serving_section(ctx, args, net):
    """Config-4 stream (Poisson arrivals at 50 jobs/s; 2-4 layers x 4-16
    wires; N in {16, 21, 23}; walks log-uniform in [1e5, --serve-walks-max])
    through three arms on the same seeded jobs: drwc_frw_run one job at a
    time in arrival order (the FDM-per-hop engine without serving), the
    server with an FDM solve on every hop, and the server with the learned
    networks (one per resolution, N = 16 from the learned section, 21 and 23
    trained here the same way) and the uniform-permittivity table for cubes
    of a single permittivity. Latency = submission to result."""
    from deeprwcap_b200 import engine
    from deeprwcap_b200 import workloads as W
    stream = W.serving_stream(n_jobs=args.serve_jobs, rate=50.0, seed=1,
                              walks=(1e5, args.serve_walks_max))
    hbm, _, _ = peaks()

    def summary(lat, hops, wall, st=None):
        lat = np.asarray(lat)
        out = {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
               "makespan_s": wall, "hops": int(hops), "hops_per_s": hops / wall}
        if st is not None:
            out.update({"busy_s": st["busy_seconds"], "hops_per_s_busy": st["hops"] / st["busy_seconds"],
                        "fdm_hops": st["fdm_hops"], "net_hops": st["net_hops"],
                        "table_hops": st["table_hops"], "fallbacks": st["fallbacks"],
                        "audits": st["audits"], "audit_kl_mean": st["audit_kl_mean"],
                        "graph_launches": st["graph_launches"],
                        "kernels_launched": st["kernels_launched"],
                        "max_running": st["max_running"], "arena_peak_bytes": st["arena_peak"],
                        "fdm_alg_GBps_over_busy": st["fdm_bytes"] / st["busy_seconds"] / 1e9})
        return out

    # (1) one job at a time through drwc_frw_run, started when it arrives
    t0 = time.perf_counter()
    lat, hops = [], 0
    for j in stream:
        dt = t0 + j.arrival - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        r = engine.extract(j.structure, W.serve_params(j), ctx)
        lat.append(time.perf_counter() - (t0 + j.arrival))
        hops += r.hops
    seq = summary(lat, hops, time.perf_counter() - t0)

    import torch
    dev = torch.device("cuda", ctx.device)

    def served(**opts):
        # every job's walk records (end net, weight by walk id) for the
        # walk-by-walk comparison of the forms
        recs = [(torch.full((j.walks,), -2, dtype=torch.int32, device=dev),
                 torch.zeros(j.walks, dtype=torch.float64, device=dev)) for j in stream]
        torch.cuda.synchronize()
        with engine.Server(ctx, **opts) as srv:
            t0 = time.perf_counter()
            ids = []
            for j, rc in zip(stream, recs):
                dt = t0 + j.arrival - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                ids.append(srv.submit(j.structure, W.serve_params(j), records=rc))
            res = [srv.wait(i, timeout=3600) for i in ids]
            wall = time.perf_counter() - t0
            lat = [srv.times(i)[1] for i in ids]
            st = srv.stats()
        torch.cuda.synchronize()
        host = [(e.cpu().numpy(), w.cpu().numpy()) for e, w in recs]
        del recs
        return summary(lat, sum(r.hops for r in res), wall, st), res, host

    plain, res_p, rec_p = served()
    plain["fdm_roofline_frac_of_measured_hbm"] = plain["fdm_alg_GBps_over_busy"] / hbm
    out = {"jobs": len(stream), "rate_jobs_per_s": 50.0,
           "walks_range": [1e5, args.serve_walks_max],
           "N_mix": {str(n): sum(1 for j in stream if j.N == n) for n in (16, 21, 23)},
           "total_walks": int(sum(j.walks for j in stream)),
           "sequential_frw_run": seq, "served_fdm": plain}
    if net is not None:
        # networks for the other served resolutions, trained here like the N = 16 one
        from deeprwcap_b200 import train
        nets, train_info = [net], {}
        for N in (21, 23):
            t0 = time.perf_counter()
            X, T, TG = train.build_dataset(ctx, args.serve_train_samples, seed=N, N=N,
                                           log=lambda *a: None)
            Xt, Tt, TGt, Xv, Tv, TGv = train.split(X, T, TG, seed=N)
            nN = engine.Net(seed=N, ctx=ctx, N=N)
            train.train(nN, Xt, Tt, TGt, epochs=args.train_epochs, batch=512, lr=1e-3,
                        log=lambda *a: None)
            train_info[str(N)] = {"samples": int(X.shape[0]), "epochs": args.train_epochs,
                                  "seconds": time.perf_counter() - t0,
                                  **train.evaluate(nN, Xv, Tv, TGv)}
            del X, T, TG, Xt, Tt, TGt, Xv, Tv, TGv
            nets.append(nN)
        out["train_21_23"] = train_info
        learned, res_l, rec_l = served(net=nets, uniform_table=1)
        # walk by walk against the FDM-served jobs (the same walk ids; the
        # FDM-served walks are drwc_frw_run's)
        per_job = [paired_accuracy(a[0], a[1], b[0], b[1], j.structure.n_nets + 1)
                   for a, b, j in zip(rec_l, rec_p, stream)]
        learned["accuracy"] = {
            "jobs": len(per_job),
            "jobs_consistent": int(sum(p["all_consistent"] for p in per_job)),
            "jobs_pass": int(sum(p["all_pass"] for p in per_job)),
            "self_rel_diff": [p["entries"]["self"]["rel_diff"] for p in per_job],
            "self_rel_3sem": [p["entries"]["self"]["rel_3sem"] for p in per_job],
            "max_abs_coupling_rel_diff": max(
                (abs(v["rel_diff"]) for p in per_job for k, v in p["entries"].items()
                 if k != "self"), default=0.0),
            "per_job": per_job}
        # capacitance agreement of the learned+served form with the FDM walk, per job
        self_diff = [abs(a.cap[0] - b.cap[0]) / abs(b.cap[0]) for a, b in zip(res_l, res_p)]
        learned["self_cap_rel_diff_vs_fdm"] = {"max": float(max(self_diff)),
                                               "mean": float(np.mean(self_diff))}
        # the two estimates are independent runs: difference over combined 1-sigma
        zs = [abs(a.cap[0] - b.cap[0]) / float(np.hypot(a.stderr[0], b.stderr[0]))
              for a, b in zip(res_l, res_p)]
        learned["self_cap_diff_over_combined_sigma"] = {"max": float(max(zs)),
                                                        "mean": float(np.mean(zs))}
        learned["self_cap_rel_stderr_fdm_mean"] = float(np.mean(
            [b.stderr[0] / abs(b.cap[0]) for b in res_p]))
        out["served_learned_table"] = learned
        out["speedup_hops_per_s_vs_sequential_fdm"] = learned["hops_per_s"] / seq["hops_per_s"]
        out["speedup_p50_vs_sequential_fdm"] = seq["p50_s"] / learned["p50_s"]
    return out


def summary_of(line):
    """The headline figures of every section in a few keys, printed last in the
    JSON line so that a truncated log keeps them."""
    g = lambda d, *ks: (None if d is None else (g(d.get(ks[0]), *ks[1:]) if len(ks) > 1
                                                 else d.get(ks[0])))
    s = {"frw_hops_per_s": line["value"], "frw_e2e_hops_per_s": g(line, "e2e", "value"),
         "roofline_frac": g(line, "roofline", "frac"),
         "roofline_bound": g(line, "roofline", "bound"),
         "job_s": g(line, "job", "seconds"), "job_converged": g(line, "job", "converged"),
         "job_walks": g(line, "job", "walks"),
         "cfg0_gpu_cubes_per_s": g(line, "fdm_config0", "gpu_cubes_per_s"),
         "cfg0_vs_ggft_cores": g(line, "fdm_config0", "gpu_vs_cpu"),
         "cfg0_max_rel_err": g(line, "fdm_config0", "max_rel_err_normwise"),
         "cfg2_cubes_per_s": g(line, "fdm_config2", "cubes_per_s"),
         "cfg2_max_rel_err": g(line, "fdm_config2", "max_rel_err_vs_fp64_oracle"),
         "cpu_baseline_hops_per_s": g(line, "cpu_baseline", "value")}
    pv = g(line, "cpu_baseline", "precision_vs_fp64_walk")
    if pv:
        s["precision_max_entry_rel_diff_vs_fp64_walk"] = max(
            (abs(v["rel_diff"]) for v in pv["entries"].values()), default=None)
    lr = line.get("learned")
    if lr:
        s["dense_gain_learned_walker"] = lr.get("gain")
        s["dense_gain_served_net"] = lr.get("gain_served_learned")
        s["dense_gain_served_net_table"] = lr.get("gain_served_learned_table")
        s["dense_accuracy_all_consistent"] = {
            k: g(lr, *path, "accuracy", "all_consistent") for k, path in
            (("learned_walker", ()), ("served_net", ("served_learned",)),
             ("served_net_table", ("served_learned_table",)))}
    sv = line.get("serving")
    if sv:
        s["stream_speedup_vs_sequential_fdm"] = sv.get("speedup_hops_per_s_vs_sequential_fdm")
        s["stream_p50_s"] = {k: g(sv, k, "p50_s") for k in
                             ("sequential_frw_run", "served_fdm", "served_learned_table")}
        s["stream_jobs_consistent"] = g(sv, "served_learned_table", "accuracy",
                                        "jobs_consistent")
    return s


def paired_accuracy(e1, w1, e0, w0, n_entries, master=0, self_tol=0.01, cpl_tol=0.02):
    """Walk-by-walk comparison of two forms of one job on the same walk ids
    (records e*, w*): per entry the relative difference of the estimates and
    3x the standard error of the walk-by-walk difference, for the self term
    and the couplings that make up 95 % of the coupling magnitude. pass:
    |difference| + 3 sigma within the tolerance (1 % self, 2 % couplings);
    consistent: |difference| within the tolerance + 3 sigma."""
    n = len(w0)
    cap = lambda e, w, j: float(np.where(e == j, w, 0.0).sum() / n)
    c0 = np.array([cap(e0, w0, j) for j in range(n_entries)])
    order = [j for j in np.argsort(-np.abs(c0)) if j != master]
    tot = np.abs(c0[order]).sum()
    cpl, acc = [], 0.0
    for j in order:
        if acc >= 0.95 * tot:
            break
        cpl.append(int(j))
        acc += abs(c0[j])
    rows = {}
    ok = True
    for j, tol in [(master, self_tol)] + [(j, cpl_tol) for j in cpl]:
        d = np.where(e1 == j, w1, 0.0) - np.where(e0 == j, w0, 0.0)
        rel = float(d.mean() / abs(c0[j]))
        sem3 = float(3 * d.std() / np.sqrt(n) / abs(c0[j]))
        rows[("self" if j == master else f"c{j}")] = {
            "rel_diff": rel, "rel_3sem": sem3, "tol": tol,
            "pass": abs(rel) + sem3 <= tol, "consistent": abs(rel) <= tol + sem3}
        ok &= abs(rel) <= tol + sem3
    return {"walks": n, "entries": rows, "all_consistent": bool(ok),
            "all_pass": bool(all(r["pass"] for r in rows.values()))}


def run_b200(args, world, rank, local):
    import torch
    from deeprwcap_b200 import engine

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local))
    ctx = engine.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    s, p = workload()
    job = engine.Job(s, p, ctx)
    B = args.walks
    dev = torch.device("cuda", local)
    end = torch.empty(B, dtype=torch.int32, device=dev)
    hops = torch.empty(B, dtype=torch.int32, device=dev)
    wt = torch.empty(B, dtype=torch.float64, device=dev)
    stats = torch.zeros((args.steps + args.warmup + 1, 5), dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    base = rank * (args.steps + args.warmup) * B

    def step(k, rec=None):
        with torch.cuda.stream(stream):
            flush.zero_()
        if rec:
            rec[0].record(stream)
        job.walks_device(base + k * B, B, end, hops, wt, stats[k])
        if rec:
            rec[1].record(stream)

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    launches0 = ctx.launches
    with ClockSampler(local) as clk:
        t_wall0 = time.perf_counter()
        for k in range(args.steps):
            step(args.warmup + k, evs[k])
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall0
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches = ctx.launches - launches0
    step_ms = [a.elapsed_time(b) for a, b in evs]
    t_dev = sum(step_ms) / 1e3
    st = stats[args.warmup:args.warmup + args.steps].cpu().numpy()
    hops_tot, iters_tot, sweeps_tot, esc_tot, fail_tot = (int(x) for x in st.sum(axis=0))
    # max over ranks of device time, sum of hops
    if world > 1:
        t = torch.tensor([t_dev, float(hops_tot)], dtype=torch.float64, device=dev)
        tmax = t.clone(); torch.distributed.all_reduce(tmax[:1], op=torch.distributed.ReduceOp.MAX)
        tsum = t.clone(); torch.distributed.all_reduce(tsum[1:], op=torch.distributed.ReduceOp.SUM)
        t_dev_all, hops_all = float(tmax[0]), float(tsum[1])
    else:
        t_dev_all, hops_all = t_dev, float(hops_tot)
    value = hops_all / t_dev_all

    # ---- end to end through the public API: host buffers, pinned copies
    e2e = None
    if rank == 0:
        from deeprwcap_b200 import abi
        import ctypes as C
        nE = max(1, min(args.steps, 3))
        h_end = torch.empty(B, dtype=torch.int32).pin_memory()
        h_hops = torch.empty(B, dtype=torch.int32).pin_memory()
        h_w = torch.empty(B, dtype=torch.float64).pin_memory()
        sc = s.to_c()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_hops = 0
        for k in range(nE):
            rc = ctx.lib.drwc_frw_walks(ctx.h, C.byref(sc), C.byref(p), 900_000_000 + k * B, B,
                                        h_end.data_ptr(), h_hops.data_ptr(), h_w.data_ptr(), None)
            abi.check(rc, "drwc_frw_walks")
            e2e_hops += int(h_hops.numpy().sum())
        t_e2e = time.perf_counter() - t0
        e2e = {"value": e2e_hops / t_e2e, "unit": "hops/s",
               "h2d_bytes_per_step": int(job.h2d_bytes),
               "d2h_bytes_per_step": int(B * (4 + 4 + 8) + 3 * 8)}

    # ---- job time to convergence (-p 1%, -c 1%, --c-ratio 0.95)
    job_info = None
    if rank == 0 and not args.no_job:
        pj = p
        pj.max_walks = args.job_max_walks
        pj.batch_walks = 1 << 17
        pj.min_walks = 1 << 17
        r = engine.extract(s, pj, ctx)
        job_info = {"seconds": r.seconds, "walks": int(r.walks), "hops": int(r.hops),
                    "converged": r.converged, "hops_per_s": r.hops_per_s,
                    "cap_fF": [float(x) for x in r.cap],
                    "stderr_fF": [float(x) for x in r.stderr]}

    # ---- the FDM Green's-function workloads on their own: 64 cubes of N = 16
    #      against the reference ggft, and the 8192-cube mixed batch
    fdm0 = fdm2 = None
    if rank == 0 and not args.no_fdm:
        fdm0 = fdm_config0_section(ctx, args)
        fdm2 = fdm_batch_section(ctx, args, 3, 2)

    # ---- learned transition kernels (network trained here on engine-generated
    #      FDM data) vs the FDM walk on the dense 24-conductor structure
    learned = None
    net = None
    if rank == 0 and not args.no_learned:
        net, learned = learned_section(ctx, args)

    # ---- serving: a Poisson stream of extraction jobs through the server
    serving = None
    if rank == 0 and not args.no_serve:
        serving = serving_section(ctx, args, net)

    # ---- roofline of the dominant kernel (the per-hop FDM solve inside the walk kernel)
    hbm, bf16, src = peaks()
    NNN = N_CUBE ** 3
    alg_bytes = (48.0 * iters_tot + 40.0 * sweeps_tot) * NNN + hops_tot * (8.0 * NNN +
                                                                          8.0 * 6 * N_CUBE ** 2)
    achieved = alg_bytes / args.steps / (t_dev / args.steps) / 1e9
    prof = profile_figures()

    # ---- CPU baseline (rank 0, N = 1 only): reference CPU path on the host cores
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        nthreads = os.cpu_count() or 1
        recs = []
        h, w, dt, kind = cpu_walks(nthreads, args.cpu_s, 50_000_000, 2 * nthreads, recs)
        cpu = {"value": h / dt, "unit": "hops/s", "cores": nthreads, "kind": kind,
               "sample": f"{w} walks ({h} hops) of the same job, ~{args.cpu_s:.0f} s; restated "
                         f"CPU walk loop + reference ggft per hop (N={N_CUBE}, tol {FDM_TOL:g})"}
        # precision form: the FP32 CG + FP64 refinement walk against the FP64
        # FDM walk (the CPU walker above, reference ggft per hop) on the same
        # walk ids, per capacitance entry
        e_c = np.concatenate([r[0] for r in recs])
        w_c = np.concatenate([r[1] for r in recs])
        e_g, _, w_g = engine.frw_walks(s, p, 50_000_000, len(w_c), ctx=ctx)
        same = (e_g == e_c)
        ent = {}
        for j in range(s.n_nets + 1):
            x_c = np.where(e_c == j, w_c, 0.0)
            x_g = np.where(e_g == j, w_g, 0.0)
            c0 = x_c.mean()
            if c0 == 0.0:
                continue
            d = x_g - x_c
            ent[str(j)] = {"rel_diff": float(d.mean() / abs(c0)),
                           "rel_3sem": float(3 * d.std() / np.sqrt(len(d)) / abs(c0))}
        cpu["precision_vs_fp64_walk"] = {
            "walks": int(len(w_c)), "same_end_net": float(same.mean()),
            "max_weight_rel_diff_same_walks": float(np.max(
                np.abs(w_g[same] - w_c[same]) / np.maximum(np.abs(w_c[same]), 1e-300))),
            "entries": ent,
            "note": "walk-by-walk: the device walk (FP32 CG + FP64 refinement to 1e-8) vs the "
                    "CPU walk with the reference FP64 ggft per hop, same Philox streams"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "hops/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_dev_all / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic",
            "config": {"workload": "two_layer_crossing_frw_fdm_per_hop", "N": N_CUBE,
                       "walks_per_step_per_gpu": B, "fdm_tol": FDM_TOL, "parallelism": f"replicas{world}",
                       "l2": "flushed between steps (256 MB write)",
                       "hops_per_step": hops_tot / args.steps,
                       "fp32_iters_per_hop": iters_tot / max(1, hops_tot),
                       "fp64_sweeps_per_hop": sweeps_tot / max(1, hops_tot),
                       "solves_escalated": esc_tot, "solves_failed": fail_tot},
            "e2e": e2e,
            "gpu_launches": int(launches),
            "roofline": walk_roofline(prof, hops_tot, t_dev, args.steps, clk.summary(),
                                      achieved, hbm, src),
            "clocks": clk.summary(),
            "wall_s_timed": t_wall,
            "job": job_info,
            "fdm_config0": fdm0,
            "fdm_config2": fdm2,
            "learned": learned,
            "serving": serving,
            "cpu_baseline": cpu,
        }
        line["summary"] = summary_of(line)
        print(json.dumps(line), flush=True)
    job.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def _fdm_timed(ctx, torch, stream, call, steps, warmup, flush):
    """Device time per call (CUDA events on the library's stream, L2 flushed
    before each call), after `warmup` untimed calls."""
    for _ in range(warmup):
        call()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        evs[k][0].record(stream)
        call()
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    return sum(x.elapsed_time(y) for x, y in evs) / 1e3 / steps


def fdm_config0_section(ctx, args):
    """64 transition cubes, N = 16 (1-4 horizontal layers with uniform-random z
    cuts and eps ~ U[2, 8], 0-2 random boxes with eps ~ U[2, 8]), each solved
    for the Poisson kernel and the three gradient codes: on the GPU in one
    batched call (inputs resident in HBM, tol 1e-10) and by the reference
    ggft (compiled from its sources, tol 1e-12, as ggft/src/main.cpp:38-57
    loops over cubes) on all host cores. Max relative error per cube and
    code (normwise and elementwise over the row's largest value)."""
    import ctypes as C
    import torch
    from deeprwcap_b200 import abi
    from deeprwcap_b200 import workloads as W
    from oracle import oracle as O
    dev = torch.device("cuda", ctx.device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    n, N = 64, 16
    eps, _ = W.fdm_cubes(n, N, seed=20260, noise_frac=0.0)
    m = 4 * n  # (cube, code) pairs
    Ns = np.full(m, N, dtype=np.int32)
    eoff = (np.arange(m, dtype=np.int64) // 4) * N ** 3
    codes = (np.arange(m) % 4).astype(np.int32)
    ooff = np.arange(m, dtype=np.int64) * 6 * N * N
    eps_d = torch.from_numpy(eps.reshape(-1).copy()).to(dev)
    out_d = torch.zeros(m * 6 * N * N, dtype=torch.float64, device=dev)
    st_d = torch.zeros(m, dtype=torch.int32, device=dev)
    opts = abi.FdmOpts(1e-10, 1e-5, 8, 0)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()

    def call():
        abi.check(ctx.lib.drwc_fdm_solve_batch_device(
            ctx.h, m, Ns.ctypes.data, eoff.ctypes.data, eps_d.data_ptr(), codes.ctypes.data,
            C.byref(opts), ooff.ctypes.data, out_d.data_ptr(), None, None, None,
            st_d.data_ptr()), "drwc_fdm_solve_batch_device")
    t_gpu = _fdm_timed(ctx, torch, stream, call, 5, 3, flush)
    got = out_d.cpu().numpy().reshape(n, 4, -1)
    out = {"workload": "64 cubes, N = 16, GFT + WVTZ/WVTX/WVTY each", "cubes": n,
           "gpu_cubes_per_s": n / t_gpu, "gpu_ms": 1e3 * t_gpu,
           "converged": int((st_d.cpu().numpy() == 0).sum()), "solves": m}
    if O.ref_available(N):
        nthreads = os.cpu_count() or 1
        ref = np.zeros((n, 4, 6 * N * N))
        t_cpu = 0.0
        for code in range(4):
            r, ok, sec = O.ggft_ref(eps, code, tol=1e-12, nthreads=nthreads)
            ref[:, code] = r
            t_cpu += sec
        nrm = np.linalg.norm(got - ref, axis=2) / np.linalg.norm(ref, axis=2)
        elt = np.abs(got - ref).max(axis=2) / np.abs(ref).max(axis=2)
        out.update({"cpu_cubes_per_s": n / t_cpu, "cpu_cores": nthreads,
                    "cpu_kind": "reference ggft, tol 1e-12",
                    "gpu_vs_cpu": t_cpu / t_gpu,
                    "max_rel_err_normwise": float(nrm.max()),
                    "max_rel_err_elementwise": float(elt.max()), "tolerance": 1e-6})
    return out


def fdm_batch_section(ctx, args, steps, warmup, rank=0):
    """8192 cubes, N drawn from {16, 21, 23}, layered permittivity with 10 % of
    cubes carrying voxel noise (eps log-uniform in [1, 12]), one mixed-
    precision solve per cube to a 1e-8 FP64 relative residual. A step is one
    drwc_fdm_solve_batch_device call over all cubes (inputs resident in HBM,
    L2 flushed between steps). Per-cube error vs the FP64 oracle on a sample;
    the reference ggft on a sample of the same cubes, all host cores."""
    import ctypes as C
    import torch
    from deeprwcap_b200 import abi
    from deeprwcap_b200 import workloads as W
    dev = torch.device("cuda", ctx.device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    b = W.mixed_fdm_batch(args.cubes, seed=2026 + rank)
    eps = torch.from_numpy(b.eps).to(dev)
    out = torch.empty(b.out_size, dtype=torch.float64, device=dev)
    n = b.ncubes
    iters = torch.zeros(n, dtype=torch.int32, device=dev)
    sweeps = torch.zeros(n, dtype=torch.int32, device=dev)
    relres = torch.zeros(n, dtype=torch.float64, device=dev)
    status = torch.zeros(n, dtype=torch.int32, device=dev)
    opts = abi.FdmOpts(FDM_TOL, 1e-5, 8, 0)
    Ns = np.ascontiguousarray(b.N, dtype=np.int32)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()

    def call():
        abi.check(ctx.lib.drwc_fdm_solve_batch_device(
            ctx.h, n, Ns.ctypes.data, b.eps_off.ctypes.data, eps.data_ptr(), None,
            C.byref(opts), b.out_off.ctypes.data, out.data_ptr(), iters.data_ptr(),
            sweeps.data_ptr(), relres.data_ptr(), status.data_ptr()), "drwc_fdm_solve_batch_device")
    l0 = ctx.launches
    t = _fdm_timed(ctx, torch, stream, call, steps, warmup, flush)
    launches = (ctx.launches - l0) // max(1, steps + warmup)
    it = iters.cpu().numpy().astype(np.int64)
    sw = sweeps.cpu().numpy().astype(np.int64)
    cells = b.N.astype(np.int64) ** 3
    alg = float(np.sum(cells * (48 * it + 40 * sw)) + 8 * cells.sum() +
                8 * 6 * np.sum(b.N.astype(np.int64) ** 2))
    hbm, _, src = peaks()
    st = status.cpu().numpy()
    res = {"workload": "mixed_fdm_batch", "cubes": n, "N": [16, 21, 23], "noise_frac": 0.1,
           "fdm_tol": FDM_TOL, "cubes_per_s": n / t, "ms_per_step": 1e3 * t,
           "launches_per_step": int(launches),
           "fp32_iters_per_cube": float(it.mean()), "fp64_sweeps_per_cube": float(sw.mean()),
           "converged": int((st == 0).sum()), "max_relres": float(relres.max().item()),
           "streamed_pcg_GBps": alg / t / 1e9, "streamed_pcg_frac_of_hbm": alg / t / 1e9 / hbm,
           "hbm_peak_source": src,
           "note": "streamed_pcg_* = the bytes a streamed (HBM-resident) PCG would move for "
                   "these iterations; the solver keeps each cube on chip"}
    if not args.no_cpu:
        from oracle import oracle as O
        nthreads = os.cpu_count() or 1
        resv = out.cpu().numpy()
        errs = []
        cps_num = cps_den = 0.0
        kind = "port"
        for N in (16, 21, 23):
            idx = np.nonzero(b.N == N)[0][:max(nthreads, 24)]
            cubes = np.stack([b.cube(int(c)) for c in idx])
            if O.ref_available(N):
                _, ok, sec = O.ggft_ref(cubes, 0, tol=FDM_TOL, nthreads=nthreads)
                kind = "reference"
            else:
                _, ok, sec = O.fdm_solve_batch(cubes, 0, tol=FDM_TOL, nthreads=nthreads)
            cps_num += len(idx) * np.mean(b.N == N)
            cps_den += sec * np.mean(b.N == N)
            for c in idx[:8]:
                ref, *_ = O.fdm_solve(b.cube(int(c)), 0, tol=1e-13)
                g = resv[b.out_off[c]:b.out_off[c] + 6 * N * N]
                errs.append(float(np.linalg.norm(g - ref) / np.linalg.norm(ref)))
        res["cpu_baseline"] = {"value": cps_num / cps_den, "unit": "cubes/s", "cores": nthreads,
                               "kind": kind,
                               "sample": "reference ggft (compiled from its sources) on up to "
                                         "24 cubes per N of the same batch, tol 1e-8"}
        res["max_rel_err_vs_fp64_oracle"] = max(errs)
        res["error_sample_cubes"] = len(errs)
    return res


def run_fdm_batch(args, world, rank, local):
    """Secondary workload alone: the batched uneven FDM (fdm_batch_section) as
    its own JSON line."""
    import torch
    from deeprwcap_b200 import engine
    torch.cuda.set_device(local)
    ctx = engine.Context(local)
    with ClockSampler(local) as clk:
        r = fdm_batch_section(ctx, args, args.steps, args.warmup, rank)
    line = {"metric": "batched uneven FDM surface Green's functions", "value": r["cubes_per_s"],
            "unit": "cubes/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["ms_per_step"], "higher_is_better": True, "dtype": "f32+f64",
            "data": "synthetic", "config": {k: v for k, v in r.items() if k != "cpu_baseline"},
            "gpu_launches": r["launches_per_step"] * args.steps,
            "clocks": clk.summary(), "cpu_baseline": r.get("cpu_baseline")}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 20; 5 for --impl reference, whose steps are ~8 s each)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--walks", type=int, default=32768)
    ap.add_argument("--cpu-s", type=float, default=15.0)
    ap.add_argument("--cpu-step-s", type=float, default=8.0)
    ap.add_argument("--job-max-walks", type=int, default=1 << 22)
    ap.add_argument("--no-job", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="frw", choices=["frw", "fdm_batch"])
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--train-samples", type=int, default=1 << 20)
    ap.add_argument("--train-epochs", type=int, default=4)
    ap.add_argument("--learned-walks", type=int, default=1 << 20)
    ap.add_argument("--cubes", type=int, default=8192)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-fdm", action="store_true")
    ap.add_argument("--serve-jobs", type=int, default=10)
    ap.add_argument("--serve-walks-max", type=float, default=1e7)
    ap.add_argument("--serve-train-samples", type=int, default=1 << 20)
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 5 if args.impl == "reference" else 20
    world, rank, local = dist_init()
    if args.workload == "fdm_batch":
        run_fdm_batch(args, world, rank, local)
    elif args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_b200(args, world, rank, local)


if __name__ == "__main__":
    main()
