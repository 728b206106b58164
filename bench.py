#!/usr/bin/env python
"""Throughput of the self-gravity Poisson solve on B200.

Workload (one "step" = one solve): the time-step call of bipoly_hydro's
potential_solver on the 130x98x256 grid (dr = dz = 1/126, isym 2, mmax 30):
a bipolytropic binary (R1 0.3, R2 0.22, separation 0.9, mass ratio 0.5, core
density x2 inside 0.4 R) rigidly rotated by one azimuthal zone per solve,
each solve warm-started from the previous potential (5 ADI steps).  Every
solve streams the FP64 Green tables (212 MB in the compact form, 660 MB in
full), so the per-step working set is larger than the 126 MB L2.

  value      solves/s with rho resident in HBM (device-array C ABI call)
  e2e        solves/s through the host-array C ABI call: pinned rho copied in
             and pot copied out inside every step
  roofline   the boundary contraction (the dominant kernel: k_green_compact
             on the compact tables, k_green_contract on the full ones)
             against measured HBM
  batched    warm solves of n independent instances per call (one pass over
             the Green tables for all n): solves/s per batch size
  converged  the same sequence solved to convergence in FP64 and in the
             mixed form (FP32 ADI cycles, FP64 residual/update refinement):
             solves/s, p50/p99 latency, and the mixed form's error vs FP64
  cpu_baseline  the CPU oracle (C restatement of the reference algorithm)
             on this host

--impl reference times that CPU restatement as the reference arm (the
Fortran reference cannot be compiled on these machines).

Multi-GPU (torchrun): every rank runs its own independent solve sequence
(weak scaling, no collective on the data path); timing is max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GRID = dict(numr=130, numz=98, numphi=256, dr=1.0 / 126.0, isym=2, mmax=30)
METRIC = "Poisson solves/s at 130x98x256 (FP64 drop-in, warm 5-step time-step solve)"
FALLBACK_HBM_GBS = 6650.0


def compulsory_bytes(numr, numz, numphi, mmax, isym, warm=True, G=1):
    """B_alg per solve: read rho, read warm Phi, write Phi, stream the tables once."""
    n = numr * numz * numphi
    nr, nz = numr - 2, numz - 2
    rows = nr + nz + (nr if isym == 1 else 0)
    return 8 * n * (1 + (1 if warm else 0) + 1) + 8 * nr * nz * rows * mmax / G


def contract_bytes(numr, numz, mmax, isym):
    """Algorithmic bytes of one k_green_contract launch: tables + moment vectors + S."""
    nr, nz = numr - 2, numz - 2
    rows = nr + nz + (nr if isym == 1 else 0)
    return 8 * (nr * nz * rows * mmax + 2 * mmax * nr * nz + 2 * mmax * rows)


def compact_dims(numr, numz, isym):
    """The compact-table layout of bph_compact.h: tiles, side-vector stride, sets."""
    nr, nz = numr - 2, numz - 2
    nb8 = (nr + 7) // 8
    kpl = (nz + 31) // 32
    return dict(nr=nr, nz=nz, npair=nb8 * (nb8 + 1) // 2, nsets=2 if isym == 1 else 1, stride=nz + 32 * kpl,
                side_ctas=(nr + 7) // 8)


def compact_table_bytes(numr, numz, mmax, isym):
    """Bytes of the compact tables: symmetric 8x8 tiles per height plus the side vectors."""
    d = compact_dims(numr, numz, isym)
    return 8 * mmax * (d["nsets"] * d["npair"] * d["nz"] * 64 + d["nr"] * 2 * d["stride"])


def compact_contract_bytes(numr, numz, mmax, isym):
    """Algorithmic bytes of one k_green_compact launch: compact tables + moment vectors
    + partial sums written and read once + S."""
    d = compact_dims(numr, numz, isym)
    nr, nz = d["nr"], d["nz"]
    rows = nr + nz + (nr if isym == 1 else 0)
    parts = mmax * (d["nsets"] * d["npair"] * 32 + d["side_ctas"] * nz * 2)
    return compact_table_bytes(numr, numz, mmax, isym) + 8 * (2 * mmax * nr * nz + 2 * parts + 2 * mmax * rows)


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def committed_traffic(kernel="k_green_contract"):
    """dram bytes per launch of the contraction kernel from its committed ncu summary, if any."""
    name = {"k_green_contract": "green_contract_130x98x256.md",
            "k_green_compact": "green_compact_130x98x256.md"}[kernel]
    path = os.path.join(ROOT, "profiles", name)
    try:
        text = open(path).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", text)
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clock/throttle samples of one GPU while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def __enter__(self):
        import tempfile

        fd, self.path = tempfile.mkstemp(prefix="bph_clocks_", suffix=".csv")
        os.close(fd)
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), float(parts[2]), parts[3:]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        smax = max(r[1] for r in rows)
        loaded = [r for r in rows if r[2] > 200.0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in loaded:
            for name, flag in zip(names, r[3][1:]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(loaded)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    """Max of a per-rank value (device time of the timed region) over ranks."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: int, world: int, ms_max: float) -> float:
    """Whole-job throughput: units all ranks processed / the slowest rank's time."""
    return world * units_per_rank / (ms_max / 1e3)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def shard_instances(n: int, world: int, rank: int) -> range:
    """The contiguous block of instance ids 0..n-1 that rank owns; block sizes
    differ by at most one and the blocks of ranks 0..world-1 cover 0..n-1
    once.  Independent solves need no exchange between ranks."""
    q, r = divmod(n, world)
    start = rank * q + min(rank, r)
    return range(start, start + q + (1 if rank < r else 0))


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def oracle_section(B, solver, base, last, args, want_cpu):
    """Parity of the timed workload with the CPU oracle, and the CPU baseline.

    * last_timed_rel_l2: the oracle's warm state is set from the potential
      of the second-to-last timed solve, and its warm solve of the last timed
      density is compared with the last timed potential;
    * sequence: a cold solve and four warm rotated solves through the
      host-array drop-in call on the GPU and on the oracle, max rel L2;
    * cpu_baseline: warm solves/s of the oracle on this host's cores.
    """
    from bipoly_hydro_b200 import fields
    from oracle import oracle as O

    O.build()
    O.set_num_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    o = O.Oracle(GRID["numr"], GRID["numz"], GRID["numphi"], GRID["dr"], GRID["isym"], GRID["mmax"])
    setup_s = time.perf_counter() - t0
    shape = (GRID["numr"], GRID["numz"], GRID["numphi"])

    def fortran(v):
        return np.asfortranarray(np.asarray(v).reshape(shape, order="F"))

    parity = {"tolerance": 1e-12, "oracle_setup_s": setup_s}
    if last["prev"] is not None:
        o.set_potential(fortran(last["prev"]))
        po = o.potential_solver(fortran(last["rho"]), last["tstep"])
        parity["last_timed_rel_l2"] = rel_l2(fortran(last["pot"]), po)
    else:
        parity["last_timed_rel_l2"] = None
    seq = []
    for k in range(5):
        rho = fields.rotate(base, k)
        seq.append(rel_l2(solver.potential_solver(rho, 0 if k == 0 else k + 1),
                          o.potential_solver(rho, 0 if k == 0 else k + 1)))
    parity["sequence_rel_l2"] = seq
    parity["sequence"] = "cold + 4 warm rotated solves through bph_potential_solver (host arrays)"
    parity["pass"] = max(seq + [parity["last_timed_rel_l2"] or 0.0]) <= 1e-12
    cpu = None
    if want_cpu:
        n, t0 = 0, time.perf_counter()
        while True:
            o.potential_solver(fields.rotate(base, 5 + n), 6 + n)
            n += 1
            el = time.perf_counter() - t0
            if el >= args.cpu_seconds or n >= 200:
                break
        cpu = {"value": n / el, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
               "sample": f"{n} warm solves of the same sequence in {el:.1f} s after an untimed setup "
                         f"(C restatement of potential_solver, OpenMP)"}
    o.close()
    return parity, cpu


def run_reference(args, world, rank):
    """--impl reference: the CPU restatement on this host's cores, rank 0 only."""
    if rank != 0:
        return
    from bipoly_hydro_b200 import fields

    base = fields.bipolytrope_pair(GRID["numr"], GRID["numz"], GRID["numphi"], GRID["dr"], GRID["isym"])
    cores = os.cpu_count() or 1
    from oracle import oracle as O

    O.build()
    O.set_num_threads(cores)
    o = O.Oracle(GRID["numr"], GRID["numz"], GRID["numphi"], GRID["dr"], GRID["isym"], GRID["mmax"])
    o.potential_solver(base, 0)
    for w in range(args.warmup):
        o.potential_solver(fields.rotate(base, 1 + w), 2 + w)
    times = []
    t_all = time.perf_counter()
    for i in range(args.steps):
        rho = fields.rotate(base, 1 + args.warmup + i)
        t0 = time.perf_counter()
        o.potential_solver(rho, 2 + args.warmup + i)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_all > args.reference_budget_s:
            break
    o.close()
    n = len(times)
    total = sum(times)
    v = n / total
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": n, "warmup": args.warmup, "ms_per_step": 1e3 * total / n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "130x98x256 warm time-step solves, bipolytrope pair rotated 1 zone/solve",
                   **GRID, "nsteps_adi": 5},
        "p50_ms": 1e3 * float(np.percentile(times, 50)), "p99_ms": 1e3 * float(np.percentile(times, 99)),
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
                         "sample": f"{n} warm solves of the sequence (steps requested {args.steps}), "
                                   f"C restatement of potential_solver with OpenMP over slots/rows"},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference Fortran+MPI cannot be compiled here (no Fortran compiler or MPI); "
                "the arm runs the C restatement of its algorithm",
    }
    print(json.dumps(line), flush=True)


def serve_bench(B, torch, dev, rhos, args):
    """Continuous-batching server under Poisson arrivals of SCF-like client requests.

    serve_clients resident clients on the 130x98x256 grid, each running an
    SCF-like sequence rho <- 0.9 rho + 0.1 rho (1 + 0.01 N(0,1)) renormalised
    to its initial mass, densities kept on the device (two buffers per
    client); the requests of all clients arrive as one Poisson process at the
    offered rate.  Latency is submit-to-completion as the server records it.
    """
    nclients, iters = args.serve_clients, args.serve_iters
    srv_solver = B.PotentialSolver(**GRID)
    srv = B.Server(srv_solver, max_clients=nclients, mem_cap_bytes=150 * 10 ** 9, device_arrays=True)
    nrot = rhos.shape[0]
    gen = torch.Generator(device=dev)
    gen.manual_seed(20261203)
    out = {"grid": "130x98x256", "clients": nclients, "requests_per_rate": nclients * iters,
           "capacity": srv.capacity, "dtype": "f64 drop-in (rates); converged FP64 vs mixed (converged)",
           "rates": []}

    def run_rate(rate):
        ids = [srv.open_client() for _ in range(nclients)]
        rho = [[rhos[(37 * c) % nrot] * (1.0 + 0.2 * c / nclients), torch.empty_like(rhos[0])] for c in range(nclients)]
        mass = [float(r[0].sum()) for r in rho]
        pot = [[torch.empty_like(rhos[0]), torch.empty_like(rhos[0])] for _ in range(nclients)]
        rng = np.random.default_rng(int(rate))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=nclients * iters))
        rid = {}
        lat = []
        st0 = srv.stats()
        t0 = time.perf_counter()
        for k in range(nclients * iters):
            c, it = k % nclients, k // nclients
            buf = it % 2
            if it >= 2:
                lat.append(srv.wait(rid.pop((c, it - 2)), timeout=120.0)[1])
            src = rho[c][1 - buf] if it > 0 else rho[c][0]
            if it > 0:
                noise = torch.randn(src.shape, generator=gen, device=dev, dtype=torch.float64)
                nxt = src * (1.0 + 0.001 * noise)
                rho[c][buf].copy_(nxt * (mass[c] / float(nxt.sum())))
            else:
                rho[c][buf] = src.clone()
            torch.cuda.current_stream().synchronize()
            while time.perf_counter() - t0 < arrivals[k]:
                pass
            rid[(c, it)] = srv.submit(ids[c], rho[c][buf], pot[c][buf])
        for key in list(rid):
            lat.append(srv.wait(rid.pop(key), timeout=120.0)[1])
        elapsed = time.perf_counter() - t0
        st = srv.stats()
        for cid in ids:
            srv.close_client(cid)
        return {"offered_req_per_s": rate, "solves_per_s": nclients * iters / elapsed,
                "p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
                "mean_batch": (st["solves"] - st0["solves"]) / max(1, st["batches"] - st0["batches"])}

    for rate in [float(x) for x in args.serve_rates.split(",") if x]:
        out["rates"].append(run_rate(rate))
    # converged serving, FP64 against mixed precision (same clients and arrivals)
    conv_rates = [float(x) for x in args.serve_conv_rates.split(",") if x]
    if conv_rates:
        out["converged"] = {"nsteps_per_cycle": args.conv_nsteps, "tol_update": args.conv_tol}
        for key, mixed in (("fp64", False), ("mixed", True)):
            srv.set_converged(args.conv_nsteps, args.conv_tol, 100, mixed)
            out["converged"][key] = [run_rate(r) for r in conv_rates]
        srv.set_converged(0)
    srv.close()
    srv_solver.close()
    return out


MIXED_GRIDS = [(66, 66, 64, 1.0 / 62.0), (130, 98, 128, 1.0 / 126.0), (130, 98, 256, 1.0 / 126.0),
               (258, 194, 256, 1.0 / 250.0)]


def serve_mixed_bench(B, torch, dev, args):
    """Serving with the clients' grids drawn uniformly over MIXED_GRIDS: one
    server (continuous batching, resident clients) per grid, each on its own
    stream, the admission cap split evenly; the requests of all clients
    arrive as one Poisson process; SCF-like sequences as in serve_bench.
    Each grid gets two base densities (drawn q, a, core jump), scaled per
    client."""
    from bipoly_hydro_b200 import fields

    nclients, iters = args.serve_clients, args.serve_iters
    rng = np.random.default_rng(20261204)
    shape_of = [int(g) for g in rng.integers(0, len(MIXED_GRIDS), nclients)]
    servers, solvers, streams, bases = [], [], [], []
    for g, (numr, numz, numphi, dr) in enumerate(MIXED_GRIDS):
        sv = B.PotentialSolver(numr, numz, numphi, dr, 2, 30)
        st = torch.cuda.Stream()
        sv.set_stream(st)
        n_g = max(1, shape_of.count(g))
        servers.append(B.Server(sv, max_clients=n_g, mem_cap_bytes=150 * 10 ** 9 // len(MIXED_GRIDS),
                                device_arrays=True))
        solvers.append(sv)
        streams.append(st)
        bases.append([torch.from_numpy(np.ascontiguousarray(fields.bipolytrope_pair(
            numr, numz, numphi, dr, 2, mass_ratio=float(rng.uniform(0.2, 1.0)),
            separation=float(rng.uniform(0.6, 1.0)), core_jump=float(rng.uniform(1.5, 3.0))).ravel(order="F"))).to(dev)
            for _ in range(2)])
    gen = torch.Generator(device=dev)
    gen.manual_seed(20261204)
    out = {"grids": {f"{a}x{b}x{c}": shape_of.count(g) for g, (a, b, c, _) in enumerate(MIXED_GRIDS)},
           "clients": nclients, "requests_per_rate": nclients * iters, "dtype": "f64", "rates": []}
    def run_rate(rate):
        ids = [servers[shape_of[c]].open_client() for c in range(nclients)]
        rho = [[bases[shape_of[c]][c % 2] * (1.0 + 0.2 * c / nclients), None] for c in range(nclients)]
        for r in rho:
            r[1] = torch.empty_like(r[0])
        mass = [float(r[0].sum()) for r in rho]
        pot = [[torch.empty_like(r[0]), torch.empty_like(r[0])] for r in rho]
        arrivals = np.cumsum(np.random.default_rng(int(rate)).exponential(1.0 / rate, size=nclients * iters))
        rid, lat, lat_g = {}, [], [[] for _ in MIXED_GRIDS]
        t0 = time.perf_counter()
        for k in range(nclients * iters):
            c, it = k % nclients, k // nclients
            srv, buf = servers[shape_of[c]], it % 2
            if it >= 2:
                v = srv.wait(rid.pop((c, it - 2)), timeout=120.0)[1]
                lat.append(v)
                lat_g[shape_of[c]].append(v)
            src = rho[c][1 - buf] if it > 0 else rho[c][0]
            if it > 0:
                noise = torch.randn(src.shape, generator=gen, device=dev, dtype=torch.float64)
                nxt = src * (1.0 + 0.001 * noise)
                rho[c][buf].copy_(nxt * (mass[c] / float(nxt.sum())))
            else:
                rho[c][buf] = src.clone()
            torch.cuda.current_stream().synchronize()
            while time.perf_counter() - t0 < arrivals[k]:
                pass
            rid[(c, it)] = srv.submit(ids[c], rho[c][buf], pot[c][buf])
        for (c, it) in list(rid):
            v = servers[shape_of[c]].wait(rid.pop((c, it)), timeout=120.0)[1]
            lat.append(v)
            lat_g[shape_of[c]].append(v)
        elapsed = time.perf_counter() - t0
        res = {
            "offered_req_per_s": rate, "solves_per_s": nclients * iters / elapsed,
            "p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
            "p50_ms_per_grid": {f"{a}x{b}x{c2}": (1e3 * float(np.percentile(lg, 50)) if lg else None)
                                for (a, b, c2, _), lg in zip(MIXED_GRIDS, lat_g)}}
        for c in range(nclients):
            servers[shape_of[c]].close_client(ids[c])
        return res

    for rate in [float(x) for x in args.serve_mixed_rates.split(",") if x]:
        out["rates"].append(run_rate(rate))
    # converged serving over the grid mix, FP64 against mixed precision
    conv_rates = [float(x) for x in args.serve_conv_rates.split(",") if x][:1]
    if conv_rates:
        out["converged"] = {"nsteps_per_cycle": args.conv_nsteps, "tol_update": args.conv_tol}
        for key, mixed in (("fp64", False), ("mixed", True)):
            for srv in servers:
                srv.set_converged(args.conv_nsteps, args.conv_tol, 100, mixed)
            out["converged"][key] = [run_rate(r) for r in conv_rates]
        for srv in servers:
            srv.set_converged(0)
    for srv in servers:
        srv.close()
    for sv in solvers:
        sv.close()
    del bases
    torch.cuda.empty_cache()
    return out


def mixed_grid_bench(B, torch, dev, args, stream):
    """Independent warm solves on a mix of grids: instances drawn uniformly over
    MIXED_GRIDS with mass ratio U(0.2,1), separation U(0.6,1) and core jump
    U(1.5,3).  One batch per grid, all recorded as one plan (one graph launch,
    the grids' branches concurrent), against the same batches called one after
    another on one stream."""
    from concurrent.futures import ThreadPoolExecutor

    from bipoly_hydro_b200 import fields

    rng = np.random.default_rng(20261203)
    n = args.mixed_grid_instances
    shape_of = rng.integers(0, len(MIXED_GRIDS), n)
    params = [(int(g), float(rng.uniform(0.2, 1.0)), float(rng.uniform(0.6, 1.0)), float(rng.uniform(1.5, 3.0)))
              for g in shape_of]

    def make(p):
        g, q, a, cj = p
        numr, numz, numphi, dr = MIXED_GRIDS[g]
        return fields.bipolytrope_pair(numr, numz, numphi, dr, 2, mass_ratio=q, separation=a, core_jump=cj)

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        fields_ = list(ex.map(make, params))
    solvers, batches, parts, counts = [], [], [], []
    t0 = time.perf_counter()
    for g, (numr, numz, numphi, dr) in enumerate(MIXED_GRIDS):
        idx = [i for i in range(n) if shape_of[i] == g]
        if not idx:
            continue
        sv = B.PotentialSolver(numr, numz, numphi, dr, 2, 30)
        sv.set_stream(stream)
        bt = B.Batch(sv, len(idx))
        d_rho = [torch.from_numpy(np.ascontiguousarray(fields_[i].ravel(order="F"))).to(dev) for i in idx]
        d_pot = [torch.empty_like(x) for x in d_rho]
        solvers.append(sv)
        batches.append(bt)
        parts.append((bt, d_rho, d_pot))
        counts.append(len(idx))
    setup_s = time.perf_counter() - t0
    del fields_
    calls = max(3, args.mixed_grid_calls)
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    # the same batches called in turn on one stream
    for bt, r, p in parts:
        bt.solve_device(r, p, 0)
    for w in range(3):
        for bt, r, p in parts:
            bt.solve_device(r, p, 2 + w)
    torch.cuda.synchronize()
    ea.record(stream)
    for k in range(calls):
        for bt, r, p in parts:
            bt.solve_device(r, p, 5 + k)
    eb.record(stream)
    torch.cuda.synchronize()
    ms_serial = ea.elapsed_time(eb) / calls

    # converged solves of every instance, FP64 against mixed precision (cold starts, so both
    # forms run their full cycle count; one batched call per grid, grids in turn)
    conv = {}
    for key, mixed in (("fp64", False), ("mixed", True)):
        for bt, r, p in parts:  # untimed: builds schedules and work arrays
            bt.solve_converged_device(r, p, args.conv_nsteps, True, args.conv_tol, 100, mixed)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cyc = []
        for bt, r, p in parts:
            cyc.append(bt.solve_converged_device(r, p, args.conv_nsteps, True, args.conv_tol, 100, mixed).cycles)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        conv[key] = {"ms": 1e3 * el, "solves_per_s": n / el, "cycles_per_grid": cyc}
        if not mixed:
            ref = [[x.clone() for x in p] for _, _, p in parts]
        else:
            conv[key]["max_rel_err_vs_fp64"] = max(float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
                                                   for (_, _, p), rp in zip(parts, ref) for a, b in zip(p, rp))
            del ref
    conv["speedup_mixed_vs_fp64"] = conv["mixed"]["solves_per_s"] / conv["fp64"]["solves_per_s"]
    conv["nsteps_per_cycle"], conv["tol_update"] = args.conv_nsteps, args.conv_tol

    plan = B.Plan(parts)
    plan.launch(0, stream)
    for w in range(3):
        plan.launch(2 + w, stream)
    plan.synchronize(stream)
    torch.cuda.synchronize()
    ea.record(stream)
    for k in range(calls):
        plan.launch(5 + k, stream)
    eb.record(stream)
    plan.synchronize(stream)
    ms_plan = ea.elapsed_time(eb) / calls
    launches = plan.launches
    plan.close()
    for bt in batches:
        bt.close()
    for sv in solvers:
        sv.close()
    del parts
    torch.cuda.empty_cache()
    return {"instances": n, "per_grid": {f"{a}x{b}x{c}": k for (a, b, c, _), k in
                                         zip([MIXED_GRIDS[g] for g in range(len(MIXED_GRIDS))
                                              if any(shape_of == g)], counts)},
            "plan_solves_per_s": n / (ms_plan / 1e3), "plan_ms_per_launch": ms_plan,
            "plan_kernel_launches": launches,
            "serial_batches_solves_per_s": n / (ms_serial / 1e3), "serial_ms_per_round": ms_serial,
            "setup_s": setup_s, "precision": "f64 drop-in (5 warm ADI steps)", "calls": calls,
            "converged": conv}


def large_grid_bench(B, torch, dev, args, stream):
    """Mixed precision against FP64 on the 258x194x512 grid (dr = 1/250,
    the bipolytrope-pair recipe of the production grid) and on the 66x66x64
    field of two n=1 polytropes: warm drop-in rate, then converged solves
    (FP64, and the FP32 refinement with FP64 residuals) with their error."""
    from bipoly_hydro_b200 import fields

    out = {}
    cases = [("258x194x512", (258, 194, 512, 1.0 / 250.0),
              lambda: fields.bipolytrope_pair(258, 194, 512, 1.0 / 250.0, 2, mass_ratio=0.5)),
             ("66x66x64", (66, 66, 64, 1.0 / 62.0), lambda: fields.two_polytropes())]
    for name, (numr, numz, numphi, dr), make in cases:
        sv = B.PotentialSolver(numr, numz, numphi, dr, 2, 30)
        sv.set_stream(stream)
        base = make()
        d = [torch.from_numpy(np.ascontiguousarray(fields.rotate(base, i).ravel(order="F"))).to(dev)
             for i in range(2)]
        pot = torch.empty_like(d[0])
        sv.potential_solver_device(d[0], pot, 0)
        for i in range(3):
            sv.potential_solver_device(d[i % 2], pot, 2 + i)
        n = 10
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ea.record(stream)
        for i in range(n):
            sv.potential_solver_device(d[i % 2], pot, 5 + i)
        eb.record(stream)
        torch.cuda.synchronize()
        ms = ea.elapsed_time(eb) / n
        res = {"dropin_ms": ms, "dropin_solves_per_s": 1e3 / ms}
        ref = None
        for key, mixed in (("fp64", False), ("mixed", True)):
            ts = []
            for rep in range(4):  # the first builds the loop graph: untimed
                sv.solve_converged_device(d[0], pot, args.conv_nsteps, True, 1e-13, 100, False)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                info = sv.solve_converged_device(d[1], pot, args.conv_nsteps, False, args.conv_tol, 100, mixed)
                torch.cuda.synchronize()
                if rep:
                    ts.append(time.perf_counter() - t0)
            r = {"ms": 1e3 * float(np.median(ts)), "solves_per_s": 1.0 / float(np.median(ts)),
                 "cycles": info.cycles}
            if mixed:
                r["rel_err_vs_fp64"] = float(torch.linalg.norm(pot - ref) / torch.linalg.norm(ref))
            else:
                ref = pot.clone()
            res[key] = r
        res["speedup_mixed_vs_fp64"] = res["mixed"]["solves_per_s"] / res["fp64"]["solves_per_s"]
        res["mixed_kind"] = sv.info()["mixed_kind"]
        out[name] = res
        sv.close()
        del d, pot, ref
        torch.cuda.empty_cache()
    return out


def run_gpu(args, world, rank, local):
    import torch

    import bipoly_hydro_b200 as B
    from bipoly_hydro_b200 import fields

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    numr, numz, numphi = GRID["numr"], GRID["numz"], GRID["numphi"]
    ntot = numr * numz * numphi
    solver = B.PotentialSolver(**GRID)
    stream = torch.cuda.current_stream()
    solver.set_stream(stream)

    # Density sequence: the numphi rotations of the pair are sharded over the
    # ranks (shard_instances); each rank keeps its shard resident and cycles
    # through it (one zone of rotation per solve within the shard).
    base = fields.bipolytrope_pair(numr, numz, numphi, GRID["dr"], GRID["isym"], mass_ratio=0.5)
    base_t = torch.from_numpy(np.ascontiguousarray(base.ravel(order="F"))).to(dev)
    c_view = base_t.view(numphi, numz, numr)  # C view of the Fortran (numr, numz, numphi) array
    total_rot = args.rotations if args.rotations > 0 else numphi
    shard = shard_instances(max(total_rot, world), world, rank)
    nrot = len(shard)
    rhos = torch.empty((nrot, ntot), dtype=torch.float64, device=dev)
    for i, rot in enumerate(shard):
        rhos[i].copy_(torch.roll(c_view, shifts=rot % numphi, dims=0).reshape(-1))
    # two output buffers, alternated by the timed solves: the last two
    # potentials stay on the device for the parity check after the timing
    d_pots = [torch.empty(ntot, dtype=torch.float64, device=dev) for _ in range(2)]
    d_pot = d_pots[0]

    # cold start, then warm-up solves
    solver.potential_solver_device(rhos[0], d_pot, 0)
    tstep = 2
    for w in range(args.warmup):
        solver.potential_solver_device(rhos[(1 + w) % nrot], d_pot, tstep)
        tstep += 1
    solver.synchronize()

    # ---- value: device-resident inputs --------------------------------
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        if not uuid.startswith("GPU-"):
            uuid = "GPU-" + uuid
    except Exception:
        uuid = None
    l0 = solver.launch_count
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(uuid) as clk:
        e0.record(stream)
        for i in range(args.steps):
            solver.potential_solver_device(rhos[(1 + args.warmup + i) % nrot], d_pots[i % 2], tstep)
            tstep += 1
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    launches = solver.launch_count - l0
    solver.synchronize()
    # the last timed solve (its density, the potential before it, its result)
    last_i = args.steps - 1
    last = {"rho": rhos[(1 + args.warmup + last_i) % nrot].cpu().numpy(),
            "prev": d_pots[(last_i - 1) % 2].cpu().numpy() if args.steps >= 2 else None,
            "pot": d_pots[last_i % 2].cpu().numpy(), "tstep": tstep - 1}
    ms_total = max_over_ranks(e0.elapsed_time(e1), world)
    ms_per_step = ms_total / args.steps
    value = job_rate(args.steps, world, ms_total)
    clocks = clk.summary()

    # ---- the same warm solve captured once into a CUDA graph and replayed -
    graph_replay = None
    if not args.no_graph:
        gbuf = rhos[1].clone()
        gpot = torch.empty_like(d_pot)
        cap = torch.cuda.Stream()
        graph = torch.cuda.CUDAGraph()
        torch.cuda.synchronize()
        with torch.cuda.graph(graph, stream=cap):
            solver.set_stream(torch.cuda.current_stream())
            solver.potential_solver_device(gbuf, gpot, tstep)
        solver.set_stream(stream)
        for _ in range(5):
            graph.replay()
        ga, gb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        nrep = max(50, args.steps // 2)
        torch.cuda.synchronize()
        ga.record(stream)
        for _ in range(nrep):
            graph.replay()
        gb.record(stream)
        torch.cuda.synchronize()
        gms = ga.elapsed_time(gb) / nrep
        graph_replay = {"solves_per_s": 1e3 / gms, "ms_per_solve": gms, "replays": nrep}
        del graph
        solver.synchronize()

    # ---- the same solve with the GPU split into two SM partitions --------
    # (green contexts: the contraction on one, the free-slot ADI on the other)
    green = None
    if rank == 0 and not args.no_green:
        green = []
        # the serialised schedule (no side stream) first, then SM partitions
        configs = [("serial", {"BPH_OVERLAP": "0"}), ("fft_dense", {"BPH_FFT_DENSE": "1"}),
                   ("serial+fft_dense", {"BPH_OVERLAP": "0", "BPH_FFT_DENSE": "1"})] + [
            (int(x), {"BPH_GREEN": "1", "BPH_GREEN_SMS": x}) for x in args.green_sms.split(",") if x]
        for sms, env in configs:
            os.environ.update(env)
            try:
                gs = B.PotentialSolver(**GRID)
            finally:
                for k in env:
                    os.environ.pop(k, None)
            gs.set_stream(stream)
            got = gs.info()["green_sms"]
            gp = torch.empty_like(d_pot)
            gs.potential_solver_device(rhos[0], gp, 0)
            for w in range(3):
                gs.potential_solver_device(rhos[(1 + w) % nrot], gp, 2 + w)
            ga, gb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            nrep = max(50, min(args.steps, 500))
            torch.cuda.synchronize()
            ga.record(stream)
            for i in range(nrep):
                gs.potential_solver_device(rhos[(4 + i) % nrot], gp, 5 + i)
            gb.record(stream)
            torch.cuda.synchronize()
            gms = ga.elapsed_time(gb) / nrep
            green.append({"requested_sms": sms, "contraction_sms": got, "solves_per_s": 1e3 / gms,
                          "ms_per_solve": gms})
            gs.close()
            del gp

    # ---- per-phase kernel times (CUDA events on the launch stream) ------
    def time_phase(phase, reps, **kw):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(3):
            solver.run_phase(phase, **kw)
        a.record(stream)
        for _ in range(reps):
            solver.run_phase(phase, **kw)
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    phases = {
        "fft_fwd_rho": time_phase(B.solver.PHASE_FFT_RHO, 50, d_rho=rhos[0]),
        "green_contract": time_phase(B.solver.PHASE_CONTRACT, 50),
        "boundary_slots_standalone": time_phase(B.solver.PHASE_SLOTS, 50),
        "adi_5steps": time_phase(B.solver.PHASE_ADI, 50, nsteps=5),
        "fft_inv": time_phase(B.solver.PHASE_FFT_INV, 50, d_pot=d_pot),
    }
    solver.synchronize()
    peak, peak_kind = hbm_peak()
    compact = solver.info()["contract_kind"] == B.solver.CONTRACT_COMPACT
    contract_kernel = "k_green_compact" if compact else "k_green_contract"
    if compact:
        cb = compact_contract_bytes(numr, numz, GRID["mmax"], GRID["isym"])
    else:
        cb = contract_bytes(numr, numz, GRID["mmax"], GRID["isym"])
    achieved = cb / (phases["green_contract"] / 1e3) / 1e9
    traffic = committed_traffic(contract_kernel)
    # compulsory bytes of the solve as the reference forms it (full tables) and as run
    b_alg_full = compulsory_bytes(numr, numz, numphi, GRID["mmax"], GRID["isym"], warm=True)
    b_alg = b_alg_full
    if compact:
        nr_, nz_ = numr - 2, numz - 2
        rows = nr_ + nz_ + (nr_ if GRID["isym"] == 1 else 0)
        b_alg = b_alg_full - 8 * nr_ * nz_ * rows * GRID["mmax"] + compact_table_bytes(
            numr, numz, GRID["mmax"], GRID["isym"])
    solve_gbs = b_alg / (ms_per_step / 1e3) / 1e9

    # ---- e2e: host-array C ABI call with pinned buffers ----------------
    n_e2e = min(args.steps, args.e2e_steps)
    npin = min(nrot, n_e2e)
    h_rho = [torch.empty(ntot, dtype=torch.float64, pin_memory=True) for _ in range(npin)]
    for i in range(npin):
        h_rho[i].copy_(rhos[(1 + i) % nrot])
    h_pot = torch.empty(ntot, dtype=torch.float64, pin_memory=True)
    rho_np = [t.numpy() for t in h_rho]
    pot_np = h_pot.numpy()
    lib = B.load_library()
    import ctypes

    for i in range(3):
        rc = lib.bph_potential_solver(solver._h, ctypes.c_void_p(rho_np[i % npin].ctypes.data),
                                      ctypes.c_void_p(pot_np.ctypes.data), tstep)
        tstep += 1
        assert rc == 0, lib.bph_last_error()
    barrier(world)
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_lat = []
    e2.record(stream)
    for i in range(n_e2e):
        t0 = time.perf_counter()
        rc = lib.bph_potential_solver(solver._h, ctypes.c_void_p(rho_np[i % npin].ctypes.data),
                                      ctypes.c_void_p(pot_np.ctypes.data), tstep)
        e2e_lat.append(time.perf_counter() - t0)
        tstep += 1
        if rc != 0:
            raise RuntimeError(lib.bph_last_error().decode())
    e3.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms_e2e = max_over_ranks(e2.elapsed_time(e3), world)
    e2e_value = job_rate(n_e2e, world, ms_e2e)

    # ---- e2e on pageable host arrays, then the same arrays registered ----
    # (a Fortran caller passes its COMMON arrays: pageable unless the shim
    # registers them, which it does once in potsetup)
    def host_rate(rho_list, pot_arr, n):
        nonlocal tstep
        lat = []
        for i in range(3):
            rc = lib.bph_potential_solver(solver._h, ctypes.c_void_p(rho_list[i % len(rho_list)].ctypes.data),
                                          ctypes.c_void_p(pot_arr.ctypes.data), tstep)
            tstep += 1
            assert rc == 0, lib.bph_last_error()
        barrier(world)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for i in range(n):
            t0 = time.perf_counter()
            rc = lib.bph_potential_solver(solver._h, ctypes.c_void_p(rho_list[i % len(rho_list)].ctypes.data),
                                          ctypes.c_void_p(pot_arr.ctypes.data), tstep)
            lat.append(time.perf_counter() - t0)
            tstep += 1
            if rc != 0:
                raise RuntimeError(lib.bph_last_error().decode())
        b.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ms = max_over_ranks(a.elapsed_time(b), world)
        return {"value": job_rate(n, world, ms), "unit": "solves/s",
                "p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99))}

    n_pg = min(n_e2e, args.e2e_pageable_steps)
    rho_pg = [np.array(rho_np[i % npin]) for i in range(min(npin, 4))]  # plain (pageable) numpy copies
    pot_pg = np.empty(ntot)
    e2e_pageable = host_rate(rho_pg, pot_pg, n_pg)
    for arr in rho_pg + [pot_pg]:
        B.register_host(arr)
    e2e_registered = host_rate(rho_pg, pot_pg, n_pg)
    for arr in rho_pg + [pot_pg]:
        B.unregister_host(arr)
    del rho_pg, pot_pg

    # ---- parity with the oracle and the CPU baseline (rank 0) ----------
    parity, cpu = None, None
    if rank == 0 and not args.no_parity:
        parity, cpu = oracle_section(B, solver, base, last, args, want_cpu=(world == 1 and not args.no_cpu_baseline))

    # The sections below are reported by rank 0 only; with several ranks the
    # others skip them (no collective follows, and the host is not shared by
    # eight copies of the serving loops).
    side = rank == 0

    # ---- batched solves: n instances per call, one table pass ----------
    batched = None
    if side and args.batch_sizes:
        batched = {}
        for nb_ in [int(x) for x in args.batch_sizes.split(",") if x]:
            bt = B.Batch(solver, nb_)
            ins = [rhos[(7 * i) % nrot] for i in range(nb_)]
            outs = [torch.empty(ntot, dtype=torch.float64, device=dev) for _ in range(nb_)]
            bt.solve_device(ins, outs, 0)
            for w in range(3):
                bt.solve_device(ins, outs, 2 + w)
            calls = max(3, args.batch_calls)
            ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            ea.record(stream)
            for k in range(calls):
                ins = [rhos[(7 * i + k + 1) % nrot] for i in range(nb_)]
                bt.solve_device(ins, outs, 5 + k)
            eb.record(stream)
            torch.cuda.synchronize()
            ms = ea.elapsed_time(eb)
            batched[str(nb_)] = {"solves_per_s": nb_ * calls / (ms / 1e3), "ms_per_call": ms / calls}
            del outs
            bt.close()

    # ---- mixed precision on the large grid and the small field --------
    large_grid = None
    if side and not args.no_large_grid:
        large_grid = large_grid_bench(B, torch, dev, args, stream)

    # ---- converged batched solves: FP64 vs mixed ------------------------
    batched_conv = None
    if side and args.batch_sizes and args.converged_steps > 0:
        nb_ = max(int(x) for x in args.batch_sizes.split(",") if x)
        ins = [rhos[(7 * i) % nrot] for i in range(nb_)]
        batched_conv = {"instances": nb_, "nsteps_per_cycle": args.conv_nsteps, "tol_update": args.conv_tol}

        def measure(ns, mixed):
            bt = B.Batch(solver, nb_)
            outs = [torch.empty(ntot, dtype=torch.float64, device=dev) for _ in range(nb_)]
            bt.solve_converged_device(ins, outs, ns, True, 1e-13, 100, mixed)
            ts, cyc = [], []
            for k in range(4):
                ins_k = [rhos[(7 * i + k + 1) % nrot] for i in range(nb_)]
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                info = bt.solve_converged_device(ins_k, outs, ns, False, args.conv_tol, 100, mixed)
                torch.cuda.synchronize()
                ts.append(time.perf_counter() - t0)
                cyc.append(info.cycles)
            bt.close()
            return ({"solves_per_s": nb_ / float(np.median(ts)), "ms_per_call": 1e3 * float(np.median(ts)),
                     "mean_cycles": float(np.mean(cyc))}, outs)

        def err_vs(outs, ref):
            return max(float(torch.linalg.norm(a - b) / torch.linalg.norm(b)) for a, b in zip(outs, ref))

        r64, ref_outs = measure(args.conv_nsteps, False)
        batched_conv["fp64"] = r64
        rmx, outs = measure(args.conv_nsteps, True)
        rmx["max_rel_err_vs_fp64"] = err_vs(outs, ref_outs)
        kind_names = {B.solver.MIXED_ADI_FORWARD: "adi_forward", B.solver.MIXED_ADI_INCREMENT: "adi_increment",
                      B.solver.MIXED_ADI_GLOBAL: "adi_global", B.solver.MIXED_ADI_WARP: "adi_warp",
                      B.solver.MIXED_DIRECT: "direct"}
        tuned = solver.info()["mixed_kind"]
        rmx["inner_solver"] = kind_names.get(tuned, str(tuned))
        batched_conv["mixed"] = rmx
        batched_conv["speedup_mixed_vs_fp64"] = rmx["solves_per_s"] / r64["solves_per_s"]
        # beside it, the ratio against the plain form: the batched 5-step drop-in of the same
        # batch size (a converged solve does more work than a 5-step one)
        if batched and str(nb_) in batched:
            plain = batched[str(nb_)]["solves_per_s"]
            batched_conv["vs_plain_form"] = {"plain_solves_per_s": plain,
                                             "mixed_over_plain": rmx["solves_per_s"] / plain}
        # the mixed form with its fastest FP32 ADI inner solver as well (the precision's share
        # of the speed-up, without the direct solve)
        if tuned == B.solver.MIXED_DIRECT:
            info0 = solver.info()
            adi_kinds = [(info0["mixed_warp_ns"], B.solver.MIXED_ADI_WARP),
                         (info0["mixed_forward_ns"], B.solver.MIXED_ADI_FORWARD),
                         (info0["mixed_increment_ns"], B.solver.MIXED_ADI_INCREMENT)]
            adi_kinds = [k for k in adi_kinds if k[0] > 0]
            if adi_kinds:
                solver.set_mixed_adi(min(adi_kinds)[1])
                radi, outs2 = measure(args.conv_nsteps, True)
                radi["max_rel_err_vs_fp64"] = err_vs(outs2, ref_outs)
                radi["inner_solver"] = kind_names[min(adi_kinds)[1]]
                batched_conv["mixed_adi"] = radi
                batched_conv["speedup_mixed_adi_vs_fp64"] = radi["solves_per_s"] / r64["solves_per_s"]
                del outs2
                solver.set_mixed_adi(tuned)
        # each form at its own best cycle length (the converged answer does not depend on it)
        sweep = sorted(set(int(x) for x in args.conv_nsteps_sweep.split(",") if x))
        if sweep:
            table = {"fp64": {}, "mixed": {}}
            for ns in sweep:
                for key, mixed in (("fp64", False), ("mixed", True)):
                    if ns == args.conv_nsteps:
                        table[key][str(ns)] = batched_conv[key]
                        continue
                    r, outs = measure(ns, mixed)
                    r["max_rel_err_vs_fp64"] = err_vs(outs, ref_outs)
                    table[key][str(ns)] = r
                    del outs
            best = {k: max(v.items(), key=lambda kv: kv[1]["solves_per_s"]) for k, v in table.items()}
            batched_conv["nsteps_sweep"] = table
            batched_conv["best"] = {k: {"nsteps_per_cycle": int(ns), **r} for k, (ns, r) in best.items()}
            batched_conv["speedup_mixed_vs_fp64_best"] = (best["mixed"][1]["solves_per_s"] /
                                                          best["fp64"][1]["solves_per_s"])
        del ref_outs

    # ---- batches over a mix of grids, one plan launch ------------------
    mixed_grid = None
    if side and args.mixed_grid_instances > 0:
        mixed_grid = mixed_grid_bench(B, torch, dev, args, stream)

    # ---- serving: Poisson arrivals of SCF-like client requests ----------
    serving = None
    if side and args.serve_rates and not args.no_serving:
        serving = serve_bench(B, torch, dev, rhos, args)

    serving_mixed = None
    if side and args.serve_mixed_rates and not args.no_serving:
        serving_mixed = serve_mixed_bench(B, torch, dev, args)

    # ---- converged solves: FP64 vs mixed (FP32 ADI + FP64 refinement) --
    conv = None
    if side and args.converged_steps > 0:
        conv = {}
        nconv = args.converged_steps
        ref_pots = []
        tuned_kind = solver.info()["mixed_kind"]
        variants = [("fp64", None), ("mixed_forward", B.solver.MIXED_ADI_FORWARD),
                    ("mixed_increment", B.solver.MIXED_ADI_INCREMENT)]
        if solver.info()["mixed_warp_ns"] > 0:
            variants.append(("mixed_warp", B.solver.MIXED_ADI_WARP))
        if solver.info()["mixed_direct_ns"] > 0:
            variants.append(("mixed_direct", B.solver.MIXED_DIRECT))
        for key, kind in variants:
            if kind is not None:
                solver.set_mixed_adi(kind)
            # every form starts from the same converged potential of rhos[0]
            solver.solve_converged_device(rhos[0], d_pot, args.conv_nsteps, True, 1e-13, 100, False)
            clat, cycles, pots = [], [], []
            for i in range(nconv):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                info = solver.solve_converged_device(rhos[(1 + i) % nrot], d_pot, args.conv_nsteps, False,
                                                     args.conv_tol, 100, kind is not None)
                torch.cuda.synchronize()
                clat.append(time.perf_counter() - t0)
                cycles.append(info.cycles)
                pots.append(d_pot.clone())
            err = None
            if kind is None:
                ref_pots = pots
            else:
                err = max(float(torch.linalg.norm(a - b) / torch.linalg.norm(b)) for a, b in zip(pots, ref_pots))
            conv[key] = {"solves_per_s": nconv / sum(clat), "p50_ms": 1e3 * float(np.percentile(clat, 50)),
                         "p99_ms": 1e3 * float(np.percentile(clat, 99)), "mean_cycles": float(np.mean(cycles)),
                         "max_rel_err_vs_fp64": err}
            if kind is not None:
                del pots
        solver.set_mixed_adi(tuned_kind)
        conv["nsteps_per_cycle"] = args.conv_nsteps
        conv["tol_update"] = args.conv_tol
        names = {B.solver.MIXED_ADI_FORWARD: "mixed_forward", B.solver.MIXED_ADI_INCREMENT: "mixed_increment",
                 B.solver.MIXED_ADI_WARP: "mixed_warp", B.solver.MIXED_DIRECT: "mixed_direct"}
        conv["autotuned_kind"] = names.get(tuned_kind, str(tuned_kind))
        best = max(conv[k]["solves_per_s"] for k, kind in variants if kind is not None)
        conv["speedup_mixed_vs_fp64"] = best / conv["fp64"]["solves_per_s"]
        del ref_pots

    solver_info = solver.info()
    solver.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "130x98x256 warm time-step solves, bipolytrope pair rotated 1 zone/solve",
                       **GRID, "nsteps_adi": 5},
            "parallelism": f"independent sequence per GPU x{world}",
            "l2": "per-solve working set (212 MB compact Green tables, 660 MB full) > 126 MB L2, no flush needed",
            "zone_updates_per_s": value * ntot * 5,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": 8 * ntot,
                    "d2h_bytes_per_step": 8 * ntot, "host_memory": "pinned (torch pin_memory)",
                    "p50_ms": 1e3 * float(np.percentile(e2e_lat, 50)),
                    "p99_ms": 1e3 * float(np.percentile(e2e_lat, 99)),
                    "pageable": e2e_pageable, "registered": e2e_registered,
                    "pageable_vs_pinned": e2e_pageable["value"] / e2e_value,
                    "registered_vs_pinned": e2e_registered["value"] / e2e_value},
            "parity": parity,
            "parity_rel_l2": parity["last_timed_rel_l2"] if parity else None,
            "roofline": {"bound": "hbm", "kernel": contract_kernel, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "alg_bytes_per_launch": cb,
                         "solve_alg_bytes": b_alg, "solve_gbs": solve_gbs, "solve_frac": solve_gbs / peak,
                         "solve_alg_bytes_full_tables": b_alg_full,
                         "solve_frac_full_tables": b_alg_full / (ms_per_step / 1e3) / 1e9 / peak},
            "phase_ms": phases,
            "converged": conv,
            "batched": batched,
            "batched_converged": batched_conv,
            "mixed_grid_batches": mixed_grid,
            "large_grid": large_grid,
            "serving": serving,
            "serving_mixed_grids": serving_mixed,
            "graph_replay": graph_replay,
            "sm_partitions": green,
            "launch_config": solver_info,
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=500)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle parity section")
    ap.add_argument("--e2e-pageable-steps", type=int, default=100,
                    help="host-array solves timed on pageable and on registered arrays")
    ap.add_argument("--reference-budget-s", type=float, default=150.0)
    ap.add_argument("--batch-sizes", default="4,16", help="batched warm solves timed per batch size (empty skips)")
    ap.add_argument("--batch-calls", type=int, default=20)
    ap.add_argument("--mixed-grid-instances", type=int, default=96,
                    help="instances of the mixed-grid plan section (0 skips)")
    ap.add_argument("--mixed-grid-calls", type=int, default=10)
    ap.add_argument("--no-large-grid", action="store_true",
                    help="skip the 258x194x512 / 66x66x64 mixed-vs-FP64 section")
    ap.add_argument("--serve-rates", default="200,1000,4000",
                    help="offered request rates (req/s) of the serving section (empty skips)")
    ap.add_argument("--serve-clients", type=int, default=64)
    ap.add_argument("--serve-conv-rates", default="300,1500",
                    help="offered rates of converged serving, FP64 and mixed (empty skips)")
    ap.add_argument("--serve-mixed-rates", default="100,400,1600",
                    help="offered rates of the mixed-grid serving section (empty skips)")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving section")
    ap.add_argument("--no-graph", action="store_true", help="skip the CUDA-graph replay section")
    ap.add_argument("--no-green", action="store_true", help="skip the SM-partition section")
    ap.add_argument("--green-sms", default="48,64,80,96",
                    help="contraction SMs of the SM-partition section (green contexts)")
    ap.add_argument("--serve-iters", type=int, default=8, help="SCF-like requests per client per rate")
    ap.add_argument("--converged-steps", type=int, default=20,
                    help="warm converged solves timed per form (FP64 and mixed); 0 skips")
    ap.add_argument("--conv-nsteps", type=int, default=10, help="ADI steps per refinement cycle")
    ap.add_argument("--conv-tol", type=float, default=1e-11, help="stop when |dphi|/|phi| <= tol")
    ap.add_argument("--conv-nsteps-sweep", default="6,8,10,14",
                    help="cycle lengths of the batched converged sweep (each form at its best; empty skips)")
    ap.add_argument("--rotations", type=int, default=0,
                    help="resident density rotations (0: numphi); small values make a small profiling case")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        # The CPU reference arm uses no GPU and no collective: rank 0 runs it.
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup()
    try:
        run_gpu(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
