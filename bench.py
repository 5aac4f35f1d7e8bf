#!/usr/bin/env python
"""Sector-solve throughput of the symmetry-resolved ED path on B200.

Workload (default ``checkerboard24``): spinless fermions on the 3x4x2
checkerboard (24 sites, 4 particles, 10,626 states, 892 orbits), translation
group of order 12; one step = all 12 momentum sectors, lowest 6 eigenvalues
each, solved in one batched block-Lanczos (FP32 matvec, FP64 recurrence and
reorthogonalisation, FP64 refinement) to |dE| < 1e-10 against the CPU oracle.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One JSON line on rank 0.  N > 1 runs independent replicas (one per GPU, no
collective in the data path); ``value`` is the total over all ranks divided
by the slowest rank's time.  ``--impl reference`` times the CPU restatement
of the reference's numpy/ARPACK path on the host cores instead.
"""

from __future__ import annotations

import os

_NCPU = os.cpu_count() or 1
for _v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
    os.environ.setdefault(_v, str(_NCPU))

import argparse  # noqa: E402
import json  # noqa: E402
import statistics  # noqa: E402
import subprocess  # noqa: E402
import sys  # noqa: E402
import threading  # noqa: E402
import time  # noqa: E402
from fractions import Fraction  # noqa: E402

import numpy as np  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "checkerboard24": dict(nev=6, desc="checkerboard 3x4x2, 24 sites, 4 fermions, |G|=12, 12 sectors"),
    "heisenberg16": dict(nev=4, desc="Heisenberg ring N=16, 8 up spins, |G|=16, 16 sectors"),
}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x: float, ws: int, device="cuda") -> float:
    """The slowest rank's value of ``x`` (all-reduce MAX over the default
    process group); ``x`` itself with one rank."""
    if ws <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(ws: int, units_per_rank: int, t_max: float) -> float:
    """Whole-job throughput of ``ws`` independent replicas, each doing
    ``units_per_rank`` units: all units over the slowest rank's time."""
    return ws * units_per_rank / t_max


# ---------------------------------------------------------------------------
# CPU side: the oracle (restatement of the reference's numpy/scipy path)
# ---------------------------------------------------------------------------


def cpu_sector_solves(model, n_filled, G, irreps, nev, budget_s=20.0, min_sectors=3, cat=None):
    """Time the reference algorithm (projection table + CSR + ARPACK per
    sector, catalog built outside the timing as in the reference benchmark)
    on a bounded sample of sectors; returns (solves/s, n_timed, eigvals)."""
    from oracle import port

    n = G.n_site
    fermion = model.particle_statistics.name == "FERMIONIC"
    if cat is None:
        perm0, eta = port.group_arrays(G)
        cat = port.catalog(n, n_filled, perm0, eta, fermion)
    # sectors in order, cycling through the workload again until the budget
    # is spent (a bounded sample of about budget_s seconds of host work)
    t_all, done, vals = 0.0, 0, {}
    s = 0
    while t_all < budget_s or done < min_sectors:
        chi = np.asarray(irreps[s].values, dtype=np.complex128)
        t0 = time.perf_counter()
        orbits = port.sector_orbits(cat, chi)
        H = port.csr_block(cat, n, orbits, model.bilinear_terms, model.density_density_terms, chi, fermion)
        w, _ = port.solve(H, nev)
        t_all += time.perf_counter() - t0
        vals[s] = w
        done += 1
        s = (s + 1) % len(irreps)
    return done / t_all, done, vals, t_all


def oracle_eigs(model, n_filled, G, irreps, nev):
    from oracle import port

    fermion = model.particle_statistics.name == "FERMIONIC"
    perm0, eta = port.group_arrays(G)
    cat = port.catalog(G.n_site, n_filled, perm0, eta, fermion)
    out = {}
    for s, ir in enumerate(irreps):
        chi = np.asarray(ir.values, dtype=np.complex128)
        orbits = port.sector_orbits(cat, chi)
        H = port.csr_block(cat, G.n_site, orbits, model.bilinear_terms, model.density_density_terms, chi,
                           fermion)
        out[s] = port.solve(H, nev)[0]
    return out


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    from realspace_exatdiagonalization_py_b200 import models
    import realspace_exatdiagonalization_py_b200.symmetry as sym

    wl = WORKLOADS[args.workload]
    model, nf = models.config_model(args.workload)
    G = sym.build_translation_group(model.lattice)
    irreps = sym.build_irrep_list(G, model.lattice)
    from oracle import port

    perm0, eta = port.group_arrays(G)
    cat = port.catalog(G.n_site, nf, perm0, eta, model.particle_statistics.name == "FERMIONIC")
    per_step = []
    for it in range(args.warmup + args.steps):
        rate, n_done, _, t = cpu_sector_solves(model, nf, G, irreps, wl["nev"], budget_s=4.0, min_sectors=2,
                                               cat=cat)
        if it >= args.warmup:
            per_step.append((n_done, t))
    tot_n = sum(n for n, _ in per_step)
    tot_t = sum(t for _, t in per_step)
    val = tot_n / tot_t
    line = {
        "impl": "reference",
        "metric": "sector-solves/s",
        "value": val,
        "unit": "sector-solves/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * tot_t / len(per_step),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "desc": wl["desc"], "nev": wl["nev"],
                   "step": "bounded sample of sectors: projection table + CSR + ARPACK eigs(which=SR)"},
        "cpu_baseline": {"value": val, "unit": "sector-solves/s", "cores": _NCPU, "kind": "port",
                         "sample": f"{tot_n} sector solves over {args.steps} steps (catalog built once, untimed)"},
        "e2e": {"value": val, "unit": "sector-solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 7:
                continue
            try:
                sm.append(float(p[0]))
                mx = float(p[1])
            except ValueError:
                continue
            for n, v in zip(names, p[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def sector_matvec_bytes(dm, sset, col_sector, x_bytes):
    """Algorithmic bytes of one apply over the given columns: per column
    (one sector matvec) D_s * (8 + 2 s) + H_s * 16 -- the representative
    mask, x read and y write per row and one 16-B table entry per hop of the
    sector's rows.  H_s comes from the projection table's row lengths."""
    import torch

    rp = dm.proj["rowptr"]
    hops_row = (rp[1:] - rp[:-1]).to(torch.float64)
    mem = sset.member
    total = 0.0
    for s in col_sector.tolist():
        on = ((mem >> int(s)) & 1).to(torch.bool)
        d = int(on.sum().item())
        h = float(hops_row[on].sum().item())
        total += d * (8 + 2 * x_bytes) + h * 16
    return total


def _zero_outside(X, sset, col_sector):
    import torch

    for c, s in enumerate(col_sector.tolist()):
        X[((sset.member >> int(s)) & 1) == 0, c] = 0
    X[:, len(col_sector):] = 0
    return X


def time_apply(dm, sset, cs, X, Y, prec, variant, n_launch, warm=3):
    """Average time of one apply (CUDA events on the current stream)."""
    import torch

    for _ in range(warm):
        dm.apply_block(sset, cs, X, Y, precision=prec, variant=variant)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(n_launch):
        dm.apply_block(sset, cs, X, Y, precision=prec, variant=variant)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / n_launch * 1e-3


def apply_roofline(ed, data, sset, solver, peak_gbs, n_launch=200):
    """The batch's FP32 matvec (all columns of the bench workload) timed with
    CUDA events, against the per-sector-matvec algorithmic bytes."""
    import torch

    dm, _ = data._device()
    b = solver.batch
    n_orb = data.orbit_catalog.n_orbits
    X = _zero_outside(torch.randn((n_orb, b.ld), dtype=torch.complex64, device="cuda"), sset, b.col_sector)
    Y = torch.empty((n_orb, b.ld), dtype=torch.complex128, device="cuda")
    t = time_apply(dm, sset, b.col_sector, X, Y, 32, 0, n_launch, warm=5)
    alg = sector_matvec_bytes(dm, sset, b.col_sector, 8)
    ach = alg / t / 1e9
    return {"kernel": "k_proj_spmv<32,*> (rsed_apply_h, projection table)", "bound": "hbm",
            "achieved": ach, "peak": peak_gbs, "unit": "GB/s", "frac": ach / peak_gbs, "traffic": None,
            "alg_bytes_per_launch": alg, "avg_launch_us": t * 1e6, "hops_per_launch": dm.proj["n_hops"],
            "columns": b.n_cols, "note": "latency-bound size (892 orbits): see matvec_at_scale"}


def matvec_at_scale(ed, models, peak_gbs, n_launch=20, precisions=(32, 64), per_sector=4, otf=True):
    """The HBM-bound matvec at the 32-site Haldane size (10.5M states, 657,756
    orbits, table 168 MB > L2): 16 sectors x 4 block columns, the shape of one
    batched Lanczos step, through the projection table (and, for comparison,
    the on-the-fly apply)."""
    import torch

    model, nf = models.config_model("haldane32")
    G = ed.build_translation_group(model.lattice)
    t0 = time.perf_counter()
    data = ed.build_ed_data(model, filling_fraction=Fraction(nf, model.lattice.n_site), symmetry_group=G)
    torch.cuda.synchronize()
    t_cat = time.perf_counter() - t0
    dm, sset = data._device()
    t0 = time.perf_counter()
    dm.build_projection(sset.sqrt_stab, precisions=precisions)
    torch.cuda.synchronize()
    t_proj = time.perf_counter() - t0
    n_orb = data.orbit_catalog.n_orbits
    ns = len(data.irrep_list)
    ncol = per_sector * ns
    ld = ncol + (ncol & 1)
    cs = torch.arange(ns, dtype=torch.int32, device="cuda").repeat_interleave(per_sector)
    nh = dm.proj["n_hops"]
    out = {"workload": f"haldane32: 32 sites, 8 bosons, C=10,518,300, |G|=16, {ns} sectors x {per_sector} columns",
           "n_orbits": n_orb, "hops_per_apply": nh, "catalog_build_s": t_cat, "projection_build_s": t_proj,
           "projection_bytes": dm.projection_bytes(), "l2": "x > L2 for every precision (no flush needed)"}
    for prec in precisions:
        dt, xb = (torch.complex128, 16) if prec == 64 else (torch.complex64, 8)
        X = _zero_outside(torch.randn((n_orb, ld), dtype=dt, device="cuda"), sset, cs)
        Y = torch.empty((n_orb, ld), dtype=torch.complex128, device="cuda")
        t = time_apply(dm, sset, cs, X, Y, prec, 0, n_launch)
        alg = sector_matvec_bytes(dm, sset, cs, xb)
        wb = 16 if prec == 64 else 8
        uniq = nh * (4 + wb) + n_orb * (8 + 8 + 16) + n_orb * ncol * (xb + 16)
        gathered = nh * ncol * xb
        r = {"avg_apply_ms": t * 1e3, "alg_bytes": alg, "alg_GBs": alg / t / 1e9,
             "frac_of_measured_hbm": alg / t / 1e9 / peak_gbs,
             "unique_bytes": uniq, "unique_GBs": uniq / t / 1e9,
             "gathered_x_bytes": gathered, "gathered_x_GBs": gathered / t / 1e9}
        if otf:
            proj = dm.proj
            dm.proj = None
            dm.refresh()
            t_otf = time_apply(dm, sset, cs, X, Y, prec, 0, max(3, n_launch // 4))
            dm.proj = proj
            dm.refresh()
            r["on_the_fly_apply_ms"] = t_otf * 1e3
        out[f"fp{prec}"] = r
        del X, Y
    return out


def serving_at_scale(ed, models, n_req=32, rate=20.0, block=2, plain_samples=2):
    """The request loop at the 32-site Haldane size: a Poisson stream (seed 0)
    of (sector, flux) requests over a 16 x 16 flux grid and 16 sectors,
    served with continuous batching (FP32 matvec + FP64 refinement, nev 4),
    against the plain FP64 path (one request at a time, block 1, no graph,
    host polling every iteration) on the first requests of the stream."""
    import torch
    from realspace_exatdiagonalization_py_b200.serving import poisson_requests

    model, nf = models.config_model("haldane32")
    sm = ed.ServingModel(model, nf, name="haldane32")
    reqs = poisson_requests(n_req, rate=rate, n_sectors=sm.n_sectors, flux_grid=16, model="haldane32", seed=0)
    srv = ed.SolveServer(sm, nev=4, precision=32, block=block, poll=16)
    srv.warm(48)  # start-up: lane buffers and captured graphs, before the stream begins
    res = srv.run([ed.SolveRequest(r.rid, r.sector, r.flux, r.model, r.arrival) for r in reqs], realtime=True)
    summ = ed.latency_summary(res)
    by_id = {r.rid: r for r in res}
    # capacity: the same requests submitted at once (the Poisson stream above
    # cannot finish faster than its own arrivals, ~n_req / rate seconds)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    burst = srv.run([ed.SolveRequest(1000 + r.rid, r.sector, r.flux, r.model) for r in reqs], realtime=False)
    torch.cuda.synchronize()
    cap_s = time.perf_counter() - t0
    cap_dE = max(float(np.max(np.abs(b.eigenvalues - by_id[b.rid - 1000].eigenvalues))) for b in burst)
    out = {"workload": f"haldane32 requests: {n_req} Poisson arrivals at {rate}/s (seed 0), uniform sector of "
                       f"{sm.n_sectors}, uniform flux on 16x16, nev 4", **summ,
           "block": block, "peak_concurrent_lanes": srv.peak_running, "flux_contexts": len(srv.contexts),
           "device_GB_in_use": srv.used_bytes() / 1e9,
           "fp32_error_before_refinement_max": float(max(r.fp32_error.max() for r in res)),
           "iterations": [min(r.iterations for r in res), max(r.iterations for r in res)],
           "capacity": {"requests": len(burst), "makespan_s": cap_s, "throughput_per_s": len(burst) / cap_s,
                        "max_abs_dE_vs_stream": cap_dE,
                        "note": "all requests submitted at once, flux contexts already warm from the stream"}}
    del srv
    torch.cuda.empty_cache()
    # plain FP64 path on the first requests
    plain_t, dE = [], []
    for r in reqs[:plain_samples]:
        ctx = ed.FluxContext(sm, sm.normalize_flux(r.flux), 64)
        p = ed.LanczosParams(block=1, n_slots=48, precision=64, check_every=1)
        b = ed.LanczosBatch(ctx.dm, ctx.sset, [r.sector], 4, p)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.load_start(None)
        b.start()
        b.run(poll=1, graph=False)
        torch.cuda.synchronize()
        plain_t.append(time.perf_counter() - t0)
        dE.append(float(np.max(np.abs(b.eigenvalues()[0] - by_id[r.rid].eigenvalues))))
        del b, ctx
        torch.cuda.empty_cache()
    plain_rate = len(plain_t) / sum(plain_t)
    out.update({"plain_fp64_solves_per_s": plain_rate, "plain_fp64_s_per_solve": plain_t,
                "served_over_plain": summ["throughput_per_s"] / plain_rate,
                "served_capacity_over_plain": out["capacity"]["throughput_per_s"] / plain_rate,
                "max_abs_dE_served_vs_plain_fp64": max(dE)})
    return out


def _laughlin_manifold(ed, model, nf, n=2):
    """The ``n`` lowest zero-flux states over all momentum sectors (the
    nu = 1/2 Laughlin pair), from one batched FP64 solve with two levels per
    sector, as ``(labels, nev_per_sector, energies)``: two sectors with one
    level each, or one sector with two."""
    G = ed.build_translation_group(model.lattice, [0.0, 0.0])
    data = ed.build_ed_data(model, filling_fraction=Fraction(nf, model.lattice.n_site), symmetry_group=G)
    res = ed.solve_sectors_batched(data, list(range(len(data.irrep_list))), nev=n, return_vectors=False)
    low = sorted((float(res[s][0][k]), s) for s in res for k in range(min(n, len(res[s][0]))))[:n]
    secs = sorted({s for _, s in low}, key=lambda s: min(e for e, t in low if t == s))
    per = n // len(secs) if n % len(secs) == 0 else 1
    if per * len(secs) != n:
        raise RuntimeError(f"lowest states {low} do not split evenly over their sectors")
    return [data.irrep_list[s].label for s in secs], per, [e for e, _ in low]


def _time_chern(ed, model, nf, labels, grid, nev=1, mode="matrixfree", engine="scan"):
    import shutil
    import tempfile

    import torch

    d = tempfile.mkdtemp(prefix="chern_")
    try:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = ed.many_body_chern_number(model, labels, filling_fraction=Fraction(nf, model.lattice.n_site),
                                      flux_grid_size=grid, nev_per_sector=nev, mode=mode, checkpoint_dir=d,
                                      engine=engine)
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0
    finally:
        shutil.rmtree(d, ignore_errors=True)


def chern_at_scale(ed, models, grid=4, peak_gbs=6650.0, cpu_grid=2, scan_grid=4):
    """The many-body Chern number of the two lowest zero-flux states of the
    32-site Haldane bosons on a grid x grid flux torus, end to end through
    ``many_body_chern_number`` with the served engine (every (flux point,
    sector) FP64 solve a request) and, on scan_grid x scan_grid, with the scan
    engine (the reference's route: flux point after flux point, checkpoints in
    a temporary directory); the overlap launch of one row of links timed alone
    against the HBM peak; and, like for like, the scan engine and the CPU
    oracle's restatement of the reference's driver on the 24-site model
    (cpu_grid x cpu_grid points)."""
    import warnings

    import torch

    from oracle import port

    model, nf = models.config_model("haldane32")
    labels, nev, e0 = _laughlin_manifold(ed, model, nf)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        _time_chern(ed, model, nf, labels, (2, 2), nev)  # warm-up: library, allocator, tuner cache
        _time_chern(ed, model, nf, labels, (2, 2), nev, engine="served")
        r, total = _time_chern(ed, model, nf, labels, (grid, grid), nev, engine="served")
        rs, ts = _time_chern(ed, model, nf, labels, (scan_grid, scan_grid), nev)
    C = int(model_basis_size(model, nf))
    n_m = len(labels) * nev
    out = {"workload": f"haldane32: 32 sites, 8 bosons, C={C:,}, sectors {labels} x {nev} level(s), "
                       f"{grid}x{grid} flux grid, FP64 solves",
           "chern_number": r.chern_number, "min_link_det": r.min_link_det, "zero_flux_E0": e0,
           "served": {"grid": [grid, grid], "total_s": total, "s_per_flux_point": total / (grid * grid)},
           "scan": {"grid": [scan_grid, scan_grid], "total_s": ts, "s_per_flux_point": ts / (scan_grid * scan_grid),
                    "chern_number": rs.chern_number}}
    out["overlap_row"] = overlap_row(ed, C, n_m, grid, peak_gbs)
    # like for like on the 24-site model: the device driver and the oracle
    m24, nf24 = models.config_model("haldane24")
    lab24, nev24, _ = _laughlin_manifold(ed, m24, nf24)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        r24, t24 = _time_chern(ed, m24, nf24, lab24, (cpu_grid, cpu_grid), nev24)
    def flux_setup(flux):
        ed.update_second_quantized_model_with_twisted_phases(m24, twisted_phases_over_2π=flux)
        G = ed.build_translation_group(m24.lattice, flux)
        return G, ed.build_irrep_list(G, m24.lattice)

    t0 = time.perf_counter()
    o24 = port.chern(m24, nf24, lab24, (cpu_grid, cpu_grid), nev24, flux_setup)
    tc = time.perf_counter() - t0
    npts = cpu_grid * cpu_grid
    out["haldane24_like_for_like"] = {
        "grid": [cpu_grid, cpu_grid], "sectors": lab24, "nev_per_sector": nev24,
        "device_scan_s_per_flux_point": t24 / npts,
        "oracle_s_per_flux_point": tc / npts, "device_chern": r24.chern_number, "oracle_chern": o24["chern_number"],
        "max_abs_curvature_diff": float(np.max(np.abs(r24.berry_curvature - o24["berry_curvature"]))),
        "oracle_threads": _NCPU, "oracle_kind": "port"}
    return out


def overlap_row(ed, C, n_m, grid, peak_gbs, reps=5):
    """One row of Chern links alone: ``rsed_fock_overlaps`` over the 2*grid
    slot pairs (x links to the next row, y links within the row) of random
    dense Fock states (complex128, ``2*grid`` slots of ``n_m`` states of ``C``
    amplitudes), CUDA-event time per call against the HBM peak.  Algorithmic
    bytes = every distinct slot once (2*grid * n_m * C * 16); each slot enters
    up to four pairs, and ``pair_bytes`` counts it once per pair."""
    import torch

    g = torch.Generator(device="cuda").manual_seed(0)
    states = torch.randn((2 * grid, n_m, C), dtype=torch.complex128, device="cuda", generator=g)
    pairs = [(iy, grid + iy) for iy in range(grid)] + [(iy, (iy + 1) % grid) for iy in range(grid)]
    for _ in range(3):
        ed.fock_overlaps(states, pairs)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    for _ in range(reps):
        ed.fock_overlaps(states, pairs)
    ev1.record()
    torch.cuda.synchronize()
    t = ev0.elapsed_time(ev1) / 1e3 / reps
    algo = len({x for pr in pairs for x in pr}) * n_m * C * 16
    del states
    torch.cuda.empty_cache()
    return {"pairs": len(pairs), "n_m": n_m, "n_states": C, "s": t, "algorithmic_bytes": algo,
            "pair_bytes": len(pairs) * 2 * n_m * C * 16, "achieved_GBs": algo / t / 1e9,
            "frac_of_measured_hbm": algo / t / 1e9 / peak_gbs}


def correlators_at_scale(ed, models):
    """The one-body density matrix and the density pairs of the lowest state
    of sector (0, 0) of the 32-site Haldane bosons (657,756 orbits, |G| = 16,
    8 bosons: 16 x 8 x 24 hops per orbit projected back into the sector), timed
    on the device with CUDA events; and, like for like on the 16-site model
    (sector (0, 1), lowest state), the device kernel against the CPU oracle's
    restatement of the reference's orbit-by-orbit loop."""
    import torch

    from oracle import port
    from realspace_exatdiagonalization_py_b200 import correlators as cr

    out = {}
    model, nf = models.config_model("haldane32")
    G = ed.build_translation_group(model.lattice, [0.0, 0.0])
    data = ed.build_ed_data(model, filling_fraction=Fraction(nf, model.lattice.n_site), symmetry_group=G)
    res = ed.solve_sectors_batched(data, [0], nev=1, precision=64)
    _, sset = data._device()
    basis = ed.Symmetry_Sector_Basis(data.irrep_list[0], data.orbit_catalog, sset, 0)
    c = res[0][1][:, 0]
    cr.one_body_density_matrix(basis, c)  # warm-up (occupancy query, allocator)
    cr.density_pairs(basis, c)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    torch.cuda.synchronize()
    ev[0].record()
    rho = cr.one_body_density_matrix(basis, c)
    ev[1].record()
    D = cr.density_pairs(basis, c)
    ev[2].record()
    torch.cuda.synchronize()
    n, k = model.lattice.n_site, nf
    hops = basis.dim * 16 * k * (n - k)
    out["haldane32"] = {"sector": [0, 0], "dim": basis.dim, "E0": float(res[0][0][0]),
                        "obdm_ms": ev[0].elapsed_time(ev[1]), "pairs_ms": ev[1].elapsed_time(ev[2]),
                        "hops_projected": hops, "trace_rho": float(np.trace(rho).real),
                        "sum_pairs_diag": float(np.trace(D))}
    # like for like: 16-site model, device vs oracle
    m16 = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[2, 4],
                                                                    params=models.params_DNSheng)
    G16 = ed.build_translation_group(m16.lattice, [0.0, 0.0])
    d16 = ed.build_ed_data(m16, filling_fraction=Fraction(4, 16), symmetry_group=G16)
    s = next(i for i, ir in enumerate(d16.irrep_list) if ir.label == (0, 1))
    r16 = ed.solve_sectors_batched(d16, [s], nev=1, precision=64)
    _, ss16 = d16._device()
    b16 = ed.Symmetry_Sector_Basis(d16.irrep_list[s], d16.orbit_catalog, ss16, s)
    c16 = r16[s][1][:, 0]
    cr.one_body_density_matrix(b16, c16)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rho16 = cr.one_body_density_matrix(b16, c16)
    t_dev = time.perf_counter() - t0
    perm0, eta = port.group_arrays(G16)
    cat = port.catalog(16, 4, perm0, eta, False)
    chi = np.asarray(d16.irrep_list[s].values, dtype=np.complex128)
    orbits = port.sector_orbits(cat, chi)
    t0 = time.perf_counter()
    rho_o = port.obdm_orbitwise(cat, orbits, np.asarray(c16), chi, perm0, eta, False, 16, 4)
    t_cpu = time.perf_counter() - t0
    out["haldane16_like_for_like"] = {"sector": [0, 1], "dim": b16.dim, "device_ms": t_dev * 1e3,
                                      "oracle_ms": t_cpu * 1e3, "oracle_threads": 1,
                                      "max_abs_diff": float(np.abs(rho16 - rho_o).max())}
    return out


def reference_benchmark(ed, models):
    """The reference's own headline benchmark, mirrored through the drop-in
    API: for every (model, size) its benchmark script lists, the orbit catalog
    is built outside the timed region and ``ed_scan_at_irrep_matrixfree`` of
    sector 0 with nev = 1 is timed (host clock around a synchronised call, as
    the reference times it); published times are the reference's matrix-free
    single-sector times on its 12-core CPU (benchmark_raw_latest_py.csv,
    committed as tests/golden/reference_benchmark.npz)."""
    import torch

    f = dict(np.load(os.path.join(ROOT, "tests", "golden", "reference_benchmark.npz")))

    def build(model, label, n_site):
        if model == "Heisenberg":
            return models.build_heisenberg_second_quantized_model(n_site, 1.0)
        ss = [int(x) for x in label.split("×")]
        if model == "Haldane_Boson":
            return models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=ss,
                                                                            params=models.params_DNSheng)
        return models.build_spinful_hubbard_second_quantized_model(ss, 1.0, 8.0)

    def data_for(i):
        m = build(str(f["model"][i]), str(f["label"][i]), int(f["n_site"][i]))
        G = ed.build_translation_group(m.lattice)
        return ed.build_ed_data(m, filling_fraction=Fraction(int(f["n_filled"][i]), int(f["n_site"][i])),
                                symmetry_group=G)

    # warm-up, as the reference warms its JIT on every code path: the smallest
    # dense-path (<= 500 rows) and Lanczos-path cases through the API (library
    # and kernel loading, allocator, graph set-up), and one dense eigen-solve at
    # the largest dense-path size, whose cuSOLVER kernels load lazily on first
    # use (about 0.1 s once per process); each timed call below gets fresh data
    dims = [int(x) for x in f["sector_dim"]]
    for i in (min(range(len(dims)), key=lambda k: dims[k]),
              min((k for k in range(len(dims)) if dims[k] > 500), key=lambda k: dims[k])):
        w = data_for(i)
        ed.ed_scan_at_irrep_matrixfree(w.irrep_list[0].label, w, nev=1)
    x = torch.randn(500, 500, dtype=torch.complex128, device="cuda")
    torch.linalg.eigh(x + x.conj().T)
    torch.cuda.synchronize()
    rows = []
    for i in range(len(f["model"])):
        data = data_for(i)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        vals, _ = ed.ed_scan_at_irrep_matrixfree(data.irrep_list[0].label, data, nev=1)
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        ref_t = float(f["elapsed_matrixfree_s"][i])
        rows.append({"model": str(f["model"][i]), "label": str(f["label"][i]), "sector_dim": int(data.sector_dims[0]),
                     "b200_s": t, "reference_s": ref_t, "speedup": ref_t / t,
                     "abs_dE": abs(float(vals[0]) - float(f["energy"][i]))})
    return {"workload": "reference benchmark: sector 0, nev 1, matrix-free, catalog untimed", "rows": rows}


def model_basis_size(model, nf):
    import math

    return math.comb(model.lattice.n_site, nf)


def step_kernel_shares(step, top=10):
    """Device time per kernel over one (untimed) step, from CUPTI through
    torch.profiler: [{kernel, launches, total_us, share}] sorted by time."""
    from torch.profiler import ProfilerActivity, profile

    import torch

    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        step()
        torch.cuda.synchronize()
    agg = {}
    for ev in prof.events():
        if ev.device_type.name != "CUDA":
            continue
        name = ev.name.replace("(anonymous namespace)::", "").replace("<unnamed>::", "").replace("void ", "")
        if "(" in name:
            name = name.split("(")[0]
        a = agg.setdefault(name, [0, 0.0])
        a[0] += 1
        a[1] += ev.device_time_total
    tot = sum(v[1] for v in agg.values()) or 1.0
    rows = sorted(agg.items(), key=lambda kv: -kv[1][1])[:top]
    return [{"kernel": k, "launches": v[0], "total_us": round(v[1], 1), "share": round(v[1] / tot, 4)}
            for k, v in rows]


def run_b200(args):
    import torch

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import _lib, models
    from realspace_exatdiagonalization_py_b200.batched import BatchedSectorSolver

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak_gbs = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    wl = WORKLOADS[args.workload]
    nev = wl["nev"]
    model, nf = models.config_model(args.workload)
    G = ed.build_translation_group(model.lattice)
    data = ed.build_ed_data(model, filling_fraction=Fraction(nf, model.lattice.n_site), symmetry_group=G)
    dm, sset = data._device()
    dm.build_projection(sset.sqrt_stab)
    sectors = list(range(len(data.irrep_list)))
    n_sec = len(sectors)
    assert all(d > 500 for d in sset.dims), "bench workload expects every sector on the Lanczos path"

    # how the batch runs (block sizes, persistent cluster or graph path,
    # projection table) is picked by the autotuner, untimed, before warm-up
    params = ed.LanczosParams(precision=args.precision)
    tuner = ed.Autotuner(trials=2)
    t0 = time.perf_counter()
    if args.solver == "auto":
        config, tune_table = tuner.tune(dm, sset, sectors, nev, precision=args.precision, params=params)
    else:  # "graph:<block>:<proj|otf>:<n_slots>" fixes the configuration (e.g. for profiling runs)
        _, bb, mv, ns = args.solver.split(":")
        config = ed.SolverConfig((int(bb),) * n_sec, 0, mv == "proj", int(ns))
        tune_table = []
    tune_s = time.perf_counter() - t0
    solver = BatchedSectorSolver(dm, sset, sectors, nev, precision=args.precision, params=params, config=config)
    b = solver.batch
    host_blocks = [ed.lanczos.start_block(sset.dims[s], b.block_sizes[i], 12345 + s)
                   for i, s in enumerate(sectors)]
    dev_blocks = [torch.from_numpy(x).cuda() for x in host_blocks]
    pinned_blocks = [torch.from_numpy(x).pin_memory() for x in host_blocks]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # oracle eigenvalues (|dE| check of every step's result)
    ref = oracle_eigs(model, nf, G, data.irrep_list, nev) if rank == 0 else None

    def step():
        return solver.solve(dev_blocks, vectors=False, host=False)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    lib = _lib.load()
    times = []
    max_de = 0.0
    launches = 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            n0 = lib.rsed_launch_count()
            r0 = b.replayed_launches
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            vals, _ = step()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
            launches += int(lib.rsed_launch_count() - n0)
            launches += b.replayed_launches - r0
            if ref is not None:
                v = vals.cpu().numpy()
                max_de = max(max_de, max(float(np.max(np.abs(v[i] - ref[s][:nev]))) for i, s in enumerate(sectors)))
    shares = step_kernel_shares(step) if rank == 0 else None
    t_step = max_over_ranks(float(np.sum(times)), ws)
    value = replica_throughput(ws, n_sec * args.steps, t_step)
    lat = sorted(times)

    # e2e through the public API: pinned host start blocks in, numpy eigenpairs out
    e2e_times = []
    h2d = sum(x.numel() * 16 for x in pinned_blocks)
    d2h = 0
    for it in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = ed.solve_sectors_batched(data, sectors, nev=nev, precision=args.precision, params=params,
                                       start_blocks=pinned_blocks, config=config)
        e1.record()
        torch.cuda.synchronize()
        if it >= args.warmup:
            e2e_times.append(e0.elapsed_time(e1) * 1e-3)
        d2h = sum(res[s][0].nbytes + res[s][1].nbytes for s in sectors)
    e2e_val = replica_throughput(ws, n_sec * len(e2e_times), max_over_ranks(sum(e2e_times), ws))

    extra = {}
    if rank == 0:
        # plain FP64 GPU path: one sector at a time, block 1, no graph, host
        # polling every iteration
        p_plain = ed.LanczosParams(block=1, n_slots=48, precision=64, check_every=1)
        plain_t = []
        for s in sectors[: max(3, min(n_sec, args.plain_sectors))]:
            pb = ed.LanczosBatch(dm, sset, [s], nev, p_plain)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            pb.load_start([dev_blocks[s][:, :1]])
            pb.start()
            pb.run(poll=1, graph=False)
            e1.record()
            torch.cuda.synchronize()
            plain_t.append(e0.elapsed_time(e1) * 1e-3)
            if ref is not None:
                max_de_plain = float(np.max(np.abs(pb.eigenvalues()[0] - ref[s][:nev])))
                extra.setdefault("plain_fp64_max_abs_dE", 0.0)
                extra["plain_fp64_max_abs_dE"] = max(extra["plain_fp64_max_abs_dE"], max_de_plain)
        plain_rate = len(plain_t) / sum(plain_t)
        ps = sorted(plain_t)
        extra.update({
            "plain_fp64_sector_solves_per_s": plain_rate,
            "plain_fp64_latency_ms": {"p50": 1e3 * ps[len(ps) // 2], "p99": 1e3 * ps[-1]},
            "batched_over_plain": value / ws / plain_rate,
        })
    # with several ranks the others wait in the closing barrier: only the
    # N = 1 run carries the longer diagnostics and the CPU baseline
    if rank == 0 and ws == 1:
        # FP64-matvec batched variant (its own tuned configuration)
        cfg64 = config if args.solver != "auto" else tuner.tune(
            dm, sset, sectors, nev, precision=64, params=ed.LanczosParams(precision=64))[0]
        extra["fp64_batched_config"] = cfg64.describe()
        s64 = BatchedSectorSolver(dm, sset, sectors, nev, precision=64,
                                  params=ed.LanczosParams(precision=64), config=cfg64)
        for _ in range(2):
            s64.solve(None, vectors=False, host=False)
        t64 = []
        for _ in range(max(3, args.steps // 2)):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            v64, _ = s64.solve(None, vectors=False, host=False)
            e1.record()
            torch.cuda.synchronize()
            t64.append(e0.elapsed_time(e1) * 1e-3)
        extra["fp64_batched_sector_solves_per_s"] = n_sec * len(t64) / sum(t64)
        extra["fp64_batched_max_abs_dE"] = max(float(np.max(np.abs(v64.cpu().numpy()[i] - ref[s][:nev])))
                                               for i, s in enumerate(sectors))
        fe = solver.fp32_error()
        if fe is not None:
            extra["fp32_matvec_error_before_refinement"] = {"max": float(fe.max()), "median": float(np.median(fe))}
    if rank == 0:
        extra["residual_norm_max"] = float(solver.residuals().max())
        extra["step_kernel_shares"] = shares
        extra["autotune"] = {"chosen": config.describe(), "tune_s": tune_s,
                             "candidates": [{"config": r["config"], "solve_ms": None if r["time_s"] is None
                                             else 1e3 * r["time_s"], "ok": r["ok"]} for r in tune_table]}
        st = b.status()
        extra["lanczos_iterations"] = {"min": int(st[:, 3].min()), "max": int(st[:, 3].max())}
        roof = apply_roofline(ed, data, sset, solver, peak_gbs)
        roof["peak_source"] = peak_src
        if not args.skip_scale and ws == 1:
            try:
                extra["matvec_at_scale"] = matvec_at_scale(ed, models, peak_gbs)
            except Exception as exc:  # noqa: BLE001 - reported, not fatal
                extra["matvec_at_scale"] = {"error": repr(exc)}
            torch.cuda.empty_cache()
            try:
                extra["serving_at_scale"] = serving_at_scale(ed, models)
            except Exception as exc:  # noqa: BLE001 - reported, not fatal
                extra["serving_at_scale"] = {"error": repr(exc)}
            torch.cuda.empty_cache()
            try:
                extra["reference_benchmark"] = reference_benchmark(ed, models)
            except Exception as exc:  # noqa: BLE001 - reported, not fatal
                extra["reference_benchmark"] = {"error": repr(exc)}
        # CPU baseline: the oracle (reference algorithm) on the host cores, N = 1 only
        cpu_base = None
        if ws == 1:
            cpu_rate, cpu_n, _, cpu_t = cpu_sector_solves(model, nf, G, data.irrep_list, nev,
                                                          budget_s=args.cpu_budget)
            cpu_base = {"value": cpu_rate, "unit": "sector-solves/s", "cores": _NCPU, "kind": "port",
                        "sample": f"{cpu_n} sector solves of the same workload (its 12 sectors, "
                                  f"cycled) in {cpu_t:.1f} s: projection table + CSR + ARPACK per "
                                  "sector, catalog untimed"}
        line = {
            "metric": "sector-solves/s",
            "value": value,
            "unit": "sector-solves/s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": 1e3 * t_step / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "c64 matvec / f64 Lanczos" if args.precision == 32 else "f64",
            "data": "synthetic",
            "config": {"workload": args.workload, "desc": wl["desc"], "nev": nev,
                       "sectors_per_step": n_sec, "solver": config.describe(), "precision": args.precision,
                       "l2": "256 MB buffer written between timed steps",
                       "parallelism": f"replicas x{ws}"},
            "latency_ms": {"p50": 1e3 * lat[len(lat) // 2], "p99": 1e3 * lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
            "parity": {"max_abs_dE_vs_oracle": max_de, "tolerance": 1e-10},
            "e2e": {"value": e2e_val, "unit": "sector-solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "api": "solve_sectors_batched(start_blocks=pinned host) -> numpy eigenpairs"},
            "roofline": roof,
            "cpu_baseline": cpu_base,
            "clocks": clk.summary(),
            "gpu_launches": launches,
            "extra": extra,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="checkerboard24", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--plain-sectors", type=int, default=12)
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--skip-scale", action="store_true")
    ap.add_argument("--solver", default="auto",
                    help='"auto" (measured by the autotuner) or "graph:<block>:<proj|otf>:<n_slots>"')
    ap.add_argument("--matvec-only", action="store_true",
                    help="only the 32-site matvec at scale (for kernel profiling)")
    ap.add_argument("--matvec-launches", type=int, default=20)
    ap.add_argument("--solve-scale", type=int, default=0,
                    help="only a batched solve of this many 32-site Haldane sectors (for kernel profiling)")
    ap.add_argument("--matvec-precision", type=int, default=0, choices=[0, 32, 64])
    ap.add_argument("--matvec-no-otf", action="store_true")
    ap.add_argument("--serving-only", action="store_true", help="only the 32-site served request stream")
    ap.add_argument("--corr", action="store_true", help="only the correlators of the 32-site Haldane ground state")
    ap.add_argument("--reference-benchmark", action="store_true",
                    help="only the reference's own single-sector benchmark, mirrored through the drop-in API")
    ap.add_argument("--overlap-only", type=int, default=0,
                    help="only the Chern link overlaps of one row of this flux grid (for kernel profiling)")
    ap.add_argument("--chern", type=int, default=0,
                    help="only the many-body Chern number of the 32-site Haldane pair on this flux grid")
    args = ap.parse_args()
    if args.solve_scale:
        import realspace_exatdiagonalization_py_b200 as ed
        import torch
        from realspace_exatdiagonalization_py_b200 import models

        model, nf = models.config_model("haldane32")
        G = ed.build_translation_group(model.lattice)
        data = ed.build_ed_data(model, filling_fraction=Fraction(nf, model.lattice.n_site), symmetry_group=G)
        secs = list(range(args.solve_scale))
        cfg = ed.SolverConfig((2,) * len(secs), 0, True, 16)
        res = ed.solve_sectors_batched(data, secs, nev=4, precision=32, config=cfg, return_vectors=False)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = ed.solve_sectors_batched(data, secs, nev=4, precision=32, config=cfg, return_vectors=False)
        torch.cuda.synchronize()
        print(json.dumps({"workload": f"haldane32: {len(secs)} sectors, FP32 + FP64 refinement, b=2, nev 4",
                          "solve_s": time.perf_counter() - t0, "E0": [float(res[s][0][0]) for s in secs]}))
        return
    if args.reference_benchmark:
        import realspace_exatdiagonalization_py_b200 as ed
        from realspace_exatdiagonalization_py_b200 import models

        print(json.dumps(reference_benchmark(ed, models)), flush=True)
        return
    if args.corr:
        import realspace_exatdiagonalization_py_b200 as ed
        from realspace_exatdiagonalization_py_b200 import models

        print(json.dumps(correlators_at_scale(ed, models)), flush=True)
        return
    if args.serving_only:
        import realspace_exatdiagonalization_py_b200 as ed
        from realspace_exatdiagonalization_py_b200 import models

        print(json.dumps(serving_at_scale(ed, models)), flush=True)
        return
    if args.overlap_only:
        import realspace_exatdiagonalization_py_b200 as ed

        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
            os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
        print(json.dumps({"workload": f"one row of Chern links: {args.overlap_only}x{args.overlap_only} grid, "
                                      "2 states per flux point, 10,518,300 amplitudes per state (32-site Haldane)",
                          **overlap_row(ed, 10_518_300, 2, args.overlap_only,
                                        float(peaks.get("hbm_gbs", 6650.0)))}), flush=True)
        return
    if args.chern:
        import realspace_exatdiagonalization_py_b200 as ed
        from realspace_exatdiagonalization_py_b200 import models

        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
            os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
        print(json.dumps(chern_at_scale(ed, models, grid=args.chern, peak_gbs=float(peaks.get("hbm_gbs", 6650.0)))),
              flush=True)
        return
    if args.matvec_only:
        import realspace_exatdiagonalization_py_b200 as ed
        from realspace_exatdiagonalization_py_b200 import models

        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
            os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
        precs = (args.matvec_precision,) if args.matvec_precision else (32, 64)
        print(json.dumps(matvec_at_scale(ed, models, float(peaks.get("hbm_gbs", 6650.0)),
                                         n_launch=args.matvec_launches, precisions=precs,
                                         otf=not args.matvec_no_otf)), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
