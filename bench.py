#!/usr/bin/env python
"""Sector-solve throughput of the symmetry-resolved ED path on B200.

Workload (default ``haldane32``): hard-core bosons on the 4x4x2 Haldane
honeycomb (32 sites, 8 bosons, 10,518,300 states, 657,756 orbits, t = 1,
t' = 0.6 exp(+-0.4 pi i), V1 = 1, zero flux), translation group of order 16;
one step = all 16 momentum sectors, lowest 4 eigenvalues each, solved in one
batched block Lanczos (FP32 matvec, FP64 recurrence and reorthogonalisation,
FP64 Rayleigh-Ritz refinement) to |dE| < 1e-10 against the reference's own
ARPACK eigenvalues (tests/golden/haldane32.npz).  ``--workload
checkerboard24`` selects the 24-site checkerboard fermions (12 sectors, nev 6).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One JSON line on rank 0.  N > 1 runs independent replicas (one per GPU, no
collective in the data path); ``value`` is the total over all ranks divided
by the slowest rank's time.  ``--impl reference`` times the reference's own
numpy/scipy path (``ed_scan_at_irrep_matrixfree``: projection table, CSR,
ARPACK) on the host cores instead.
"""

from __future__ import annotations

import os

_NCPU = os.cpu_count() or 1
for _v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
    os.environ.setdefault(_v, str(_NCPU))

import argparse  # noqa: E402
import contextlib  # noqa: E402
import io  # noqa: E402
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

HALDANE_PARAMS = {"t": 1.0, "t'": 0.6, "t''": 0.0, "phi_over_2pi": 0.2, "V1": 1.0, "V2": 0.0}
WORKLOADS = {
    "haldane32": dict(nev=4, golden="haldane32", golden_key="zf_eig",
                      desc="Haldane bosons 4x4x2 = 32 sites, 8 bosons (nu = 1/2), t=1, t'=0.6 e^{+-0.4 pi i}, "
                           "t''=0, V1=1, zero flux; C(32,8) = 10,518,300 states, 657,756 orbits, |G|=16, "
                           "all 16 momentum sectors"),
    "checkerboard24": dict(nev=6, golden="checkerboard24", golden_key="eig_vals",
                           desc="checkerboard 3x4x2 = 24 sites, 4 fermions, |G|=12, all 12 sectors"),
    "heisenberg16": dict(nev=4, golden="heisenberg16", golden_key="eig_vals",
                         desc="Heisenberg ring N=16, 8 up spins, |G|=16, all 16 sectors"),
}
# DRAM bytes per launch of the dominant kernels from one ncu capture each
# (dram__bytes_read.sum + dram__bytes_write.sum); the capture commands and the
# workloads are in the named profiles/ summaries.
NCU_TRAFFIC: dict = {
    ("haldane32", "k_proj_spmv<32>"): {"bytes_per_launch": 2.93e9 + 0.32535e9,
                                       "profile": "profiles/k_proj_spmv_fp32_haldane32_bench.md"},
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


def golden_eigs(name: str):
    """``{sector: lowest eigenvalues}`` of a workload from the reference's own
    ARPACK results committed under tests/golden (None if absent)."""
    wl = WORKLOADS[name]
    path = os.path.join(ROOT, "tests", "golden", wl["golden"] + ".npz")
    if not os.path.isfile(path):
        return None
    f = np.load(path)
    vals = f[wl["golden_key"]]
    secs = f["eig_sectors"] if "eig_sectors" in f else np.arange(len(vals))
    return {int(s): np.asarray(v, dtype=np.float64) for s, v in zip(secs, vals)}


# ---------------------------------------------------------------------------
# CPU side: the reference's own numpy/scipy path (or the oracle port)
# ---------------------------------------------------------------------------


def _reference_model(R, name):
    """The workload's model built by the reference's own model builders."""
    if name == "haldane32":
        return R.bosonic.build_zero_flux_bosonic_fci_second_quantized_model(
            sample_size=[4, 4], params=dict(HALDANE_PARAMS)), 8
    if name == "checkerboard24":
        p = dict(R.fermionic.params_Sun_Gu_Katsura_Sarma)
        p.update({"V1": 1.0, "V2": 0.0, "V3": 0.0})
        with contextlib.redirect_stdout(io.StringIO()):
            return R.fermionic.build_zero_flux_fermionic_fci_second_quantized_model(
                sample_size=[3, 4], params=p), 4
    if name == "heisenberg16":
        with contextlib.redirect_stdout(io.StringIO()):
            return R.heisenberg.build_heisenberg_second_quantized_model(16, 1.0), 8
    raise ValueError(name)


class CpuSectorSolver:
    """Times whole sector solves of a workload on the host cores.

    ``kind == "reference"``: the reference package itself (installed under
    baseline/_ref by oracle/install_reference.py, loaded through
    oracle/ref_shim.py), one ``ed_scan_at_irrep_matrixfree(label, ed_data,
    nev)`` per sector -- its projection table, CSR and ARPACK ``eigs``, the
    unit its own benchmark times.  ``kind == "port"``: the oracle's
    restatement of the same steps, used only where the reference package is
    absent.  The orbit catalog is built once in the constructor (untimed, as
    in the reference's benchmark)."""

    # below this sector size the reference's ARPACK/BLAS calls are tiny and
    # multi-threaded BLAS only adds synchronisation (measured: 0.055 s per
    # 892-row sector with one thread, 0.2-7 s with eight); above it all cores
    # help (657,756 rows: 45 s with eight threads, 50 s with one)
    SMALL_SECTOR = 20000

    def __init__(self, name: str, nev: int):
        from oracle import ref_shim

        self.name, self.nev = name, nev
        t0 = time.perf_counter()
        if ref_shim.available():
            self.kind = "reference"
            R = ref_shim.load()
            self.sre = R.sre
            model, nf = _reference_model(R, name)
            G = R.sre.build_translation_group(model.lattice, None)
            with contextlib.redirect_stdout(io.StringIO()):
                self.data = R.sre.build_ed_data(model, filling_fraction=Fraction(nf, model.lattice.n_site),
                                                symmetry_group=G)
            self.labels = [ir.label for ir in self.data.irrep_list]
        else:
            from oracle import port
            from realspace_exatdiagonalization_py_b200 import models
            import realspace_exatdiagonalization_py_b200.symmetry as sym

            self.kind = "port"
            model, nf = models.config_model(name)
            G = sym.build_translation_group(model.lattice)
            self.irreps = sym.build_irrep_list(G, model.lattice)
            self.model, self.n = model, G.n_site
            self.fermion = model.particle_statistics.name == "FERMIONIC"
            perm0, eta = port.group_arrays(G)
            self.cat = port.catalog(G.n_site, nf, perm0, eta, self.fermion)
            self.labels = [ir.label for ir in self.irreps]
        self.catalog_s = time.perf_counter() - t0
        n_orb = (len(self.data.orbit_catalog.representative_mask_list) if self.kind == "reference"
                 else len(self.cat["reprs"]))
        self.threads = 1 if n_orb < self.SMALL_SECTOR else _NCPU

    def solve(self, s: int) -> tuple[np.ndarray, float]:
        """Eigenvalues of sector ``s`` and the seconds the solve took."""
        from threadpoolctl import threadpool_limits

        with threadpool_limits(limits=self.threads):
            return self._solve(s)

    def _solve(self, s: int) -> tuple[np.ndarray, float]:
        t0 = time.perf_counter()
        if self.kind == "reference":
            with contextlib.redirect_stdout(io.StringIO()):
                w, _ = self.sre.ed_scan_at_irrep_matrixfree(self.labels[s], self.data, nev=self.nev)
        else:
            from oracle import port

            chi = np.asarray(self.irreps[s].values, dtype=np.complex128)
            orbits = port.sector_orbits(self.cat, chi)
            H = port.csr_block(self.cat, self.n, orbits, self.model.bilinear_terms,
                               self.model.density_density_terms, chi, self.fermion)
            w, _ = port.solve(H, self.nev)
        return np.asarray(w, dtype=np.float64), time.perf_counter() - t0

    def sample(self, budget_s: float, min_solves: int = 1, start: int = 0):
        """Sector solves in order (from ``start``, cycling) until ``budget_s``
        seconds of solving are spent; returns (solves/s, solves, seconds,
        {sector: eigenvalues})."""
        t_all, done, vals = 0.0, 0, {}
        s = start % len(self.labels)
        while t_all < budget_s or done < min_solves:
            w, t = self.solve(s)
            t_all += t
            vals[s] = w
            done += 1
            s = (s + 1) % len(self.labels)
        return done / t_all, done, t_all, vals


def run_reference(args):
    """``--impl reference``: the reference's own path on the host cores, on
    rank 0 only (the other ranks exit without work).  One reference sector
    solve of the 32-site workload takes tens of seconds, so the arm times
    whole sector solves until ``--ref-budget`` seconds are spent (at least
    one) instead of ``--steps`` full steps of 16 sectors each; ``ms_per_step``
    is the measured time per sector times the sectors of one step."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    wl = WORKLOADS[args.workload]
    cpu = CpuSectorSolver(args.workload, wl["nev"])
    n_sec = len(cpu.labels)
    budget = getattr(args, "ref_budget", 150.0)
    if args.workload != "haldane32":
        budget = min(budget, 4.0 * max(1, args.steps))
    rate, n_done, t, _ = cpu.sample(budget, min_solves=1)
    line = {
        "impl": "reference",
        "metric": "sector-solves/s",
        "value": rate,
        "unit": "sector-solves/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * n_sec / rate,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "desc": wl["desc"], "nev": wl["nev"], "sectors_per_step": n_sec,
                   "step": "one sector solve = ed_scan_at_irrep_matrixfree (projection table + CSR + "
                           "ARPACK eigs(which='SR', tol=1e-10)); ms_per_step = seconds per sector x sectors"},
        "cpu_baseline": {"value": rate, "unit": "sector-solves/s", "cores": cpu.threads, "kind": cpu.kind,
                         "sample": f"{n_done} whole sector solve(s) in {t:.1f} s, sectors in order from 0 "
                                   f"(the reference's catalog built once in {cpu.catalog_s:.1f} s, untimed); "
                                   f"the arm times solves up to a {budget:.0f} s budget rather than "
                                   f"{args.steps} steps of {n_sec} sectors"},
        "e2e": {"value": rate, "unit": "sector-solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
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
    """Per-column bytes of one apply over the given columns, counted per
    sector matvec: D_s * (8 + 2 s) + H_s * 16 -- the representative
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


def proj_apply_unique_bytes(n_hops: int, n_orb: int, n_cols: int, prec: int) -> int:
    """Bytes one projection-table apply must move at least once: the table
    (per hop the 4-B target/group word and the 8-B or 16-B weight, 8-B row
    offsets), per row the 8-B sector membership and the 16-B diagonal, x read
    once (8 or 16 B per element) and y written once (16 B per element)."""
    wb = 8 if prec == 32 else 16
    return n_hops * (4 + wb) + (n_orb + 1) * 8 + n_orb * (8 + 16) + n_orb * n_cols * (wb + 16)


def lanczos_step_bytes(n_orb: int, batch, state) -> dict:
    """Algorithmic bytes of the Gram reductions and block updates of one
    batched solve, from the counters the kernels keep per instance
    (state[:, 12] = basis blocks + W read by every executed Gram-Schmidt
    pass, state[:, 13] = executed passes).  A reduction reads its nb blocks
    and W once ((nb + 1) n b 16 B); the update after it reads them once more
    and writes W or the new basis block once ((nb + 2) n b 16 B), plus the
    FP32 copy of every new block (n b 8 B) in an FP32-matvec solve."""
    red = upd = 0
    for i, b in enumerate(batch.block_sizes):
        blk = n_orb * b * 16
        blocks, passes, steps = int(state[i, 12]), int(state[i, 13]), int(state[i, 3])
        red += blocks * blk
        upd += (blocks + passes) * blk + (steps * n_orb * b * 8 if batch.p.precision == 32 else 0)
    return {"reduce": red, "update": upd}


def cupti_kernels(step):
    """Device time per kernel over one (untimed) call of ``step``, from CUPTI
    through torch.profiler: {kernel name: [launches, total_us]}."""
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
    return agg


def kernel_shares(agg, top=10):
    tot = sum(v[1] for v in agg.values()) or 1.0
    rows = sorted(agg.items(), key=lambda kv: -kv[1][1])[:top]
    return [{"kernel": k, "launches": v[0], "total_us": round(v[1], 1), "share": round(v[1] / tot, 4)}
            for k, v in rows]


def _family(agg, prefix, contains=""):
    n = us = 0.0
    for k, (c, t) in agg.items():
        if k.startswith(prefix) and contains in k:
            n += c
            us += t
    return int(n), us


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


def serving_at_scale(ed, models, n_req=32, rate=20.0, block=2, plain_samples=2, n_slots=16):
    """The request loop at the 32-site Haldane size: a Poisson stream (seed 0)
    of (sector, flux) requests over a 16 x 16 flux grid and 16 sectors,
    served with continuous batching (FP32 matvec + FP64 refinement, nev 4),
    against the plain FP64 path (one request at a time, block 1, no graph,
    the solver's default check schedule) on the first requests of the stream."""
    import torch
    from realspace_exatdiagonalization_py_b200.serving import poisson_requests

    model, nf = models.config_model("haldane32")
    sm = ed.ServingModel(model, nf, name="haldane32")
    reqs = poisson_requests(n_req, rate=rate, n_sectors=sm.n_sectors, flux_grid=16, model="haldane32", seed=0)
    srv = ed.SolveServer(sm, nev=4, precision=32, block=block, n_slots=n_slots, poll=16)
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
        p = ed.LanczosParams(block=1, precision=64)
        b = ed.LanczosBatch(ctx.dm, ctx.sset, [r.sector], 4, p)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.load_start(None)
        b.start()
        b.run(graph=False)
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


def _load_peaks():
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        peaks = {}
    if "hbm_gbs" in peaks:
        return float(peaks["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (6.65 TB/s, no MEASURED_PEAKS.json)"


def small_config_line(ed, models, name, precision=32, steps=10):
    """A short batched run of a small workload (all sectors, autotuned) with
    parity against the reference's goldens: the latency-bound end of the
    range, beside the HBM-bound headline."""
    import torch
    from realspace_exatdiagonalization_py_b200.batched import BatchedSectorSolver

    wl = WORKLOADS[name]
    nev = wl["nev"]
    model, nf = models.config_model(name)
    G = ed.build_translation_group(model.lattice)
    data = ed.build_ed_data(model, filling_fraction=Fraction(nf, model.lattice.n_site), symmetry_group=G)
    dm, sset = data._device()
    dm.build_projection(sset.sqrt_stab)
    sectors = list(range(len(data.irrep_list)))
    params = ed.LanczosParams(precision=precision)
    config, _ = ed.Autotuner(trials=2).tune(dm, sset, sectors, nev, precision=precision, params=params)
    solver = BatchedSectorSolver(dm, sset, sectors, nev, precision=precision, params=params, config=config)
    blocks = [torch.from_numpy(ed.lanczos.start_block(sset.dims[s], solver.batch.block_sizes[i], 12345 + s)).cuda()
              for i, s in enumerate(sectors)]
    for _ in range(3):
        solver.solve(blocks, vectors=False, host=False)
    ref = golden_eigs(name)
    times, de = [], 0.0
    for _ in range(steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        vals, _ = solver.solve(blocks, vectors=False, host=False)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
        v = vals.cpu().numpy()
        if ref is not None:
            de = max(de, max(float(np.max(np.abs(v[i] - ref[s][:nev]))) for i, s in enumerate(sectors)))
    return {"workload": name, "desc": wl["desc"], "nev": nev, "precision": precision,
            "solver": config.describe(), "sector_solves_per_s": len(sectors) * steps / sum(times),
            "ms_per_step": 1e3 * sum(times) / steps, "max_abs_dE_vs_reference": de if ref is not None else None}


def config5_line(ed, models, n_sectors=4, nev=6, cpp_threads=0):
    """The 48-site checkerboard (4x6x2, 8 fermions, C(48,8) = 377,348,994
    states, |G| = 24): device catalog, then a batched solve (FP32 matvec + FP64
    refinement, nev 6) of ``n_sectors`` sectors, timed; the C++ restatement
    (oracle/cpu_ref.cpp, OpenMP on the host cores -- the reference cannot rank
    beyond 42 sites) builds the same catalog, compared by SHA-256 digests of
    the tables, and applies the first sector's operator once to a seeded
    vector, compared with the device's apply; its catalog and apply times are
    the CPU figures, a sector solve extrapolated from one apply times the
    device solve's matvec count (labelled: not the reference, extrapolated)."""
    import hashlib

    import torch

    from oracle import cpu, port

    model, nf = models.config_model("checkerboard48")
    G = ed.build_translation_group(model.lattice)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    data = ed.build_ed_data(model, filling_fraction=Fraction(nf, 48), symmetry_group=G)
    dm, sset = data._device()
    torch.cuda.synchronize()
    t_cat = time.perf_counter() - t0
    secs = list(range(n_sectors))
    cfg = ed.SolverConfig((2,) * n_sectors, 0, True, 16)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = ed.solve_sectors_batched(data, secs, nev=nev, precision=32, config=cfg, return_vectors=False)
    torch.cuda.synchronize()
    t_solve = time.perf_counter() - t0
    solver = next(iter(data.__dict__.get("_solvers", {}).values()), None)
    st = solver.batch.status() if solver is not None else None
    iters = [int(x) - 1 for x in st[:, 3]] if st is not None else []
    cat = data.orbit_catalog
    def amp_bits(a32):  # components below 1e-15 (signed zeros included) as +0
        a = np.ascontiguousarray(a32).view(np.float32).copy()
        a[np.abs(a) < 1e-15] = 0
        return a.tobytes()

    tab = cat.table.cpu().numpy()
    dev_digest = {k: hashlib.sha256(np.ascontiguousarray(tab[:, i]).tobytes()).hexdigest()
                  for k, i in (("rep_rank", 0), ("rep_sym", 1))}
    dev_digest.update({k: hashlib.sha256(amp_bits(tab[:, i])).hexdigest()
                       for k, i in (("rep_amp_re", 2), ("rep_amp_im", 3))})
    dev_digest["reprs"] = hashlib.sha256(cat.repr_masks.cpu().numpy().view(np.uint64).tobytes()).hexdigest()
    del tab
    perm0, eta = port.group_arrays(G)
    t0 = time.perf_counter()
    ref = cpu.catalog(48, nf, perm0, eta, True, nthreads=cpp_threads)
    t_cpp_cat = time.perf_counter() - t0
    amp = ref["rep_amp"].view(np.int32).reshape(-1, 2)
    cpp_digest = {"rep_rank": hashlib.sha256(ref["rep_rank"].tobytes()).hexdigest(),
                  "rep_sym": hashlib.sha256(ref["rep_sym"].tobytes()).hexdigest(),
                  "rep_amp_re": hashlib.sha256(amp_bits(amp[:, 0])).hexdigest(),
                  "rep_amp_im": hashlib.sha256(amp_bits(amp[:, 1])).hexdigest(),
                  "reprs": hashlib.sha256(ref["reprs"].tobytes()).hexdigest()}
    del amp
    chi = np.asarray(data.irrep_list[0].values, dtype=np.complex128)
    op = cpu.SectorOperator(ref, chi, model.bilinear_terms, model.density_density_terms, nthreads=cpp_threads)
    x = np.random.default_rng(48).standard_normal(op.n) + 1j * np.random.default_rng(49).standard_normal(op.n)
    t0 = time.perf_counter()
    y_cpp = op(x)
    t_cpp_apply = time.perf_counter() - t0
    basis = ed.Symmetry_Sector_Basis(data.irrep_list[0], cat, sset, 0)
    H = ed.MatrixFreeHamiltonian(basis, model.bilinear_terms, model.density_density_terms, None, model=dm)
    y_dev = H.adjoint_device(torch.from_numpy(x).cuda()).cpu().numpy()[:, 0]
    mv_err = float(np.abs(y_dev - y_cpp).max() / np.abs(y_cpp).max())
    applies = (max(iters) + 1) if iters else None
    return {"workload": "checkerboard48: 4x6x2 = 48 sites, 8 fermions, C(48,8) = 377,348,994 states, |G| = 24, "
                        f"{cat.n_orbits:,} orbits; {n_sectors} sectors, nev {nev}, FP32 matvec + FP64 refinement",
            "sector_dims": [int(sset.dims[s]) for s in secs],
            "device": {"catalog_s": t_cat, "solve_s": t_solve, "sector_solves_per_s": n_sectors / t_solve,
                       "lanczos_steps": iters, "single_pass_steps": None if st is None else int(st[:, 11].sum()),
                       "E0": [float(res[s][0][0]) for s in secs]},
            "cpp_restatement": {"kind": "port", "label": "C++ restatement of the reference's algorithm, not the "
                                "reference (which cannot rank beyond 42 sites)", "threads": cpp_threads or _NCPU,
                                "catalog_s": t_cpp_cat, "apply_s": t_cpp_apply,
                                "sector_solve_s_extrapolated": None if applies is None else t_cpp_apply * applies,
                                "extrapolation": "one apply x (device Lanczos steps + 1) of the slowest sector"},
            "parity": {"catalog_digests_equal": {k: dev_digest[k] == cpp_digest[k] for k in dev_digest},
                       "amplitudes": "components below 1e-15 (signed zeros included) compared as +0",
                       "apply_max_rel_diff": mv_err}}


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
    from realspace_exatdiagonalization_py_b200.batched import BatchedSectorSolver, projection_precisions

    peak_gbs, peak_src = _load_peaks()
    wl = WORKLOADS[args.workload]
    nev = wl["nev"]
    model, nf = models.config_model(args.workload)
    G = ed.build_translation_group(model.lattice)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    data = ed.build_ed_data(model, filling_fraction=Fraction(nf, model.lattice.n_site), symmetry_group=G)
    dm, sset = data._device()
    torch.cuda.synchronize()
    t_cat = time.perf_counter() - t0
    t0 = time.perf_counter()
    dm.build_projection(sset.sqrt_stab, precisions=projection_precisions(dm, args.precision))
    torch.cuda.synchronize()
    t_proj = time.perf_counter() - t0
    sectors = list(range(len(data.irrep_list)))
    n_sec = len(sectors)
    n_orb = data.orbit_catalog.n_orbits
    assert all(d > 500 for d in sset.dims), "bench workload expects every sector on the Lanczos path"

    # how the batch runs (block sizes, persistent cluster or graph path,
    # projection table, basis length) is picked by the autotuner, untimed
    params = ed.LanczosParams(precision=args.precision, single_pass=not args.two_pass, stream=not args.no_stream,
                              stream_update=args.stream_update)
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
    host_blocks = [ed.lanczos.start_block(sset.dims[s], b.block_sizes[i], 12345 + s) for i, s in enumerate(sectors)]
    dev_blocks = [torch.from_numpy(x).cuda() for x in host_blocks]
    pinned_blocks = [torch.from_numpy(x).pin_memory() for x in host_blocks]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ref = golden_eigs(args.workload) if rank == 0 else None

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
    if ws > 1:
        torch.distributed.barrier()
    t_step = max_over_ranks(float(np.sum(times)), ws)
    value = replica_throughput(ws, n_sec * args.steps, t_step)
    lat = sorted(times)
    st = b.status()
    iters = [int(x) - 1 for x in st[:, 3]]
    fe = solver.fp32_error()
    resid_max = float(solver.residuals().max())

    # e2e through the public API: pinned host start blocks in, numpy eigenpairs out
    e2e_times = []
    h2d = sum(x.numel() * 16 for x in pinned_blocks)
    d2h = 0
    e2e_de = 0.0
    for it in range(min(args.warmup, 2) + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = ed.solve_sectors_batched(data, sectors, nev=nev, precision=args.precision, params=params,
                                       start_blocks=pinned_blocks, config=config)
        e1.record()
        torch.cuda.synchronize()
        if it >= min(args.warmup, 2):
            e2e_times.append(e0.elapsed_time(e1) * 1e-3)
        d2h = sum(res[s][0].nbytes + res[s][1].nbytes for s in sectors)
        if ref is not None:
            e2e_de = max(e2e_de, max(float(np.max(np.abs(res[s][0] - ref[s][:nev]))) for s in sectors))
    data.__dict__.pop("_solvers", None)
    torch.cuda.empty_cache()
    if ws > 1:
        torch.distributed.barrier()
    e2e_val = replica_throughput(ws, n_sec * len(e2e_times), max_over_ranks(sum(e2e_times), ws))

    extra = {"setup_s": {"catalog": t_cat, "projection_table": t_proj, "autotune": tune_s,
                         "note": "untimed: the catalog and the projection table are built once per catalog and "
                                 "shared by all sectors and steps"}}
    roof = None
    if rank == 0:
        # per-kernel device time of one step (CUPTI) and algorithmic bytes
        agg = cupti_kernels(step)
        st_prof = b.status()  # the kernels' counters for the profiled step
        extra["step_kernel_shares"] = kernel_shares(agg)
        fams = {}
        nh = dm.proj["n_hops"]
        n_mv, us_mv = _family(agg, "k_proj_spmv<" + str(args.precision))
        if n_mv:
            fams["k_proj_spmv<%d>" % args.precision] = {
                "kernel": f"k_proj_spmv<{args.precision},...> (FP{args.precision} projection-table matvec, all "
                          f"{b.n_cols} columns of the batch)",
                "launches": n_mv, "avg_launch_us": us_mv / n_mv,
                "alg_bytes_per_launch": proj_apply_unique_bytes(nh, n_orb, b.n_cols, args.precision),
                "unit_bytes": "per hop 4 + 8 B table, per row 8 + 8 + 16 B, per element x 8 B + y 16 B, once each"}
        lb = lanczos_step_bytes(n_orb, b, st_prof)
        # the streamed forms: k_lz_gram_stream + k_lz_finalize (reduction),
        # k_lz_update_stream (update); the per-instance forms k_lz_reduce,
        # k_lz_update / k_lz_update_rows
        for key, fam, extra_fam in (("reduce", "k_lz_reduce", ("k_lz_gram_stream", "k_lz_finalize")),
                                    ("update", "k_lz_update", ())):
            n_k, us_k = _family(agg, fam)
            names = [fam + "*"] if n_k else []
            for ef in extra_fam:
                n_e, us_e = _family(agg, ef)
                us_k += us_e
                if n_e:
                    names.append(ef)
                if ef != "k_lz_finalize":
                    n_k += n_e
            if n_k:
                fams[fam] = {"kernel": " + ".join(names) + " (FP64 block Gram-Schmidt, "
                                       + ("two passes" if args.two_pass else "adaptive single pass") + ")",
                             "launches": n_k, "avg_launch_us": us_k / n_k,
                             "alg_bytes_per_launch": lb[key] / n_k,
                             "unit_bytes": "per executed pass (nb + 1) resp. (nb + 2) blocks of n_orb x b x 16 B, "
                                           "+ n_orb x b x 8 B FP32 copy per new block (kernel-side counters)"}
        for k, f in fams.items():
            f["achieved_GBs"] = f["alg_bytes_per_launch"] / (f["avg_launch_us"] * 1e-6) / 1e9
            f["frac"] = f["achieved_GBs"] / peak_gbs
            f["share_of_step"] = f["avg_launch_us"] * f["launches"] / max(1e-9, sum(v[1] for v in agg.values()))
        extra["kernel_rooflines"] = fams
        if fams:
            top = max(fams, key=lambda k: fams[k]["share_of_step"])
            f = fams[top]
            tr = NCU_TRAFFIC.get((args.workload, top))
            roof = {"bound": "hbm", "achieved": f["achieved_GBs"], "peak": peak_gbs, "unit": "GB/s",
                    "frac": f["frac"], "traffic": None if tr is None else tr["bytes_per_launch"],
                    "kernel": f["kernel"], "avg_launch_us": f["avg_launch_us"],
                    "alg_bytes_per_launch": f["alg_bytes_per_launch"], "timing": "CUPTI kernel durations, one step",
                    "peak_source": peak_src, "share_of_step": f["share_of_step"]}
            if tr is not None:
                roof["traffic_source"] = tr["profile"]
        extra["lanczos_iterations"] = {"min": min(iters), "max": max(iters), "steps": int(sum(iters)),
                                       "single_pass_steps": int(st[:, 11].sum()),
                                       "gram_schmidt": "two passes" if args.two_pass else "adaptive single pass"}
        extra["residual_norm_max"] = resid_max
        if fe is not None:
            extra["fp32_matvec_error_before_refinement"] = {"max": float(fe.max()), "median": float(np.median(fe))}
        extra["autotune"] = {"chosen": config.describe(), "tune_s": tune_s,
                             "candidates": [{"config": r["config"], "solve_ms": None if r["time_s"] is None
                                             else 1e3 * r["time_s"], "ok": r["ok"]} for r in tune_table]}
        # plain FP64 GPU path: one sector at a time, block 1, FP64 matvec, no
        # graph, the solver's default check schedule (Ritz checks at restarts)
        p_plain = ed.LanczosParams(block=1, precision=64)
        plain_t, plain_de = [], 0.0
        for s in sectors[: max(1, min(n_sec, args.plain_sectors))]:
            pb = ed.LanczosBatch(dm, sset, [s], nev, p_plain)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            pb.load_start([dev_blocks[s][:, :1]])
            pb.start()
            pb.run(graph=False)
            e1.record()
            torch.cuda.synchronize()
            plain_t.append(e0.elapsed_time(e1) * 1e-3)
            if ref is not None:
                plain_de = max(plain_de, float(np.max(np.abs(pb.eigenvalues()[0] - ref[s][:nev]))))
            del pb
        plain_rate = len(plain_t) / sum(plain_t)
        ps = sorted(plain_t)
        extra.update({
            "plain_fp64": {"sector_solves_per_s": plain_rate, "sectors_timed": len(plain_t),
                           "latency_ms": {"p50": 1e3 * ps[len(ps) // 2], "p99": 1e3 * ps[-1]},
                           "max_abs_dE_vs_reference": plain_de if ref is not None else None,
                           "path": "one sector per solve, block 1, FP64 projection-table matvec, no graph, "
                                   "default check schedule"},
            "batched_over_plain": value / ws / plain_rate,
            "e2e_over_plain": e2e_val / ws / plain_rate,
        })
        torch.cuda.empty_cache()
    # only the N = 1 run carries the longer diagnostics and the CPU baseline,
    # so no rank waits in the closing barrier for rank 0's extra work
    cpu_base = None
    if rank == 0 and ws == 1:
        if not args.skip_fp64:
            s64 = BatchedSectorSolver(dm, sset, sectors, nev, precision=64,
                                      params=ed.LanczosParams(precision=64), config=config)
            s64.solve(dev_blocks, vectors=False, host=False)
            t64 = []
            for _ in range(3):
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                v64, _ = s64.solve(dev_blocks, vectors=False, host=False)
                e1.record()
                torch.cuda.synchronize()
                t64.append(e0.elapsed_time(e1) * 1e-3)
            extra["fp64_batched"] = {"sector_solves_per_s": n_sec * len(t64) / sum(t64), "config": config.describe(),
                                     "max_abs_dE_vs_reference": None if ref is None else max(
                                         float(np.max(np.abs(v64.cpu().numpy()[i] - ref[s][:nev])))
                                         for i, s in enumerate(sectors))}
            del s64
        del solver
        torch.cuda.empty_cache()
        if not args.skip_scale:
            for key, fn in (("serving_at_scale", lambda: serving_at_scale(ed, models)),
                            ("config2_checkerboard24", lambda: small_config_line(ed, models, "checkerboard24")),
                            ("reference_benchmark", lambda: reference_benchmark(ed, models))):
                if key == "config2_checkerboard24" and args.workload == "checkerboard24":
                    continue
                try:
                    extra[key] = fn()
                except Exception as exc:  # noqa: BLE001 - reported, not fatal
                    extra[key] = {"error": repr(exc)}
                torch.cuda.empty_cache()
    if rank == 0 and ws == 1 and not args.no_cpu:
        # CPU baseline: the reference's own path on the host cores, N = 1 only
        cpu = CpuSectorSolver(args.workload, nev)
        rate, n_done, t_cpu, cvals = cpu.sample(args.cpu_budget, min_solves=1)
        cpu_de = None
        if ref is not None:
            cpu_de = max(float(np.max(np.abs(cvals[s][:nev] - ref[s][:nev]))) for s in cvals)
        cpu_base = {"value": rate, "unit": "sector-solves/s", "cores": cpu.threads, "kind": cpu.kind,
                    "sample": f"{n_done} whole sector solve(s) of this workload in {t_cpu:.1f} s: "
                              + ("the reference's ed_scan_at_irrep_matrixfree (projection table + CSR + ARPACK)"
                                 if cpu.kind == "reference" else "the oracle port of the reference's steps")
                              + f", catalog built once ({cpu.catalog_s:.1f} s, untimed)",
                    "max_abs_dE_vs_golden": cpu_de}
    if rank == 0:
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
                       "l2": "inputs larger than L2 (Lanczos blocks of 0.17-0.67 GB); 256 MB buffer also "
                             "written between timed steps",
                       "parallelism": f"replicas x{ws}"},
            "latency_ms": {"p50": 1e3 * lat[len(lat) // 2], "p99": 1e3 * lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                           "unit": "one step (all sectors)"},
            "parity": {"max_abs_dE_vs_reference": max_de if ref is not None else None, "tolerance": 1e-10,
                       "e2e_max_abs_dE": e2e_de if ref is not None else None,
                       "reference": f"tests/golden/{wl['golden']}.npz (the reference's ARPACK eigenvalues)"},
            "e2e": {"value": e2e_val, "unit": "sector-solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "api": "solve_sectors_batched(start_blocks=pinned host) -> numpy eigenvalues + eigenvectors"},
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
    ap.add_argument("--workload", default="haldane32", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--plain-sectors", type=int, default=3)
    ap.add_argument("--cpu-budget", type=float, default=30.0,
                    help="seconds of reference sector solves for cpu_baseline (at least one solve)")
    ap.add_argument("--ref-budget", type=float, default=150.0,
                    help="seconds of reference sector solves for --impl reference (at least one solve)")
    ap.add_argument("--skip-scale", action="store_true", help="skip the serving / config-2 / benchmark extras")
    ap.add_argument("--skip-fp64", action="store_true", help="skip the FP64-matvec batched variant")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (e.g. for kernel profiling)")
    ap.add_argument("--two-pass", action="store_true",
                    help="always two Gram-Schmidt passes per step (no adaptive single pass)")
    ap.add_argument("--no-stream", action="store_true",
                    help="per-instance Gram-Schmidt kernels instead of the streamed whole-row panels")
    ap.add_argument("--stream-update", action="store_true",
                    help="the streamed update after the streamed Gram reduction (default: the row-group update)")
    ap.add_argument("--config5", type=int, default=0,
                    help="only the 48-site checkerboard line for this many sectors (device vs C++ restatement)")
    ap.add_argument("--solver", default="auto",
                    help='"auto" (measured by the autotuner) or "graph:<block>:<proj|otf>:<n_slots>"')
    ap.add_argument("--matvec-only", action="store_true",
                    help="only the 32-site matvec at scale (for kernel profiling)")
    ap.add_argument("--matvec-launches", type=int, default=20)
    ap.add_argument("--solve-scale", type=int, default=0,
                    help="only a batched solve of this many 32-site Haldane sectors (for kernel profiling)")
    ap.add_argument("--scale-slots", type=int, default=16,
                    help="basis slots of the --solve-scale solve (fewer slots, smaller footprint)")
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
    peak_gbs = None
    if args.solve_scale:
        import realspace_exatdiagonalization_py_b200 as ed
        import torch
        from realspace_exatdiagonalization_py_b200 import models

        model, nf = models.config_model("haldane32")
        G = ed.build_translation_group(model.lattice)
        data = ed.build_ed_data(model, filling_fraction=Fraction(nf, model.lattice.n_site), symmetry_group=G)
        secs = list(range(args.solve_scale))
        cfg = ed.SolverConfig((2,) * len(secs), 0, True, args.scale_slots)
        prm = ed.LanczosParams(block=2, precision=32, single_pass=not args.two_pass, stream=not args.no_stream,
                               stream_update=args.stream_update)
        res = ed.solve_sectors_batched(data, secs, nev=4, precision=32, params=prm, config=cfg,
                                       return_vectors=False)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = ed.solve_sectors_batched(data, secs, nev=4, precision=32, params=prm, config=cfg,
                                       return_vectors=False)
        torch.cuda.synchronize()
        print(json.dumps({"workload": f"haldane32: {len(secs)} sectors, FP32 + FP64 refinement, b=2, nev 4",
                          "solve_s": time.perf_counter() - t0, "E0": [float(res[s][0][0]) for s in secs]}))
        return
    if args.impl == "reference":
        run_reference(args)
        return
    special = args.reference_benchmark or args.corr or args.serving_only or args.overlap_only or args.chern \
        or args.matvec_only or args.config5
    if special:
        import realspace_exatdiagonalization_py_b200 as ed
        from realspace_exatdiagonalization_py_b200 import models

        peak_gbs, _ = _load_peaks()
    if args.reference_benchmark:
        print(json.dumps(reference_benchmark(ed, models)), flush=True)
    elif args.corr:
        print(json.dumps(correlators_at_scale(ed, models)), flush=True)
    elif args.serving_only:
        print(json.dumps(serving_at_scale(ed, models)), flush=True)
    elif args.overlap_only:
        print(json.dumps({"workload": f"one row of Chern links: {args.overlap_only}x{args.overlap_only} grid, "
                                      "2 states per flux point, 10,518,300 amplitudes per state (32-site Haldane)",
                          **overlap_row(ed, 10_518_300, 2, args.overlap_only, peak_gbs)}), flush=True)
    elif args.chern:
        print(json.dumps(chern_at_scale(ed, models, grid=args.chern, peak_gbs=peak_gbs)), flush=True)
    elif args.config5:
        print(json.dumps(config5_line(ed, models, n_sectors=args.config5)), flush=True)
    elif args.matvec_only:
        precs = (args.matvec_precision,) if args.matvec_precision else (32, 64)
        print(json.dumps(matvec_at_scale(ed, models, peak_gbs, n_launch=args.matvec_launches, precisions=precs,
                                         otf=not args.matvec_no_otf)), flush=True)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
