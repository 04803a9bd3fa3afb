"""Benchmark of the CHAPSim periodic-channel time step on B200.

Workload (one "step" = one RK3 time step: CFL/dt + 3 substeps, the CpuT
boundary of src/SOLVE.f90:76,137): periodic plane channel at Re_tau ~ 395
(REN = 6875), domain 2pi x 2 x pi, grid 384 x 256 x 384, tanh-stretched y
(STR2 = 2), FP64 throughout, seeded perturbed-Poiseuille start projected by
the NS = 0 substep, CFL 0.5.  Metric: grid-point * RK3-steps per second.
The line's variants are the same grid in mixed precision (FP32 stencils and
CN sweeps, FP64 Poisson y-solve and projection), the 128^3 channel at
Re_tau ~ 180 in both precisions, and the heated main-domain channel with
table-search and with learned properties.

  python bench.py [--gpus N --steps K --warmup W]        # B200 arm
  python bench.py --impl reference [...]                 # CPU reference arm

With N > 1 (launched by torch.distributed.run) every rank advances its own
independent channel (replicas: the path has no data-parallel exchange) and
the time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "chapsim1.0_b200"))

from chapsim.mesh import channel_setup  # noqa: E402
from chapsim.fields import initial_field  # noqa: E402

METRIC = "grid-pt·RK3-steps/s: mixed/learned vs plain FP64 on 1 B200 at stated error"
UNIT = "grid-pt*RK3-steps/s"
WORKLOADS = {
    # name: (L, M, N, HX, HZ, STR2, REN, DT0, CFLGV)
    "channel128_retau180_fp64": (128, 128, 128, 4 * math.pi, 4 * math.pi / 3, 2.0, 2800.0, 0.05, 0.5),
    "channel64_retau180_fp64": (64, 64, 64, 2 * math.pi, math.pi, 2.0, 2800.0, 0.05, 0.5),
    "channel384x256x384_retau395_fp64": (384, 256, 384, 2 * math.pi, math.pi, 2.0, 6875.0, 0.05, 0.5),
}
DEFAULT_WORKLOAD = "channel384x256x384_retau395_fp64"
ENSEMBLE_WORKLOAD = "ensemble12_uneven"


def ensemble_members(seed=2025, n=12):
    """Twelve periodic channels of uneven size (64^3 .. 192 x 128 x 192, domain
    2pi x 2 x pi), Re_tau drawn uniformly from 180-395 and converted to REN by
    Dean's correlation Re_tau = 0.09 (2 Re_b)^0.88; seeds base + member."""
    rng = np.random.default_rng(seed)
    xs, ys = [64, 96, 128, 192], [64, 96, 128]
    out = []
    for c in range(n):
        L, N = int(rng.choice(xs)), int(rng.choice(xs))
        M = int(rng.choice(ys))
        if c == 0:
            L, M, N = 64, 64, 64
        if c == n - 1:
            L, M, N = 192, 128, 192
        re_tau = float(rng.uniform(180.0, 395.0))
        ren = (re_tau / 0.09) ** (1.0 / 0.88) / 2.0
        out.append((L, M, N, 2 * math.pi, math.pi, 2.0, ren, seed + c))
    return out
L2_BYTES = 126 * 1024 * 1024

# algorithmic FP64 words per grid point moved by one launch of each kernel
# (reads + writes of the arrays the reference's algorithm needs; the
# spectral arrays hold (L/2+1)/L complex values per point)
HEATED_WORKLOAD = "heated256x192x128_retau180_cn"
# heated main-domain channel: grid, domain, REN, DT0, CFLGV, wall heat flux, rho*h perturbation
HEATED = {"L": 256, "M": 192, "N": 128, "HX": 4 * math.pi, "HZ": 4 * math.pi / 3, "STR2": 2.0, "REN": 2800.0,
          "DT0": 1e-3, "CFLGV": 0.5, "qw": 0.5, "dh_amp": 1e-3}
# training schedule of the learned property model: (Adam iterations, learning rate)
MLP_SCHEDULE = [(8000, 3e-3), (8000, 1e-3), (8000, 3e-4), (4000, 1e-4)]
MLP_BOUND = 2e-2  # stated max error of each model output: |model - table| / max(|table|, output scale)


def heated_case():
    """Seeded heated channel: perturbed Poiseuille G, rho*h = table origin +
    a seeded perturbation, the 2048-row synthetic property table."""
    from chapsim import thermo
    h = HEATED
    s = channel_setup(h["L"], h["M"], h["N"], h["HX"], h["HZ"], h["STR2"], h["REN"])
    Q, PR = initial_field(s, 1973, 0.1)
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    cthecd = 1.0 / h["REN"] / (tab.ref["M0"] * tab.ref["CP0"] / tab.ref["K0"])
    DH = np.zeros((h["N"], h["M"] + 2, h["L"]))
    DH[:, 1:h["M"] + 1, :] = h["dh_amp"] * np.random.default_rng(5).uniform(-1.0, 1.0, (h["N"], h["M"], h["L"]))
    return s, Q, PR, tab, cthecd, DH


def heated_kernel_words(L, M):
    """Algorithmic FP64 words per grid point per launch of the heated main-domain
    step (Crank-Nicolson momentum, thermal solver on)."""
    spec = 2.0 * (L // 2 + 1) / L
    return {
        "k_io_cfl": 5.0, "k_dt": 0.0,                 # Q x3, Viscousity, DENSITY
        "k_eng_rhs": 10.0,                            # H, T, kappa, G x3, DH, RHS_E0 in; DH, RHS_E0 out
        "k_eng_props": 11.0, "k_mlp_infer": 11.0,     # DH, DENSITY, Viscousity in; 8 property fields out
        "k_eng_bc": 22.0 / M,                         # the two ghost planes
        "k_drhodt": 7.0,                              # G x3, G0 x3 in; DrhoDt out
        "k_io_props": 8.0,                            # DENSITY0, Viscousity0 in; D_STG x3, MU_STG x3 out
        "k_g0_velocity": 12.0,                        # G, D_STG in; G0, Q out (x3 each)
        "k_io_rhs_cn": 20.0,                          # G, Q, MU_STG, EXPLT0 (x3), Viscousity, PR in; EXPLT0, RHS out
        "k_io_cn_xsweep": 12.0,                       # RHS x3 in/out; 2 coefficient fields per component
        "k_io_cn_zysweep": 27.0,                      # z: as x; y: coefficients, RHS in, G in/out
        "k_io_div_fftx": 5.0 + spec,                  # G x3, DrhoDt in; RHSLLPHI, spectrum out
        "k_fftz_fwd": 2.0 * spec, "k_ysolve": 2.0 * spec, "k_fftz_inv": 2.0 * spec,
        "k_fftx_inv": spec + 1.0,                     # spectrum in; DPH out
        "k_io_correct": 16.0,                         # DPH, G, PR, D_STG, RHSLLPHI in; PR, G, Q out
    }


def heated_cpu_rate(time_budget_s, threads):
    """The heated step on the CPU FP64 restatement (table search, Crank-Nicolson), bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from oracle import Oracle
    h = HEATED
    s, Q, PR, tab, cthecd, DH = heated_case()
    ones = np.ones_like(PR)
    o = Oracle(h["L"], h["M"], h["N"], h["HX"], h["HZ"], h["STR2"], h["REN"], DT0=h["DT0"], DTMIN=1e-6,
               CFLGV=h["CFLGV"], threads=threads)
    o.io_set_fields(Q, PR, ones, ones, ones)
    o.io_set_vis_scheme(1)
    ot = orc.PropTable(tab.lists)
    o.thermal_enable(ot, DH, h["qw"], h["qw"], cthecd)
    o.set_dt(h["DT0"])
    t0 = time.perf_counter()
    n = 0
    while True:
        o.io_run_steps(1)
        n += 1
        if time.perf_counter() - t0 > time_budget_s:
            break
    dt = time.perf_counter() - t0
    o.close()
    return h["L"] * h["M"] * h["N"] * n / dt, n, dt


def run_heated(args):
    """Config 4 as its own bench line (--workload heated256x192x128_retau180_cn)."""
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    line = heated_measure(args, local, dist, ws, args.steps)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, n, dt = heated_cpu_rate(float(os.environ.get("CHAPSIM_CPU_SAMPLE_S", "15")), threads)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{n} RK3 steps of {HEATED_WORKLOAD} on the CPU FP64 restatement (OpenMP)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def heated_measure(args, local, dist, ws, steps):
    """Config 4: heated main-domain channel, Crank-Nicolson momentum, energy
    equation and property update every substep; properties by the table
    search (the plain method) and by the learned model (trained here on the
    table and on rho*h samples of the running field, judged against the
    table search).  Returns the bench line (without the CPU baseline)."""
    from chapsim import gpu
    import torch
    h = HEATED
    L, M, N, DT0, CFLGV, DTMIN = h["L"], h["M"], h["N"], h["DT0"], h["CFLGV"], 1e-6
    s, Q, PR, tab, cthecd, DH = heated_case()
    ones = np.ones_like(PR)
    ch = gpu.ChannelIO(s, device=local, ivisscheme=gpu.VIS_IMPLICIT)
    ch.upload_io(Q, PR, ones, ones, ones)
    ch.set_dt(DT0)
    ch.thermal_init(tab, DH, h["qw"], h["qw"], cthecd)
    stream = torch.cuda.ExternalStream(ch.stream_handle(), device=local)
    pts = L * M * N

    def timed(nsteps):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ch.launch_count()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)
        with ClockSampler(local) as clk:
            ev0.record(stream)
            ch.advance(nsteps, DT0, DTMIN, CFLGV)
            ev1.record(stream)
            torch.cuda.synchronize(local)
        ms = max_over_ranks(ev0.elapsed_time(ev1), dist, f"cuda:{local}")
        return ms, ch.launch_count() - l0, clk.summary()

    def kernel_profile():
        n = max(1, min(10, steps))
        kms = ch.profile_steps(n, DT0, DTMIN, CFLGV)
        return {k: v / n for k, v in kms.items()}

    # ---- plain method: table search ----
    ch.advance(args.warmup, DT0, DTMIN, CFLGV)
    ms_t, launches, clk = timed(steps)
    v_table = pts * steps * ws / (ms_t / 1000.0)
    k_table = kernel_profile()

    # ---- end to end through the public API with host buffers (table search) ----
    try:
        pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
        gh, ph, dhh = pin((3,) + PR.shape), pin(PR.shape), pin(PR.shape)
        rh, mh, qh = pin(PR.shape), pin(PR.shape), pin((3,) + PR.shape)
    except Exception:
        gh, ph, dhh = np.empty((3,) + PR.shape), np.empty(PR.shape), np.empty(PR.shape)
        rh, mh, qh = np.empty(PR.shape), np.empty(PR.shape), np.empty((3,) + PR.shape)
    G0, _, P0 = ch.download_io()
    th = ch.download_thermal()
    gh[...], ph[...], dhh[...], rh[...], mh[...] = G0, P0, th["DH"], th["D"], th["M"]
    ne = max(1, min(steps, args.e2e_steps))
    ch.sync()
    t0 = time.perf_counter()
    for _ in range(ne):
        # H2D: the flow and rho*h state of a restart; the properties follow from rho*h
        ch.lib.chapsim_upload_io_fields(ch.h, gpu._ptr(gh), gpu._ptr(ph), gpu._ptr(rh), gpu._ptr(mh), gpu._ptr(mh))
        ch.lib.chapsim_thermal_init(ch.h, gpu._ptr(dhh), h["qw"], h["qw"], cthecd)
        ch.advance(1, DT0, DTMIN, CFLGV)
        # D2H: the step's result
        ch.lib.chapsim_download_io_fields(ch.h, gpu._ptr(gh), gpu._ptr(qh), gpu._ptr(ph))
        ch.lib.chapsim_download_thermal_fields(ch.h, gpu._ptr(dhh), None, None, None, None, None, None)
    ch.sync()
    te = time.perf_counter() - t0
    e2e = pts * ne * ws / te
    h2d = int(gh.nbytes + ph.nbytes + rh.nbytes + 2 * mh.nbytes + dhh.nbytes)
    d2h = int(gh.nbytes + qh.nbytes + ph.nbytes + dhh.nbytes)

    # ---- learned property model: trained on the table and the running field ----
    dh_list = tab.lists["DH"]
    lo = float(dh_list[0] + 0.02 * (dh_list[-1] - dh_list[0]))
    hi = float(dh_list[-1] - 0.02 * (dh_list[-1] - dh_list[0]))
    field = ch.download_thermal()["DH"][:, 1:M + 1].reshape(-1)
    rng = np.random.default_rng(6)
    knots = dh_list[(dh_list >= lo) & (dh_list <= hi)]
    train = np.concatenate([knots, rng.choice(field, 4000, replace=False), rng.uniform(lo, hi, 2000)])
    ch.mlp_init(lo, hi, seed=11)
    act = gpu.MLP_CUBIC if args.mlp_activation == "cubic" else gpu.MLP_TANH
    ch.mlp_set_activation(act)
    t0 = time.perf_counter()
    loss = None
    for it, lr in MLP_SCHEDULE:
        loss = ch.mlp_train(train, it, lr=lr)
    t_train = time.perf_counter() - t0
    ch.thermal_use_mlp(True)
    ch.advance(args.warmup, DT0, DTMIN, CFLGV)
    ms_m, launches_m, clk_m = timed(steps)
    v_mlp = pts * steps * ws / (ms_m / 1000.0)
    judge = ch.mlp_judge()
    k_mlp = kernel_profile()

    # ---- the same channel in mixed precision (FP32 flow fields, FP64 properties, thermal
    #      fields and Poisson solve), with the table search and with the trained model ----
    params, _norm = ch.mlp_params()
    chm = gpu.ChannelIO(s, device=local, ivisscheme=gpu.VIS_IMPLICIT, precision="mixed")
    chm.upload_io(Q, PR, ones, ones, ones)
    chm.set_dt(DT0)
    chm.thermal_init(tab, DH, h["qw"], h["qw"], cthecd)
    stream_m = torch.cuda.ExternalStream(chm.stream_handle(), device=local)

    def timed_m(nsteps):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)
        ev0.record(stream_m)
        chm.advance(nsteps, DT0, DTMIN, CFLGV)
        ev1.record(stream_m)
        torch.cuda.synchronize(local)
        return max_over_ranks(ev0.elapsed_time(ev1), dist, f"cuda:{local}")

    chm.advance(args.warmup, DT0, DTMIN, CFLGV)
    ms_mt = timed_m(steps)
    chm.mlp_init(lo, hi, seed=11)
    chm.mlp_set_activation(act)
    chm.mlp_set_params(params)
    chm.thermal_use_mlp(True)
    chm.advance(args.warmup, DT0, DTMIN, CFLGV)
    ms_ml = timed_m(steps)
    judge_m = chm.mlp_judge()
    chm.close()

    # ---- roofline of the dominant kernel (table-search step) ----
    words = heated_kernel_words(L, M)
    per_step = {k: (1 if k in ("k_io_cfl", "k_dt") else 3) for k in k_table}
    peak, peak_kind = load_peaks()
    dom = max(k_table, key=lambda k: k_table[k])
    per_launch_ms = k_table[dom] / per_step[dom]
    dom_bytes = words[dom] * 8.0 * pts
    achieved = dom_bytes / (per_launch_ms / 1000.0) / 1e9
    traffic = load_traffic(HEATED_WORKLOAD).get(dom)
    step_bytes = sum(words[k] * 8.0 * pts * per_step[k] for k in k_table)
    step_ms = ms_t / steps
    line = {
        "metric": METRIC, "value": v_table, "unit": UNIT, "n_gpus": ws, "steps": steps, "warmup": args.warmup,
        "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": HEATED_WORKLOAD, "grid": [L, M, N], "domain": "4pi x 2 x 4pi/3", "REN": h["REN"],
                   "STR2": h["STR2"], "iVisScheme": 1, "thermal": "constant wall heat flux %.2f, table of 2048 rows"
                   % h["qw"], "properties": "table search", "cuda_graph": True,
                   "parallelism": "replicas" if ws > 1 else "single",
                   "l2": "no flush: per-step working set %.1f GB > 126 MB L2" % (40 * 8.0 * (M + 2) * L * N / 1e9)},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": ne,
                "api": "chapsim_upload_io_fields + chapsim_thermal_init + chapsim_advance_tg(1) + "
                       "chapsim_download_io_fields + chapsim_download_thermal_fields"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": dom_bytes, "share_of_step": k_table[dom] / sum(k_table.values())},
        "step_roofline": {"bytes_per_point_step": step_bytes / pts,
                          "achieved_gbs": step_bytes / (step_ms / 1000) / 1e9,
                          "frac": step_bytes / (step_ms / 1000) / 1e9 / peak},
        "kernel_ms_per_step": {k: round(v, 5) for k, v in sorted(k_table.items())},
        "clocks": clk,
        "variants": {"learned_properties": {
            "value": v_mlp, "unit": UNIT, "ms_per_step": ms_m / steps, "speedup_vs_table": v_mlp / v_table,
            "activation": args.mlp_activation,
            "judge_max_rel_err": judge, "bound": MLP_BOUND, "within_bound": max(judge.values()) <= MLP_BOUND,
            "training": {"samples": int(train.size), "iterations": sum(i for i, _ in MLP_SCHEDULE),
                         "seconds": t_train, "final_loss": loss},
            "property_update_ms_per_step": {"table": k_table.get("k_eng_props"), "model": k_mlp.get("k_mlp_infer")},
            "gpu_launches": int(launches_m), "clocks": clk_m},
            "mixed": {"value_table": pts * steps * ws / (ms_mt / 1000.0),
                      "value_learned": pts * steps * ws / (ms_ml / 1000.0), "unit": UNIT,
                      "ms_per_step_table": ms_mt / steps, "ms_per_step_learned": ms_ml / steps,
                      "speedup_vs_fp64_table": ms_t / ms_mt, "speedup_learned_vs_fp64_table": ms_t / ms_ml,
                      "judge_max_rel_err": judge_m,
                      "precision": "FP32 flow fields (G, Q, PR, EXPLT0, RHS, D_STG, MU_STG, DivU); FP64 "
                                   "properties, thermal fields, Poisson solve and projection"}},
    }
    ch.close()
    return line


# TG + main-domain run with inflow and outflow (iDomain = 3): a 128^3 periodic TG channel (4 pi x 2 x 4 pi/3)
# feeding a main domain twice its length
XINOUT = {"LT": 128, "L": 256, "M": 128, "N": 128, "HXT": 4 * math.pi, "HZ": 4 * math.pi / 3, "STR2": 2.0,
          "REN": 2800.0, "DT0": 0.01, "CFLGV": 0.5}


def xinout_measure(args, local, steps):
    """The coupled TG + inflow/outflow step (chapsim_advance_xinout), timed with CUDA events from the TG
    stream's first launch to the main-domain stream's last (the two streams join every substep)."""
    import torch
    from chapsim import gpu
    from chapsim.mesh import xinout_setup
    from chapsim.fields import xinout_fields_from_tg
    c = XINOUT
    dx = c["HXT"] / c["LT"]
    st = channel_setup(c["LT"], c["M"], c["N"], c["HXT"], c["HZ"], c["STR2"], c["REN"])
    Q, PR = initial_field(st, 7, 0.2)
    tg = gpu.ChannelTG(st)
    tg.upload(Q, PR)
    tg.set_dt(c["DT0"])
    tg.SOLVERRK3_MOM_tg(0)
    Qt, _ = tg.download()
    io = gpu.ChannelXinout(xinout_setup(c["L"], c["M"], c["N"], c["L"] * dx, c["HZ"], c["STR2"], c["REN"]), tg=tg)
    G, P = xinout_fields_from_tg(Qt, c["L"])
    ones = np.ones(io.field_shape())
    io.upload_io(G, P, ones, ones, ones)
    io.set_dt(c["DT0"])
    io.advance(args.warmup, c["DT0"], 1e-6, c["CFLGV"])
    s_tg = torch.cuda.ExternalStream(tg.stream_handle(), device=local)
    s_io = torch.cuda.ExternalStream(io.stream_handle(), device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(local)
    l0 = io.launch_count() + tg.launch_count()
    e0.record(s_tg)
    dt, cfl = io.advance(steps, c["DT0"], 1e-6, c["CFLGV"])
    e1.record(s_io)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    launches = io.launch_count() + tg.launch_count() - l0
    div = io.DIVGCK_io()
    u_out, scaling = io.outlet_state()
    pts = (c["LT"] + c["L"]) * c["M"] * c["N"]
    io.close()
    tg.close()
    return {"grids": {"tg": [c["LT"], c["M"], c["N"]], "main": [c["L"], c["M"], c["N"]]},
            "value": pts * 1e3 / ms, "unit": UNIT, "ms_per_step": ms, "steps": steps, "gpu_launches": int(launches),
            "final_dt": dt, "final_cfl": cfl, "maxdiv_ranges": [float(x) for x in div], "u_outlet": u_out,
            "outflow_scaling": scaling,
            "note": "TG + main domain with inflow/outflow (iDomain = 3), explicit viscous main domain, FP64; "
                    "value counts the points of both domains"}


def kernel_bytes(L, precision="fp64"):
    """Algorithmic bytes per grid point moved by one launch of each periodic-
    channel kernel, keyed by the kernel names profile_steps reports: reads +
    writes of the arrays the reference's algorithm needs.  The spectrum holds
    (L/2+1)/L complex values per point.  FP64: 8-byte words.  Mixed: Q, PR,
    CONVH0, RHS, RHSLLPHI, the spectrum and DPH are stored in 4-byte words."""
    w = 8.0 if precision == "fp64" else 4.0
    spec = 2.0 * (L // 2 + 1) / L * w  # complex spectrum, bytes per point
    return {
        "k_cfl": 3 * w, "k_dt_factors": 0.0,
        "k_rhs_xsweep": 13 * w,            # Q x3, PR, H0 x3 in; H0 x3, RHS x3 out (x sweep in registers)
        "k_rhs_xsweep_bulk": 13 * w,       # the same, rows staged by bulk copies
        "k_rhs_point+k_xsweep": 19 * w,    # the same, plus the RHS round trip of the separate x sweep
        "k_zsweep": 6 * w,                 # RHS x3 in/out
        "k_ysweep": 9 * w,                 # RHS x3, Q x3 in; Q x3 out
        "k_div_fftx": 4 * w + spec,        # Q x3 in; RHSLLPHI, spectrum out
        "k_div_fft2": 4 * w + spec,        # the same with the z transforms of the plane
        "k_div_fft2c": 4 * w + spec,       # the same, the plane split over a thread-block cluster
        "k_fftz_fwd": 2 * spec, "k_fftz_inv": 2 * spec,
        "k_ysolve_warp": 2 * spec, "k_ysolve_seq": 2 * spec, "k_ysolve_2w": 2 * spec,
        "k_ysolve_scan": 2 * spec,         # the factors it reads are not algorithmic bytes
        "k_fftx_inv": spec + w,            # spectrum in; DPH out
        "k_fft2_inv": spec + w,            # the same with the inverse z transforms of the plane
        "k_fft2c_inv": spec + w,           # the same, the plane split over a thread-block cluster
        "k_correct": 10 * w,               # DPH, Q x3, PR, RHSLLPHI in; Q x3, PR out
    }


def step_launches(name):
    """Launches of kernel `name` per RK3 step (CFL and the dt rule run once, the rest per substep)."""
    return 1 if name in ("k_cfl", "k_dt_factors") else 3


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(workload):
    """Per-launch DRAM bytes of each kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", f"dram_traffic_{workload}.txt")
    out = {}
    if os.path.exists(p):
        for line in open(p):
            s = line.split()
            if len(s) >= 2 and not line.startswith("#"):
                try:
                    out[s[0]] = float(s[1])
                except ValueError:
                    pass
    return out


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def replica_seed(rank):
    """Seed of the channel rank `rank` advances: replicas are independent channels, one per GPU."""
    return 1973 + rank


def max_over_ranks(x, dist, device):
    """The largest x over all ranks (a job's time is its slowest rank's); x itself when not distributed."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(points, steps, ws, ms):
    """Whole-job grid-pt*RK3-steps/s: each of the ws ranks advanced points x steps in at most ms."""
    return points * steps * ws / (ms / 1000.0)


def cpu_reference_rate(wl, steps_cap, time_budget_s, threads):
    """Timed CPU restatement of the step (oracle port, all host threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle
    L, M, N, HX, HZ, STR2, REN, DT0, CFLGV = WORKLOADS[wl]
    s = channel_setup(L, M, N, HX, HZ, STR2, REN)
    Q, PR = initial_field(s, 1973, 0.1)
    o = Oracle(L, M, N, HX, HZ, STR2, REN, DT0=DT0, CFLGV=CFLGV, threads=threads)
    o.set_fields(Q, PR)
    o.substep(0)
    o.run_steps(1)  # warm-up
    t0 = time.perf_counter()
    n = 0
    while n < steps_cap:
        o.run_steps(1)
        n += 1
        if time.perf_counter() - t0 > time_budget_s:
            break
    dt = time.perf_counter() - t0
    o.close()
    return L * M * N * n / dt, n, dt


def run_reference(args):
    ws, rank, local = dist_setup()
    wl = args.workload
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    budget = float(os.environ.get("CHAPSIM_REF_BUDGET_S", "60"))
    if wl == HEATED_WORKLOAD:
        rate, n, dt = heated_cpu_rate(budget, threads)
        L, M, N = HEATED["L"], HEATED["M"], HEATED["N"]
    else:
        rate, n, dt = cpu_reference_rate(wl, max(args.steps, 1), budget, threads)
        L, M, N = WORKLOADS[wl][:3]
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl, "grid": [L, M, N], "precision": "fp64", "parallelism": "replicas"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n} of {args.steps} RK3 steps of {wl} (CPU FP64 restatement, OpenMP)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ensemble(args):
    """Config 5: the members advanced together (one graph per step, one branch per
    member) against the same members advanced one after another."""
    from chapsim import gpu
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:  # replicas: every rank advances its own ensemble (other seeds)
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    members = ensemble_members(2025 + 100 * rank)
    DT0, DTMIN, CFLGV = 0.05, 1e-6, 0.5

    def build():
        chans = []
        for (L, M, N, HX, HZ, STR2, REN, seed) in members:
            s = channel_setup(L, M, N, HX, HZ, STR2, REN)
            Q, PR = initial_field(s, seed, 0.1)
            c = gpu.ChannelTG(s, device=local, precision=args.precision)
            c.upload(Q, PR)
            c.set_dt(1e-3)
            c.SOLVERRK3_MOM_tg(0)
            chans.append(c)
        return chans

    pts = sum(L * M * N for (L, M, N, *_r) in members)
    # sequential: each member's own graph, one after another
    seq = build()
    tune = [c.autotune(force=args.tune) for c in seq]
    for c in seq:
        c.advance(args.warmup, DT0, DTMIN, CFLGV)
    torch.cuda.synchronize(local)
    if dist is not None:
        dist.barrier()
    # each member's K steps timed with CUDA events on its own stream, one member after another
    ms_seq = 0.0
    for c in seq:
        st_c = torch.cuda.ExternalStream(c.stream_handle(), device=local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st_c)
        c.advance(args.steps, DT0, DTMIN, CFLGV)
        e1.record(st_c)
        torch.cuda.synchronize(local)
        ms_seq += e0.elapsed_time(e1)
    t_seq = max_over_ranks(ms_seq / 1000.0, dist, f"cuda:{local}")
    for c in seq:
        c.close()
    # batched: one graph per step over all members
    grp = build()
    for c, (choice, _ms) in zip(grp, tune):
        c.autotune(force=choice)
    ens = gpu.Ensemble(grp)
    ens.advance(args.warmup, DT0, DTMIN, CFLGV)
    stream = torch.cuda.ExternalStream(ens.stream_handle(), device=local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(local)
    if dist is not None:
        dist.barrier()
    launches0 = sum(c.launch_count() for c in grp)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        ens.advance(args.steps, DT0, DTMIN, CFLGV)
        ev1.record(stream)
        torch.cuda.synchronize(local)
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist, f"cuda:{local}")
    launches = sum(c.launch_count() for c in grp) - launches0
    value = aggregate_rate(pts, args.steps, ws, ms)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
        "config": {"workload": ENSEMBLE_WORKLOAD, "members": [[L, M, N, round(REN, 1)] for (L, M, N, _a, _b, _c, REN, _s)
                                                               in members],
                   "precision": args.precision, "total_points": pts,
                   "autotuned_choice_bits": [t[0] for t in tune], "l2": "no flush: members total %.0f MB" % (pts * 8 * 20 / 1e6)},
        "sequential": {"value": pts * args.steps * ws / t_seq, "unit": UNIT, "ms_per_step": 1000.0 * t_seq / args.steps,
                       "timing": "sum over the members of CUDA-event time around each member's own K graph "
                                 "replays on its stream, one member after another (the batched leg is timed "
                                 "with CUDA events on the ensemble stream)"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    line["speedup_vs_sequential"] = line["value"] / line["sequential"]["value"]
    if rank == 0:
        print(json.dumps(line), flush=True)
    ens.close()
    for c in grp:
        c.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def channel_roofline(ch, L, precision, pts, prof_steps, DT0, DTMIN, CFLGV, ms_per_step, traffic_key):
    """Per-kernel CUDA-event durations of the step (the kernels of the variants in
    use), the roofline of the kernel with the largest share and of the whole step."""
    kms = ch.profile_steps(prof_steps, DT0, DTMIN, CFLGV)
    kb = kernel_bytes(L, precision)
    peak, peak_kind = load_peaks()
    total_ms = sum(kms.values())
    dom = max(kms, key=lambda k: kms[k])
    per_launch_ms = kms[dom] / (prof_steps * step_launches(dom))
    dom_bytes = kb[dom] * pts
    achieved = dom_bytes / (per_launch_ms / 1000.0) / 1e9
    traffic = load_traffic(traffic_key).get(dom)
    step_bytes = sum(kb[k] * pts * step_launches(k) for k in kms)
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": dom_bytes, "launch_ms": per_launch_ms,
            "share_of_step": kms[dom] / total_ms}
    step = {"bytes_per_point_step": step_bytes / pts, "achieved_gbs": step_bytes / (ms_per_step / 1000) / 1e9,
            "frac": step_bytes / (ms_per_step / 1000) / 1e9 / peak,
            "survey_model_1344B_frac": (1344.0 if precision == "fp64" else 672.0) * pts / (ms_per_step / 1000) / 1e9
            / peak}
    per_kernel = {k: {"ms_per_step": kms[k] / prof_steps, "launch_ms": kms[k] / (prof_steps * step_launches(k)),
                      "frac": kb[k] * pts / (kms[k] / (prof_steps * step_launches(k)) / 1000.0) / 1e9 / peak}
                  for k in sorted(kms)}
    return roof, step, per_kernel


def channel_measure(args, wl, precision, local, dist, ws, seed, steps, keep=False):
    """One periodic-channel workload on this rank's GPU: autotune, warm-up, K
    graph replays timed with CUDA events on the library's stream (max over
    ranks), then the per-kernel profile.  Returns the measurement and, with
    keep, the open context."""
    from chapsim import gpu
    import torch
    L, M, N, HX, HZ, STR2, REN, DT0, CFLGV = WORKLOADS[wl]
    DTMIN = 1e-6
    s = channel_setup(L, M, N, HX, HZ, STR2, REN)
    Q0, PR0 = initial_field(s, seed, 0.1)
    ch = gpu.ChannelTG(s, device=local, precision=precision, pdl=not args.no_pdl)
    ch.upload(Q0, PR0)
    ch.set_dt(DT0)
    ch.SOLVERRK3_MOM_tg(0)
    # keeps the fastest y-solve, right-hand-side and pressure-stage variants for this grid; --tune pins them instead
    tuned, tune_ms = ch.autotune(force=args.tune)
    stream = torch.cuda.ExternalStream(ch.stream_handle(), device=local)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)

    # the clock sampler runs over the warm-up and the timed region (a window of several 100 ms samples)
    with ClockSampler(local) as clk:
        ch.advance(max(args.warmup, 1), DT0, DTMIN, CFLGV)  # warm-up (also captures the step graph)
        launches0 = ch.launch_count()
        barrier()
        # an NVTX range around the timed steps, so that a profiler can select them alone
        # (ncu --nvtx --nvtx-include "timed_steps/")
        torch.cuda.nvtx.range_push("timed_steps")
        ev0.record(stream)
        dt_last, cfl_last = ch.advance(steps, DT0, DTMIN, CFLGV)
        ev1.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize(local)
    barrier()
    launches = ch.launch_count() - launches0
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist, f"cuda:{local}")
    pts = L * M * N
    value = aggregate_rate(pts, steps, ws, ms)
    prof_steps = max(1, min(20, steps))
    roof, step, per_kernel = channel_roofline(ch, L, precision, pts, prof_steps, DT0, DTMIN, CFLGV, ms / steps,
                                              wl if precision == "fp64" else wl + "_mixed")
    out = {"value": value, "ms": ms, "ms_per_step": ms / steps, "launches": launches, "clocks": clk.summary(),
           "choice": tuned, "tune_ms": {k: round(v, 4) for k, v in tune_ms.items()}, "roofline": roof,
           "step_roofline": step, "kernels": per_kernel, "max_div": ch.DIVGCK_tg(), "final_dt": dt_last,
           "final_cfl": cfl_last, "grid": [L, M, N], "REN": REN, "STR2": STR2, "CFLGV": CFLGV,
           "Q0": Q0, "PR0": PR0, "pts": pts, "DT0": DT0, "DTMIN": DTMIN}
    if keep:
        out["ch"] = ch
    else:
        ch.close()
    return out


def run_b200(args):
    from chapsim import gpu
    ws, rank, local = dist_setup()
    dist = None
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    import torch
    torch.cuda.set_device(local)
    wl = args.workload
    m = channel_measure(args, wl, args.precision, local, dist, ws, replica_seed(rank), args.steps, keep=True)
    ch = m["ch"]
    L, M, N = m["grid"]
    pts, DT0, DTMIN, CFLGV = m["pts"], m["DT0"], m["DTMIN"], WORKLOADS[wl][8]
    Q0, PR0 = m["Q0"], m["PR0"]

    # ---- end to end through the public API with host buffers ----
    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)

    try:
        qh = torch.empty(Q0.shape, dtype=torch.float64, pin_memory=True).numpy()
        ph = torch.empty(PR0.shape, dtype=torch.float64, pin_memory=True).numpy()
    except Exception:
        qh, ph = np.empty_like(Q0), np.empty_like(PR0)
    qh[...], ph[...] = ch.download()
    ne = max(1, min(args.steps, args.e2e_steps))
    barrier()
    t0 = time.perf_counter()
    for _ in range(ne):
        ch.upload(qh, ph)                      # H2D: this step's input fields
        ch.advance(1, DT0, DTMIN, CFLGV)
        ch.lib.chapsim_download_fields(ch.h, gpu._ptr(qh), gpu._ptr(ph), None)  # D2H: the step's result
    ch.sync()
    te = max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{local}")
    e2e_chained = pts * ne * ws / te
    # pipelined through the asynchronous transfer calls: every step uploads its input fields and
    # downloads its result, the H2D copy of step s + 1's input and the D2H copy of step s - 1's
    # result running during step s (each step's input is the same host field set, not the last
    # step's result)
    try:
        qo = [torch.empty(Q0.shape, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
        po = [torch.empty(PR0.shape, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
    except Exception:
        qo, po = [np.empty_like(Q0) for _ in range(2)], [np.empty_like(PR0) for _ in range(2)]
    barrier()
    t0 = time.perf_counter()
    ch.upload_async(qh, ph)
    for s_ in range(ne):
        if s_ + 1 < ne:
            ch.upload_async(qh, ph)        # H2D: the next step's input fields
        ch.advance(1, DT0, DTMIN, CFLGV)   # takes the oldest uploaded fields, then steps
        ch.download_async(qo[s_ % 2], po[s_ % 2])  # D2H: this step's result
    ch.io_wait()
    tp = max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{local}")
    ch.close()
    e2e = pts * ne * ws / tp
    hbytes = int(qh.nbytes + ph.nbytes)
    del qh, ph, qo, po

    grid_desc = {128: "4pi x 2 x 4pi/3", 64: "2pi x 2 x pi", 384: "2pi x 2 x pi"}.get(L)
    line = {
        "metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
        "config": {"workload": wl, "grid": [L, M, N], "domain": grid_desc, "REN": m["REN"], "STR2": m["STR2"],
                   "CFLGV": CFLGV, "precision": args.precision,
                   "parallelism": "replicas" if ws > 1 else "single", "cuda_graph": True,
                   "programmatic_dependent_launch": not args.no_pdl,
                   "l2": "no flush: per-step working set %.0f MB > 126 MB L2" % (
                       (12 * 8 * (M + 2) * L * N + 4 * 8 * L * M * N + 24 * (L // 2 + 1) * M * N) / 1e6),
                   "final_dt": m["final_dt"], "final_cfl": m["final_cfl"], "max_div": m["max_div"],
                   "autotuned": {"choice_bits": m["choice"], "kernels": sorted(m["kernels"]), "ms": m["tune_ms"]}},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": hbytes, "d2h_bytes_per_step": hbytes,
                "steps": ne, "api": "chapsim_upload_fields_async + chapsim_advance_tg(1) + "
                                    "chapsim_download_fields_async, chapsim_io_wait at the end (copies of "
                                    "both directions overlap the steps; each step's input is the same host "
                                    "field set)",
                "chained": {"value": e2e_chained, "api": "chapsim_upload_fields + chapsim_advance_tg(1) + "
                                                         "chapsim_download_fields (each step's input is the "
                                                         "last step's downloaded result)"}},
        "gpu_launches": int(m["launches"]),
        "roofline": m["roofline"],
        "step_roofline": m["step_roofline"],
        "kernels": m["kernels"],
        "clocks": m["clocks"],
    }
    if args.precision == "fp64" and not args.no_variants:
        variants = {}
        # the same workload in mixed precision (FP32 stencils / CN sweeps, FP64 Poisson and projection)
        mm = channel_measure(args, wl, "mixed", local, dist, ws, replica_seed(rank), args.steps)
        variants["mixed"] = {
            "value": mm["value"], "unit": UNIT, "ms_per_step": mm["ms_per_step"],
            "speedup_vs_fp64": mm["value"] / m["value"], "max_div": mm["max_div"],
            "autotuned_choice_bits": mm["choice"], "autotuned_ms": {k: round(v, 4) for k, v in mm["tune_ms"].items()},
            "roofline": mm["roofline"], "step_roofline": mm["step_roofline"],
            "kernels": mm["kernels"], "gpu_launches": int(mm["launches"]), "clocks": mm["clocks"],
            "precision": "FP32 storage, stencils, CN sweeps, x/z transforms and pressure increment; "
                         "FP64 y-solve, divergence, projection, bulk sums"}
        # the 128^3 channel as a variant when the line is another grid
        small = "channel128_retau180_fp64"
        if wl != small:
            s64 = channel_measure(args, small, "fp64", local, dist, ws, replica_seed(rank), args.steps)
            s32 = channel_measure(args, small, "mixed", local, dist, ws, replica_seed(rank), args.steps)
            variants["channel128"] = {
                "workload": small, "grid": s64["grid"], "value_fp64": s64["value"], "value_mixed": s32["value"],
                "unit": UNIT, "ms_per_step_fp64": s64["ms_per_step"], "ms_per_step_mixed": s32["ms_per_step"],
                "speedup_mixed_vs_fp64": s32["value"] / s64["value"],
                "choice_bits": {"fp64": s64["choice"], "mixed": s32["choice"]},
                "roofline_fp64": s64["roofline"], "roofline_mixed": s32["roofline"],
                "step_roofline_fp64": s64["step_roofline"], "step_roofline_mixed": s32["step_roofline"],
                "kernels_fp64": s64["kernels"], "kernels_mixed": s32["kernels"]}
        # config 4: heated main domain, table search against the learned property model
        hl = heated_measure(args, local, dist, ws, min(args.steps, 100))
        lv = hl["variants"]["learned_properties"]
        variants["heated_learned"] = {
            "workload": HEATED_WORKLOAD, "grid": hl["config"]["grid"], "steps": hl["steps"],
            "value_table": hl["value"], "value_learned": lv["value"], "unit": UNIT,
            "ms_per_step_table": hl["ms_per_step"], "ms_per_step_learned": lv["ms_per_step"],
            "speedup_learned_vs_table": lv["speedup_vs_table"],
            "property_update_ms_per_step": lv["property_update_ms_per_step"],
            "judge_max_rel_err": lv["judge_max_rel_err"], "bound": lv["bound"], "within_bound": lv["within_bound"],
            "mixed": hl["variants"]["mixed"],
            "step_roofline_frac": hl["step_roofline"]["frac"],
            "note": "main domain (Crank-Nicolson momentum, energy equation, property update every substep), FP64; "
                    "the full line: --workload " + HEATED_WORKLOAD}
        variants["developing"] = xinout_measure(args, local, min(args.steps, 100))
        line["variants"] = variants
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, n, dt = cpu_reference_rate(wl, 1000, float(os.environ.get("CHAPSIM_CPU_SAMPLE_S", "15")), threads)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{n} RK3 steps of {wl} on the CPU FP64 restatement (OpenMP), after the "
                                          f"NS = 0 projection and one untimed step"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD,
                    choices=sorted(WORKLOADS) + [ENSEMBLE_WORKLOAD, HEATED_WORKLOAD])
    ap.add_argument("--e2e-steps", type=int, default=50)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-variants", action="store_true", help="skip the mixed-precision comparison of an FP64 run")
    ap.add_argument("--tune", type=int, default=-1,
                    help="kernel variant bits instead of timing them (bit 0: sequential y-solve; bits 1-2: "
                         "right-hand side 0 fused, 1 split, 2 fused with bulk-copy staging; bit 3: fused plane "
                         "transforms; bit 4: two-way y-solve); -1 times the variants and keeps the fastest")
    ap.add_argument("--mlp-activation", default="cubic", choices=["cubic", "tanh"],
                    help="hidden-layer activation of the learned property model (the clamped cubic needs no "
                         "special-function unit)")
    ap.add_argument("--no-pdl", action="store_true",
                    help="launch the step's kernels without programmatic dependent launch")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if args.workload == ENSEMBLE_WORKLOAD:
            print(json.dumps({"impl": "reference", "unavailable": "the CPU restatement is timed on the single-channel "
                                                                  "workloads only"}))
            return 0
        return run_reference(args)
    if args.workload == ENSEMBLE_WORKLOAD:
        return run_ensemble(args)
    if args.workload == HEATED_WORKLOAD:
        return run_heated(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
