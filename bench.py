#!/usr/bin/env python
"""Benchmark of the ECHO-QGP step path on B200.

Workload: 3+1D ideal RMHD in Milne coordinates on a 97x97x81 grid
(x, y, eta; dx = deta = 0.15), tabulated crossover EoS (2048 log-spaced
points), WENO5 + HLL + GLM divergence cleaning, RK3.  A "step" is one full
time step of the grid (three RK stages, con2prim included).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

value:   cell-updates/s with the state resident in HBM (the library's CUDA
         graph per step), timed with CUDA events on the library's stream,
         for the faster of the con2prim paths (Newton from the previous
         stage's primitives); the BRENTM and MLP-seeded variants are timed
         beside it in `variants`.
e2e:     the same metric through the C-ABI with host buffers: every step
         copies v and u from page-locked host memory to the device, runs one
         step and copies v and u back (echo_gpu_advance_host, whose copy of
         u overlaps the first flux sweeps).
--impl reference: the reference algorithm on the host cores (the CPU
         restatement in oracle/, all threads), on a bounded sample of the
         same workload.
Multi-GPU: the step does not shard in this workload (one grid per GPU), so
N GPUs run N independent replicas (weak scaling, no collective on the data
path); the timed region is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "echo-qgp-mhd-devel_b200"))

import numpy as np  # noqa: E402

METRIC = "cell-updates/s on 1 B200: MLP-seeded vs plain con2prim at equal 1e-10 residual"
UNIT = "cell-updates/s"
B_ALG_STEP = 1008  # algorithmic HBM bytes per cell-update of a stage-fused RK3 step, nv = 9


COUNTERS = os.path.join(ROOT, "profiles", "roofline_counters_rmhd_97x97x81.json")


def config_of(cfg) -> dict:
    """The `config` object of both arms (the headline workload)."""
    return {"workload": cfg.name, "grid": [cfg.nx, cfg.ny, cfg.nz], "nv": cfg.nv,
            "scheme": "WENO5+HLL+GLM, RK3, tabulated EoS (2048 pts)",
            "l2": "working set per step (2x v, 2x u, 3 face-flux arrays ~ 440 MB) exceeds the 126 MB L2"}


def peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "src": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "src": "fallback"}


def workload():
    from echo_gpu import initial as I
    from echo_gpu import params as P

    cfg = P.config1()
    tab = I.eos_table_loaded()
    przero = float(I.table_pressure(tab, np.array([cfg.enezero]))[0])
    return cfg, tab, przero


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        os.remove(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# CPU side: the reference algorithm (oracle restatement)
# ---------------------------------------------------------------------------
def cpu_rate(cfg, tab, przero, threads: int, target_s: float, steps: int | None = None,
             warmup: int = 0, state=None):
    """cell-updates/s of the reference algorithm on the host on a z-slab of
    the workload sized so one step takes about target_s seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O  # the CPU restatement of the reference (baseline only)
    from echo_gpu import initial as I
    from echo_gpu import params as P

    def slab(nz):
        z1, z2 = P._grid(nz, (cfg.z2 - cfg.z1) / cfg.nz)
        return cfg.replace(nz=nz, z1=z1, z2=z2)

    state = state or (lambda c: I.primitives(c, tab))
    if cfg.nz == 1:
        c = cfg  # a 2+1D grid: the whole grid
    else:
        probe = slab(6)
        o = O.Oracle(probe.to_c(przero=przero), tab, threads=threads)
        o.set_state(state(probe), None, probe.tstart)
        t0 = time.perf_counter()
        o.step()
        rate = probe.ncell / (time.perf_counter() - t0)
        nz = int(max(6, min(cfg.nz, round(target_s * rate / (cfg.nx * cfg.ny)))))
        c = slab(nz)
    o = O.Oracle(c.to_c(przero=przero), tab, threads=threads)
    o.set_state(state(c), None, c.tstart)
    for _ in range(warmup):
        o.step()
    n = steps if steps is not None else 2
    t0 = time.perf_counter()
    for _ in range(n):
        o.step()
    el = time.perf_counter() - t0
    what = "the whole grid" if c.nz == cfg.nz else "a slab"
    sample = (f"{n} full steps of {what} ({c.nx}x{c.ny}x{c.nz}) of the workload "
              f"(same spacing, EoS, scheme), after {warmup} untimed steps")
    return c.ncell * n / el, el, sample


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg, tab, przero = workload()
    threads = os.cpu_count() or 1
    # each step is one time step of a slab sized to ~1 s of work on all cores
    rate, el, sample = cpu_rate(cfg, tab, przero, threads, target_s=1.0, steps=args.steps,
                                warmup=args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (optical-Glauber Au+Au b=7 fm x Gaussian eta profile, B_y ~ exp(-x^2/2/2.5^2))",
        "config": dict(config_of(cfg), con2prim="BRENTM (the reference's ALG_SOLV=1)",
                       build="oracle/liboracle_echo.so (gcc -O2, OpenMP over pencils and cells)"),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
def algorithmic_bytes(kclass: str, cfg) -> float:
    """Compulsory HBM bytes of one launch of a kernel class (each array it
    reads or writes counted once)."""
    nv, nc = cfg.nv, cfg.ncell
    nf = [(cfg.nx + 1) * cfg.ny * cfg.nz, cfg.nx * (cfg.ny + 1) * cfg.nz, cfg.nx * cfg.ny * (cfg.nz + 1)]
    if kclass.startswith("faces"):
        d = "xyz".index(kclass[-1])
        return 8.0 * nv * (nc + nf[d])  # read v, write the face fluxes
    if kclass == "update_c2p":
        # read F(x,y,z), v, u and (two stages in three) u0; write u and v
        return 8.0 * nv * (sum(nf) + nc * (2 + 2.0 / 3.0) + 2 * nc) + nc
    return 0.0


B_ALG_RES = 1896  # bytes per cell-update of a stage-fused IMEX-SSP3(4,3,3) resistive step, nv = 12


def run_ideal_hd(args, torch, barrier, world, rank):
    """The 2+1D ideal-hydro workload: p = e/3, 101x101 (dx = 0.2 fm),
    optical-Glauber Au+Au at b = 7 fm, WENO5 + HLL, RK2 at CFL 0.4, its 100
    steps from tau = 0.4 fm/c (10 k cells: the step is launch-bound and runs
    as captured step graphs), beside the CPU restatement on one core."""
    from echo_gpu import params as P
    from echo_gpu.lib import Evolve
    from echo_gpu import initial as I

    cfg = P.config0()
    przero = cfg.enezero / 3.0
    v0 = I.primitives(cfg, None)
    ev = Evolve(cfg.to_c(przero=przero), None, exact=False)
    ev.upload(v0, None, cfg.tstart)
    stream = torch.cuda.ExternalStream(ev.stream_handle())
    ev.run(max(args.warmup, 3))
    ev.sync()
    ev.upload(v0, None, cfg.tstart)
    ev.run(1)  # the step graphs exist; time the workload's own 100 steps from tau0
    ev.upload(v0, None, cfg.tstart)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ev.run(cfg.steps)
    e1.record(stream)
    ev.sync()
    barrier()
    ms = float(e0.elapsed_time(e1))
    st = ev.stats()
    prof = ev.profile_step()
    ev.close()
    out = {"workload": cfg.name, "grid": [cfg.nx, cfg.ny], "nv": cfg.nv, "scheme": "WENO5+HLL, RK2, p = e/3",
           "value": cfg.ncell * cfg.steps * world / (ms / 1e3), "unit": UNIT, "steps": cfg.steps,
           "ms_per_step": ms / cfg.steps, "t_end": st.t, "errcode": int(st.errcode),
           "kernels_ms_per_step": {k: round(v[0], 4) for k, v in prof.items() if v[1]}}
    if world == 1 and rank == 0:
        rate, el, sample = cpu_rate(cfg, None, przero, threads=1, target_s=2.0, steps=20,
                                    state=lambda c: I.primitives(c, None))
        out["cpu_oracle"] = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample}
    return out


def run_resistive(args, torch, barrier, world, rank):
    """The resistive workload: 3+1D resistive RMHD (MHD = 2) on 193x193x129
    (dx = deta = 0.1), sigma_el = 5.8 MeV and the chiral term, IMEX-SSP3(4,3,3)
    with the implicit Ohm's law in every implicit stage's con2prim, GLM,
    WENO5 + HLL, tabulated EoS; the plain (warm-started) inversion and the
    MLP-seeded one (six invariants, E^2/U among them, trained on pairs of
    resistive runs), timed back to back.  The reference cannot run this path
    (its con2prim has no branch for MHD = 2); the CPU figure beside it is
    the oracle's statement of the same scheme on a slab of the grid."""
    from echo_gpu import initial as I
    from echo_gpu import params as P
    from echo_gpu import seed as S
    from echo_gpu.lib import Evolve

    cfg = P.config4()
    tab = I.eos_table_loaded()
    przero = float(I.table_pressure(tab, np.array([cfg.enezero]))[0])
    v0 = I.primitives(cfg, tab)
    t0 = time.perf_counter()
    Xp, Tp = S.generate_pairs(n_target=args.pairs // 2, steps=6, every=3, resistive=True)
    t1 = time.perf_counter()
    w, norm, losses = S.train(Xp, Tp, steps=args.train_steps)
    t2 = time.perf_counter()
    training = {"pairs": int(len(Xp)), "pair_generation_s": t1 - t0, "train_steps": args.train_steps,
                "train_s": t2 - t1, "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
                "source": "resistive runs of this workload at half resolution (97x97x65 over the same extent), "
                          "3 energy scales x 2 magnetisations x 3 flow amplitudes"}
    steps = max(3, min(args.steps, 20))

    def timed(algo):
        c = cfg.replace(algo_solver=algo)
        ev = Evolve(c.to_c(przero=przero), tab, exact=False)
        if algo == P.C2P_MLP:
            ev.set_seed_network(w, norm)
        ev.upload(v0, None, cfg.tstart)
        stream = torch.cuda.ExternalStream(ev.stream_handle())
        ev.run(max(args.warmup, 3))
        ev.sync()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ev.run(steps)
        e1.record(stream)
        ev.sync()
        torch.cuda.synchronize()
        barrier()
        ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
        if world > 1:
            import torch.distributed as dist

            dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        ms = float(ms.item())
        st = ev.stats()
        prof = ev.profile_step()
        ev.sync()
        ev.close()
        return ms, st, prof

    pk = peaks()
    variants = {}
    for algo, name in ((P.C2P_NEWTON, "plain"), (P.C2P_MLP, "mlp_seeded")):
        ms, st, prof = timed(algo)
        value = cfg.ncell * steps * world / (ms / 1e3)
        variants[name] = {
            "value": value, "ms_per_step": ms / steps,
            "step_roofline": {"bytes_per_cell_update": B_ALG_RES, "achieved_gbs": value / world * B_ALG_RES / 1e9,
                              "frac": value / world * B_ALG_RES / 1e9 / pk["hbm_gbs"],
                              "peak_src": pk["src"] + " (hbm_gbs)"},
            "kernels_ms_per_step": {k: round(v[0], 4) for k, v in prof.items()},
            "c2p_iters_per_cell_last_stage": st.c2p_iters / max(cfg.ncell, 1),
            "seed_fallbacks_total": int(st.seed_fallbacks), "bracket_fallbacks_total": int(st.bracket_fallbacks),
            "errcode": int(st.errcode), "repairs": int(st.repairs)}
    out = {
        "workload": cfg.name, "grid": [cfg.nx, cfg.ny, cfg.nz], "nv": cfg.nv,
        "scheme": "WENO5+HLL (light-cone speeds)+GLM, IMEX-SSP3(4,3,3), implicit Ohm's law, tabulated EoS",
        "sigma_el": cfg.sigma_el, "sigma_chiral": cfg.sigma_chiral,
        "value": variants["plain"]["value"], "unit": UNIT, "steps": steps,
        "ms_per_step": variants["plain"]["ms_per_step"],
        "value_variant": "plain (faster than mlp_seeded)",
        "variants": variants, "seed_training": training,
        "c2p_iters": "Newton steps per cell summed over the fixed point's passes: the stage-4 solve and the "
                     "final combination",
        "parity": "unpinned against the reference (no runnable resistive path); device = oracle at 1e-12",
    }
    if world == 1 and rank == 0:
        rate, el, sample = cpu_rate(cfg, tab, przero, threads=1, target_s=4.0, steps=1)
        out["cpu_oracle"] = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample}
    return out


def run_viscous(args, torch, barrier, world, rank, X1, T1):
    """The 2+1D viscous workload: Israel-Stewart shear hydro on 201x201
    (dx = 0.1 fm), eta/s = 0.12, tau_pi = 5 eta/(e+p), IMEX RK2, tabulated
    EoS, MC-Glauber Pb+Pb at b = 8 fm; the plain (warm-started) nested
    inversion and the MLP-seeded one, the network trained on pairs of the
    ideal-RMHD workload (X1, T1) and of viscous runs of this one.  40 k
    cells: the step is latency-bound, so it runs as captured step graphs."""
    from echo_gpu import initial as I
    from echo_gpu import params as P
    from echo_gpu import seed as S
    from echo_gpu.lib import Evolve

    cfg = P.config2().replace(imex=1)
    tab = I.eos_table_loaded()
    przero = float(I.table_pressure(tab, np.array([cfg.enezero]))[0])
    pcut = I.table_temperature_to_pressure(tab, cfg.smooth_temp)
    v0 = I.primitives(cfg, tab)
    t0 = time.perf_counter()
    Xv, Tv = S.generate_pairs(n_target=args.pairs // 2, viscous=True)
    X = np.concatenate([X1, Xv])
    T = np.concatenate([T1, Tv])
    t1 = time.perf_counter()
    w, norm, losses = S.train(X, T, steps=args.train_steps)
    t2 = time.perf_counter()
    training = {"pairs": int(len(X)), "viscous_pairs": int(len(Xv)), "pair_generation_s": t1 - t0,
                "train_steps": args.train_steps, "train_s": t2 - t1,
                "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
                "source": "the ideal-RMHD workload's pairs plus viscous runs of this workload "
                          "(3 energy scales x b = 0, 5, 10 fm)"}
    steps = max(20, min(args.steps * 4, 200))

    def timed(algo):
        c = cfg.replace(algo_solver=algo)
        ev = Evolve(c.to_c(przero=przero, smooth_pressure=pcut), tab, exact=False)
        if algo == P.C2P_MLP:
            ev.set_seed_network(w, norm)
        ev.upload(v0, None, cfg.tstart)
        stream = torch.cuda.ExternalStream(ev.stream_handle())
        ev.run(max(args.warmup, 3))
        ev.sync()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ev.run(steps)
        e1.record(stream)
        ev.sync()
        torch.cuda.synchronize()
        barrier()
        ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
        if world > 1:
            import torch.distributed as dist

            dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        st = ev.stats()
        prof = ev.profile_step()
        ev.sync()
        ev.close()
        return float(ms.item()), st, prof

    variants = {}
    for algo, name in ((P.C2P_NEWTON, "plain"), (P.C2P_MLP, "mlp_seeded")):
        ms, st, prof = timed(algo)
        variants[name] = {
            "value": cfg.ncell * steps * world / (ms / 1e3), "ms_per_step": ms / steps,
            "kernels_ms_per_step": {k: round(v[0], 4) for k, v in prof.items()},
            "c2p_iters_per_cell_last_stage": st.c2p_iters / max(cfg.ncell, 1),
            "seed_fallbacks_total": int(st.seed_fallbacks), "bracket_fallbacks_total": int(st.bracket_fallbacks),
            "errcode": int(st.errcode)}
    return {
        "workload": cfg.name, "grid": [cfg.nx, cfg.ny], "nv": cfg.nv, "scheme": "WENO5+HLL, IMEX RK2",
        "value": variants["plain"]["value"], "unit": UNIT, "steps": steps,
        "ms_per_step": variants["plain"]["ms_per_step"], "value_variant": "plain (faster than mlp_seeded)",
        "variants": variants, "seed_training": training,
        "c2p_iters": "Newton steps per cell summed over the nested iteration's passes, last stage",
    }, (Xv, Tv)


def run_batched(args, torch, barrier, world, rank, net=None):
    """The batched event-by-event workload: 512 Monte Carlo Glauber Pb+Pb
    events (viscous 2+1D, grids 61^2..161^2) from tau = 0.4 to 10 fm/c in
    one batch, beside the same events run one after another through the
    single-grid path, and again with the MLP-seeded inversion (net: the
    2+1D viscous workload's training pairs, joined by pairs of this one's
    events).  With N ranks the events are split across the
    GPUs by cell count (no collective on the data path): the whole job's
    cell-updates over the slowest rank's time."""
    from echo_gpu import events as EV
    from echo_gpu import initial as I
    from echo_gpu import params as P
    from echo_gpu import seed as S
    from echo_gpu import shard as SH
    from echo_gpu.batch import Batch, event_grid
    from echo_gpu.lib import Evolve

    full = EV.batched_viscous()
    mine = SH.partition_by_cells(full.cells, world)[rank]
    es = EV.EventSet(cfg=full.cfg, b=full.b[mine], n=full.n[mine], dx=full.dx, tmax=full.tmax)
    tab = EV.batched_eos_table()
    przero = float(I.table_pressure(tab, np.array([es.cfg.enezero]))[0])
    pcut = I.table_temperature_to_pressure(tab, es.cfg.smooth_temp)
    pc = es.cfg.to_c(przero=przero, smooth_pressure=pcut)
    t0 = time.perf_counter()
    srcs_all = EV.event_sources(full)
    srcs = [srcs_all[int(e)] for e in mine]
    sampling_s = time.perf_counter() - t0
    b = Batch(pc, tab, [event_grid(*es.grid(e)) for e in range(es.nev)])
    t0 = time.perf_counter()
    b.glauber(srcs, es.cfg.tstart, es.tmax)
    ic_s = time.perf_counter() - t0
    tune_ms = b.autotune(3)
    tune_rows = b.autotune_report()
    tune_choice = b.tuning()
    best_stage = {}
    for r in tune_rows:
        if r["slot"] == "stage" and (r["mode"] not in best_stage or r["ms"] < best_stage[r["mode"]]["ms"]):
            best_stage[r["mode"]] = r
    b.run(max(args.warmup, 3))  # builds the step graphs
    b.glauber(srcs, es.cfg.tstart, es.tmax)
    stream = torch.cuda.ExternalStream(b.stream_handle())
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    nsteps = b.run_to_end(chunk=16)
    e1.record(stream)
    b.sync()
    barrier()
    ms = SH.reduce_max(e0.elapsed_time(e1), device="cuda")
    st_local = b.status()
    cu = SH.reduce_sum(b.cell_updates(), device="cuda")
    st = SH.gather_status(mine, st_local, full.nev)
    seeded = None
    if net is not None:
        # the seed for this workload: pairs from a sample of its own events run
        # to the end time (dilute late stages, its EoS table) with the viscous
        # workload's pairs, one network
        t0 = time.perf_counter()
        Xe, Te = S.generate_event_pairs(full, tab, przero, pcut, n_target=args.pairs // 2, sources=srcs_all)
        Xb = np.concatenate([net[0], Xe])
        Tb = np.concatenate([net[1], Te])
        t1 = time.perf_counter()
        wb, nb, lb = S.train(Xb, Tb, steps=args.train_steps)
        t2 = time.perf_counter()
        training = {"pairs": int(len(Xb)), "event_pairs": int(len(Xe)), "pair_generation_s": t1 - t0,
                    "train_s": t2 - t1, "loss_first": float(lb[0]), "loss_last": float(lb[-1]),
                    "source": "every 32nd event of the batch run alone to the end time (8 samples each) plus the "
                              "2+1D viscous workload's pairs"}
        pcm = es.cfg.replace(algo_solver=P.C2P_MLP).to_c(przero=przero, smooth_pressure=pcut)
        bm = Batch(pcm, tab, [event_grid(*es.grid(e)) for e in range(es.nev)])
        bm.set_seed_network(wb, nb)
        bm.glauber(srcs, es.cfg.tstart, es.tmax)
        bm.autotune(3)
        bm.run(max(args.warmup, 3))
        bm.glauber(srcs, es.cfg.tstart, es.tmax)
        sm = torch.cuda.ExternalStream(bm.stream_handle())
        barrier()
        torch.cuda.synchronize()
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        m0.record(sm)
        bm.run_to_end(chunk=16)
        m1.record(sm)
        bm.sync()
        barrier()
        ms_m = SH.reduce_max(m0.elapsed_time(m1), device="cuda")
        cu_m = SH.reduce_sum(bm.cell_updates(), device="cuda")
        stm = bm.status()
        fb = SH.reduce_sum(sum(s["seed_fallbacks"] for s in stm), device="cuda")
        crashed = SH.reduce_sum(sum(1 for s in stm if s["state"] == 2), device="cuda")
        bm.close()
        seeded = {"value": cu_m / (ms_m / 1e3), "ms": ms_m, "cell_updates": int(cu_m),
                  "seed_fallbacks_total": int(fb), "events_crashed": int(crashed), "seed_training": training}
    # the same events one at a time through the single-grid path (a sample)
    b.glauber(srcs, es.cfg.tstart, es.tmax)
    v0 = b.split(b.download()[0])
    prof, _ = b.profile_step()
    b.close()
    seq_cu, seq_ms = 0, 0.0
    for e in range(0, es.nev, 16):
        cfg = es.event_config(e)
        g = Evolve(cfg.to_c(przero=przero, smooth_pressure=pcut), tab)
        g.upload(v0[e], None, cfg.tstart)
        g.set_tout(es.tmax)
        g.run(3)
        g.sync()
        gs = torch.cuda.ExternalStream(g.stream_handle())
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(gs)
        g.run(20)
        f1.record(gs)
        g.sync()
        seq_ms += f0.elapsed_time(f1)
        seq_cu += 20 * cfg.ncell
        g.close()
    seq = seq_cu / (seq_ms / 1e3)
    if rank != 0:
        return None
    plain = cu / (ms / 1e3)
    value = plain
    states = np.bincount([s["state"] for s in st], minlength=4)
    return {
        "workload": f"{full.nev} MC-Glauber Pb+Pb events (b in [0,12] fm), viscous 2+1D IS, grids "
                    f"{int(full.n.min())}^2..{int(full.n.max())}^2 at dx={full.dx}, tau {full.cfg.tstart} -> "
                    f"{full.tmax} fm/c, CFL dt per event, IMEX RK2, WENO5+HLL, crossover EoS to 1e-7 GeV/fm^3, "
                    f"ENEZERO {full.cfg.enezero}",
        "cells": int(full.cells.sum()),
        "value": value, "unit": UNIT, "ms": ms, "batched_steps": nsteps,
        "variants": {"plain": {"value": plain, "ms": ms}, "mlp_seeded": seeded},
        "scaling": "strong" if world > 1 else None,
        "sharding": f"events split over {world} GPU(s) by cell count, no data-path collective",
        "cell_updates": int(cu), "events_done": int(states[1]), "events_crashed": int(states[2]),
        "crashed": [{"event": int(e), "b": float(full.b[e]), "n": int(full.n[e]), "errcode": int(x["errcode"]),
                     "t": round(float(x["t"]), 4)} for e, x in enumerate(st) if x["state"] == 2],
        "event_steps_min_max": [int(min(s["steps"] for s in st)), int(max(s["steps"] for s in st))],
        "sequential_single_grid": {"value": seq, "unit": UNIT,
                                   "sample": "every 16th event of rank 0's share, 20 steps each, one GPU"},
        "speedup_vs_sequential": plain / world / seq,
        "speedup_vs_sequential_note": "plain batched over plain single-grid, both on one GPU",
        "kernels_ms_per_step_at_start": {k: round(x, 4) for k, x in prof.items()},
        "autotuned_ms_per_launch": {k: round(x, 4) for k, x in tune_ms.items()},
        "autotune": {"candidates_timed": len(tune_rows),
                     "search_space": "per slot: tile of 128/256/512 faces or cells x (one CTA per tile, or "
                                     "1..occupancy CTAs per SM); per stage: one launch per phase (7 launches) or "
                                     "one cooperative launch (1..occupancy CTAs per SM)",
                     "choice": tune_choice,
                     "best_stage_ms": {k: {"ms": round(v["ms"], 4), "ctas": v["ctas"]} for k, v in best_stage.items()},
                     "launches_per_stage": 1 if tune_choice["mode"] == "cooperative" else
                     (7 if es.cfg.viscosity and es.cfg.smooth_temp > 0 else 6)},
        "ic": {"nucleon_sampling_s_host": sampling_s, "smearing_and_eos_s_device": ic_s},
        "con2prim": "viscous nested Newton (system.f90:564-666), plain and from the learned seed "
                    "(the 2+1D viscous workload's network)",
    }


def run_b200(args):
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from echo_gpu import initial as I
    from echo_gpu import params as P
    from echo_gpu import seed as S
    from echo_gpu.lib import Evolve

    def barrier():
        if world > 1:
            dist.barrier()

    cfg0, tab, przero = workload()
    v0 = I.primitives(cfg0, tab)

    # the learned seed: pairs from the solver, trained by the library's kernels
    t0 = time.perf_counter()
    Xp, Tp = S.generate_pairs(n_target=args.pairs)
    t1 = time.perf_counter()
    w, norm, losses = S.train(Xp, Tp, steps=args.train_steps)
    t2 = time.perf_counter()
    training = {"pairs": int(len(Xp)), "pair_generation_s": t1 - t0, "train_steps": args.train_steps,
                "train_s": t2 - t1, "loss_first": float(losses[0]), "loss_last": float(losses[-1])}

    dev_id = str(local)
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        dev_id = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:
        pass
    clk = Clocks(dev_id)
    clk.start()

    def timed(algo):
        cfg = cfg0.replace(algo_solver=algo)
        ev = Evolve(cfg.to_c(przero=przero), tab, exact=False)
        if algo == P.C2P_MLP:
            ev.set_seed_network(w, norm)
        ev.upload(v0, None, cfg.tstart)
        stream = torch.cuda.ExternalStream(ev.stream_handle())
        ev.run(max(args.warmup, 0))  # warm-up (also builds the step graphs)
        ev.sync()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ev.run(args.steps)
        e1.record(stream)
        ev.sync()
        torch.cuda.synchronize()
        barrier()
        ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        st = ev.stats()
        return ev, stream, float(ms.item()), st

    variants = {}
    names = {P.C2P_BRENT: "reference_brentm", P.C2P_NEWTON: "plain_newton", P.C2P_MLP: "mlp_seeded"}
    keep = None
    for algo in (P.C2P_BRENT, P.C2P_NEWTON, P.C2P_MLP):
        ev, stream, ms, st = timed(algo)
        it = st.c2p_iters / max(cfg0.ncell, 1)
        variants[names[algo]] = {
            "value": cfg0.ncell * args.steps * world / (ms / 1e3), "ms_per_step": ms / args.steps,
            "c2p_iters_per_cell_last_stage": it,
            "c2p_iters": "BRENTM function evaluations" if algo == P.C2P_BRENT else "Newton steps",
            "seed_fallbacks_total": int(st.seed_fallbacks), "bracket_fallbacks_total": int(st.bracket_fallbacks),
            "errcode": int(st.errcode)}
        if algo == P.C2P_NEWTON:
            keep = (ev, stream, ms, st)
        else:
            ev.close()
    clocks = clk.stop()
    ev, stream, ms_max, st = keep
    value = variants["plain_newton"]["value"]
    prof = ev.profile_step()  # one real step, per-kernel device times
    ev.sync()

    # end to end through the C-ABI with host buffers
    nbytes = cfg0.nv * cfg0.ncell * 8
    hv = torch.empty(cfg0.nv * cfg0.ncell, dtype=torch.float64, pin_memory=True)
    hu = torch.empty(cfg0.nv * cfg0.ncell, dtype=torch.float64, pin_memory=True)
    ev.get_state(hv.data_ptr(), hu.data_ptr())
    ev.sync()
    e2e_steps = max(3, min(args.steps, 20))
    barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        # the host owns the whole state between steps: copied in, one step, copied out
        ev.advance_host(hv.data_ptr(), hu.data_ptr(), hv.data_ptr(), hu.data_ptr(), 1)
    f1.record(stream)
    ev.sync()
    barrier()
    e2e_ms = torch.tensor([f0.elapsed_time(f1)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
    e2e_value = cfg0.ncell * e2e_steps * world / (float(e2e_ms.item()) / 1e3)
    st2 = ev.stats()
    viscous, vnet = run_viscous(args, torch, barrier, world, rank, Xp, Tp) if args.viscous else (None, None)
    batched = run_batched(args, torch, barrier, world, rank, vnet) if args.batched else None
    resistive = run_resistive(args, torch, barrier, world, rank) if args.resistive else None
    ideal_hd = run_ideal_hd(args, torch, barrier, world, rank) if args.ideal_hd else None

    if world > 1:
        dist.barrier()
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    # roofline of the dominant kernel: HBM (its own compulsory bytes, and the
    # stage-fused B_alg of one stage) and FP64 (ncu FLOPs over the measured
    # FP64 peak of this GPU)
    pk = peaks()
    dom = max((k for k in prof if prof[k][1] > 0), key=lambda k: prof[k][0])
    dom_ms, dom_n = prof[dom]
    per_launch_s = dom_ms / dom_n / 1e3
    alg = algorithmic_bytes(dom, cfg0)
    achieved = alg / per_launch_s / 1e9
    stage_bytes = B_ALG_STEP / cfg0.nrk * cfg0.ncell  # one RK3 stage of a stage-fused implementation
    from echo_gpu import counters as CT
    from echo_gpu.lib import fp64_peak

    fp64_gflops, _ = fp64_peak()
    cnt, fresh = (CT.load(COUNTERS) if os.path.exists(COUNTERS) else ({}, False))
    krec = cnt.get("kernels", {})
    traffic = krec.get(dom, {}).get("dram_bytes")
    flop_dom = krec.get(dom, {}).get("fp64_flop")
    flop_step = None
    if all(k in krec for k, (_, n) in prof.items() if n and k in ("faces_x", "faces_y", "faces_z", "update_c2p")):
        flop_step = sum(krec[k]["fp64_flop"] * n for k, (_, n) in prof.items() if k in krec and n)
    counters_src = {"file": os.path.relpath(COUNTERS, ROOT), "build_hash": cnt.get("build_hash"),
                    "this_build": CT.build_hash(), "same_build": fresh}
    launches_per_step = sum(n for (_, n) in prof.values())

    cpu = None
    if world == 1:
        rate, el, sample = cpu_rate(cfg0, tab, przero, threads=1, target_s=6.0, steps=2)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (optical-Glauber Au+Au b=7 fm x Gaussian eta profile, B_y ~ exp(-x^2/2/2.5^2))",
        "config": dict(config_of(cfg0),
                       con2prim="Newton from the previous stage's primitives, residual 1e-10 (BRENTM fallback)",
                       build="libechogpu.so (--fmad=true)", parallelism=f"replicas x{world}"),
        "variants": variants,
        "training": training,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": pk["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "traffic": traffic,
                     "algorithmic_bytes_per_launch": alg,
                     "algorithmic_bytes": "the kernel's own compulsory bytes: read v once, write its face fluxes "
                                          "(faces), or read 3 face arrays, v, u, u0 and write u, v (update)",
                     "launch_ms": dom_ms / dom_n, "peak_src": pk["src"] + " (hbm_gbs)",
                     "traffic_src": counters_src,
                     "stage_b_alg": {"bytes_per_stage": stage_bytes,
                                     "note": "336 B per cell per RK3 stage of a stage-fused implementation (nv = 9)",
                                     "achieved_gbs_over_dominant_launch": stage_bytes / per_launch_s / 1e9,
                                     "frac": stage_bytes / per_launch_s / 1e9 / pk["hbm_gbs"]}},
        "fp64_roofline": {"bound": "fp64", "kernel": dom, "peak_gflops": fp64_gflops,
                          "peak_src": "measured on this GPU by echo_gpu_fp64_peak (independent DFMA chains)",
                          "flop_per_launch": flop_dom,
                          "achieved_gflops": (flop_dom / per_launch_s / 1e9) if flop_dom else None,
                          "frac": (flop_dom / per_launch_s / 1e9 / fp64_gflops) if flop_dom else None,
                          "step_flop_per_cell_update": (flop_step / cfg0.ncell) if flop_step else None,
                          "step_achieved_gflops": (flop_step / cfg0.ncell * value / world / 1e9) if flop_step else None,
                          "step_frac": (flop_step / cfg0.ncell * value / world / 1e9 / fp64_gflops) if flop_step
                          else None,
                          "flop_src": counters_src},
        "step_roofline": {"bytes_per_cell_update": B_ALG_STEP,
                          "achieved_gbs": value / world * B_ALG_STEP / 1e9,
                          "frac": value / world * B_ALG_STEP / 1e9 / pk["hbm_gbs"]},
        "kernels_ms_per_step": {k: round(v[0], 4) for k, v in prof.items()},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * nbytes, "d2h_bytes_per_step": 2 * nbytes,
                "steps": e2e_steps},
        "viscous": viscous,
        "batched": batched,
        "resistive": resistive,
        "ideal_hd": ideal_hd,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
        "stats": {"errcode": st.errcode, "repairs": st.repairs, "t": st2.t, "dt": st.dt},
    }
    print(json.dumps(line), flush=True)
    ev.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--pairs", type=int, default=600_000, help="training pairs for the con2prim seed")
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--batched", type=int, default=1, help="also run the batched event-by-event workload")
    ap.add_argument("--resistive", type=int, default=1, help="also run the resistive RMHD workload")
    ap.add_argument("--viscous", type=int, default=1, help="also run the 2+1D viscous workload")
    ap.add_argument("--ideal-hd", type=int, default=1, help="also run the 2+1D ideal-hydro workload")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
